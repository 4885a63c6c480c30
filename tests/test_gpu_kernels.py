"""CUDA kernels through the C ABI against NumPy complex128 (FP64 tolerance
stated per test)."""

import ctypes

import numpy as np
import pytest
import torch

from quatrex_b200 import _native
from quatrex_b200._interop import mat
from quatrex_b200.obc import inverse

pytestmark = pytest.mark.gpu


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _rand(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def _op(x, op):
    return x.conj().swapaxes(-2, -1) if op else x


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (2, 3, 5), (17, 33, 9), (64, 64, 64), (100, 70, 130),
                                   (256, 256, 256), (65, 129, 257)])
@pytest.mark.parametrize("op_a,op_b", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_zgemm_matches_numpy(cuda_device, m, n, k, op_a, op_b):
    rng = np.random.default_rng(m * 1000 + n * 10 + k + op_a * 2 + op_b)
    B = 3
    a = _rand(rng, B, *((k, m) if op_a else (m, k)))
    b = _rand(rng, B, *((n, k) if op_b else (k, n)))
    d = _rand(rng, B, n, m)
    ref = (0.5 - 2j) * (_op(a, op_a) @ _op(b, op_b)) + (1.5 + 0.25j) * _op(d, 1)
    A = torch.from_numpy(a).to(cuda_device)
    Bt = torch.from_numpy(b).to(cuda_device)
    D = torch.from_numpy(d).to(cuda_device)
    C = torch.empty((B, m, n), dtype=torch.complex128, device=cuda_device)
    _native.check(_native.load().qtx_zgemm_batched(m, n, k, B, 0.5, -2.0, mat(A), op_a, mat(Bt), op_b, 1.5,
                                                   0.25, mat(D), 1, mat(C), _stream()))
    got = C.cpu().numpy()
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err < 1e-14 * max(1.0, np.sqrt(k)), err


@pytest.mark.parametrize("op_a,op_b", [(0, 0), (1, 0), (0, 1)])
def test_zgemm_grouped_matches_numpy(cuda_device, op_a, op_b):
    """qtx_zgemm_grouped: per-entry pointers from device tables, a broadcast
    A block (the same pointer in two entries), accumulation into C (D = C) and
    a plain store; against NumPy."""
    rng = np.random.default_rng(31 + op_a * 2 + op_b)
    b, lib = 24, _native.load()
    X = torch.from_numpy(_rand(rng, 5, b, b)).to(cuda_device)
    C0 = _rand(rng, 3, b, b)
    Y = torch.from_numpy(C0).to(cuda_device)
    stride = b * b * 16
    tab = lambda addrs: torch.tensor(addrs, dtype=torch.int64, device=cuda_device)  # noqa: E731
    pa = tab([X.data_ptr(), X.data_ptr(), X.data_ptr() + stride])
    pb = tab([X.data_ptr() + 2 * stride, X.data_ptr() + 3 * stride, X.data_ptr() + 4 * stride])
    pc = tab([Y.data_ptr() + e * stride for e in range(3)])
    x = X.cpu().numpy()
    a_idx, b_idx = [0, 0, 1], [2, 3, 4]
    _native.check(lib.qtx_zgemm_grouped(b, b, b, 3, 0.5, -1.0, pa.data_ptr(), b, op_a, pb.data_ptr(), b, op_b,
                                        1.0, 0.0, pc.data_ptr(), b, 0, pc.data_ptr(), b, _stream()))
    ref = np.stack([C0[e] + (0.5 - 1j) * (_op(x[a_idx[e]], op_a) @ _op(x[b_idx[e]], op_b)) for e in range(3)])
    got = Y.cpu().numpy()
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-14
    # plain store (no addend table)
    _native.check(lib.qtx_zgemm_grouped(b, b, b, 3, 1.0, 0.0, pa.data_ptr(), b, op_a, pb.data_ptr(), b, op_b,
                                        0.0, 0.0, None, 0, 0, pc.data_ptr(), b, _stream()))
    ref = np.stack([_op(x[a_idx[e]], op_a) @ _op(x[b_idx[e]], op_b) for e in range(3)])
    assert np.linalg.norm(Y.cpu().numpy() - ref) / np.linalg.norm(ref) < 1e-14
    with pytest.raises(_native.QtxError):
        _native.check(lib.qtx_zgemm_grouped(b, b, 0, 3, 1.0, 0.0, pa.data_ptr(), b, 0, pb.data_ptr(), b, 0, 0.0,
                                            0.0, None, 0, 0, pc.data_ptr(), b, _stream()))


def test_zgemm_zero_k_and_null_operand(cuda_device):
    rng = np.random.default_rng(5)
    d = _rand(rng, 2, 8, 8)
    D = torch.from_numpy(d).to(cuda_device)
    C = torch.empty_like(D)
    _native.check(_native.load().qtx_zgemm_batched(8, 8, 8, 2, 1.0, 0.0, _native.NULL_MAT, 0, mat(D), 0, 2.0,
                                                   0.0, mat(D), 0, mat(C), _stream()))
    np.testing.assert_allclose(C.cpu().numpy(), 2 * d, rtol=1e-15)


@pytest.mark.parametrize("n", [1, 2, 3, 16, 17, 64, 100, 256, 300, 512, 600, 768, 1024])
def test_zinv_matches_numpy(cuda_device, n):
    rng = np.random.default_rng(n)
    B = 4 if n <= 512 else 2
    a = _rand(rng, B, n, n)  # general matrices: pivoting is exercised
    x = inverse(torch.from_numpy(a).to(cuda_device)).cpu().numpy()
    ref = np.linalg.inv(a)
    err = np.linalg.norm(x - ref) / np.linalg.norm(ref)
    cond = np.linalg.cond(a).max()
    assert err < 1e-15 * cond * n, (err, cond)
    res = np.linalg.norm(a @ x - np.eye(n)) / np.sqrt(n)
    assert res < 1e-15 * cond * n


def test_zinv_in_place_and_pivot_needed(cuda_device):
    # zero leading diagonal entries force row exchanges
    a = np.array([[[0, 1, 2], [1, 0, 3], [4, 5, 0]]], dtype=np.complex128) * (1 + 0.5j)
    t = torch.from_numpy(a).to(cuda_device)
    lib = _native.load()
    info = torch.zeros(1, dtype=torch.int32, device=cuda_device)
    _native.check(lib.qtx_zinv_batched(3, 1, mat(t), mat(t), info.data_ptr(), _stream()))
    np.testing.assert_allclose(t.cpu().numpy(), np.linalg.inv(a), rtol=1e-14, atol=1e-15)
    assert int(info.item()) == 0


def test_zinv_singular_reports(cuda_device):
    a = np.zeros((2, 4, 4), dtype=np.complex128)
    a[0] = np.eye(4)
    a[1, :, :2] = 1.0  # rank 2
    with pytest.raises(np.linalg.LinAlgError):
        inverse(torch.from_numpy(a).to(cuda_device))


def test_coo_densify_sparsify_roundtrip(cuda_device):
    rng = np.random.default_rng(0)
    B, m, n = 3, 5, 7
    mask = rng.random((m, n)) < 0.5
    r, c = np.nonzero(mask)
    nnz = r.size
    data = _rand(rng, B, nnz + 3)
    D = torch.from_numpy(data).to(cuda_device)
    rows = torch.from_numpy(r.astype(np.int32)).to(cuda_device)
    cols = torch.from_numpy(c.astype(np.int32)).to(cuda_device)
    out = torch.full((B, m, n), 9.0 + 0j, dtype=torch.complex128, device=cuda_device)
    lib = _native.load()
    _native.check(lib.qtx_coo_densify(B, D.data_ptr() + 16, D.stride(0), nnz, rows.data_ptr(), cols.data_ptr(),
                                      mat(out), m, n, _stream()))
    ref = np.zeros((B, m, n), dtype=np.complex128)
    ref[:, r, c] = data[:, 1:nnz + 1]
    np.testing.assert_array_equal(out.cpu().numpy(), ref)
    D2 = torch.zeros_like(D)
    _native.check(lib.qtx_coo_sparsify(B, mat(out), nnz, rows.data_ptr(), cols.data_ptr(), D2.data_ptr() + 16,
                                       D2.stride(0), _stream()))
    np.testing.assert_array_equal(D2.cpu().numpy()[:, 1:nnz + 1], data[:, 1:nnz + 1])


def test_assemble_diag(cuda_device):
    rng = np.random.default_rng(1)
    h = _rand(rng, 6, 6)
    z = np.array([0.5 + 1e-4j, -1.0 + 1e-4j])
    H = torch.from_numpy(h).to(cuda_device)
    Z = torch.from_numpy(z).to(cuda_device)
    out = torch.empty((2, 6, 6), dtype=torch.complex128, device=cuda_device)
    _native.check(_native.load().qtx_assemble_diag(6, 2, _native.QtxMat(H.data_ptr(), 6, 0), Z.data_ptr(),
                                                   mat(out), _stream()))
    np.testing.assert_array_equal(out.cpu().numpy(), z[:, None, None] * np.eye(6) - h[None])
