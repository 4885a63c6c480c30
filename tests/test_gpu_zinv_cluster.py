"""Cluster Gauss-Jordan inverse (one thread-block cluster per matrix, the
matrix in distributed shared memory, TMA-loaded) against NumPy and against
the one-CTA-per-matrix kernel with the same pivot rule; replaces the batched
inverse of qttools kernels/linalg/inv.py:6-40 for n <= 256."""

import ctypes

import numpy as np
import pytest
import torch

from quatrex_b200 import _native
from quatrex_b200._interop import mat
from quatrex_b200._native import QtxMat

pytestmark = pytest.mark.gpu


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _rand(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.fixture
def path():
    lib = _native.load()

    def set_path(mode):
        _native.check(lib.qtx_set_inverse_path(mode))

    yield set_path
    set_path(0)


def _inv(a_mat, x_mat, n, B, device):
    lib = _native.load()
    info = torch.zeros(B, dtype=torch.int32, device=device)
    _native.check(lib.qtx_zinv_batched(n, B, a_mat, x_mat, info.data_ptr(), _stream()))
    torch.cuda.synchronize()
    assert lib.qtx_inverse_status() == 0
    return info.cpu().numpy()


@pytest.mark.parametrize("n", [1, 3, 16, 17, 31, 32, 33, 64, 100, 128, 200, 255, 256])
def test_cluster_inverse_matches_numpy(cuda_device, path, n):
    path(3)
    rng = np.random.default_rng(9100 + n)
    B = 5
    a = _rand(rng, B, n, n)
    A = torch.from_numpy(a).to(cuda_device)
    X = torch.empty_like(A)
    info = _inv(mat(A), mat(X), n, B, cuda_device)
    assert (info == 0).all()
    np.testing.assert_array_equal(A.cpu().numpy(), a)  # out of place: input untouched
    x = X.cpu().numpy()
    ref = np.linalg.inv(a)
    cond = np.linalg.cond(a).max()
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-15 * cond * n
    assert np.linalg.norm(a @ x - np.eye(n)) / np.sqrt(n) < 1e-15 * cond * n


@pytest.mark.parametrize("n", [48, 256])
def test_cluster_inverse_agrees_with_one_cta_kernel(cuda_device, path, n):
    """Same pivot rule, same algebra: the two kernels agree to rounding; in
    place (X = A) and with a strided stack (ld > n) that the tensor map
    covers."""
    rng = np.random.default_rng(n)
    B = 7
    big = torch.from_numpy(_rand(rng, B, n, n + 8)).to(cuda_device)
    ref = big.clone()
    view = QtxMat(big.data_ptr(), n + 8, n * (n + 8))
    path(1)
    _inv(view, view, n, B, cuda_device)
    one = big.clone()
    big.copy_(ref)
    path(3)
    _inv(view, view, n, B, cuda_device)
    got = big.cpu().numpy()
    assert np.linalg.norm(got[..., :n] - one.cpu().numpy()[..., :n]) / np.linalg.norm(got[..., :n]) < 1e-12
    np.testing.assert_array_equal(got[..., n:], ref.cpu().numpy()[..., n:])  # padding untouched


def test_cluster_inverse_broadcast_input_and_singular_report(cuda_device, path):
    """A stride-0 input (one matrix for the whole batch) takes the plain-load
    path; an exactly singular matrix reports the 1-based column of its first
    zero pivot like the one-CTA kernel."""
    n, B = 96, 4
    rng = np.random.default_rng(5)
    a = _rand(rng, n, n)
    A = torch.from_numpy(a).to(cuda_device)
    X = torch.empty((B, n, n), dtype=torch.complex128, device=cuda_device)
    path(3)
    info = _inv(QtxMat(A.data_ptr(), n, 0), mat(X), n, B, cuda_device)
    assert (info == 0).all()
    ref = np.linalg.inv(a)
    for b in range(B):
        assert np.linalg.norm(X[b].cpu().numpy() - ref) / np.linalg.norm(ref) < 1e-11
    s = a.copy()
    s[:, 40] = 0.0  # column 40 is zero: the pivot search of column 40 finds nothing
    S = torch.from_numpy(np.stack([s, a])).to(cuda_device)
    Y = torch.empty_like(S)
    reports = {}
    for mode in (1, 3):
        path(mode)
        reports[mode] = _inv(mat(S), mat(Y), n, 2, cuda_device)
    assert reports[3][0] == reports[1][0] == 41
    assert reports[3][1] == 0
