"""Column-split inverse: the one-CTA Gauss-Jordan kernel launched as a
cluster of C CTAs per matrix, each factoring every panel itself and
updating its own range of columns (replaces the batched inverse of qttools
kernels/linalg/inv.py:6-40 for small batches of blocks up to 400 wide).

Every CTA of a cluster runs the same panel arithmetic on the same data, and
each column is updated by exactly one CTA with the same instruction sequence
as in the single-CTA kernel, so the results must be BIT-identical to the
single-CTA path (inverse path 1), pivots and singular reports included."""

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
    return info.cpu().numpy()


@pytest.mark.parametrize("n", [16, 64, 100, 200, 255, 256, 300, 384, 400])
def test_split_is_bit_identical_to_one_cta(cuda_device, path, n):
    rng = np.random.default_rng(4400 + n)
    B = 5
    a = _rand(rng, B, n, n)
    A = torch.from_numpy(a).to(cuda_device)
    outs, infos = {}, {}
    for mode in (1, 4):
        path(mode)
        X = torch.empty_like(A)
        infos[mode] = _inv(mat(A), mat(X), n, B, cuda_device)
        outs[mode] = X.cpu().numpy()
    np.testing.assert_array_equal(A.cpu().numpy(), a)  # out of place: input untouched
    np.testing.assert_array_equal(outs[4], outs[1])
    np.testing.assert_array_equal(infos[4], infos[1])
    ref = np.linalg.inv(a)
    cond = np.linalg.cond(a).max()
    assert np.linalg.norm(outs[4] - ref) / np.linalg.norm(ref) < 1e-15 * cond * n


@pytest.mark.parametrize("n", [96, 256])
def test_split_in_place_strided_and_permuted(cuda_device, path, n):
    """In place on a strided stack (ld > n, padding untouched), on
    row-permuted diagonally dominant matrices whose pivots come from rows
    spread over the whole block."""
    rng = np.random.default_rng(n)
    B = 6
    core = _rand(rng, B, n, n) + 4.0 * n * np.eye(n)
    for b in range(B):
        core[b] = core[b][rng.permutation(n)]
    big = np.concatenate([core, _rand(rng, B, n, 8)], axis=-1)
    res = {}
    for mode in (1, 4):
        path(mode)
        T = torch.from_numpy(big).to(cuda_device)
        view = QtxMat(T.data_ptr(), n + 8, n * (n + 8))
        assert (_inv(view, view, n, B, cuda_device) == 0).all()
        res[mode] = T.cpu().numpy()
    np.testing.assert_array_equal(res[4], res[1])
    np.testing.assert_array_equal(res[4][..., n:], big[..., n:])
    ref = np.linalg.inv(core)
    assert np.linalg.norm(res[4][..., :n] - ref) / np.linalg.norm(ref) < 1e-13


def test_split_singular_report_and_automatic_choice(cuda_device, path):
    """A zero column reports its 1-based index from every path; at a small
    batch the automatic choice (column split for n <= 400) gives the
    single-CTA bits."""
    n, B = 256, 16
    rng = np.random.default_rng(3)
    a = _rand(rng, B, n, n)
    a[2, :, 77] = 0.0
    A = torch.from_numpy(a).to(cuda_device)
    outs, infos = {}, {}
    for mode in (1, 4, 0):
        path(mode)
        X = torch.empty_like(A)
        infos[mode] = _inv(mat(A), mat(X), n, B, cuda_device)
        outs[mode] = X.cpu().numpy()
    for mode in (4, 0):
        np.testing.assert_array_equal(infos[mode], infos[1])
        ok = np.arange(B) != 2
        np.testing.assert_array_equal(outs[mode][ok], outs[1][ok])
    assert infos[1][2] == 78 and (infos[1][np.arange(B) != 2] == 0).all()
