"""Multi-CTA blocked Gauss-Jordan inverse (the large-block / small-batch
path) against NumPy and against the one-CTA-per-matrix kernel."""

import ctypes

import numpy as np
import pytest
import torch

from quatrex_b200 import EnergyPointSolver, _native, synthetic
from quatrex_b200._interop import mat

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


def _inv(a_t, x_t, n, B):
    lib = _native.load()
    info = torch.zeros(B, dtype=torch.int32, device=a_t.device)
    ws = torch.empty(lib.qtx_zinv_workspace(n, B), dtype=torch.uint8, device=a_t.device)
    _native.check(lib.qtx_zinv_batched_ws(n, B, mat(a_t), mat(x_t), info.data_ptr(), ws.data_ptr(), ws.numel(),
                                          _stream()))
    torch.cuda.synchronize()
    return info.cpu().numpy()


@pytest.mark.parametrize("n", [1, 3, 17, 64, 100, 384, 520, 768, 832, 833, 1024])
def test_wide_inverse_matches_numpy(cuda_device, path, n):
    path(2)
    rng = np.random.default_rng(7000 + n)
    B = 3 if n <= 520 else 2
    a = _rand(rng, B, n, n)
    A = torch.from_numpy(a).to(cuda_device)
    X = torch.empty_like(A)
    info = _inv(A, X, n, B)
    assert (info == 0).all()
    np.testing.assert_array_equal(A.cpu().numpy(), a)  # out of place: input untouched
    x = X.cpu().numpy()
    ref = np.linalg.inv(a)
    cond = np.linalg.cond(a).max()
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-15 * cond * n
    assert np.linalg.norm(a @ x - np.eye(n)) / np.sqrt(n) < 1e-15 * cond * n


def test_wide_matches_single_cta(cuda_device, path):
    rng = np.random.default_rng(11)
    n, B = 400, 5
    a = _rand(rng, B, n, n)
    out = {}
    for mode in (1, 2):
        path(mode)
        t = torch.from_numpy(a).to(cuda_device)
        _inv(t, t, n, B)  # in place
        out[mode] = t.cpu().numpy()
    assert np.linalg.norm(out[2] - out[1]) / np.linalg.norm(out[1]) < 1e-12


def test_wide_pivoting_and_singular_info(cuda_device, path):
    path(2)
    a = np.array([[[0, 1, 2], [1, 0, 3], [4, 5, 0]]], dtype=np.complex128) * (1 + 0.5j)
    t = torch.from_numpy(a).to(cuda_device)
    assert _inv(t, t, 3, 1)[0] == 0
    np.testing.assert_allclose(t.cpu().numpy(), np.linalg.inv(a), rtol=1e-14, atol=1e-15)
    # a zero column: both paths report the same first zero pivot
    rng = np.random.default_rng(3)
    n = 40
    s = _rand(rng, 2, n, n)
    s[1, :, 21] = 0.0
    infos = {}
    for mode in (1, 2):
        path(mode)
        t = torch.from_numpy(s).to(cuda_device)
        infos[mode] = _inv(t, t, n, 2)
    assert infos[1][0] == 0 and infos[1][1] > 0
    np.testing.assert_array_equal(infos[1], infos[2])


def test_energy_points_through_wide_inverse(cuda_device, path):
    dev = synthetic.make_device(3, 400, np.linspace(-1.0, 1.0, 4), seed=21)
    res = {}
    for mode in (1, 2):
        path(mode)
        s = EnergyPointSolver(dev.h_diag, dev.coupling, eta=dev.eta, sr_tol=1e-12, per_energy=True,
                              store_blocks=False)
        r = s.solve(dev.energies, dev.fermi_left(), dev.fermi_right())
        res[mode] = (r.transmission.cpu().numpy().copy(), r.density.cpu().numpy().copy())
        del s
    # The two paths round differently in the last bits; the Sancho-Rubio
    # decimation amplifies that to ~1e-8 (the same noise floor as LAPACK vs
    # Gauss-Jordan inverses in the end-to-end parity tests).
    for k in range(2):
        assert np.linalg.norm(res[2][k] - res[1][k]) / np.linalg.norm(res[1][k]) < 1e-7
