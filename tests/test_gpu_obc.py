"""Sancho-Rubio, the OBCSystem memoizer and the contact self-energies on the
GPU. Mirrors tests/qttools/boundary_conditions/obc/test_sancho_rubio.py:9-50
(fixed-point property, batched, max_iterations warning, memoizer modes) on
synthetic leads (the reference fixture reads an HDF5 example that is not
available), plus parity with the oracle."""

import numpy as np
import pytest
import torch

from oracle import negf_oracle as o
from quatrex_b200 import OBCSystem, SanchoRubio, contact_self_energy, synthetic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def leads():
    dev = synthetic.cfg0()
    e = dev.energies[::4]
    diag, upper, lower = dev.system_blocks(e)
    return dev, e, diag, upper, lower


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_convergence_single(cuda_device, leads):
    _, _, diag, upper, lower = leads
    sr = SanchoRubio(convergence_tol=1e-10)
    a_ii, a_ij, a_ji = diag[0][0], upper[0][0], lower[0][0]
    x = sr(a_ii, a_ij, a_ji, contact="")
    assert x.shape == a_ii.shape and isinstance(x, np.ndarray)
    assert np.allclose(x, np.linalg.inv(a_ii - a_ji @ x @ a_ij))


def test_convergence_batch_matches_oracle(cuda_device, leads):
    _, _, diag, upper, lower = leads
    sr = SanchoRubio(convergence_tol=1e-12)
    x = sr(diag[0], upper[0], lower[0], contact="")
    assert np.allclose(x, np.linalg.inv(diag[0] - lower[0] @ x @ upper[0]))
    ref, it, conv = o.sancho_rubio(diag[0], upper[0], lower[0], convergence_tol=1e-12)
    assert conv and abs(sr.last_iterations - it) <= 1
    # The decimation amplifies rounding (1e-14 perturbations of an inverse
    # move the result by up to ~1e-8 on these 64x64 leads).
    assert _rel(x, ref) < 1e-7, _rel(x, ref)


def test_per_energy_convergence_close_to_batchwide(cuda_device, leads):
    _, _, diag, upper, lower = leads
    a = [torch.from_numpy(np.ascontiguousarray(m)).to(cuda_device) for m in (diag[0], upper[0], lower[0])]
    xb, itb, _ = SanchoRubio(convergence_tol=1e-12).solve_device(*a)
    xp, itp, conv = SanchoRubio(convergence_tol=1e-12, per_energy=True).solve_device(*a)
    assert conv and itp == itb
    assert _rel(xp.cpu().numpy(), xb.cpu().numpy()) < 1e-12


def test_max_iterations_warns(cuda_device, leads):
    _, _, diag, upper, lower = leads
    sr = SanchoRubio(max_iterations=1, convergence_tol=1e-8)
    with pytest.warns(RuntimeWarning):
        sr(diag[0], upper[0], lower[0], contact="")


@pytest.mark.parametrize("mode", ["off", "auto", "force-after-first"])
def test_memoizer(cuda_device, leads, mode):
    _, _, diag, upper, lower = leads
    system = OBCSystem(SanchoRubio(convergence_tol=1e-10), memoization_mode=mode)
    a_ii, a_ij, a_ji = diag[0], upper[0], lower[0]
    x, rel, ab = system((a_ii, a_ij, a_ji), contact="contact")
    assert np.allclose(x, np.linalg.inv(a_ii - a_ji @ x @ a_ij), atol=1e-5)
    a_ii, a_ij, a_ji = a_ii * (1 + 1e-6), a_ij * (1 + 1e-6), a_ji * (1 + 1e-6)
    x, rel, ab = system((a_ii, a_ij, a_ji), contact="contact")
    assert np.allclose(x, np.linalg.inv(a_ii - a_ji @ x @ a_ij), atol=1e-5)
    assert rel.shape == a_ii.shape[:1]


def test_contact_self_energy_matches_oracle(cuda_device, leads):
    dev, e, diag, upper, lower = leads
    f = dev.fermi_left(e)
    ref = o.contact_self_energies(diag[0], upper[0], lower[0], f, convergence_tol=1e-12)
    g = ref[3]
    sig, sl, sg = contact_self_energy(upper[0], lower[0], g, f)
    for got, want in zip((sig, sl, sg), ref[:3]):
        assert _rel(got, want) < 1e-13


def test_memoizer_force_mode_semantics(cuda_device, leads):
    """'force' starts from inv(a_ii) and applies the residual step
    (boundary_system.py:270-278): the result is one fixed-point step from
    inv(a_ii), reported with a high-error warning."""
    _, _, diag, upper, lower = leads
    system = OBCSystem(SanchoRubio(convergence_tol=1e-10), memoization_mode="force")
    a = (diag[0], upper[0], lower[0])
    with pytest.warns(RuntimeWarning):
        x, rel, ab = system(a, contact="c")
    x0 = np.linalg.inv(diag[0])
    x1 = np.linalg.inv(diag[0] - lower[0] @ x0 @ upper[0])
    x2 = np.linalg.inv(diag[0] - lower[0] @ x1 @ upper[0])
    assert _rel(x, x2) < 1e-10


def test_sancho_rubio_multi_matches_single_systems(cuda_device, leads):
    """Both contacts in one decimation loop equal two separate solves."""
    import ctypes

    from quatrex_b200 import _native
    from quatrex_b200._interop import mat
    from quatrex_b200._native import QtxMat

    _, _, diag, upper, lower = leads
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(cuda_device)  # noqa: E731
    left = (t(diag[0]), t(upper[0]), t(lower[0]))
    right = (t(diag[-1]), t(lower[-1]), t(upper[-1]))
    sr = SanchoRubio(convergence_tol=1e-12, per_energy=True)
    xl, _, _ = sr.solve_device(*left)
    xr, _, _ = sr.solve_device(*right)
    lib = _native.load()
    B, n = left[0].shape[0], left[0].shape[-1]
    outs = [torch.empty_like(left[0]), torch.empty_like(right[0])]
    ws = torch.empty(lib.qtx_sancho_rubio_workspace(n, 2 * B), dtype=torch.uint8, device=cuda_device)
    it, conv = ctypes.c_int(0), ctypes.c_int(0)
    _native.check(lib.qtx_sancho_rubio_multi(
        n, 2, (ctypes.c_int64 * 2)(B, B), (QtxMat * 2)(mat(left[0]), mat(right[0])),
        (QtxMat * 2)(mat(left[1]), mat(right[1])), (QtxMat * 2)(mat(left[2]), mat(right[2])),
        (QtxMat * 2)(mat(outs[0]), mat(outs[1])), 100, 1e-12, 1, ctypes.byref(it), ctypes.byref(conv), None,
        ws.data_ptr(), ws.numel(), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    assert conv.value == 1
    assert _rel(outs[0].cpu().numpy(), xl.cpu().numpy()) < 1e-13
    assert _rel(outs[1].cpu().numpy(), xr.cpu().numpy()) < 1e-13
