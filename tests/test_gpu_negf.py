"""The whole energy point (both-contact Sancho-Rubio OBC, selected solve with
G^R, G^<, G^>, Meir-Wingreen current, Caroli transmission, density) on the
GPU against the reference golden vectors and the oracle.

Tolerance (FP64): 1e-10 relative for the RGF outputs given the same
boundary self-energies; the Sancho-Rubio surface Green's function itself is
rounding-sensitive at eta = 1e-4 (the reference's own left/right
orientation flip moves Sigma_R by 1.4e-10 relative), so the end-to-end
energy-point results are checked at 1e-9."""

import numpy as np
import pytest
import torch

from oracle import negf_oracle as o
from quatrex_b200 import EnergyPointSolver, synthetic

pytestmark = pytest.mark.gpu

TOL_E2E = 1e-9


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def cfg0_gpu(cuda_device):
    dev = synthetic.cfg0()
    s = EnergyPointSolver(dev.h_diag, dev.coupling, eta=dev.eta, sr_tol=1e-12, per_energy=False)
    r = s.solve(dev.energies, dev.fermi_left(), dev.fermi_right())
    torch.cuda.synchronize()
    return dev, s, r


def test_cfg0_observables_match_reference(golden, cfg0_gpu):
    g = golden("cfg0")
    _, _, r = cfg0_gpu
    errs = {
        "transmission": _rel(r.transmission.cpu().numpy(), g["transmission"]),
        "density": _rel(r.density.cpu().numpy(), g["density"]),
        "current": _rel(r.current.cpu().numpy(), g["current"]),
        "sigma_left": _rel(r.sigma_left.cpu().numpy()[g["pick"]], g["sigma_left"]),
        "sigma_right": _rel(r.sigma_right.cpu().numpy()[g["pick"]], g["sigma_right"]),
    }
    print("cfg0 errors vs reference:", errs)
    assert all(v < TOL_E2E for v in errs.values()), errs


def test_cfg0_blocks_match_reference(golden, cfg0_gpu):
    g = golden("cfg0")
    _, _, r = cfg0_gpu
    pick = g["pick"]
    xr = r.blocks["xr_diag"].cpu().numpy()
    xl = r.blocks["xl_diag"].cpu().numpy()
    errs = {}
    for k, i in enumerate(g["pick_blocks"]):
        errs[f"xr{i}"] = _rel(xr[i][pick], g["xr_diag"][k])
        errs[f"xl{i}"] = _rel(xl[i][pick], g["xl_diag"][k])
    errs["xg8"] = _rel(r.blocks["xg_diag"][8].cpu().numpy()[pick], g["xg_diag8"])
    errs["xl01"] = _rel(r.blocks["xl_upper"][0].cpu().numpy()[pick], g["xl_upper01"])
    errs["xl10"] = _rel(r.blocks["xl_lower"][0].cpu().numpy()[pick], g["xl_lower10"])
    print("cfg0 block errors vs reference:", errs)
    assert all(v < TOL_E2E for v in errs.values()), errs


def test_cfg0_rgf_given_same_obc_matches_oracle(cfg0_gpu):
    """Isolates the RGF part: the oracle solve fed with the GPU's boundary
    self-energies must agree to 1e-10."""
    dev, s, r = cfg0_gpu
    e = dev.energies[:8]
    diag, upper, lower = dev.system_blocks(e)
    n = dev.num_blocks
    sl = r.sigma_left.cpu().numpy()[:8]
    sr = r.sigma_right.cpu().numpy()[:8]
    fl, fr = dev.fermi_left(e), dev.fermi_right(e)
    gam = lambda x: 1j * (x - x.conj().swapaxes(-2, -1))  # noqa: E731
    obr, obl, obg = [None] * n, [None] * n, [None] * n
    obr[0], obr[-1] = sl, sr
    obl[0], obl[-1] = 1j * gam(sl) * fl[:, None, None], 1j * gam(sr) * fr[:, None, None]
    obg[0], obg[-1] = 1j * gam(sl) * (fl - 1)[:, None, None], 1j * gam(sr) * (fr - 1)[:, None, None]
    z = [np.zeros_like(d) for d in diag]
    zu = [np.zeros_like(u) for u in upper]
    ref = o.selected_solve(diag, upper, lower, z, zu, zu, z, zu, zu, obr, obl, obg, return_current=True)
    errs = {
        "current": _rel(r.current.cpu().numpy()[:8], ref["current"]),
        "xr0": _rel(r.blocks["xr_diag"][0].cpu().numpy()[:8], ref["xr_diag"][0]),
        "xl5": _rel(r.blocks["xl_diag"][5].cpu().numpy()[:8], ref["xl_diag"][5]),
        "xg_up3": _rel(r.blocks["xg_upper"][3].cpu().numpy()[:8], ref["xg_upper"][3]),
        "xl_lo3": _rel(r.blocks["xl_lower"][3].cpu().numpy()[:8], ref["xl_lower"][3]),
        "density": _rel(r.density.cpu().numpy()[:8], o.density(ref["xl_diag"])),
    }
    print("cfg0 RGF errors vs oracle (same OBC):", errs)
    assert all(v < 1e-10 for v in errs.values()), errs


def test_cfg0_transmission_equals_boundary_current(cfg0_gpu):
    """Ballistic check: -Re I_0 = (f_L - f_R) T where f_L != f_R."""
    dev, _, r = cfg0_gpu
    fl, fr = dev.fermi_left(), dev.fermi_right()
    sel = np.abs(fl - fr) > 1e-3
    t = r.transmission.cpu().numpy()
    i0 = r.current.cpu().numpy()[:, 0]
    assert sel.any()
    np.testing.assert_allclose(-i0.real[sel] / (fl - fr)[sel], t[sel], rtol=1e-8)


def test_batch_independence(cuda_device, cfg0_gpu):
    """Each energy's result is the same alone and inside a batch."""
    dev, _, r = cfg0_gpu
    s = EnergyPointSolver(dev.h_diag, dev.coupling, eta=dev.eta, sr_tol=1e-12, per_energy=True)
    idx = [3, 17]
    one = s.solve(dev.energies[idx], dev.fermi_left()[idx], dev.fermi_right()[idx])
    t1 = one.transmission.cpu().numpy()
    assert _rel(t1, r.transmission.cpu().numpy()[idx]) < 1e-10


def test_cfg1_sample_matches_reference(cuda_device, golden):
    g = golden("cfg1_sample")
    dev = synthetic.cfg1()
    e = dev.energies[g["energy_index"]]
    s = EnergyPointSolver(dev.h_diag, dev.coupling, eta=dev.eta, sr_tol=1e-12, per_energy=False)
    r = s.solve(e, dev.fermi_left(e), dev.fermi_right(e))
    errs = {
        "transmission": _rel(r.transmission.cpu().numpy(), g["transmission"]),
        "density": _rel(r.density.cpu().numpy(), g["density"]),
        "current": _rel(r.current.cpu().numpy(), g["current"]),
        "xr_fro": _rel(np.linalg.norm(r.blocks["xr_diag"].cpu().numpy(), axis=(-2, -1)).T, g["xr_fro"]),
        "xl_fro": _rel(np.linalg.norm(r.blocks["xl_diag"].cpu().numpy(), axis=(-2, -1)).T, g["xl_fro"]),
    }
    print("cfg1 sample errors vs reference:", errs)
    assert all(v < TOL_E2E for v in errs.values()), errs
