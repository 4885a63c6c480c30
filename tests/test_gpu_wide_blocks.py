"""512-wide blocks (the block size of the 64 x 512 mixed-precision workload)
on every precision of the GPU path, against the complex128 oracle.

A 4-block device of 512 x 512 blocks, built like the other synthetic
devices, on two energies of the [-3, 3] window; the oracle runs the whole
reference energy point (both-contact Sancho-Rubio to 1e-12, OBCSystem step,
contact self-energies, selected solve with current, Caroli transmission,
density) on the CPU.

Stated tolerances against the oracle (relative; transmission per energy):

==========  ============  =======  ===========  =========================
precision   transmission  density  G^R diagonal  why
==========  ============  =======  ===========  =========================
fp64        1e-7          1e-7     1e-6         the reference's own decimation
                                                noise floor (see
                                                test_oracle_noise_floor.py);
                                                1e-10 given the same boundary
                                                self-energies
emulated 6  1e-6          1e-6     1e-5         + ~1e-12 per product
emulated 5  1e-6          5e-6     5e-6         + ~3e-10 per product
mixed       2e-3          2e-2     2e-2         FP32-level products at eta=1e-4
==========  ============  =======  ===========  =========================
"""

import numpy as np
import pytest
import torch

from oracle import negf_oracle as o
from quatrex_b200 import EnergyPointSolver, synthetic

pytestmark = pytest.mark.gpu

TOL = {
    ("fp64", 0): dict(transmission=1e-7, density=1e-7, xr_diag=1e-6),
    ("emulated", 6): dict(transmission=1e-6, density=1e-6, xr_diag=1e-5),
    ("emulated", 5): dict(transmission=1e-6, density=5e-6, xr_diag=5e-6),
    ("mixed", 0): dict(transmission=2e-3, density=2e-2, xr_diag=2e-2),
}


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def wide_case(cuda_device):
    dev = synthetic.make_device(4, 512, np.array([-1.0, 0.62]), seed=0, name="wide")
    diag, upper, lower = dev.system_blocks()
    ref = o.energy_point_solve(diag, upper, lower, dev.fermi_left(), dev.fermi_right())
    return dev, ref


def _solve(dev, precision, slices):
    kw = dict(slices=slices) if precision == "emulated" else {}
    s = EnergyPointSolver(dev.h_diag, dev.coupling, eta=dev.eta, sr_tol=1e-12, per_energy=False,
                          precision=precision, **kw)
    r = s.solve(dev.energies, dev.fermi_left(), dev.fermi_right())
    torch.cuda.synchronize()
    return r


@pytest.mark.parametrize("precision,slices", list(TOL))
def test_wide_blocks_vs_oracle(wide_case, precision, slices):
    dev, ref = wide_case
    r = _solve(dev, precision, slices)
    t = r.transmission.cpu().numpy()
    xr = r.blocks["xr_diag"].cpu().numpy().astype(np.complex128)
    errs = {
        "transmission": float(np.max(np.abs(t - ref["transmission"]) / np.abs(ref["transmission"]))),
        "density": _rel(r.density.cpu().numpy(), ref["density"]),
        "xr_diag": max(_rel(xr[i], ref["xr_diag"][i]) for i in range(dev.num_blocks)),
    }
    print(f"512-wide {precision}/{slices} vs oracle:", errs)
    tol = TOL[(precision, slices)]
    assert all(errs[k] < tol[k] for k in tol), (errs, tol)


def test_wide_blocks_fp64_rgf_given_same_obc(wide_case):
    """The 1e-10 plain-FP64 gate at 512 x 512: the oracle's selected solve fed
    with the GPU's boundary self-energies."""
    dev, _ = wide_case
    r = _solve(dev, "fp64", 0)
    diag, upper, lower = dev.system_blocks()
    n = dev.num_blocks
    sl, sr = r.sigma_left.cpu().numpy(), r.sigma_right.cpu().numpy()
    fl, fr = dev.fermi_left()[:, None, None], dev.fermi_right()[:, None, None]
    gam = lambda x: 1j * (x - x.conj().swapaxes(-2, -1))  # noqa: E731
    obr, obl, obg = [None] * n, [None] * n, [None] * n
    obr[0], obr[-1] = sl, sr
    obl[0], obl[-1] = 1j * gam(sl) * fl, 1j * gam(sr) * fr
    obg[0], obg[-1] = 1j * gam(sl) * (fl - 1), 1j * gam(sr) * (fr - 1)
    z = [np.zeros_like(d) for d in diag]
    zu = [np.zeros_like(u) for u in upper]
    ref = o.selected_solve(diag, upper, lower, z, zu, zu, z, zu, zu, obr, obl, obg, return_current=True)
    errs = {
        "current": _rel(r.current.cpu().numpy(), ref["current"]),
        "density": _rel(r.density.cpu().numpy(), o.density(ref["xl_diag"])),
        "xr_diag": max(_rel(r.blocks["xr_diag"][i].cpu().numpy(), ref["xr_diag"][i]) for i in range(n)),
        "xl_upper": max(_rel(r.blocks["xl_upper"][i].cpu().numpy(), ref["xl_upper"][i]) for i in range(n - 1)),
        "transmission": _rel(r.transmission.cpu().numpy(),
                             o.transmission_caroli_rgf(diag, upper, lower, obr, sl, sr)),
    }
    print("512-wide fp64 RGF vs oracle (same OBC):", errs)
    assert all(v < 1e-10 for v in errs.values()), errs
