"""The oracle's screened-interaction (W) solve against the reference's own
``CoulombScreeningSolver.solve`` (src/quatrex/coulomb_screening/solver.py:
724-889), recorded in ``tests/golden/w_solve.npz`` by
``tests/golden/make_w_solve_golden.py``: the superblock system matrix
I - V P^R with the contact spillover, L^< and L^> (V P V with the spillover),
the contact boundary self-energies, and W^<, W^> without and with the DOS
peak filter. CPU only."""

import numpy as np
import pytest

from oracle import negf_oracle as o


@pytest.fixture(scope="module")
def case(golden):
    g = golden("w_solve")

    def bt(k):
        return (list(g[f"{k}_diag"]), list(g[f"{k}_upper"]), list(g[f"{k}_lower"]))

    def run(limit):
        return o.w_solve(bt("v"), bt("p_lesser"), bt("p_greater"), bt("p_retarded_hermitian"),
                         int(g["num_connected_blocks"]), g["energies"],
                         lambda t: o.obc_system_solve(t[0], t[1], t[2], 100, 1e-12)[0],
                         lambda b, q: o.lyapunov_system_solve(b, q)[0], dos_peak_limit=limit)

    return g, run(None), run(float(g["dos_peak_limit"]))


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def test_w_system_and_boundary_conditions_match_reference(case):
    g, plain, _ = case
    for key in ("m", "ll", "lg"):
        for t, name in enumerate(("diag", "upper", "lower")):
            assert _rel(np.stack(plain[key][t]), g[f"plain_{key}_{name}"]) < 1e-14, (key, name)
    for side, end in (("left", "first"), ("right", "last")):
        for t, name in enumerate(("retarded", "lesser", "greater")):
            assert _rel(plain["obc"][side][t], g[f"plain_obc_{name}_{end}"]) < 1e-13, (side, name)


@pytest.mark.parametrize("which", ["plain", "filtered"])
def test_w_matches_reference(case, which):
    g, plain, filtered = case
    got = plain if which == "plain" else filtered
    for w in ("wl", "wg"):
        for name in ("diag", "upper", "lower"):
            assert _rel(np.stack(got[f"{w}_{name}"]), g[f"{which}_{w}_{name}"]) < 1e-13, (w, name)


def test_peak_filter_mask(case):
    g, _, filtered = case
    np.testing.assert_array_equal(filtered["mask"], [True, False, False, True, True])
    zero = np.array([np.abs(g["filtered_wl_diag"][:, e]).max() == 0 for e in range(g["energies"].size)])
    np.testing.assert_array_equal(zero, filtered["mask"])  # energy 0 is also zeroed unconditionally
