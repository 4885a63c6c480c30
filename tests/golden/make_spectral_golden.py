"""Generates ``spectral.npz``: the reference's spectral OBC (Beyn's contour
method) on strip leads, the fixture that pins the oracle's restatement of
``src/qttools/nevp/beyn.py`` and ``src/qttools/boundary_conditions/obc/
spectral.py``.

Usage (needs the quatrex reference sources)::

    QTX_REFERENCE_SRC=<quatrex checkout>/src python tests/golden/make_spectral_golden.py

Cases: strip leads (``quatrex_b200.synthetic.strip_lead``) of 4 x 4 and
8 x 8 sites per block on 9 energies in [-3.2, 3.2], with the quatrex
configuration defaults of the spectral OBC (``quatrex/core/config.py``:
r_o = 10, r_i = 0.8, 20 quadrature points, min_decay 1e-3, max_decay
1.5 ln r_o, 2 refinement iterations, min_propagation 1e-2, residual
tolerance 1e-3, eta_decay 1e-12) and a subspace of m_0 modes.
"""

from __future__ import annotations

import os
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
if "QTX_REFERENCE_SRC" not in os.environ:
    sys.exit("set QTX_REFERENCE_SRC to the reference's src/ directory (it holds qttools/ and quatrex/)")
os.environ["QTX_ARRAY_MODULE"] = "numpy"
sys.path.insert(0, str(HERE / "_stubs"))
sys.path.insert(0, os.environ["QTX_REFERENCE_SRC"])
sys.path.insert(0, str(HERE.parent.parent))

import numpy as np  # noqa: E402

from qttools.comm import comm  # noqa: E402

_CFG = {k: "device_mpi" for k in ("all_to_all", "all_gather", "all_reduce", "bcast")}
comm.configure(block_comm_size=1, block_comm_config=_CFG, stack_comm_config=_CFG, override=True)

from qttools.boundary_conditions.obc import Spectral  # noqa: E402
from qttools.nevp import Beyn  # noqa: E402

from quatrex_b200 import synthetic  # noqa: E402

CASES = {"w4l4": (4, 4, 10), "w8l8": (8, 8, 20)}
ENERGIES = np.linspace(-3.2, 3.2, 9)


def main() -> None:
    out: dict = {"energies": ENERGIES}
    for tag, (w, slices, m0) in CASES.items():
        a_ii, a_ij, a_ji = synthetic.strip_lead(w, slices, ENERGIES, seed=1)
        solver = Spectral(Beyn(10.0, 0.8, m0, 20), min_decay=1e-3, max_decay=1.5 * np.log(10.0),
                          num_ref_iterations=2, min_propagation=1e-2, residual_tolerance=1e-3,
                          residual_normalization=True, eta_decay=1e-12)
        x1 = solver(a_ii, a_ij, a_ji, "left")
        x2 = solver(a_ii, a_ij, a_ji, "left")  # second call: the subspace guess advances
        out[f"{tag}_shape"] = np.array([w, slices, m0])
        out[f"{tag}_x_ii"] = x1
        out[f"{tag}_x_ii_second"] = x2
    np.savez_compressed(HERE / "spectral.npz", **out)
    print("wrote", HERE / "spectral.npz", sorted(out))


if __name__ == "__main__":
    main()
