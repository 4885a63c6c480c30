"""Generates ``screening.npz``: the reference's boundary conditions of the
screened interaction W (the Lyapunov doubling solver, the memoizing
Lyapunov system and CoulombScreeningSolver._compute_contact_obc), the
fixture that pins the oracle's restatement.

Usage (needs the quatrex reference sources)::

    QTX_REFERENCE_SRC=<quatrex checkout>/src python tests/golden/make_screening_golden.py

Case: the synthetic W lead of ``quatrex_b200.synthetic.screened_lead``
(block size 16, 3 energies, seed 4). The contact glue is the reference's own
method, called with a minimal solver object that holds exactly the
attributes it reads (block sections and connected blocks 1, the Coulomb
matrix, OBCSystem(SanchoRubio) and LyapunovSystem(Doubling) with memoization
off).
"""

from __future__ import annotations

import os
import sys
from pathlib import Path
from types import SimpleNamespace

HERE = Path(__file__).resolve().parent
if "QTX_REFERENCE_SRC" not in os.environ:
    sys.exit("set QTX_REFERENCE_SRC to the reference's src/ directory (it holds qttools/ and quatrex/)")
os.environ["QTX_ARRAY_MODULE"] = "numpy"
sys.path.insert(0, str(HERE / "_stubs"))
sys.path.insert(0, os.environ["QTX_REFERENCE_SRC"])
sys.path.insert(0, str(HERE.parent.parent))

import numpy as np  # noqa: E402
import scipy.sparse as sps  # noqa: E402

from qttools.comm import comm  # noqa: E402

_CFG = {k: "device_mpi" for k in ("all_to_all", "all_gather", "all_reduce", "bcast")}
comm.configure(block_comm_size=1, block_comm_config=_CFG, stack_comm_config=_CFG, override=True)

# The contact-ordering helpers quatrex.coulomb_screening.solver imports pull
# in the meshing module of the electrostatics subsystem (gmsh, ase, pyvista),
# which the W boundary conditions never call: an empty stand-in module with
# the one name imported from it keeps that chain out.
import types  # noqa: E402

_meshing = types.ModuleType("quatrex.electrostatics.meshing")
_meshing.inside_shape = None
sys.modules["quatrex.electrostatics.meshing"] = _meshing

from qttools.boundary_conditions.lyapunov import Doubling, LyapunovSystem  # noqa: E402
from qttools.boundary_conditions.obc import OBCSystem, SanchoRubio  # noqa: E402
from qttools.datastructures import DSDBCOO  # noqa: E402
from quatrex.coulomb_screening.solver import CoulombScreeningSolver  # noqa: E402

from quatrex_b200 import synthetic  # noqa: E402

B, NE, SEED = 16, 3, 4


def two_block(blocks, stack):
    """DSDBCOO of two b x b blocks holding (x_10, x_00, x_01) as blocks
    (1, 0), (0, 0), (0, 1) (block (1, 1) = block (0, 0))."""
    pattern = sps.coo_matrix(np.ones((2 * B, 2 * B), dtype=np.complex128))
    m = DSDBCOO.from_sparray(pattern, np.array([B, B]), stack)
    x10, x00, x01 = blocks
    m.blocks[0, 0] = x00
    m.blocks[1, 1] = x00
    m.blocks[0, 1] = x01
    m.blocks[1, 0] = x10
    return m


def main() -> None:
    w = synthetic.screened_lead(B, NE, seed=SEED)
    out = {}
    # Lyapunov doubling on its own: a random contraction a and a stacked q.
    rng = np.random.default_rng(9)
    a = (rng.standard_normal((NE, B, B)) + 1j * rng.standard_normal((NE, B, B))) * 0.08
    q = rng.standard_normal((2, NE, B, B)) + 1j * rng.standard_normal((2, NE, B, B))
    out["lyap_a"], out["lyap_q"] = a, q
    out["lyap_x"] = Doubling()(a, q, "test")
    x, rel, ab = LyapunovSystem(Doubling(), memoization_mode="off")((a, q), "test")
    out["lyap_system_x"], out["lyap_system_rel"], out["lyap_system_abs"] = x, rel, ab
    # The contact glue of the W solve.
    stub = SimpleNamespace(
        small_block_sections=1, num_connected_blocks=1,
        coulomb_matrix=two_block(tuple(np.broadcast_to(x, (1, B, B)) for x in w["v"]), (1,)),
        obc=OBCSystem(SanchoRubio(max_iterations=100, convergence_tol=1e-12), memoization_mode="off"),
        lyapunov=LyapunovSystem(Doubling(), memoization_mode="off"))
    p = {k: two_block(w[k], (NE,)) for k in ("p_lesser", "p_greater", "p_retarded")}
    obc_r, obc_l, obc_g = CoulombScreeningSolver._compute_contact_obc(
        stub, "left", p["p_lesser"], p["p_greater"], p["p_retarded"], diagonal_inds=(0, 0), upper_inds=(0, 1))
    out["obc_retarded"], out["obc_lesser"], out["obc_greater"] = obc_r, obc_l, obc_g
    np.savez_compressed(HERE / "screening.npz", **out)
    print("wrote", HERE / "screening.npz", sorted(out))


if __name__ == "__main__":
    main()
