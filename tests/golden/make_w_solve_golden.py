"""Generates ``w_solve.npz``: the reference's screened-interaction (W) solve,
``CoulombScreeningSolver.solve`` (src/quatrex/coulomb_screening/solver.py:
724-889), on a synthetic device, the fixture that pins the oracle's
restatement ``oracle.negf_oracle.w_solve`` and the GPU solve.

Usage (needs the quatrex reference sources)::

    QTX_REFERENCE_SRC=<quatrex checkout>/src python tests/golden/make_w_solve_golden.py

Case: ``quatrex_b200.synthetic.screened_device`` with 9 small blocks of 8,
5 energies, seed 1, three connected blocks (superblocks of 24), OBC block
sections 1, non-symmetric storage. The solver object is built without its
configuration-driven constructor: it holds exactly the attributes ``solve``
and the methods it calls read, with the containers allocated the way the
constructor allocates them (solver.py:61-196: sparsity patterns of V P and
V P V from the module's own ``_compute_sparsity_pattern``, the system
matrix and L^<, L^> in superblocks, P^R in small blocks), OBCSystem
(SanchoRubio, tol 1e-12) and LyapunovSystem(Doubling) with memoization off,
and the reference's RGF wrapped to record the system it is handed. Two
solves: without the peak filter, and with it at a threshold between the
DOS gradients of the energies so that some are filtered (energies 0, 3, 4).
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

import types  # noqa: E402

import numpy as np  # noqa: E402
import scipy.sparse as sps  # noqa: E402

from qttools.comm import comm  # noqa: E402

_CFG = {k: "device_mpi" for k in ("all_to_all", "all_gather", "all_reduce", "bcast")}
comm.configure(block_comm_size=1, block_comm_config=_CFG, stack_comm_config=_CFG, override=True)

# See make_screening_golden.py: the contact-ordering helpers pull in the
# electrostatics meshing module, which the W solve never calls.
_meshing = types.ModuleType("quatrex.electrostatics.meshing")
_meshing.inside_shape = None
sys.modules["quatrex.electrostatics.meshing"] = _meshing

from qttools.boundary_conditions.lyapunov import Doubling, LyapunovSystem  # noqa: E402
from qttools.boundary_conditions.obc import OBCSystem, SanchoRubio  # noqa: E402
from qttools.datastructures import DSDBCOO  # noqa: E402
from qttools.greens_function_solver import RGF  # noqa: E402
from qttools.greens_function_solver.solver import OBCBlocks  # noqa: E402
from quatrex.coulomb_screening import solver as cs  # noqa: E402

from quatrex_b200 import synthetic  # noqa: E402

NS, B, NC, NE, SEED = 9, 8, 3, 5, 1


def bt_pattern(n, b):
    mask = np.zeros((n * b, n * b))
    for i in range(n):
        for j in (i - 1, i, i + 1):
            if 0 <= j < n:
                mask[i * b:(i + 1) * b, j * b:(j + 1) * b] = 1.0
    return sps.coo_matrix(mask)


def container(blocks, stack):
    diag, upper, lower = blocks
    m = DSDBCOO.from_sparray(bt_pattern(NS, B).astype(np.complex128), np.full(NS, B), stack)
    for i in range(NS):
        m.blocks[i, i] = np.broadcast_to(diag[i], stack + (B, B))
        if i + 1 < NS:
            m.blocks[i, i + 1] = np.broadcast_to(upper[i], stack + (B, B))
            m.blocks[i + 1, i] = np.broadcast_to(lower[i], stack + (B, B))
    return m


class RecordingRGF:
    """The reference's RGF, recording the superblock system it solves."""

    def __init__(self):
        self.inner = RGF()
        self.seen = {}

    def selected_solve(self, a, sigma_lesser, sigma_greater, obc_blocks, out, return_retarded=False):
        n = a.num_blocks
        for name, m in (("m", a), ("ll", sigma_lesser), ("lg", sigma_greater)):
            self.seen[f"{name}_diag"] = np.stack([np.array(m.blocks[i, i]) for i in range(n)])
            self.seen[f"{name}_upper"] = np.stack([np.array(m.blocks[i, i + 1]) for i in range(n - 1)])
            self.seen[f"{name}_lower"] = np.stack([np.array(m.blocks[i + 1, i]) for i in range(n - 1)])
        for key in ("retarded", "lesser", "greater"):
            self.seen[f"obc_{key}_first"] = np.array(getattr(obc_blocks, key)[0])
            self.seen[f"obc_{key}_last"] = np.array(getattr(obc_blocks, key)[-1])
        return self.inner.selected_solve(a=a, sigma_lesser=sigma_lesser, sigma_greater=sigma_greater,
                                         obc_blocks=obc_blocks, out=out, return_retarded=return_retarded)


def make_solver(d, energies, dos_peak_limit, filtering):
    s = cs.CoulombScreeningSolver.__new__(cs.CoulombScreeningSolver)
    small = np.full(NS, B)
    s.coulomb_matrix = container(d["v"], (1,))
    s.small_block_sizes = small
    s.num_connected_blocks = NC
    s.block_sizes = small[: NS // NC] * NC
    dummy = DSDBCOO.from_sparray(bt_pattern(NS, B).astype(np.float32), small, (1,))
    vp = cs._compute_sparsity_pattern(dummy, dummy, dtype=np.float32)
    s.system_matrix = DSDBCOO.from_sparray(vp.astype(np.complex128), s.block_sizes, energies.shape)
    s.system_matrix.free_data()
    lp = cs._compute_sparsity_pattern(dummy, dummy, dummy, dtype=np.float32)
    s.l_lesser = DSDBCOO.from_sparray(lp.astype(np.complex128), s.block_sizes, energies.shape)
    s.l_greater = DSDBCOO.zeros_like(s.l_lesser)
    s.l_lesser.free_data()
    s.l_greater.free_data()
    s.p_retarded = DSDBCOO.from_sparray(bt_pattern(NS, B).astype(np.complex128), small, energies.shape)
    s.p_retarded.free_data()
    s.energies = energies
    s.dos_peak_limit = dos_peak_limit
    s.obc_blocks = OBCBlocks(num_blocks=NS // NC)
    s.block_sections = 1
    s.small_block_sections = 1
    s.flatband = False
    s.solve_call_count = 0
    s.filtering_iteration_limit = 1 if filtering else 0
    s.max_batch_size = None
    s.obc = OBCSystem(SanchoRubio(max_iterations=100, convergence_tol=1e-12), memoization_mode="off")
    s.lyapunov = LyapunovSystem(Doubling(), memoization_mode="off")
    s.solver = RecordingRGF()
    return s


def run(d, energies, dos_peak_limit, filtering):
    s = make_solver(d, energies, dos_peak_limit, filtering)
    p = {k: container(d[k], energies.shape) for k in ("p_lesser", "p_greater", "p_retarded_hermitian")}
    w_pattern = bt_pattern(NS // NC, NC * B).astype(np.complex128)
    outs = tuple(DSDBCOO.from_sparray(w_pattern, s.block_sizes, energies.shape) for _ in range(2))
    s.solve(p["p_lesser"], p["p_greater"], p["p_retarded_hermitian"], out=outs)
    res = dict(s.solver.seen)
    n = NS // NC
    for name, w in zip(("wl", "wg"), outs):
        res[f"{name}_diag"] = np.stack([np.array(w.blocks[i, i]) for i in range(n)])
        res[f"{name}_upper"] = np.stack([np.array(w.blocks[i, i + 1]) for i in range(n - 1)])
        res[f"{name}_lower"] = np.stack([np.array(w.blocks[i + 1, i]) for i in range(n - 1)])
    return res


def main() -> None:
    d = synthetic.screened_device(NS, B, NE, seed=SEED)
    energies = np.linspace(0.1, 0.5, NE)
    out = {"energies": energies, "num_connected_blocks": np.array(NC)}
    for k in ("v", "p_lesser", "p_greater", "p_retarded_hermitian"):
        for t, name in enumerate(("diag", "upper", "lower")):
            out[f"{k}_{name}"] = np.stack(d[k][t])
    plain = run(d, energies, 0.0, filtering=False)
    out.update({f"plain_{k}": v for k, v in plain.items()})
    # Threshold of the peak filter (solver.py:695-715) between the energies'
    # largest DOS gradients of this case (0.0082 / 0.0096 eV^-1; 0.0033,
    # 0.0099 and 0.0105 for the others), so that energies 0, 3 and 4 are
    # filtered with a margin of about 8 % on either side.
    limit = 0.0089
    out["dos_peak_limit"] = np.array(limit)
    filt = run(d, energies, limit, filtering=True)
    out.update({f"filtered_{k}": v for k, v in filt.items() if k.startswith("w")})
    np.savez_compressed(HERE / "w_solve.npz", **out)
    print("wrote", HERE / "w_solve.npz", sorted(out))


if __name__ == "__main__":
    main()
