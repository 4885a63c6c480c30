"""Records qttools ``DSDBCOO`` containers and the reference solver's outputs on
them, for the plugin test that runs without the reference installed.

The GPU tests run where the reference package is not available, so they
cannot construct qttools' own ``DSDBCOO``. This script builds them with the
reference package (NumPy backend; single-rank ``mpi4py`` / ``h5py``
stand-ins from ``_stubs/``) and writes ``qttools_dsdbcoo.npz`` with, for
every container, exactly the attributes the plugin reads
(``data`` with its stack shape, the block-sorted ``rows`` / ``cols``,
``block_sizes``, ``num_blocks``, ``shape``, ``symmetry``,
``global_stack_shape``), plus the ``data`` arrays that the reference's
``RGF.selected_solve`` and ``RGF.selected_inv`` write into fresh
``DSDBCOO.zeros_like`` containers. ``tests/test_gpu_qttools_containers.py``
rebuilds containers with those attributes and checks the plugin writes the
same ``data`` (same nonzero order) as the reference.

Usage (needs the quatrex reference sources)::

    QTX_REFERENCE_SRC=<quatrex checkout>/src python tests/golden/make_qttools_containers.py
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
import scipy.sparse as sps  # noqa: E402

from qttools.comm import comm  # noqa: E402

_CFG = {k: "device_mpi" for k in ("all_to_all", "all_gather", "all_reduce", "bcast")}
comm.configure(block_comm_size=1, block_comm_config=_CFG, stack_comm_config=_CFG, override=True)

from qttools.datastructures import DSDBCOO  # noqa: E402
from qttools.greens_function_solver import RGF  # noqa: E402
from qttools.greens_function_solver.solver import OBCBlocks  # noqa: E402

from quatrex_b200 import synthetic  # noqa: E402

FIELDS = ("rows", "cols", "block_sizes")


def record(out: dict, name: str, m) -> None:
    assert type(m).__name__ == "DSDBCOO"
    out[f"{name}_data"] = np.asarray(m.data)
    for f in FIELDS:
        out[f"{name}_{f}"] = np.asarray(getattr(m, f))
    out[f"{name}_num_blocks"] = np.array(m.num_blocks)
    out[f"{name}_shape"] = np.array(m.shape)
    out[f"{name}_global_stack_shape"] = np.array(m.global_stack_shape)
    out[f"{name}_symmetry"] = np.array(bool(m.symmetry))


def main() -> None:
    out: dict = {}
    bs = np.array([2, 2, 2, 4, 4, 2, 2, 2])
    dense = synthetic.random_bt_dense(bs, seed=11)
    stack = (5,)
    bl = sps.coo_matrix(dense)
    bl = sps.coo_matrix(bl - bl.conj().T)
    bg = sps.coo_matrix(1j * dense)
    bg = sps.coo_matrix(bg - bg.conj().T)
    A = DSDBCOO.from_sparray(sps.coo_matrix(dense), bs, stack)
    Bl = DSDBCOO.from_sparray(bl, bs, stack)
    Bg = DSDBCOO.from_sparray(bg, bs, stack)
    # Energy dependence: scale the diagonal blocks differently per stack entry.
    rng = np.random.default_rng(3)
    for i in range(len(bs)):
        A.blocks[i, i] = A.blocks[i, i] * (1.0 + 0.1 * rng.random(stack))[:, None, None]
    n = len(bs)
    obc = OBCBlocks(num_blocks=n)
    obc.retarded[0] = 0.3 * (rng.random((*stack, bs[0], bs[0])) + 1j * rng.random((*stack, bs[0], bs[0])))
    obc.retarded[-1] = 0.2 * (rng.random((*stack, bs[-1], bs[-1])) + 1j * rng.random((*stack, bs[-1], bs[-1])))
    for layer, occupancy in ((0, 0.7), (-1, 0.2)):
        sigma = obc.retarded[layer]
        gamma = 1j * (sigma - sigma.conj().swapaxes(-2, -1))
        obc.lesser[layer] = 1j * occupancy * gamma
        obc.greater[layer] = 1j * (occupancy - 1.0) * gamma
    record(out, "a", A)
    record(out, "sigma_lesser", Bl)
    record(out, "sigma_greater", Bg)
    for key in ("retarded", "lesser", "greater"):
        out[f"obc_{key}_first"] = getattr(obc, key)[0]
        out[f"obc_{key}_last"] = getattr(obc, key)[-1]

    # Batched over the stack (2 + 2 + 1 entries), as the plugin must split it.
    xl, xg, xr = RGF(max_batch_size=2).selected_solve(A, Bl, Bg, obc_blocks=obc, return_retarded=True)
    for name, x in (("xl", xl), ("xg", xg), ("xr", xr)):
        record(out, name, x)
    # The reference's boundary current terms (rgf.py:414-428) use the whole
    # OBC stacks, so the current is taken with one batch covering the stack.
    # (without out= the current is returned only together with X^R, rgf.py:430-435)
    *_, current = RGF(max_batch_size=stack[0]).selected_solve(A, Bl, Bg, obc_blocks=obc, return_retarded=True,
                                                              return_current=True)
    assert isinstance(current, np.ndarray) and current.dtype == np.complex128
    out["current"] = current
    x = RGF(max_batch_size=3).selected_inv(A, obc_blocks=obc)
    record(out, "inv", x)
    np.savez_compressed(HERE / "qttools_dsdbcoo.npz", **out)
    print("wrote", HERE / "qttools_dsdbcoo.npz", sorted(out))


if __name__ == "__main__":
    main()
