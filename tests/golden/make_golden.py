"""Generates the golden fixtures in this directory from the reference package.

Run with the quatrex reference sources (Python, NumPy backend) at
``$QTX_REFERENCE_SRC`` (the reference's ``src/`` directory, required)::

    QTX_REFERENCE_SRC=<quatrex checkout>/src python tests/golden/make_golden.py

The reference needs ``mpi4py`` and ``h5py`` at import time; neither is on the
solver path, so the single-rank stand-ins under ``_stubs/`` are put first on
``sys.path``. Outputs (all small, committed):

* ``bt_small.npz`` -- the reference GF-solver test construction
  (``tests/qttools/greens_function_solver/conftest.py:58-104``) on both test
  block layouts, solved by the reference ``RGF.selected_inv`` and
  ``RGF.selected_solve`` through ``DSDBCOO`` on a (4,) energy stack.
* ``cfg0.npz`` -- 16 blocks of 64x64, 32 energies in [-2, 2]: reference
  Sancho-Rubio + ``OBCSystem`` boundary self-energies of both contacts, the
  reference ``selected_solve`` with ``return_current=True``, the density and
  the dense Caroli transmission built from the reference outputs.
* ``cfg1_sample.npz`` -- 32 blocks of 256x256 on 3 energies of the
  1024-point [-3, 3] grid: current, density, transmission and per-block
  checksums of G^R / G^< (full blocks would be tens of MB).
"""

from __future__ import annotations

import os
import sys
import time
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

from qttools.boundary_conditions.obc import OBCSystem, SanchoRubio  # noqa: E402
from qttools.datastructures import DSDBCOO  # noqa: E402
from qttools.greens_function_solver import RGF  # noqa: E402
from qttools.greens_function_solver.solver import OBCBlocks  # noqa: E402

from quatrex_b200 import synthetic  # noqa: E402


def _h(x):
    return x.conj().swapaxes(-2, -1)


def bt_small(out: dict):
    for tag, bs in (("const", [2] * 10), ("mixed", [2, 2, 2, 4, 4, 2, 2, 2])):
        bs = np.array(bs)
        dense = synthetic.random_bt_dense(bs, seed=7)
        stack = (4,)
        coo = sps.coo_matrix(dense)
        a = DSDBCOO.from_sparray(coo, bs, stack)
        x = RGF(max_batch_size=2).selected_inv(a)
        out[f"{tag}_block_sizes"] = bs
        out[f"{tag}_a"] = dense
        out[f"{tag}_inv"] = x.to_dense()[0]
        bl = sps.coo_matrix(dense)
        bl = bl - bl.conj().T
        bl = sps.coo_matrix(bl)
        bg = sps.coo_matrix(1j * dense)
        bg = sps.coo_matrix(bg - bg.conj().T)
        A = DSDBCOO.from_sparray(coo, bs, stack)
        Bl = DSDBCOO.from_sparray(bl, bs, stack)
        Bg = DSDBCOO.from_sparray(bg, bs, stack)
        xl, xg, xr = RGF(max_batch_size=100).selected_solve(A, Bl, Bg, return_retarded=True)
        out[f"{tag}_sigma_lesser"] = bl.toarray()
        out[f"{tag}_sigma_greater"] = bg.toarray()
        out[f"{tag}_xl"] = xl.to_dense()[0]
        out[f"{tag}_xg"] = xg.to_dense()[0]
        out[f"{tag}_xr"] = xr.to_dense()[0]


def _bt_pattern(n, b):
    rows, cols = [], []
    for i in range(n):
        for j in (i - 1, i, i + 1):
            if 0 <= j < n:
                r, c = np.meshgrid(np.arange(b) + i * b, np.arange(b) + j * b, indexing="ij")
                rows.append(r.ravel())
                cols.append(c.ravel())
    rows = np.concatenate(rows)
    cols = np.concatenate(cols)
    return sps.coo_matrix((np.ones(rows.size, dtype=np.complex128), (rows, cols)), shape=(n * b, n * b))


def physics_case(dev, energy_index, tol=1e-12):
    """Runs the reference electron-solve path on the selected energies."""
    n, b = dev.num_blocks, dev.block_size
    energies = dev.energies[energy_index]
    ne = energies.size
    diag, upper, lower = dev.system_blocks(energies)
    pattern = _bt_pattern(n, b)
    bs = dev.block_sizes
    A = DSDBCOO.from_sparray(pattern, bs, (ne,))
    A.data[:] = 0
    for i in range(n):
        A.blocks[i, i] = diag[i]
        if i + 1 < n:
            A.blocks[i, i + 1] = upper[i]
            A.blocks[i + 1, i] = lower[i]

    f_l = dev.fermi_left(energies)
    f_r = dev.fermi_right(energies)
    obc = OBCSystem(SanchoRubio(max_iterations=100, convergence_tol=tol), memoization_mode="off")

    def contact(a_ii, a_ij, a_ji, occ, name):
        g, *_ = obc((a_ii, a_ij, a_ji), contact=name)
        sigma = a_ji @ g @ a_ij
        gamma = 1j * (sigma - _h(sigma))
        return sigma, 1j * gamma * occ[:, None, None], 1j * gamma * (occ - 1)[:, None, None], g

    # Left contact: (A00, A01, A10). Right contact: the reference flips both
    # axes of (A_NN, A_N,N-1, A_N-1,N) and flips the result back.
    sl, ll, gl, g_left = contact(A.blocks[0, 0], A.blocks[0, 1], A.blocks[1, 0], f_l, "left")
    fl = lambda x: np.flip(x, axis=(-2, -1))  # noqa: E731
    sr, lr, gr, g_right = contact(fl(A.blocks[n - 1, n - 1]), fl(A.blocks[n - 1, n - 2]),
                                  fl(A.blocks[n - 2, n - 1]), f_r, "right")
    sr, lr, gr, g_right = fl(sr), fl(lr), fl(gr), fl(g_right)

    obc_blocks = OBCBlocks(num_blocks=n)
    obc_blocks.retarded[0], obc_blocks.lesser[0], obc_blocks.greater[0] = sl, ll, gl
    obc_blocks.retarded[-1], obc_blocks.lesser[-1], obc_blocks.greater[-1] = sr, lr, gr
    SL = DSDBCOO.zeros_like(A)
    SG = DSDBCOO.zeros_like(A)
    xl, xg, xr, current = RGF(max_batch_size=ne).selected_solve(
        A, SL, SG, obc_blocks=obc_blocks, return_retarded=True, return_current=True)
    density = xl.diagonal().imag
    return dict(A=A, xl=xl, xg=xg, xr=xr, current=current, density=density, sigma_left=sl,
                sigma_right=sr, g_left=g_left, g_right=g_right, diag=diag, upper=upper, lower=lower)


def caroli_from_blocks(diag, upper, lower, sigma_l, sigma_r):
    n = len(diag)
    b = diag[0].shape[-1]
    ne = diag[0].shape[0]
    t = np.zeros(ne)
    for e in range(ne):
        a = np.zeros((n * b, n * b), dtype=np.complex128)
        for i in range(n):
            a[i * b:(i + 1) * b, i * b:(i + 1) * b] = diag[i][e]
            if i + 1 < n:
                a[i * b:(i + 1) * b, (i + 1) * b:(i + 2) * b] = upper[i][e]
                a[(i + 1) * b:(i + 2) * b, i * b:(i + 1) * b] = lower[i][e]
        a[:b, :b] -= sigma_l[e]
        a[-b:, -b:] -= sigma_r[e]
        g = np.linalg.inv(a)
        g0n = g[:b, -b:]
        gl = 1j * (sigma_l[e] - sigma_l[e].conj().T)
        gr = 1j * (sigma_r[e] - sigma_r[e].conj().T)
        t[e] = np.trace(gl @ g0n @ gr @ g0n.conj().T).real
    return t


def cfg0(out: dict):
    dev = synthetic.cfg0()
    idx = np.arange(dev.energies.size)
    r = physics_case(dev, idx)
    n = dev.num_blocks
    out["energies"] = dev.energies
    out["h00_checksum"] = np.array([dev.h_diag.sum(), np.abs(dev.h_diag).sum(), dev.coupling.sum()])
    out["h_corner"] = dev.h_diag[0, :4, :4]
    out["t_corner"] = dev.coupling[:4, :4]
    out["current"] = r["current"]
    out["density"] = r["density"]
    pick = np.array([0, 13])
    out["pick"] = pick
    blocks = [0, n - 1]
    out["pick_blocks"] = np.array(blocks)
    out["xr_diag"] = np.stack([r["xr"].blocks[i, i][pick] for i in blocks])
    out["xl_diag"] = np.stack([r["xl"].blocks[i, i][pick] for i in blocks])
    out["xg_diag8"] = r["xg"].blocks[8, 8][pick]
    out["xl_upper01"] = r["xl"].blocks[0, 1][pick]
    out["xl_lower10"] = r["xl"].blocks[1, 0][pick]
    out["sigma_left"] = r["sigma_left"][pick]
    out["sigma_right"] = r["sigma_right"][pick]
    out["transmission"] = caroli_from_blocks(r["diag"], r["upper"], r["lower"], r["sigma_left"],
                                             r["sigma_right"])
    # Reference selected_inv of A - Sigma_L - Sigma_R.
    x = RGF().selected_inv(r["A"], obc_blocks=_slice_obc(r, n))
    out["inv_diag8"] = x.blocks[8, 8][pick]
    out["inv_upper01"] = x.blocks[0, 1][pick]


def _slice_obc(r, n):
    ob = OBCBlocks(num_blocks=n)
    ob.retarded[0] = r["sigma_left"]
    ob.retarded[-1] = r["sigma_right"]
    return ob


def cfg1_sample(out: dict):
    dev = synthetic.cfg1()
    idx = np.array([100, 511, 900])
    r = physics_case(dev, idx)
    n = dev.num_blocks
    out["energy_index"] = idx
    out["energies"] = dev.energies[idx]
    out["current"] = r["current"]
    out["density"] = r["density"]
    out["transmission"] = caroli_from_blocks(r["diag"], r["upper"], r["lower"], r["sigma_left"],
                                             r["sigma_right"])
    out["xr_trace"] = np.stack([np.trace(r["xr"].blocks[i, i], axis1=-2, axis2=-1) for i in range(n)], -1)
    out["xr_fro"] = np.stack([np.linalg.norm(r["xr"].blocks[i, i], axis=(-2, -1)) for i in range(n)], -1)
    out["xl_fro"] = np.stack([np.linalg.norm(r["xl"].blocks[i, i], axis=(-2, -1)) for i in range(n)], -1)
    out["xl_upper_fro"] = np.stack(
        [np.linalg.norm(r["xl"].blocks[i, i + 1], axis=(-2, -1)) for i in range(n - 1)], -1)
    out["xg_fro"] = np.stack([np.linalg.norm(r["xg"].blocks[i, i], axis=(-2, -1)) for i in range(n)], -1)
    out["sigma_left_fro"] = np.linalg.norm(r["sigma_left"], axis=(-2, -1))
    out["sigma_right_fro"] = np.linalg.norm(r["sigma_right"], axis=(-2, -1))
    out["sigma_left_trace"] = np.trace(r["sigma_left"], axis1=-2, axis2=-1)
    out["xr_block0_corner"] = r["xr"].blocks[0, 0][:, :8, :8]


def main():
    for name, fn in (("bt_small", bt_small), ("cfg0", cfg0), ("cfg1_sample", cfg1_sample)):
        t0 = time.time()
        out = {}
        fn(out)
        np.savez_compressed(HERE / f"{name}.npz", **out)
        print(f"{name}: {time.time() - t0:.1f} s, {(HERE / f'{name}.npz').stat().st_size / 1e6:.2f} MB")


if __name__ == "__main__":
    main()
