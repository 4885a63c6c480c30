"""The screened-interaction (W) solve of a Coulomb-screening step on the GPU:
``CoulombScreeningSolver.solve`` (src/quatrex/coulomb_screening/solver.py:
724-889) for one rank, without flat-band homogenisation, with OBC
``block_sections = 1``.

Per batch of energies, every block operation is a library kernel:

* the retarded polarization P^R = P^R_h + (P^> - P^<) / 2 block by block
  (solver.py:448-493; ``qtx_zcombine``);
* the system matrix M = I - V P^R (solver.py:542-578): the blocks (i, j),
  |i - j| <= 2, of the small-block product (qttools ``bd_matmul``,
  src/qttools/datastructures/routines.py:354-467) accumulated by batched
  GEMMs straight into their quadrant of the superblock of ``nc`` small
  blocks that holds them (the reference regroups the same storage by
  changing the block sizes, solver.py:82-96,800-803), with the contacts'
  spillover terms (solver.py:495-539);
* the contact boundary self-energies (solver.py:211-446) from the expanded
  periodic superblocks of the boundary blocks (src/qttools/toeplitz/
  toeplitz.py:114-226) through ``lyapunov.screened_contact_obc``;
* L^< and L^> = V P^< V, V P^> V (qttools ``_bd_sandwich``,
  routines.py:8-102, blocks |i - j| <= 3) with their spillover
  (solver.py:580-678), into superblock quadrants likewise;
* the selected solve on the superblocks (``qtx_selected_solve``, the
  reference's ``RGF.selected_solve`` with ``return_retarded=False``).

After all batches the DOS peak filter zeroes the energies whose local DOS
gradient exceeds ``dos_peak_limit`` (solver.py:680-722) while
``solve_call_count < filtering_iteration_limit``, and the first energy is
zeroed (solver.py:884-886).
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _native
from ._interop import default_device, from_device, mat, to_device
from ._native import NULL_MAT, QtxBT, QtxMat
from .lyapunov import Doubling, LyapunovSystem, screened_contact_obc
from .obc import OBCSystem, SanchoRubio, _stream
from .utils import get_batches, workspace_pool

_C128 = torch.complex128


def _bt_lists(x, n, device):
    """(diag, upper, lower) block lists of a block-tridiagonal input: a
    triple of lists, or a container with ``blocks[i, j]`` (DSDBCOO)."""
    if hasattr(x, "blocks"):
        diag = [x.blocks[i, i] for i in range(n)]
        upper = [x.blocks[i, i + 1] for i in range(n - 1)]
        lower = [x.blocks[i + 1, i] for i in range(n - 1)]
    else:
        diag, upper, lower = x

    def dev(t):
        return to_device(t, device).to(_C128).contiguous()
    return [dev(t) for t in diag], [dev(t) for t in upper], [dev(t) for t in lower]


class _Grouped:
    """Grouped GEMM launches (``qtx_zgemm_grouped``) of b x b blocks: every
    launch is a list of (A, B, C) device addresses with C (+)= alpha A B; the
    pointer tables of all launches go to the device in one copy, then the
    launches run in the order they were added."""

    def __init__(self, b: int, device: torch.device):
        self.b, self.device = b, device
        self.launches = []  # (alpha, accumulate, lda, ldb, ldc, a, b, c)

    def add(self, alpha, accumulate, lda, ldb, ldc, a, bb, c):
        """a, bb, c: lists of int64 address arrays (concatenated in order)."""
        if a:
            self.launches.append((alpha, accumulate, lda, ldb, ldc, np.concatenate(a), np.concatenate(bb),
                                  np.concatenate(c)))

    def run(self):
        if not self.launches:
            return
        lib = _native.load()
        tables, offs = [], []
        pos = 0
        for *_, a, bb, c in self.launches:
            n = len(a)
            pad = n + (n & 1)  # each table starts 16-byte aligned
            for t in (a, bb, c):
                offs.append(pos)
                tables.append(t)
                if pad > n:
                    tables.append(np.zeros(1, dtype=np.int64))
                pos += pad
        dev = torch.from_numpy(np.concatenate(tables)).to(self.device)
        base = dev.data_ptr()
        stream = _stream(self.device)
        for li, (alpha, acc, lda, ldb, ldc, a, bb, c) in enumerate(self.launches):
            pa, pb, pc = (base + 8 * offs[3 * li + t] for t in range(3))
            _native.check(lib.qtx_zgemm_grouped(self.b, self.b, self.b, len(a), alpha, 0.0, pa, lda, 0, pb, ldb, 0,
                                                1.0 if acc else 0.0, 0.0, pc if acc else None, ldc, 0, pc, ldc,
                                                stream))
        self._keep = dev  # the tables live until the launches have run (stream order)
        self.launches = []


class CoulombScreeningSolve:
    """GPU W solve for one rank (``CoulombScreeningSolver.solve``).

    Parameters
    ----------
    coulomb_matrix
        V in small blocks: a (diag, upper, lower) triple of block lists of
        (b, b) (or (1, b, b)) blocks, or a DSDBCOO container.
    num_connected_blocks
        Small blocks per superblock of the solve (solver.py:74-96); the
        number of small blocks must be a multiple of it.
    energies
        All energies of the solve (the peak filter's abscissa).
    obc, lyapunov
        Boundary solvers of M's lead and of the Lyapunov equation (default:
        ``OBCSystem(SanchoRubio(100, 1e-12))`` and
        ``LyapunovSystem(Doubling())``, memoization off).
    dos_peak_limit, filtering_iteration_limit, max_batch_size
        As the reference's configuration (``coulomb_screening`` section).
    """

    def __init__(self, coulomb_matrix, num_connected_blocks: int, energies, obc: OBCSystem | None = None,
                 lyapunov: LyapunovSystem | None = None, dos_peak_limit: float = 100.0,
                 filtering_iteration_limit: int = 1000, max_batch_size: int | None = None,
                 device: torch.device | None = None):
        self.device = device or default_device()
        self.energies = np.asarray(energies, dtype=np.float64)
        v = coulomb_matrix
        n = len(v[0]) if isinstance(v, (tuple, list)) else int(v.num_blocks)
        self.v = tuple([t.reshape(t.shape[-2:]).unsqueeze(0).contiguous() for t in lst]
                       for lst in _bt_lists(v, n, self.device))
        self.num_small = n
        self.b = int(self.v[0][0].shape[-1])
        self.nc = int(num_connected_blocks)
        if n % self.nc != 0:
            raise ValueError(f"Number of blocks must be divisible by {self.nc}.")
        if n < 2 * self.nc:
            raise ValueError("the device needs at least two superblocks")
        self.obc = obc or OBCSystem(SanchoRubio(max_iterations=100, convergence_tol=1e-12),
                                    memoization_mode="off")
        self.lyapunov = lyapunov or LyapunovSystem(Doubling(), memoization_mode="off")
        self.dos_peak_limit = float(dos_peak_limit)
        self.filtering_iteration_limit = int(filtering_iteration_limit)
        self.max_batch_size = max_batch_size
        self.solve_call_count = 0

    # ------------------------------------------------------------------
    def _v(self, i, j):
        d, u, lo = self.v
        return d[i] if i == j else (u[i] if j == i + 1 else lo[j])

    def _gemm(self, a, b, out, alpha=1.0, accumulate=True):
        """out (+)= alpha a b for (B, b, b) stacks or views; a V block (1, b, b)
        is broadcast over the batch."""
        lib = _native.load()
        batch = max(a.shape[0], b.shape[0], out.shape[0])
        ma = mat(a, stride=0) if a.shape[0] == 1 and batch > 1 else mat(a)
        mb = mat(b, stride=0) if b.shape[0] == 1 and batch > 1 else mat(b)
        mo = mat(out)
        _native.check(lib.qtx_zgemm_batched(self.b, self.b, self.b, batch, alpha, 0.0, ma, 0, mb, 0,
                                            1.0 if accumulate else 0.0, 0.0, mo if accumulate else NULL_MAT, 0,
                                            mo, _stream(self.device)))

    def _quad(self, sup, i, j):
        """The (B, b, b) view of small block (i, j) inside its superblock."""
        nc, b = self.nc, self.b
        d, u, lo = sup
        I, J = i // nc, j // nc
        blk = d[I] if I == J else (u[I] if J == I + 1 else lo[J])
        a, c = i % nc, j % nc
        return blk[:, a * b:(a + 1) * b, c * b:(c + 1) * b]

    def _superblocks(self, batch, identity=False):
        ns, nb = self.num_small // self.nc, self.nc * self.b
        z = lambda: torch.zeros((batch, nb, nb), dtype=_C128, device=self.device)  # noqa: E731
        d = [z() for _ in range(ns)]
        if identity:
            for t in d:
                t.diagonal(dim1=-2, dim2=-1).fill_(1.0)
        return d, [z() for _ in range(ns - 1)], [z() for _ in range(ns - 1)]

    def _expand(self, a_ji, a_ii, a_ij):
        """Expanded periodic superblocks (toeplitz.py:114-226, block sections 1)."""
        nc, b = self.nc, self.b
        if nc == 1:
            return a_ji.contiguous(), a_ii.contiguous(), a_ij.contiguous()
        shape = a_ii.shape[:-2] + (nc * b, nc * b)
        ji, ii, ij = (torch.zeros(shape, dtype=_C128, device=self.device) for _ in range(3))
        for r in range(nc):
            ii[..., r * b:(r + 1) * b, r * b:(r + 1) * b] = a_ii
        for r in range(nc - 1):
            ii[..., r * b:(r + 1) * b, (r + 1) * b:(r + 2) * b] = a_ij
            ii[..., (r + 1) * b:(r + 2) * b, r * b:(r + 1) * b] = a_ji
        ij[..., -b:, :b] = a_ij
        ji[..., :b, -b:] = a_ji
        return ji, ii, ij

    # ------------------------------------------------------------------
    def _batch(self, pl, pg, prh, out_l, out_g, sl):
        n, b, dev = self.num_small, self.b, self.device
        lib = _native.load()
        stream = _stream(dev)
        batch = pl[0][0].shape[0]

        def blk(m, i, j):
            d, u, lo = m
            return d[i] if i == j else (u[i] if j == i + 1 else lo[j])

        # P^R = P^R_h + (P^> - P^<) / 2 (solver.py:473-493)
        coefs = (ctypes.c_double * 6)(1.0, 0.0, 0.5, 0.0, -0.5, 0.0)
        pr = tuple([] for _ in range(3))
        for t in range(3):
            for x_h, x_g, x_l in zip(prh[t], pg[t], pl[t]):
                o = torch.empty_like(x_h)
                terms = (QtxMat * 3)(mat(x_h), mat(x_g), mat(x_l))
                _native.check(lib.qtx_zcombine(b, b, batch, mat(o), 3, terms, coefs, None, stream))
                pr[t].append(o)
        nb = self.nc * b
        es = np.arange(batch, dtype=np.int64)
        zb = b * b * 16  # bytes per small block of one energy

        def a_v(i, j):  # an energy-independent V block, broadcast over the batch
            return np.full(batch, self._v(i, j).data_ptr(), dtype=np.int64)

        def a_blk(t):  # the energies of a (batch, b, b) stack
            return t.data_ptr() + es * zb

        def a_quad(sup, i, j):  # small block (i, j) of its superblock, every energy
            return self._quad(sup, i, j).data_ptr() + es * (nb * nb * 16)

        # M = I - V P^R - spillover, in superblocks (solver.py:542-578): one
        # grouped launch per (k - i, j - i) over all block rows and energies,
        # k ascending for every output block as bd_matmul sums it
        msup = self._superblocks(batch, identity=True)
        grp = _Grouped(b, dev)
        for dk in (-1, 0, 1):
            for dj in range(dk - 1, dk + 2):
                if abs(dj) > 2:
                    continue
                A, B_, C = [], [], []
                for i in range(n):
                    k, j = i + dk, i + dj
                    # blocks outside the superblock tridiagonal band (only for
                    # nc < 3) are not read by the selected solve: skipped
                    if 0 <= k < n and 0 <= j < n and abs(i // self.nc - j // self.nc) <= 1:
                        A.append(a_v(i, k))
                        B_.append(a_blk(blk(pr, k, j)))
                        C.append(a_quad(msup, i, j))
                grp.add(-1.0, True, b, b, nb, A, B_, C)
        grp.run()
        self._gemm(self._v(1, 0), blk(pr, 0, 1), self._quad(msup, 0, 0), alpha=-1.0)
        self._gemm(self._v(n - 2, n - 1), blk(pr, n - 1, n - 2), self._quad(msup, n - 1, n - 1), alpha=-1.0)
        # contact boundary self-energies (solver.py:380-446)
        obc = {}
        for side in ("left", "right"):
            if side == "left":
                def tri(m):
                    return blk(m, 1, 0), blk(m, 0, 0), blk(m, 0, 1)
                vt = (self._v(1, 0), self._v(0, 0), self._v(0, 1))
            else:
                def tri(m):
                    return tuple(torch.flip(x, dims=(-2, -1)) for x in
                                 (blk(m, n - 2, n - 1), blk(m, n - 1, n - 1), blk(m, n - 1, n - 2)))
                vt = tuple(torch.flip(x, dims=(-2, -1)) for x in
                           (self._v(n - 2, n - 1), self._v(n - 1, n - 1), self._v(n - 1, n - 2)))
            trips = [self._expand(*tri(m)) for m in (pr, pl, pg)]
            vexp = tuple(x[0] for x in self._expand(*vt))
            r, lo, g = screened_contact_obc(trips[0], trips[1], trips[2], vexp, self.obc, self.lyapunov,
                                            contact=f"{side}-{sl}", device=dev)
            r, lo, g = (to_device(x, dev).contiguous() for x in (r, lo, g))
            if side == "right":
                r, lo, g = (torch.flip(x, dims=(-2, -1)).contiguous() for x in (r, lo, g))
            obc[side] = (r, lo, g)
        # L = V P V with the spillover (solver.py:823-838, 580-678)
        lsup = []
        tmp = torch.empty((n, 5, batch, b, b), dtype=_C128, device=dev)  # ab[i][k - i + 2]
        for p_ in (pl, pg):
            sup = self._superblocks(batch)
            tmp.zero_()
            # ab[i][k] = sum over m (ascending) of V[i, m] P[m, k]
            grp = _Grouped(b, dev)
            for dm in (-1, 0, 1):
                for dk in (-1, 0, 1):
                    A, B_, C = [], [], []
                    for i in range(n):
                        m, k = i + dm, i + dm + dk
                        if 0 <= m < n and 0 <= k < n:
                            A.append(a_v(i, m))
                            B_.append(a_blk(blk(p_, m, k)))
                            C.append(a_blk(tmp[i, k - i + 2]))
                    grp.add(1.0, True, b, b, b, A, B_, C)
            # L[i, j] = sum over k (ascending) of ab[i][k] V[k, j]
            for dj in range(-3, 4):
                for dkj in (-1, 0, 1):
                    A, B_, C = [], [], []
                    for i in range(n):
                        j, k = i + dj, i + dj + dkj
                        if 0 <= j < n and 0 <= k < n and abs(k - i) <= 2 and abs(i // self.nc - j // self.nc) <= 1:
                            A.append(a_blk(tmp[i, k - i + 2]))
                            B_.append(a_v(k, j))
                            C.append(a_quad(sup, i, j))
                    grp.add(1.0, True, b, b, nb, A, B_, C)
            grp.run()
            t1 = torch.empty((batch, b, b), dtype=_C128, device=dev)
            for (a0, a1) in ((0, 1), (n - 1, n - 2)):
                # left: v10 = V[1,0], v01 = V[0,1]; right: the flipped-order blocks
                v10, v00, v01 = self._v(a1, a0), self._v(a0, a0), self._v(a0, a1)
                p10, p00, p01 = blk(p_, a1, a0), blk(p_, a0, a0), blk(p_, a0, a1)
                for x, y, z, i, j in ((v10, p01, v00, a0, a0), (v00, p10, v01, a0, a0), (v10, p00, v01, a0, a0),
                                      (v10, p01, v01, a0, a1), (v10, p10, v01, a1, a0)):
                    self._gemm(x, y, t1, accumulate=False)
                    self._gemm(t1, z, self._quad(sup, i, j))
            lsup.append(sup)
        # selected solve on the superblocks (solver.py:843-864)
        ns = n // self.nc
        keep = []

        def bt(diag, upper, lower):
            bs = (ctypes.c_int32 * ns)(*([nb] * ns))
            d = (QtxMat * ns)(*[mat(x) for x in diag])
            u = (QtxMat * (ns - 1))(*[mat(x) if x is not None else NULL_MAT for x in upper])
            lo = (QtxMat * (ns - 1))(*[mat(x) if x is not None else NULL_MAT for x in lower])
            keep.extend([bs, d, u, lo])
            return QtxBT(ns, bs, d, u, lo)

        A = bt(*msup)
        SL = bt(lsup[0][0], lsup[0][1], [None] * (ns - 1))
        SG = bt(lsup[1][0], lsup[1][1], [None] * (ns - 1))
        XL = bt(*[[x[sl] for x in lst] for lst in out_l])
        XG = bt(*[[x[sl] for x in lst] for lst in out_g])
        obcs = []
        for k in range(3):
            arr = (QtxMat * ns)(*([NULL_MAT] * ns))
            arr[0] = mat(obc["left"][k])
            arr[ns - 1] = mat(obc["right"][k])
            obcs.append(arr)
        bs = (ctypes.c_int32 * ns)(*([nb] * ns))
        ws = workspace_pool.get(lib.qtx_selected_solve_workspace(ns, bs, batch, 0), dev, "rgf")
        info = torch.zeros(batch, dtype=torch.int32, device=dev)
        _native.check(lib.qtx_selected_solve(
            ctypes.byref(A), ctypes.byref(SL), ctypes.byref(SG), obcs[0], obcs[1], obcs[2], ctypes.byref(XL),
            ctypes.byref(XG), None, None, NULL_MAT, None, 0, batch, info.data_ptr(), ws.data_ptr(), ws.numel(),
            stream))
        if int(info.max()) != 0:
            raise np.linalg.LinAlgError("singular Schur complement in the W solve")

    # ------------------------------------------------------------------
    def solve(self, p_lesser, p_greater, p_retarded_hermitian, out=None):
        """W^<, W^> of all energies (solver.py:724-889).

        Each polarization is a (diag, upper, lower) triple of block lists of
        (E, b, b) stacks in small blocks, or a DSDBCOO container. Returns
        (w_lesser, w_greater), each a (diag, upper, lower) triple of device
        superblock stacks (E, nc b, nc b); with ``out`` (two containers with
        ``blocks[i, j]`` in superblocks) the results are also written there.
        """
        n, dev = self.num_small, self.device
        pl = _bt_lists(p_lesser, n, dev)
        pg = _bt_lists(p_greater, n, dev)
        prh = _bt_lists(p_retarded_hermitian, n, dev)
        ne = pl[0][0].shape[0]
        for name, m in (("p_lesser", pl), ("p_greater", pg), ("p_retarded_hermitian", prh)):
            counts = (len(m[0]), len(m[1]), len(m[2]))
            if counts != (n, n - 1, n - 1):
                raise ValueError(f"{name}: expected {n} diagonal and {n - 1} off-diagonal blocks, got {counts}")
            for lst in m:
                for x in lst:
                    if tuple(x.shape) != (ne, self.b, self.b):
                        raise ValueError(f"{name}: blocks must be ({ne}, {self.b}, {self.b}) stacks, got "
                                         f"{tuple(x.shape)}")
        ns, nb = n // self.nc, self.nc * self.b
        w = []
        for _ in range(2):
            z = lambda: torch.zeros((ne, nb, nb), dtype=_C128, device=dev)  # noqa: E731
            w.append(([z() for _ in range(ns)], [z() for _ in range(ns - 1)], [z() for _ in range(ns - 1)]))
        sizes, offsets = get_batches(ne, self.max_batch_size or ne)
        for bi in range(len(sizes)):
            sl = slice(int(offsets[bi]), int(offsets[bi + 1]))

            def cut(m):
                return tuple([x[sl] for x in lst] for lst in m)

            self._batch(cut(pl), cut(pg), cut(prh), w[0], w[1], sl)
        if self.solve_call_count < self.filtering_iteration_limit:
            self._filter_peaks(w)
        for lst in (*w[0], *w[1]):
            for x in lst:
                x[0] = 0.0
        self.solve_call_count += 1
        if out is not None:
            for container, ww in zip(out, w):
                like = container.data
                for i in range(ns):
                    container.blocks[i, i] = from_device(ww[0][i], like)
                    if i + 1 < ns:
                        container.blocks[i, i + 1] = from_device(ww[1][i], like)
                        container.blocks[i + 1, i] = from_device(ww[2][i], like)
        return w[0], w[1]

    def _filter_peaks(self, w):
        """solver.py:680-722 on one rank: zero the energies whose largest
        local-DOS gradient over the superblocks exceeds dos_peak_limit."""
        wl, wg = w
        dos = []
        for i in range(len(wl[0])):
            lesser = torch.diagonal(wl[0][i], dim1=-2, dim2=-1).imag.mean(-1)
            greater = -torch.diagonal(wg[0][i], dim1=-2, dim2=-1).imag.mean(-1)
            dos.append(0.5 * (greater - lesser))
        dos = torch.stack(dos)
        e = torch.as_tensor(self.energies, dtype=torch.float64, device=self.device)
        grad = torch.gradient(dos, spacing=(e,), dim=1)[0].abs()
        mask = grad.max(dim=0).values > self.dos_peak_limit
        self.last_mask = mask
        for lst in (*wl, *wg):
            for x in lst:
                x[mask] = 0.0
