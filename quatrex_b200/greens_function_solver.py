"""Green's-function solvers with the qttools plugin interface.

``RGF`` is a drop-in for ``qttools.greens_function_solver.RGF``
(``src/qttools/greens_function_solver/rgf.py:10-438``): same constructor,
same ``selected_inv`` / ``selected_solve`` signatures, return conventions
and errors; the recursions run in libqtx_b200 on the GPU. ``OBCBlocks`` and
``GFSolver`` mirror ``src/qttools/greens_function_solver/solver.py:12-113``.
"""

from __future__ import annotations

import ctypes
from abc import ABC, abstractmethod

import numpy as np
import torch

from . import _native
from ._interop import BTView, default_device, from_device, kind, obc_mats
from ._native import NULL_MAT, QtxMat
from .emulation import gemm_path
from .utils import get_batches, workspace_pool


class OBCBlocks:
    """Per-layer open-boundary blocks (solver.py:12-27)."""

    def __init__(self, num_blocks: int):
        self.retarded: list = [None] * num_blocks
        self.lesser: list = [None] * num_blocks
        self.greater: list = [None] * num_blocks


class GFSolver(ABC):
    """Abstract Green's-function solver (solver.py:31-113)."""

    @abstractmethod
    def selected_inv(self, a, obc_blocks: OBCBlocks | None = None, out=None):
        ...

    @abstractmethod
    def selected_solve(self, a, sigma_lesser, sigma_greater, obc_blocks: OBCBlocks | None = None,
                       out: tuple | None = None, return_retarded: bool = False,
                       return_current: bool = False):
        ...


def _raise_if_singular(info: torch.Tensor) -> None:
    if info.numel() and bool((info != 0).any()):
        # numpy.linalg.inv raises LinAlgError on an exactly singular block,
        # which is what the reference solver propagates.
        raise np.linalg.LinAlgError("Singular matrix")


def _stream(device: torch.device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


class RGF(GFSolver):
    """Selected inversion / selected solve of block-tridiagonal stacks on
    the GPU (recursive Green's function).

    Parameters
    ----------
    max_batch_size : int, optional
        Maximum number of stack entries (energies) processed together, as in
        the reference (default 100).
    device : torch.device, optional
        CUDA device; defaults to the current device.
    precision : "fp64" (default), "mixed" or "emulated"
        "mixed": ``selected_solve`` runs on complex64 copies of the blocks with
        split-TF32 tensor-core products and FP64 inverses of the Schur
        complements (``qtx_selected_solve_mixed``); inputs and outputs keep
        the containers' complex128 type. ``selected_inv`` is always FP64.
        "emulated": complex128 throughout, every product formed on the int8
        tensor cores from ``slices`` digit planes per operand (FP64-class
        accuracy: ~1e-12 relative per product at 6 slices, FP64 level at 7).
        "fp64" and "mixed" use the FP64 DMMA products whatever GEMM path the
        calling thread selected with ``emulation.gemm_path``.
    slices : int
        Digit planes per operand of the "emulated" precision (3-8).
    """

    def __init__(self, max_batch_size: int = 100, device: torch.device | None = None,
                 precision: str = "fp64", slices: int = 6) -> None:
        if precision not in ("fp64", "mixed", "emulated"):
            raise ValueError(f"precision must be 'fp64', 'mixed' or 'emulated', got {precision!r}")
        if precision == "emulated" and not 3 <= int(slices) <= 8:
            raise ValueError(f"slices must be 3-8, got {slices}")
        self.max_batch_size = max_batch_size
        self.device = device
        self.precision = precision
        self.slices = int(slices)

    def _path(self):
        return gemm_path(self.slices if self.precision == "emulated" else 0)

    def _dev(self) -> torch.device:
        return self.device if self.device is not None else default_device()

    # ------------------------------------------------------------------
    def selected_inv(self, a, obc_blocks: OBCBlocks | None = None, out=None):
        """rgf.py:25-113: diagonal and first off-diagonal blocks of A^{-1}."""
        with self._path():
            return self._selected_inv(a, obc_blocks, out)

    def _selected_inv(self, a, obc_blocks, out):
        lib = _native.load()
        device = self._dev()
        n = int(a.num_blocks)
        if obc_blocks is None:
            obc_blocks = OBCBlocks(num_blocks=n)
        sizes, slices = get_batches(a.shape[0], self.max_batch_size)
        x = out if out is not None else a.__class__.zeros_like(a)
        st = _stream(device)
        for b in range(len(sizes)):
            sl = slice(int(slices[b]), int(slices[b + 1]), 1)
            A = BTView(a, sl, device, st.value, "in")
            X = BTView(x, sl, device, st.value, "out")
            keep: list = []
            obc = obc_mats(obc_blocks.retarded, sl, n, device, keep)
            batch = A.batch
            abi_a, abi_x = A.abi(), X.abi()
            ws_bytes = lib.qtx_selected_inv_workspace(n, abi_a.block_sizes, batch)
            ws = workspace_pool.get(ws_bytes, device, "rgf")
            info = torch.zeros(batch, dtype=torch.int32, device=device)
            _native.check(lib.qtx_selected_inv(ctypes.byref(abi_a), obc, ctypes.byref(abi_x), batch,
                                               info.data_ptr(), ws.data_ptr(), ws.numel(), st))
            _raise_if_singular(info)
            X.finalize()
        if out is None:
            return x
        return None

    # ------------------------------------------------------------------
    def selected_solve(self, a, sigma_lesser, sigma_greater, obc_blocks: OBCBlocks | None = None,
                       out: tuple | None = None, return_retarded: bool = False,
                       return_current: bool = False):
        """rgf.py:115-438: X^R, X^< and X^> on the block-tridiagonal pattern,
        optionally with the Meir-Wingreen layer current."""
        with self._path():
            return self._selected_solve(a, sigma_lesser, sigma_greater, obc_blocks, out, return_retarded,
                                        return_current)

    def _selected_solve(self, a, sigma_lesser, sigma_greater, obc_blocks, out, return_retarded,
                        return_current):
        lib = _native.load()
        device = self._dev()
        n = int(sigma_lesser.num_blocks)
        if obc_blocks is None:
            obc_blocks = OBCBlocks(num_blocks=n)

        if out is not None:
            xl, xg, *xr = out
            if return_retarded:
                if len(xr) != 1:
                    raise ValueError("Invalid number of output matrices.")
                xr = xr[0]
            else:
                xr = None
        else:
            xl = a.__class__.zeros_like(a)
            xg = a.__class__.zeros_like(a)
            xr = a.__class__.zeros_like(a) if return_retarded else None

        current = None
        if return_current:
            cshape = (*sigma_lesser.shape[:-2], n + 1)
            current = _zeros_like_array(sigma_lesser.data, cshape)

        sizes, slices = get_batches(sigma_lesser.shape[0], self.max_batch_size)
        if len(sizes) > 1 and all(_on_host(m) for m in (a, sigma_lesser, sigma_greater, xl, xg)):
            return self._selected_solve_pipelined(a, sigma_lesser, sigma_greater, obc_blocks, xl, xg, xr,
                                                  current, sizes, slices, out, return_retarded,
                                                  return_current)
        st = _stream(device)
        for b in range(len(sizes)):
            sl = slice(int(slices[b]), int(slices[b + 1]), 1)
            A = BTView(a, sl, device, st.value, "in")
            SL = BTView(sigma_lesser, sl, device, st.value, "in", need=("diag", "upper"))
            SG = BTView(sigma_greater, sl, device, st.value, "in", need=("diag", "upper"))
            XL = BTView(xl, sl, device, st.value, "out")
            XG = BTView(xg, sl, device, st.value, "out")
            XR = BTView(xr, sl, device, st.value, "out", need=("diag",)) if xr is not None else None
            keep: list = []
            orr = obc_mats(obc_blocks.retarded, sl, n, device, keep)
            ol = obc_mats(obc_blocks.lesser, sl, n, device, keep)
            og = obc_mats(obc_blocks.greater, sl, n, device, keep)
            batch = A.batch
            cur = torch.zeros((batch, n + 1), dtype=torch.complex128, device=device) if return_current else None
            abi = [v.abi() if v is not None else None for v in (A, SL, SG, XL, XG, XR)]
            info = torch.zeros(batch, dtype=torch.int32, device=device)
            sym = bool(getattr(xl, "symmetry", False)) or bool(getattr(xg, "symmetry", False))
            flags = _native.QTX_SOLVE_SYMMETRIC_OUT if sym else 0
            _solve_call(lib, self.precision, abi, (orr, ol, og), cur, info,
                        lambda nb: workspace_pool.get(nb, device, "rgf"), flags, batch, st, device)
            _raise_if_singular(info)
            XL.finalize(write_lower=not getattr(xl, "symmetry", False))
            XG.finalize(write_lower=not getattr(xg, "symmetry", False))
            if XR is not None:
                XR.finalize()
            if return_current:
                _assign_rows(current, sl, cur)

        if out is None:
            if return_retarded:
                if return_current:
                    return xl, xg, xr, current
                return xl, xg, xr
            return xl, xg
        if return_current:
            return current
        return None

    def _selected_solve_pipelined(self, a, sigma_lesser, sigma_greater, obc_blocks, xl, xg, xr, current, sizes,
                                  slices, out, return_retarded, return_current):
        """selected_solve for host (CPU torch) containers with more than one
        batch: uploads run on a copy stream two batches ahead and write-backs
        on a third stream while a batch is solved. The batches are shifted
        by half a batch so that the first and the last are half as large:
        the upload before the first solve and the write-back after the last
        one (the parts nothing overlaps) are short. The copy streams persist across calls, so the caching
        allocator reuses their buffers instead of allocating new ones each
        call. Same results and conventions; a singular block raises after the
        last batch."""
        lib = _native.load()
        device = self._dev()
        n = int(sigma_lesser.num_blocks)
        comp = torch.cuda.current_stream(device)
        up_s, down_s = _copy_streams(device)
        up_s.wait_stream(comp)
        down_s.wait_stream(comp)
        slices = _split_ends(slices)
        sizes = np.diff(slices)
        sym_l = bool(getattr(xl, "symmetry", False))
        sym_g = bool(getattr(xg, "symmetry", False))
        flags = _native.QTX_SOLVE_SYMMETRIC_OUT if (sym_l or sym_g) else 0
        keep, infos, curs, deferred = [], [], [], []

        def stage(b):
            sl = slice(int(slices[b]), int(slices[b + 1]), 1)
            with torch.cuda.stream(up_s):
                hs = up_s.cuda_stream
                views = (BTView(a, sl, device, hs, "in"),
                         BTView(sigma_lesser, sl, device, hs, "in", need=("diag", "upper")),
                         BTView(sigma_greater, sl, device, hs, "in", need=("diag", "upper")),
                         BTView(xl, sl, device, hs, "out"), BTView(xg, sl, device, hs, "out"),
                         BTView(xr, sl, device, hs, "out", need=("diag",)) if xr is not None else None)
                obc_keep: list = []
                obcs = (obc_mats(obc_blocks.retarded, sl, n, device, obc_keep),
                        obc_mats(obc_blocks.lesser, sl, n, device, obc_keep),
                        obc_mats(obc_blocks.greater, sl, n, device, obc_keep))
                ev = torch.cuda.Event()
                ev.record(up_s)
            return sl, views, obcs, obc_keep, ev

        staged = [stage(b) for b in range(min(2, len(sizes)))]
        for b in range(len(sizes)):
            sl, views, obcs, obc_keep, ev = staged.pop(0)
            if b + 2 < len(sizes):
                staged.append(stage(b + 2))
            comp.wait_event(ev)
            A, SL, SG, XL, XG, XR = views
            batch = A.batch
            cur = torch.zeros((batch, n + 1), dtype=torch.complex128, device=device) if return_current else None
            info = torch.zeros(batch, dtype=torch.int32, device=device)
            abi = [v.abi() if v is not None else None for v in views]
            _solve_call(lib, self.precision, abi, obcs, cur, info,
                        lambda nb: workspace_pool.get(nb, device, "rgf"), flags, batch,
                        ctypes.c_void_p(comp.cuda_stream), device)
            keep.append(abi)
            done = torch.cuda.Event()
            done.record(comp)
            with torch.cuda.stream(down_s):
                down_s.wait_event(done)
                for v, lower in ((XL, not sym_l), (XG, not sym_g), (XR, True)):
                    if v is None:
                        continue
                    if v.can_finalize_async():
                        post = v.finalize_async(write_lower=lower)
                        if post is not None:
                            deferred.append(post)
                    else:
                        down_s.synchronize()
                        v.finalize(write_lower=lower)
            keep.append((views, obc_keep, abi))
            infos.append(info)
            curs.append((sl, cur))
        down_s.synchronize()
        comp.synchronize()
        for post in deferred:
            post()
        for info in infos:
            _raise_if_singular(info)
        if return_current:
            for sl, cur in curs:
                _assign_rows(current, sl, cur)
        if out is None:
            if return_retarded:
                if return_current:
                    return xl, xg, xr, current
                return xl, xg, xr
            return xl, xg
        if return_current:
            return current
        return None


def _block_shapes(bs, n):
    return ([(bs[i], bs[i]) for i in range(n)], [(bs[i], bs[i + 1]) for i in range(n - 1)],
            [(bs[i + 1], bs[i]) for i in range(n - 1)])


def _convert(lib, rows, cols, batch, src, src_t, dst, dst_t, stream):
    _native.check(lib.qtx_convert(rows, cols, batch, src, src_t, dst, dst_t, stream))


def _solve_call(lib, precision, abi, obcs, cur, info, ws_getter, flags, batch, stream, device):
    """One selected-solve call on the given complex128 block views; the mixed
    precision converts them to complex64 copies, solves, and converts the
    outputs back into the views."""
    n = abi[0].num_blocks
    bs = [int(abi[0].block_sizes[i]) for i in range(n)]
    if precision in ("fp64", "emulated"):  # the caller's scope selects the GEMM path
        ws = ws_getter(lib.qtx_selected_solve_workspace(n, abi[0].block_sizes, batch, int(cur is not None)))
        _native.check(lib.qtx_selected_solve(
            ctypes.byref(abi[0]), ctypes.byref(abi[1]), ctypes.byref(abi[2]), obcs[0], obcs[1], obcs[2],
            ctypes.byref(abi[3]), ctypes.byref(abi[4]), ctypes.byref(abi[5]) if abi[5] is not None else None,
            cur.data_ptr() if cur is not None else None, NULL_MAT, None, flags, batch,
            info.data_ptr(), ws.data_ptr(), ws.numel(), stream))
        return
    c128, c64 = _native.QTX_C128, _native.QTX_C64
    keep: list = []
    shapes = _block_shapes(bs, n)

    def low(bt, role):
        """complex64 twin of a block-tridiagonal view (inputs converted)."""
        parts = []
        for k, arr in enumerate((bt.diag, bt.upper, bt.lower)):
            cnt = n if k == 0 else n - 1
            out = []
            for i in range(max(cnt, 0)):
                m = arr[i]
                if not m.ptr:
                    out.append(NULL_MAT)
                    continue
                r, c = shapes[k][i]
                t = (torch.empty if role == "in" else torch.zeros)((batch, r, c), dtype=torch.complex64,
                                                                   device=device)
                keep.append(t)
                q = QtxMat(t.data_ptr(), c, r * c)
                if role == "in":
                    _convert(lib, r, c, batch, m, c128, q, c64, stream)
                out.append(q)
            parts.append(out)
        d = (QtxMat * n)(*parts[0])
        u = (QtxMat * max(n - 1, 1))(*(parts[1] or [NULL_MAT]))
        lo = (QtxMat * max(n - 1, 1))(*(parts[2] or [NULL_MAT]))
        keep.extend([d, u, lo])
        return _native.QtxBT(n, bt.block_sizes, d, u, lo), parts

    def low_obc(arr):
        if arr is None:
            return None
        out = (QtxMat * n)(*([NULL_MAT] * n))
        for i in range(n):
            m = arr[i]
            if m.ptr:
                t = torch.empty((batch, bs[i], bs[i]), dtype=torch.complex64, device=device)
                keep.append(t)
                q = QtxMat(t.data_ptr(), bs[i], bs[i] * bs[i])
                _convert(lib, bs[i], bs[i], batch, m, c128, q, c64, stream)
                out[i] = q
        keep.append(out)
        return out

    lo_in = [low(abi[k], "in")[0] for k in range(3)]
    lo_out = [low(abi[k], "out") if abi[k] is not None else None for k in (3, 4, 5)]
    lo_obc = [low_obc(o) for o in obcs]
    ws = ws_getter(lib.qtx_selected_solve_mixed_workspace(n, abi[0].block_sizes, batch, int(cur is not None)))
    _native.check(lib.qtx_selected_solve_mixed(
        ctypes.byref(lo_in[0]), ctypes.byref(lo_in[1]), ctypes.byref(lo_in[2]), lo_obc[0], lo_obc[1], lo_obc[2],
        ctypes.byref(lo_out[0][0]), ctypes.byref(lo_out[1][0]),
        ctypes.byref(lo_out[2][0]) if lo_out[2] is not None else None,
        cur.data_ptr() if cur is not None else None, NULL_MAT, None, flags, batch,
        info.data_ptr(), ws.data_ptr(), ws.numel(), stream))
    symmetric = bool(flags & _native.QTX_SOLVE_SYMMETRIC_OUT)
    for k, lo in zip((3, 4, 5), lo_out):
        if lo is None:
            continue
        bt, parts = abi[k], lo[1]
        for kk, arr in enumerate((bt.diag, bt.upper, bt.lower)):
            if kk == 2 and symmetric:
                continue  # not written by the solve: the container keeps its values
            for i, q in enumerate(parts[kk]):
                if q.ptr and arr[i].ptr:
                    r, c = shapes[kk][i]
                    _convert(lib, r, c, batch, q, c64, arr[i], c128, stream)


_streams: dict = {}


def _copy_streams(device: torch.device):
    """The upload and write-back streams of a device (created once)."""
    key = (device.type, device.index)
    if key not in _streams:
        _streams[key] = (torch.cuda.Stream(device), torch.cuda.Stream(device))
    return _streams[key]


def _split_ends(slices) -> np.ndarray:
    """Pipeline batch boundaries: the reference's batches shifted by half a
    batch, so that the first and the last pipeline batch are half as large
    (short upload before the first solve and write-back after the last one)
    and every other batch keeps the full size (no batch exceeds the
    caller's max_batch_size)."""
    b = [int(x) for x in slices]
    if len(b) < 3:  # a single batch: nothing to overlap
        return np.asarray(b)
    size = max(b[i + 1] - b[i] for i in range(len(b) - 1))
    half = max(size // 2, 1)
    total = b[-1]
    out = [0, half]
    while out[-1] + size < total:
        out.append(out[-1] + size)
    if out[-1] < total:
        out.append(total)
    return np.asarray(out)


def _on_host(m) -> bool:
    d = getattr(m, "data", None)
    return isinstance(d, torch.Tensor) and d.device.type == "cpu"


def _zeros_like_array(like, shape):
    k = kind(like)
    if k == "torch":
        return torch.zeros(shape, dtype=torch.complex128, device=like.device)
    if k == "cupy":
        import cupy  # noqa: PLC0415

        return cupy.zeros(shape, dtype=np.complex128)
    return np.zeros(shape, dtype=np.complex128)


def _assign_rows(dst, sl: slice, src: torch.Tensor) -> None:
    view = dst[sl]
    val = src.reshape(view.shape)
    k = kind(dst)
    if k == "torch":
        view.copy_(val)
    else:
        view[...] = from_device(val, dst)
