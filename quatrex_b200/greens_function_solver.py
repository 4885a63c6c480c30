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
    """

    def __init__(self, max_batch_size: int = 100, device: torch.device | None = None) -> None:
        self.max_batch_size = max_batch_size
        self.device = device

    def _dev(self) -> torch.device:
        return self.device if self.device is not None else default_device()

    # ------------------------------------------------------------------
    def selected_inv(self, a, obc_blocks: OBCBlocks | None = None, out=None):
        """rgf.py:25-113: diagonal and first off-diagonal blocks of A^{-1}."""
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
            ws_bytes = lib.qtx_selected_solve_workspace(n, abi[0].block_sizes, batch, int(return_current))
            ws = workspace_pool.get(ws_bytes, device, "rgf")
            info = torch.zeros(batch, dtype=torch.int32, device=device)
            sym = bool(getattr(xl, "symmetry", False)) or bool(getattr(xg, "symmetry", False))
            flags = _native.QTX_SOLVE_SYMMETRIC_OUT if sym else 0
            _native.check(lib.qtx_selected_solve(
                ctypes.byref(abi[0]), ctypes.byref(abi[1]), ctypes.byref(abi[2]), orr, ol, og,
                ctypes.byref(abi[3]), ctypes.byref(abi[4]),
                ctypes.byref(abi[5]) if abi[5] is not None else None,
                cur.data_ptr() if cur is not None else None, NULL_MAT, None, flags, batch,
                info.data_ptr(), ws.data_ptr(), ws.numel(), st))
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
