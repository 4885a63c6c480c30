"""Torch-backed DSDBCOO: a stack of block-sparse matrices in block-sorted
COO storage, with the block/stack access API of qttools' ``DSDBCOO``
(``src/qttools/datastructures/dsdbcoo.py``, ``dsdbsparse.py``).

Only the single-rank ("stack" distribution, one block rank) part of the
reference container is provided: it is what the solvers of this package
read and write. ``data`` has shape ``(*stack_shape, nnz)``; ``rows`` /
``cols`` are global indices sorted by block row, then block column, then
row-major inside each block (``compute_block_sort_index``,
``src/qttools/kernels/datastructure/numba/dsdbcoo.py``).
"""

from __future__ import annotations

import numpy as np
import torch

from ._interop import BlockLayout, kind


def block_sort_index(rows: np.ndarray, cols: np.ndarray, block_sizes: np.ndarray) -> np.ndarray:
    """Stable permutation sorting COO entries by (block row, block column),
    keeping the incoming (row-major) order inside each block."""
    offs = np.concatenate(([0], np.cumsum(block_sizes)))
    bi = np.searchsorted(offs, rows, side="right") - 1
    bj = np.searchsorted(offs, cols, side="right") - 1
    return np.lexsort((bj, bi))


class _BlockIndexer:
    def __init__(self, m: "DSDBCOO"):
        self.m = m

    def __getitem__(self, idx):
        i, j = idx
        m = self.m
        n = m.num_blocks
        i, j = (i + n) % n, (j + n) % n
        lead = tuple(m.data.shape[:-1])
        bi, bj = int(m.block_sizes[i]), int(m.block_sizes[j])
        e = m._layout.entries.get((i, j)) if abs(i - j) <= 1 else _generic_entry(m, i, j)
        pin = m.data.device.type == "cpu" and m.data.is_pinned()
        if e is not None and e.dense:
            # block-sorted dense block: a fresh copy of its contiguous range
            # (pinned when the container is, so an upload is a plain DMA)
            out = torch.empty(lead + (bi, bj), dtype=m.data.dtype, device=m.data.device, pin_memory=pin)
            out.copy_(m.data[..., e.start:e.stop].reshape(lead + (bi, bj)))
            return out
        out = torch.zeros(lead + (bi, bj), dtype=m.data.dtype, device=m.data.device, pin_memory=pin)
        if e is None:
            return out
        r = torch.from_numpy(e.rows.astype(np.int64)).to(m.data.device)
        c = torch.from_numpy(e.cols.astype(np.int64)).to(m.data.device)
        out[..., r, c] = m.data[..., e.start:e.stop]
        return out

    def __setitem__(self, idx, value):
        i, j = idx
        m = self.m
        n = m.num_blocks
        i, j = (i + n) % n, (j + n) % n
        e = m._layout.entries.get((i, j)) if abs(i - j) <= 1 else _generic_entry(m, i, j)
        if e is None:
            return
        v = value if isinstance(value, torch.Tensor) else torch.as_tensor(np.asarray(value))
        v = v.to(device=m.data.device, dtype=m.data.dtype)
        r = torch.from_numpy(e.rows.astype(np.int64)).to(m.data.device)
        c = torch.from_numpy(e.cols.astype(np.int64)).to(m.data.device)
        v = torch.broadcast_to(v, tuple(m.data.shape[:-1]) + v.shape[-2:])
        m.data[..., e.start:e.stop] = v[..., r, c]


def _generic_entry(m, i, j):
    offs = m.block_offsets
    rows, cols = m.rows, m.cols
    sel = np.nonzero((rows >= offs[i]) & (rows < offs[i + 1]) & (cols >= offs[j]) & (cols < offs[j + 1]))[0]
    if sel.size == 0:
        return None
    from ._interop import BlockEntry

    return BlockEntry(int(sel[0]), int(sel[-1]) + 1, False, (rows[sel] - offs[i]).astype(np.int32),
                      (cols[sel] - offs[j]).astype(np.int32))


class _StackIndexer:
    def __init__(self, m: "DSDBCOO"):
        self.m = m

    def __getitem__(self, sl):
        m = self.m
        if not isinstance(sl, tuple):
            sl = (sl,)
        data = m.data[sl + (Ellipsis, slice(None))] if sl else m.data
        if data.dim() == 1:
            data = data.unsqueeze(0)
        return DSDBCOO(data, m.rows, m.cols, m.block_sizes, _layout=m._layout)


class DSDBCOO:
    """Block-sorted COO stack with qttools-style block and stack indexers."""

    def __init__(self, data: torch.Tensor, rows, cols, block_sizes, global_stack_shape=None,
                 symmetry: bool = False, _layout: BlockLayout | None = None):
        if symmetry:
            raise NotImplementedError("symmetric storage is only read through the reference container")
        self.data = data
        self.rows = np.asarray(rows, dtype=np.int64)
        self.cols = np.asarray(cols, dtype=np.int64)
        self.block_sizes = np.asarray(block_sizes, dtype=np.int64)
        self.block_offsets = np.concatenate(([0], np.cumsum(self.block_sizes)))
        self.num_blocks = len(self.block_sizes)
        self.symmetry = False
        self.stack_shape = tuple(data.shape[:-1])
        self.global_stack_shape = tuple(global_stack_shape) if global_stack_shape else self.stack_shape
        size = int(self.block_offsets[-1])
        self.shape = self.stack_shape + (size, size)
        self.dtype = data.dtype
        self._layout = _layout if _layout is not None else BlockLayout(self.rows, self.cols, self.block_sizes)
        self._qtx_layout = self._layout
        self.blocks = _BlockIndexer(self)
        self.stack = _StackIndexer(self)

    @property
    def nnz(self) -> int:
        return int(self.data.shape[-1])

    @classmethod
    def from_sparray(cls, sparray, block_sizes, global_stack_shape, symmetry: bool = False,
                     device=None, dtype=torch.complex128) -> "DSDBCOO":
        """Mirrors ``DSDBCOO.from_sparray`` (dsdbcoo.py:886-977), single rank."""
        coo = sparray.tocoo()
        if not coo.has_canonical_format:
            coo.sum_duplicates()
        block_sizes = np.asarray(block_sizes, dtype=np.int64)
        order = block_sort_index(coo.row, coo.col, block_sizes)
        vals = torch.from_numpy(np.ascontiguousarray(coo.data[order]).astype(np.complex128))
        if isinstance(global_stack_shape, int):
            global_stack_shape = (global_stack_shape,)
        data = vals.to(dtype).reshape((1,) * len(global_stack_shape) + (-1,)).expand(
            tuple(global_stack_shape) + (vals.numel(),)).clone()
        if device is not None:
            data = data.to(device)
        return cls(data, coo.row[order], coo.col[order], block_sizes, global_stack_shape, symmetry)

    @classmethod
    def zeros_like(cls, other: "DSDBCOO") -> "DSDBCOO":
        return cls(torch.zeros_like(other.data), other.rows, other.cols, other.block_sizes,
                   other.global_stack_shape, _layout=other._layout)

    def to_dense(self) -> torch.Tensor:
        out = torch.zeros(self.shape, dtype=self.data.dtype, device=self.data.device)
        r = torch.from_numpy(self.rows).to(self.data.device)
        c = torch.from_numpy(self.cols).to(self.data.device)
        out[..., r, c] = self.data
        return out

    def diagonal(self) -> torch.Tensor:
        """Main diagonal (zeros where the pattern has no entry)."""
        size = self.shape[-1]
        out = torch.zeros(self.stack_shape + (size,), dtype=self.data.dtype, device=self.data.device)
        sel = np.nonzero(self.rows == self.cols)[0]
        if sel.size:
            idx = torch.from_numpy(sel).to(self.data.device)
            pos = torch.from_numpy(self.rows[sel]).to(self.data.device)
            out[..., pos] = self.data[..., idx]
        return out

    def __repr__(self) -> str:
        return (f"DSDBCOO(shape={self.shape}, block_sizes={self.block_sizes.tolist()}, "
                f"device={self.data.device})")


def is_host(x) -> bool:
    return kind(x) == "numpy" or (isinstance(x, torch.Tensor) and x.device.type == "cpu")
