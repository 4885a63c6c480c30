"""Array interop and the DSDBSparse <-> device block-view boundary.

The solvers accept the reference's ``DSDBSparse`` objects (NumPy- or
CuPy-backed) as well as this package's torch-backed :class:`DSDBCOO`, and
any stack of dense blocks given as NumPy, CuPy or torch arrays. Device
arrays are used in place (CuPy through DLPack, torch directly); host arrays
are copied to the GPU and results copied back.

For block-sorted COO storage (qttools ``DSDBCOO``,
``src/qttools/datastructures/dsdbcoo.py:297-331``) a block whose nonzeros
are the full ``b_i x b_j`` block in row-major order is handed to the CUDA
kernels as a strided view of the ``data`` array itself (no copy). Other
blocks are densified / sparsified on the device (``qtx_coo_densify`` /
``qtx_coo_sparsify``). Any other DSDBSparse type goes through its own
``.blocks[i, j]`` indexer.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _native
from ._native import NULL_MAT, QtxMat

_C128 = torch.complex128
_ELEM = 16  # bytes of one complex128

# Bytes moved between host and device memory by this module (the plugin's
# inputs, outputs and boundary blocks); read by the end-to-end benchmark.
transfer_bytes = {"h2d": 0, "d2h": 0}


def _count(direction: str, t) -> None:
    transfer_bytes[direction] += int(t.numel()) * int(t.element_size())


# ---------------------------------------------------------------------------
# Arrays
# ---------------------------------------------------------------------------
def default_device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("quatrex_b200 requires a CUDA device (sm_100a); none is visible")
    return torch.device("cuda", torch.cuda.current_device())


def kind(x) -> str:
    if isinstance(x, torch.Tensor):
        return "torch"
    if isinstance(x, np.ndarray):
        return "numpy"
    if hasattr(x, "__cuda_array_interface__") or type(x).__module__.startswith("cupy"):
        return "cupy"
    return "numpy"


def to_device(x, device: torch.device, dtype=_C128) -> torch.Tensor:
    """Device tensor viewing (or holding a copy of) ``x``."""
    k = kind(x)
    if k == "torch":
        t = x
        if t.device != device:
            t = t.to(device, non_blocking=True)
            if x.device.type == "cpu":
                _count("h2d", x)
    elif k == "cupy":
        t = torch.from_dlpack(x)
    else:
        arr = np.asarray(x)
        t = torch.from_numpy(np.ascontiguousarray(arr)).to(device, non_blocking=False)
        _count("h2d", t)
    if t.dtype != dtype:
        t = t.to(dtype)
    return t


def from_device(t: torch.Tensor, like):
    """Returns ``t`` as the array type of ``like``."""
    k = kind(like)
    if k == "torch":
        if t.device == like.device:
            return t
        if like.device.type == "cpu" and t.is_cuda:
            # pinned host result: the copy is a DMA, and so is a later upload
            out = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
            out.copy_(t, non_blocking=True)
            _count("d2h", t)
            torch.cuda.current_stream(t.device).synchronize()
            return out
        return t.to(like.device)
    if k == "cupy":
        import cupy  # noqa: PLC0415 - only present when the caller uses CuPy

        return cupy.from_dlpack(t)
    if t.is_cuda:
        _count("d2h", t)
    return t.detach().cpu().numpy()


def assign(dst, src: torch.Tensor) -> None:
    """``dst[...] = src`` for a NumPy / CuPy / torch destination view."""
    k = kind(dst)
    if k == "torch":
        if dst.device.type == "cpu" and src.is_cuda:
            _count("d2h", src)
        dst.copy_(src.reshape(dst.shape))
    elif k == "cupy":
        import cupy  # noqa: PLC0415

        dst[...] = cupy.from_dlpack(src.contiguous()).reshape(dst.shape)
    else:
        if src.is_cuda:
            _count("d2h", src)
        dst[...] = src.detach().cpu().numpy().reshape(dst.shape)


def merged_spans(entries) -> list[list[int]]:
    """Sorted element ranges [start, stop) of the given block entries, with
    touching ranges merged (block-sorted storage keeps (i, i) and (i, i+1)
    adjacent)."""
    spans: list[list[int]] = []
    for a, b in sorted((e.start, e.stop) for e in entries):
        if spans and spans[-1][1] == a:
            spans[-1][1] = b
        else:
            spans.append([a, b])
    return spans


def copy_spans(dst: torch.Tensor, src: torch.Tensor, spans, stream) -> None:
    """Copies the element ranges ``spans`` of every row of the (rows, nnz)
    tensors src -> dst on ``stream`` (raw handle) with qtx_copy_ranges; one
    of them may be host memory (pinned: an asynchronous DMA)."""
    from ctypes import c_int64

    if not spans:
        return
    esz = src.element_size()
    rows = int(src.shape[0])
    off = (c_int64 * len(spans))(*[a * esz for a, _ in spans])
    ln = (c_int64 * len(spans))(*[(b - a) * esz for a, b in spans])
    _native.check(_native.load().qtx_copy_ranges(dst.data_ptr(), dst.stride(0) * esz, src.data_ptr(),
                                                 src.stride(0) * esz, rows, off, ln, len(spans), stream))
    moved = rows * sum(b - a for a, b in spans) * esz
    if src.device.type == "cpu" and dst.is_cuda:
        transfer_bytes["h2d"] += moved
    elif src.is_cuda and dst.device.type == "cpu":
        transfer_bytes["d2h"] += moved


def mat(t: torch.Tensor, offset_elems: int = 0, ld: int | None = None,
        stride: int | None = None) -> QtxMat:
    """qtx_mat of a (batch, rows, cols) tensor, or of a view into a
    (batch, nnz) data tensor starting at ``offset_elems``."""
    if t is None:
        return NULL_MAT
    if t.dtype not in (_C128, torch.complex64):
        raise TypeError(f"expected complex128 or complex64 device data, got {t.dtype}")
    if ld is None:
        ld = t.stride(-2)
    if stride is None:
        stride = t.stride(0)
    return QtxMat(t.data_ptr() + offset_elems * t.element_size(), int(ld), int(stride))


def stack3(x: torch.Tensor) -> torch.Tensor:
    """Flattens leading stack dimensions: (..., m, n) -> (B, m, n)."""
    return x.reshape(-1, x.shape[-2], x.shape[-1])


# ---------------------------------------------------------------------------
# Block layout of block-sorted COO storage
# ---------------------------------------------------------------------------
@dataclass
class BlockEntry:
    start: int
    stop: int
    dense: bool  # full block in row-major order
    rows: np.ndarray  # block-local int32
    cols: np.ndarray


class BlockLayout:
    """Slices and local indices of every tridiagonal block of a block-sorted
    COO pattern (the work of ``compute_block_slice``,
    ``kernels/datastructure/numba/dsdbcoo.py``)."""

    def __init__(self, rows, cols, block_sizes):
        rows = np.asarray(_host(rows)).astype(np.int64)
        cols = np.asarray(_host(cols)).astype(np.int64)
        self.block_sizes = np.asarray(_host(block_sizes)).astype(np.int64)
        self.block_offsets = np.concatenate(([0], np.cumsum(self.block_sizes)))
        self.nnz = int(rows.size)
        n = len(self.block_sizes)
        bi = np.searchsorted(self.block_offsets, rows, side="right") - 1
        bj = np.searchsorted(self.block_offsets, cols, side="right") - 1
        self.entries: dict[tuple[int, int], BlockEntry | None] = {}
        for i in range(n):
            for j in (i - 1, i, i + 1):
                if j < 0 or j >= n:
                    continue
                idx = np.nonzero((bi == i) & (bj == j))[0]
                if idx.size == 0:
                    self.entries[(i, j)] = None
                    continue
                start, stop = int(idx[0]), int(idx[-1]) + 1
                if stop - start != idx.size:
                    raise ValueError(f"block ({i}, {j}) is not contiguous in the data; "
                                     "the storage is not block-sorted")
                r = (rows[start:stop] - self.block_offsets[i]).astype(np.int32)
                c = (cols[start:stop] - self.block_offsets[j]).astype(np.int32)
                m, k = int(self.block_sizes[i]), int(self.block_sizes[j])
                dense = (stop - start == m * k) and np.array_equal(
                    r.astype(np.int64) * k + c, np.arange(m * k))
                self.entries[(i, j)] = BlockEntry(start, stop, bool(dense), r, c)
        self._dev: dict = {}

    def device_index(self, key, device):
        cached = self._dev.get((key, device))
        if cached is None:
            e = self.entries[key]
            cached = (torch.from_numpy(e.rows).to(device), torch.from_numpy(e.cols).to(device))
            self._dev[(key, device)] = cached
        return cached


def _host(x):
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy()
    if hasattr(x, "get") and type(x).__module__.startswith("cupy"):
        return x.get()
    return x


_layout_cache: dict[int, tuple[object, BlockLayout]] = {}


def layout_of(m) -> BlockLayout | None:
    """BlockLayout for block-sorted COO matrices (None for other formats)."""
    if hasattr(m, "_qtx_layout"):
        return m._qtx_layout
    if not (hasattr(m, "rows") and hasattr(m, "cols")) or getattr(m, "symmetry", False):
        return None
    if type(m).__name__ not in ("DSDBCOO",):
        return None
    key = id(m.rows)
    hit = _layout_cache.get(key)
    if hit is not None and hit[0] is m.rows:
        return hit[1]
    lay = BlockLayout(m.rows, m.cols, m.block_sizes)
    _layout_cache[key] = (m.rows, lay)
    return lay


# ---------------------------------------------------------------------------
# Device block views of one stack batch
# ---------------------------------------------------------------------------
class BTView:
    """Device block views (qtx_mat) of a block-tridiagonal DSDBSparse for the
    stack slice ``sl``. ``role`` is "in" (read) or "out" (written)."""

    def __init__(self, m, sl: slice, device: torch.device, stream, role: str = "in",
                 need=("diag", "upper", "lower")):
        self.m = m
        self.sl = sl
        self.device = device
        self.stream = stream
        self.role = role
        self.num_blocks = int(m.num_blocks)
        self.block_sizes = [int(b) for b in np.asarray(_host(m.block_sizes))]
        self.keep: list = []
        self.pending: list = []  # (kind, key, dense tensor)
        self.layout = layout_of(m)
        n = self.num_blocks
        self.diag = [NULL_MAT] * n
        self.upper = [NULL_MAT] * max(n - 1, 0)
        self.lower = [NULL_MAT] * max(n - 1, 0)
        self.data = None
        self.data_src = None
        if self.layout is not None:
            self._setup_coo(need)
        else:
            self._setup_generic(need)

    # -- block-sorted COO fast path -------------------------------------
    def _setup_coo(self, need):
        src = self.m.data[self.sl]
        lead = tuple(src.shape[:-1])
        nnz = int(src.shape[-1])
        self.lead_shape = lead
        k = kind(src)
        host = k == "numpy" or (k == "torch" and src.device.type == "cpu")
        self._host = host
        self._need = need
        # Inputs cross the bus as one contiguous copy (a DMA at full link
        # speed; per-block strided copies would be staged through pageable
        # memory).
        needed = [e for (i, j), e in self.layout.entries.items() if e is not None and (
            "diag" if i == j else ("upper" if j == i + 1 else "lower")) in need]
        partial = len(needed) < sum(e is not None for e in self.layout.entries.values())
        if (self.role == "in" and host and k == "torch" and partial and src.is_contiguous()
                and src.dtype == _C128 and src.numel()):
            # only the blocks the solver reads cross the bus
            t = torch.empty(src.shape, dtype=_C128, device=self.device)
            copy_spans(t.reshape(-1, nnz), src.reshape(-1, nnz), merged_spans(needed), self.stream)
        elif self.role == "in" or (k in ("torch", "cupy") and not host):
            t = to_device(src, self.device)
        else:
            # host output: nothing is uploaded; finalize() returns the written blocks
            t = torch.zeros(src.shape, dtype=_C128, device=self.device)
        t2 = t.reshape(-1, nnz) if t.numel() else t.reshape(0, nnz)
        if self.role == "out" and k in ("torch", "cupy") and t2.data_ptr() != t.data_ptr():
            t2 = t2.contiguous()
        if t2.stride(-1) != 1:
            t2 = t2.contiguous()
        self.data = t2
        self.data_src = src
        self.batch = t2.shape[0]
        self._inplace_out = (self.role == "out" and k in ("torch", "cupy")
                             and t2.data_ptr() == _data_ptr(src) and t2.is_contiguous())
        for (i, j), e in self.layout.entries.items():
            which = "diag" if i == j else ("upper" if j == i + 1 else "lower")
            if which not in need:
                continue
            idx = i if which != "lower" else j
            if e is None:
                if self.role == "out":
                    continue
                qm = NULL_MAT
            elif e.dense:
                qm = QtxMat(t2.data_ptr() + e.start * _ELEM, self.block_sizes[j], t2.stride(0))
            else:
                dense = torch.empty((self.batch, self.block_sizes[i], self.block_sizes[j]), dtype=_C128,
                                    device=self.device)
                self.keep.append(dense)
                if self.role == "in":
                    rows, cols = self.layout.device_index((i, j), self.device)
                    _native.check(_native.load().qtx_coo_densify(
                        self.batch, t2.data_ptr() + e.start * _ELEM, t2.stride(0), e.stop - e.start,
                        rows.data_ptr(), cols.data_ptr(), mat(dense), self.block_sizes[i],
                        self.block_sizes[j], self.stream))
                else:
                    dense.zero_()
                    self.pending.append(((i, j), dense))
                qm = mat(dense)
            getattr(self, which)[idx] = qm

    # -- generic DSDBSparse: use the container's own block indexer --------
    def _setup_generic(self, need):
        stack = self.m.stack[self.sl] if hasattr(self.m, "stack") else self.m
        self._stack_view = stack
        n = self.num_blocks
        self.batch = None
        for i in range(n):
            for j in (i - 1, i, i + 1):
                if j < 0 or j >= n:
                    continue
                which = "diag" if i == j else ("upper" if j == i + 1 else "lower")
                if which not in need:
                    continue
                idx = i if which != "lower" else j
                if self.role == "in":
                    blk = stack.blocks[i, j]
                    t = stack3(to_device(blk, self.device)).contiguous()
                    self.lead_shape = tuple(blk.shape[:-2])
                else:
                    lead = tuple(self.m.data[self.sl].shape[:-1])
                    self.lead_shape = lead
                    bsz = int(np.prod(lead)) if lead else 1
                    t = torch.zeros((bsz, self.block_sizes[i], self.block_sizes[j]), dtype=_C128,
                                    device=self.device)
                    self.pending.append(((i, j), t))
                self.batch = t.shape[0]
                self.keep.append(t)
                getattr(self, which)[idx] = mat(t)
        if self.batch is None:
            lead = tuple(self.m.data[self.sl].shape[:-1])
            self.lead_shape = lead
            self.batch = int(np.prod(lead)) if lead else 1

    # -- ABI struct -------------------------------------------------------
    def abi(self):
        from ctypes import c_int32

        n = self.num_blocks
        self._bs = (c_int32 * n)(*self.block_sizes)
        self._d = (QtxMat * n)(*self.diag)
        self._u = (QtxMat * max(n - 1, 1))(*(self.upper or [NULL_MAT]))
        self._l = (QtxMat * max(n - 1, 1))(*(self.lower or [NULL_MAT]))
        return _native.QtxBT(n, self._bs, self._d, self._u, self._l)

    def can_finalize_async(self) -> bool:
        """True when finalize_async() applies: a block-sorted COO host
        container whose blocks are all dense in place (no sparsify pass)."""
        return (self.role == "out" and self.layout is not None and not self.pending
                and getattr(self, "_host", False) and kind(self.m.data) == "torch")

    def finalize_async(self, write_lower: bool = True) -> None:
        """finalize() without synchronising: the device-to-host copies of the
        written blocks are enqueued on the current stream; the caller keeps
        this view alive, synchronises, then calls the returned callable (if
        any) before reading the container."""
        written = [e for (i, j), e in self.layout.entries.items() if e is not None and (
            (i == j and "diag" in self._need) or (j == i + 1 and "upper" in self._need)
            or (j == i - 1 and "lower" in self._need and write_lower))]
        total = sum(e is not None for e in self.layout.entries.values())
        dst = self.m.data[self.sl]
        src = self.data.reshape(self.data_src.shape)
        if len(written) == total:
            dst.copy_(src, non_blocking=True)
            _count("d2h", src)
            return None
        if dst.is_contiguous() and dst.is_pinned():
            # the written blocks go straight into the container (one DMA per span)
            nnz = int(self.data.shape[-1])
            copy_spans(dst.reshape(-1, nnz), self.data, merged_spans(written),
                       torch.cuda.current_stream(self.device).cuda_stream)
            return None
        # Some blocks must keep the container's values: one contiguous DMA
        # into pinned staging now, the written ranges copied on the host by
        # the returned callable once the stream has been synchronised.
        stage = torch.empty(src.shape, dtype=src.dtype, pin_memory=True)
        stage.copy_(src, non_blocking=True)

        def scatter():
            for e in written:
                dst[..., e.start:e.stop] = stage[..., e.start:e.stop]

        return scatter

    def finalize(self, write_lower: bool = True) -> None:
        """Writes results back to the container (role "out")."""
        if self.role != "out":
            return
        if self.layout is not None:
            lib = _native.load()
            for (i, j), dense in self.pending:
                if j == i - 1 and not write_lower:
                    continue
                e = self.layout.entries[(i, j)]
                rows, cols = self.layout.device_index((i, j), self.device)
                _native.check(lib.qtx_coo_sparsify(
                    self.batch, mat(dense), e.stop - e.start, rows.data_ptr(), cols.data_ptr(),
                    self.data.data_ptr() + e.start * _ELEM, self.data.stride(0), self.stream))
            if not self._inplace_out:
                written = [e for (i, j), e in self.layout.entries.items() if e is not None and (
                    (i == j and "diag" in self._need) or (j == i + 1 and "upper" in self._need)
                    or (j == i - 1 and "lower" in self._need and write_lower))]
                total = sum(e is not None for e in self.layout.entries.values())
                if self._host and len(written) < total:
                    # only the blocks the solver wrote go back to the host container
                    dst = self.m.data[self.sl]
                    nnz = int(self.data.shape[-1])
                    hd = dst if kind(dst) == "torch" else torch.from_numpy(dst) if (
                        isinstance(dst, np.ndarray) and dst.dtype == np.complex128) else None
                    if hd is not None and hd.is_contiguous():
                        copy_spans(hd.reshape(-1, nnz), self.data, merged_spans(written),
                                   torch.cuda.current_stream(self.device).cuda_stream)
                    else:
                        src = self.data.reshape(self.data_src.shape)
                        for e in written:
                            dst[..., e.start:e.stop] = src[..., e.start:e.stop].cpu().numpy()
                            transfer_bytes["d2h"] += int(src[..., e.start:e.stop].numel()) * _ELEM
                    torch.cuda.current_stream(self.device).synchronize()
                else:
                    torch.cuda.current_stream(self.device).synchronize()
                    assign(self.m.data[self.sl], self.data.reshape(self.data_src.shape))
            return
        torch.cuda.current_stream(self.device).synchronize()
        stack = self._stack_view
        for (i, j), dense in self.pending:
            if j == i - 1 and not write_lower:
                continue
            val = dense.reshape(*self.lead_shape, dense.shape[-2], dense.shape[-1])
            like = self.m.data
            stack.blocks[i, j] = from_device(val, like)


def _data_ptr(x) -> int:
    if isinstance(x, torch.Tensor):
        return x.data_ptr()
    cai = getattr(x, "__cuda_array_interface__", None)
    if cai is not None:
        return int(cai["data"][0])
    return -1


def obc_mats(blocks, sl: slice, num_blocks: int, device: torch.device, keep: list, sign: float = 1.0):
    """qtx_mat array for one OBCBlocks list (None entries -> NULL)."""
    if blocks is None:
        return None
    arr = (QtxMat * num_blocks)()
    anyset = False
    for i, blk in enumerate(blocks):
        if blk is None:
            arr[i] = NULL_MAT
            continue
        t = stack3(to_device(blk[sl], device)).contiguous()
        if sign != 1.0:
            t = t * sign
        keep.append(t)
        arr[i] = mat(t)
        anyset = True
    return arr if anyset else None
