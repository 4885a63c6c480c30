"""Complex128 products on the int8 tensor cores (FP64 emulation).

``zgemm_emulated`` evaluates ``alpha op(A) op(B) + beta op(D)`` for stacks of
complex128 matrices with the tcgen05 ``kind::i8`` kernel of
``csrc/zgemm_oz.cu``: every operand is split into ``slices`` int8 planes of
balanced base-256 digits under a power-of-two scale per row of op(A) / column
of op(B), digit pairs are multiplied exactly in int32 and combined in FP64.
The error of an element is below ``2 * slices * k * 2**(4 - 8 * slices) *
max|op(A)_i.| * max|op(B)_.j|`` (k: complex inner dimension) (about 1e-12 relative at 6 slices, FP64 level
at 7).

``gemm_path(slices)`` routes every complex128 product of the drivers called
from this thread (selected inversion / solve, Sancho-Rubio, OBC refinement,
contact self-energy) through the same kernel; the drivers' workspace queries
include its scratch while the path is selected.
"""

from __future__ import annotations

import ctypes
from contextlib import contextmanager

import torch

from . import _native
from ._interop import mat, stack3

DEFAULT_SLICES = 6


def _stream() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


@contextmanager
def gemm_path(slices: int):
    """Selects the calling thread's complex128 GEMM path for the scope:
    0 = FP64 DMMA, 3-8 = the int8 emulation with that many slices."""
    lib = _native.load()
    prev = lib.qtx_get_gemm_path()
    _native.check(lib.qtx_set_gemm_path(int(slices)))
    try:
        yield
    finally:
        _native.check(lib.qtx_set_gemm_path(prev))


def workspace_bytes(m: int, n: int, k: int, batch: int, slices: int = DEFAULT_SLICES) -> int:
    return int(_native.load().qtx_zgemm_emulated_workspace(m, n, k, batch, slices))


def zgemm_emulated(a: torch.Tensor, b: torch.Tensor, *, op_a: int = 0, op_b: int = 0,
                   alpha: complex = 1.0, beta: complex = 0.0, d: torch.Tensor | None = None,
                   op_d: int = 0, slices: int = DEFAULT_SLICES, out: torch.Tensor | None = None,
                   workspace: torch.Tensor | None = None) -> torch.Tensor:
    """Batched ``alpha op(a) op(b) + beta op(d)`` (op = identity or conjugate
    transpose) on (batch, rows, cols) complex128 CUDA tensors."""
    a3, b3 = stack3(a), stack3(b)
    batch = a3.shape[0]
    m = a3.shape[2] if op_a else a3.shape[1]
    k = a3.shape[1] if op_a else a3.shape[2]
    n = b3.shape[1] if op_b else b3.shape[2]
    kb = b3.shape[2] if op_b else b3.shape[1]
    if kb != k or b3.shape[0] != batch:
        raise ValueError("zgemm_emulated: operand shapes do not match")
    for t in (a3, b3):
        if t.dtype != torch.complex128 or not t.is_cuda or t.stride(-1) != 1:
            raise TypeError("zgemm_emulated: complex128 CUDA tensors with unit column stride required")
    if out is None:
        out = torch.empty((batch, m, n), dtype=torch.complex128, device=a3.device)
    if workspace is None:
        workspace = torch.empty(workspace_bytes(m, n, k, batch, slices), dtype=torch.uint8, device=a3.device)
    d3 = stack3(d) if d is not None else None
    _native.check(_native.load().qtx_zgemm_emulated_batched(
        m, n, k, batch, float(complex(alpha).real), float(complex(alpha).imag), mat(a3), int(op_a), mat(b3),
        int(op_b), float(complex(beta).real), float(complex(beta).imag), mat(d3), int(op_d), mat(out),
        int(slices), workspace.data_ptr(), workspace.numel(), _stream()))
    return out


def status() -> int:
    """1 if a bounded wait inside an emulated GEMM timed out since the last
    call (the flag is cleared), else 0. Synchronises the device."""
    st = _native.load().qtx_emulated_gemm_status()
    if st < 0:
        _native.check(st)
    return st
