"""The allocation-free selected inversion (qtx_selected_inv_static).

Some callers cannot call cudaMalloc / cudaFree while they solve: both calls
synchronise the device, and once a caching pool or a framework has reserved
the GPU's memory a fresh allocation fails or fragments it. This entry point
takes its scratch from a 64 MiB device array inside the library instead of a
caller workspace. The test calls it through the C ABI twice in a row (the
array keeps the previous call's contents) and compares each result with
the workspace-based qtx_selected_inv at the FP64 tolerance of the RGF tests
and, once, with the CPU oracle's selected inversion; it checks that the entry
point keeps to the FP64 products when the calling thread selected the
int8-emulated GEMM path, and that an oversize request is refused with
nothing enqueued or written.
This file is collected last so that a stop at the first failure has run every
other test already; it also passes when run alone.
"""

import ctypes

import numpy as np
import pytest
import torch

from oracle import negf_oracle as o
from quatrex_b200 import _native
from quatrex_b200._interop import mat
from quatrex_b200._native import NULL_MAT, QtxBT, QtxMat

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _problem(block_sizes, batch, device, seed):
    rng = np.random.default_rng(seed)
    n = len(block_sizes)

    def rnd(m, k):
        return torch.from_numpy(rng.standard_normal((batch, m, k)) + 1j * rng.standard_normal((batch, m, k))).to(device)

    diag = [rnd(b, b) + 4 * max(block_sizes) * torch.eye(b, dtype=torch.complex128, device=device)
            for b in block_sizes]
    upper = [rnd(block_sizes[i], block_sizes[i + 1]) for i in range(n - 1)]
    lower = [rnd(block_sizes[i + 1], block_sizes[i]) for i in range(n - 1)]
    obc = [None] * n
    obc[0] = rnd(block_sizes[0], block_sizes[0]) * 0.1
    obc[-1] = rnd(block_sizes[-1], block_sizes[-1]) * 0.1
    return diag, upper, lower, obc


def _bt(diag, upper, lower, keep):
    n = len(diag)
    bs = (ctypes.c_int32 * n)(*[d.shape[-1] for d in diag])
    d = (QtxMat * n)(*[mat(x) for x in diag])
    u = (QtxMat * max(n - 1, 1))(*([mat(x) for x in upper] or [NULL_MAT]))
    lo = (QtxMat * max(n - 1, 1))(*([mat(x) for x in lower] or [NULL_MAT]))
    keep += [bs, d, u, lo]
    return QtxBT(n, bs, d, u, lo)


def _outputs(diag, upper, lower):
    return ([torch.zeros_like(x) for x in diag], [torch.zeros_like(x) for x in upper],
            [torch.zeros_like(x) for x in lower])


def _solve(lib, block_sizes, batch, prob, static, device):
    diag, upper, lower, obc = prob
    keep = []
    a = _bt(diag, upper, lower, keep)
    xd, xu, xl = _outputs(diag, upper, lower)
    x = _bt(xd, xu, xl, keep)
    n = len(block_sizes)
    o = (QtxMat * n)(*[mat(t) if t is not None else NULL_MAT for t in obc])
    info = torch.zeros(batch, dtype=torch.int32, device=device)
    if static:
        st = lib.qtx_selected_inv_static(ctypes.byref(a), o, ctypes.byref(x), batch, info.data_ptr(), _stream())
    else:
        nbytes = lib.qtx_selected_inv_workspace(n, a.block_sizes, batch)
        ws = torch.empty(nbytes, dtype=torch.uint8, device=device)
        st = lib.qtx_selected_inv(ctypes.byref(a), o, ctypes.byref(x), batch, info.data_ptr(), ws.data_ptr(),
                                  nbytes, _stream())
    _native.check(st)
    torch.cuda.synchronize()
    assert int(info.abs().sum()) == 0
    return [t.cpu().numpy() for t in xd + xu + xl]


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_static_scratch_matches_workspace_version_twice(cuda_device):
    lib = _native.load()
    cases = [([64] * 8, 6, 1), ([48, 64, 17, 64, 32], 5, 2)]
    for block_sizes, batch, seed in cases:  # two calls in a row, different layouts
        prob = _problem(block_sizes, batch, cuda_device, seed)
        ref = _solve(lib, block_sizes, batch, prob, static=False, device=cuda_device)
        got = _solve(lib, block_sizes, batch, prob, static=True, device=cuda_device)
        for g, r in zip(got, ref):
            assert _rel(g, r) < RTOL
    # and the first layout once more, after the array holds the second one
    prob = _problem([64] * 8, 6, cuda_device, 1)
    ref = _solve(lib, [64] * 8, 6, prob, static=False, device=cuda_device)
    got = _solve(lib, [64] * 8, 6, prob, static=True, device=cuda_device)
    for g, r in zip(got, ref):
        assert _rel(g, r) < RTOL


def test_static_scratch_matches_oracle(cuda_device):
    """Diagonal and off-diagonal blocks of (A - OBC)^{-1} against the oracle's
    restatement of rgf.py:25-113 on the same blocks."""
    lib = _native.load()
    block_sizes, batch = [48, 64, 17, 64, 32], 3
    prob = _problem(block_sizes, batch, cuda_device, 4)
    got = _solve(lib, block_sizes, batch, prob, static=True, device=cuda_device)
    diag, upper, lower, obc = ([None if t is None else t.cpu().numpy() for t in x] for x in prob)
    xd, xu, xl = o.selected_inv(diag, upper, lower, obc)
    n = len(block_sizes)
    refs = list(xd) + list(xu) + list(xl)
    assert len(got) == len(refs) == 3 * n - 2
    for g, r in zip(got, refs):
        assert _rel(g, r) < 1e-10


def test_static_scratch_ignores_emulated_gemm_path(cuda_device):
    """With the int8-emulated products selected on the calling thread, the
    entry point still runs the FP64 products (its array holds no digit
    planes) and leaves the thread's selection as it was."""
    lib = _native.load()
    block_sizes, batch = [64] * 6, 4
    prob = _problem(block_sizes, batch, cuda_device, 9)
    fp64 = _solve(lib, block_sizes, batch, prob, static=False, device=cuda_device)
    _native.check(lib.qtx_set_gemm_path(5))
    try:
        got = _solve(lib, block_sizes, batch, prob, static=True, device=cuda_device)
        assert lib.qtx_get_gemm_path() == 5
        emulated = _solve(lib, block_sizes, batch, prob, static=False, device=cuda_device)
    finally:
        _native.check(lib.qtx_set_gemm_path(0))
    for g, r in zip(got, fp64):
        assert _rel(g, r) < RTOL
    # the workspace path did switch to the emulated products (differs at ~1e-10)
    assert max(_rel(e, r) for e, r in zip(emulated, fp64)) > 0.0


def test_static_scratch_rejects_oversize(cuda_device):
    lib = _native.load()
    keep = []
    n, b, batch = 4, 1024, 4
    inp = torch.ones((batch, b, b), dtype=torch.complex128, device=cuda_device)
    out = torch.full((batch, b, b), 7.0 + 3.0j, dtype=torch.complex128, device=cuda_device)
    bs = (ctypes.c_int32 * n)(*([b] * n))
    m_in = (QtxMat * n)(*([mat(inp)] * n))
    m_out = (QtxMat * n)(*([mat(out)] * n))
    a = QtxBT(n, bs, m_in, m_in, m_in)
    x = QtxBT(n, bs, m_out, m_out, m_out)
    keep.append((bs, m_in, m_out))
    info = torch.full((batch,), -77, dtype=torch.int32, device=cuda_device)
    st = lib.qtx_selected_inv_static(ctypes.byref(a), None, ctypes.byref(x), batch, info.data_ptr(), _stream())
    torch.cuda.synchronize()
    assert st == _native.QTX_ERR_WORKSPACE
    assert b"static scratch" in lib.qtx_last_error()
    # refused before anything was enqueued: outputs and info keep their sentinels
    assert bool((out == 7.0 + 3.0j).all())
    assert bool((info == -77).all())
