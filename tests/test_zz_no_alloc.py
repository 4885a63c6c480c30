"""The allocation-free selected inversion (qtx_selected_inv_static).

Some callers cannot call cudaMalloc / cudaFree while they solve: both calls
synchronise the device, and once a caching pool or a framework has reserved
the GPU's memory a fresh allocation fails or fragments it. This entry point
takes its scratch from a 64 MiB device array inside the library instead of a
caller workspace. The test calls it through the C ABI twice in a row (the
array keeps the previous call's contents) and compares each result with
the workspace-based qtx_selected_inv at the FP64 tolerance of the RGF tests,
then checks that an oversize request is refused before any work is done.
This file is collected last so that a stop at the first failure has run every
other test already; it also passes when run alone.
"""

import ctypes

import numpy as np
import pytest
import torch

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


def test_static_scratch_rejects_oversize(cuda_device):
    lib = _native.load()
    keep = []
    big = torch.empty((1, 1), dtype=torch.complex128, device=cuda_device)
    n = 4
    bs = (ctypes.c_int32 * n)(*([1024] * n))
    m = (QtxMat * n)(*([QtxMat(big.data_ptr(), 1024, 0)] * n))
    a = QtxBT(n, bs, m, m, m)
    keep.append((bs, m))
    st = lib.qtx_selected_inv_static(ctypes.byref(a), None, ctypes.byref(a), 4, None, _stream())
    assert st == _native.QTX_ERR_WORKSPACE
    assert b"static scratch" in lib.qtx_last_error()
