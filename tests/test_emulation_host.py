"""Host-side behaviour of the int8 GEMM emulation (no GPU): the thread-local
path selection, its effect on the drivers' workspace queries, and argument
checks."""

import ctypes
import threading

from quatrex_b200 import _native
from quatrex_b200.emulation import gemm_path, workspace_bytes


def test_gemm_path_scope_restores_and_sizes_workspace():
    lib = _native.load()
    bs = (ctypes.c_int32 * 3)(64, 64, 64)
    base = lib.qtx_selected_solve_workspace(3, bs, 8, 1)
    inv_base = lib.qtx_selected_inv_workspace(3, bs, 8)
    sr_base = lib.qtx_sancho_rubio_workspace(64, 8)
    plane = workspace_bytes(64, 64, 64, 8, 6)
    assert plane > 6 * 8 * (128 + 2 * 64) * 128
    with gemm_path(6):
        assert lib.qtx_get_gemm_path() == 6
        assert lib.qtx_selected_solve_workspace(3, bs, 8, 1) >= base + plane - 1024
        assert lib.qtx_selected_inv_workspace(3, bs, 8) >= inv_base + plane - 1024
        assert lib.qtx_sancho_rubio_workspace(64, 8) >= sr_base + plane - 1024
        # the mixed (complex64) solve keeps its own products
        assert lib.qtx_selected_solve_mixed_workspace(3, bs, 8, 1) > 0
    assert lib.qtx_get_gemm_path() == 0
    assert lib.qtx_selected_solve_workspace(3, bs, 8, 1) == base


def test_gemm_path_is_thread_local():
    lib = _native.load()
    seen = []
    with gemm_path(5):
        t = threading.Thread(target=lambda: seen.append(lib.qtx_get_gemm_path()))
        t.start()
        t.join()
        assert lib.qtx_get_gemm_path() == 5
    assert seen == [0]


def test_emulation_argument_errors():
    lib = _native.load()
    assert lib.qtx_set_gemm_path(2) == _native.QTX_ERR_ARG
    assert lib.qtx_set_gemm_path(9) == _native.QTX_ERR_ARG
    assert lib.qtx_get_gemm_path() == 0
    assert workspace_bytes(64, 64, 64, 4, 2) == 0
    # slices * 2k * 2^14 must stay below 2^31
    assert workspace_bytes(64, 64, 20000, 1, 8) == 0
    assert workspace_bytes(64, 64, 8000, 1, 8) > 0
    st = lib.qtx_zgemm_emulated_batched(8, 8, 8, 1, 1.0, 0.0, _native.NULL_MAT, 0, _native.NULL_MAT, 0,
                                        0.0, 0.0, _native.NULL_MAT, 0, _native.NULL_MAT, 6, None, 0, None)
    assert st == _native.QTX_ERR_ARG
