"""The C-ABI library loads without a GPU and exports every entry point that
include/qtx_b200.h declares, with the signatures the ctypes binding uses."""

import re
from pathlib import Path

from quatrex_b200 import _native, build

HEADER = Path(__file__).resolve().parent.parent / "include" / "qtx_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(qtx_[a-z0-9_]+)\s*\(", text)))


def test_library_builds_and_loads():
    path = build.build()
    assert path.exists()
    lib = _native.load()
    assert lib.qtx_version() == 100


def test_every_declared_symbol_is_exported_and_bound():
    lib = _native.load()
    names = declared_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), f"{name} is declared but not exported"
        assert name in _native.SIGNATURES, f"{name} has no ctypes signature"
    assert sorted(_native.SIGNATURES) == names


def test_workspace_queries_need_no_gpu():
    import ctypes

    lib = _native.load()
    bs = (ctypes.c_int32 * 4)(64, 64, 32, 64)
    w1 = lib.qtx_selected_inv_workspace(4, bs, 8)
    w2 = lib.qtx_selected_solve_workspace(4, bs, 8, 0)
    w3 = lib.qtx_selected_solve_workspace(4, bs, 8, 1)
    assert 0 < w1 < w2 < w3
    assert lib.qtx_sancho_rubio_workspace(64, 8) >= 10 * 64 * 64 * 16 * 8
    assert lib.qtx_obc_workspace(64, 8) > 0
    assert lib.qtx_selected_inv_workspace(0, bs, 8) == 0


def test_argument_errors_are_reported_without_gpu():
    lib = _native.load()
    st = lib.qtx_zgemm_batched(-1, 1, 1, 1, 1.0, 0.0, _native.NULL_MAT, 0, _native.NULL_MAT, 0, 0.0, 0.0,
                               _native.NULL_MAT, 0, _native.NULL_MAT, None)
    assert st == _native.QTX_ERR_ARG
    assert b"invalid" in lib.qtx_last_error()
    st = lib.qtx_selected_inv(None, None, None, 1, None, None, 0, None)
    assert st == _native.QTX_ERR_ARG
