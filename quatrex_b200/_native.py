"""ctypes binding of libqtx_b200.so (include/qtx_b200.h).

The library is the only compute path: there is no CPU or library fallback.
Importing this module works without a GPU (so the exported symbols can be
inspected), but every call that launches work requires CUDA and raises a
``RuntimeError`` if the library is missing.
"""

from __future__ import annotations

import ctypes
from ctypes import POINTER, Structure, c_double, c_int, c_int32, c_int64, c_size_t, c_void_p
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libqtx_b200.so"

QTX_OK = 0
QTX_ERR_ARG = -1
QTX_ERR_CUDA = -2
QTX_ERR_WORKSPACE = -3
QTX_ERR_SINGULAR = -4
QTX_ERR_UNSUPPORTED = -5
QTX_SOLVE_SYMMETRIC_OUT = 1
QTX_C128 = 0
QTX_C64 = 1

KERNEL_CLASSES = {"zgemm": 0, "zinv": 1, "blockops": 2, "reduce": 3, "format": 4, "cgemm": 5,
                  "zgemm_emu": 6, "split": 7}


class QtxMat(Structure):
    _fields_ = [("ptr", c_void_p), ("ld", c_int64), ("stride", c_int64)]


class QtxBT(Structure):
    _fields_ = [
        ("num_blocks", c_int32),
        ("block_sizes", POINTER(c_int32)),
        ("diag", POINTER(QtxMat)),
        ("upper", POINTER(QtxMat)),
        ("lower", POINTER(QtxMat)),
    ]


NULL_MAT = QtxMat(None, 0, 0)

# name -> (restype, argtypes)
SIGNATURES = {
    "qtx_version": (c_int, []),
    "qtx_last_error": (ctypes.c_char_p, []),
    "qtx_zgemm_batched": (c_int, [c_int, c_int, c_int, c_int64, c_double, c_double, QtxMat, c_int,
                                  QtxMat, c_int, c_double, c_double, QtxMat, c_int, QtxMat, c_void_p]),
    "qtx_cgemm_batched": (c_int, [c_int, c_int, c_int, c_int64, ctypes.c_float, ctypes.c_float, QtxMat, c_int,
                                  QtxMat, c_int, ctypes.c_float, ctypes.c_float, QtxMat, c_int, QtxMat, c_void_p,
                                  c_void_p]),
    "qtx_zgemm_grouped": (c_int, [c_int, c_int, c_int, c_int64, c_double, c_double, c_void_p, c_int64, c_int,
                                  c_void_p, c_int64, c_int, c_double, c_double, c_void_p, c_int64, c_int, c_void_p,
                                  c_int64, c_void_p]),
    "qtx_zcombine": (c_int, [c_int, c_int, c_int64, QtxMat, c_int, POINTER(QtxMat), POINTER(c_double),
                             c_void_p, c_void_p]),
    "qtx_zinv_batched": (c_int, [c_int, c_int64, QtxMat, QtxMat, c_void_p, c_void_p]),
    "qtx_zinv_workspace": (c_size_t, [c_int, c_int64]),
    "qtx_zinv_batched_ws": (c_int, [c_int, c_int64, QtxMat, QtxMat, c_void_p, c_void_p, c_size_t, c_void_p]),
    "qtx_set_inverse_path": (c_int, [c_int]),
    "qtx_inverse_status": (c_int, []),
    "qtx_zgemm_emulated_workspace": (c_size_t, [c_int, c_int, c_int, c_int64, c_int]),
    "qtx_zgemm_emulated_batched": (c_int, [c_int, c_int, c_int, c_int64, c_double, c_double, QtxMat, c_int,
                                           QtxMat, c_int, c_double, c_double, QtxMat, c_int, QtxMat, c_int,
                                           c_void_p, c_size_t, c_void_p]),
    "qtx_set_gemm_path": (c_int, [c_int]),
    "qtx_get_gemm_path": (c_int, []),
    "qtx_emulated_gemm_status": (c_int, []),
    "qtx_selected_inv_workspace": (c_size_t, [c_int32, POINTER(c_int32), c_int64]),
    "qtx_selected_inv": (c_int, [POINTER(QtxBT), POINTER(QtxMat), POINTER(QtxBT), c_int64, c_void_p,
                                 c_void_p, c_size_t, c_void_p]),
    "qtx_selected_inv_static": (c_int, [POINTER(QtxBT), POINTER(QtxMat), POINTER(QtxBT), c_int64, c_void_p,
                                        c_void_p]),
    "qtx_selected_solve_workspace": (c_size_t, [c_int32, POINTER(c_int32), c_int64, c_int]),
    "qtx_selected_solve": (c_int, [POINTER(QtxBT), POINTER(QtxBT), POINTER(QtxBT), POINTER(QtxMat),
                                   POINTER(QtxMat), POINTER(QtxMat), POINTER(QtxBT), POINTER(QtxBT),
                                   POINTER(QtxBT), c_void_p, QtxMat, c_void_p, c_int, c_int64,
                                   c_void_p, c_void_p, c_size_t, c_void_p]),
    "qtx_selected_solve_mixed_workspace": (c_size_t, [c_int32, POINTER(c_int32), c_int64, c_int]),
    "qtx_selected_solve_mixed": (c_int, [POINTER(QtxBT), POINTER(QtxBT), POINTER(QtxBT), POINTER(QtxMat),
                                         POINTER(QtxMat), POINTER(QtxMat), POINTER(QtxBT), POINTER(QtxBT),
                                         POINTER(QtxBT), c_void_p, QtxMat, c_void_p, c_int, c_int64,
                                         c_void_p, c_void_p, c_size_t, c_void_p]),
    "qtx_convert": (c_int, [c_int, c_int, c_int64, QtxMat, c_int, QtxMat, c_int, c_void_p]),
    "qtx_sancho_rubio_workspace": (c_size_t, [c_int, c_int64]),
    "qtx_sancho_rubio": (c_int, [c_int, c_int64, QtxMat, QtxMat, QtxMat, QtxMat, c_int, c_double, c_int,
                                 POINTER(c_int), POINTER(c_int), c_void_p, c_void_p, c_void_p, c_size_t,
                                 c_void_p]),
    "qtx_sancho_rubio_multi": (c_int, [c_int, c_int, POINTER(c_int64), POINTER(QtxMat), POINTER(QtxMat),
                                       POINTER(QtxMat), POINTER(QtxMat), c_int, c_double, c_int, POINTER(c_int),
                                       POINTER(c_int), c_void_p, c_void_p, c_size_t, c_void_p]),
    "qtx_sancho_rubio_multi_async": (c_int, [c_int, c_int, POINTER(c_int64), POINTER(QtxMat), POINTER(QtxMat),
                                             POINTER(QtxMat), POINTER(QtxMat), c_int, c_double, c_int, c_void_p,
                                             c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "qtx_obc_workspace": (c_size_t, [c_int, c_int64]),
    "qtx_contact_self_energy": (c_int, [c_int, c_int64, QtxMat, QtxMat, QtxMat, c_void_p, QtxMat, QtxMat,
                                        QtxMat, c_void_p, c_size_t, c_void_p]),
    "qtx_obc_refine": (c_int, [c_int, c_int64, QtxMat, QtxMat, QtxMat, QtxMat, QtxMat, c_void_p, c_void_p,
                               c_void_p, c_void_p, c_size_t, c_void_p]),
    "qtx_transmission": (c_int, [c_int, c_int, c_int64, QtxMat, QtxMat, QtxMat, c_void_p, c_void_p,
                                 c_size_t, c_void_p]),
    "qtx_coo_densify": (c_int, [c_int64, c_void_p, c_int64, c_int64, c_void_p, c_void_p, QtxMat, c_int,
                                c_int, c_void_p]),
    "qtx_coo_sparsify": (c_int, [c_int64, QtxMat, c_int64, c_void_p, c_void_p, c_void_p, c_int64,
                                 c_void_p]),
    "qtx_beyn_moments_workspace": (c_size_t, [c_int, c_int64, c_int]),
    "qtx_beyn_moments": (c_int, [c_int, c_int64, QtxMat, QtxMat, QtxMat, c_double, c_double, c_int, QtxMat, QtxMat,
                                 c_void_p, c_void_p, c_size_t, c_void_p]),
    "qtx_lyapunov_workspace": (c_size_t, [c_int, c_int64]),
    "qtx_lyapunov_doubling": (c_int, [c_int, c_int64, QtxMat, QtxMat, QtxMat, c_int, c_double, c_double,
                                      POINTER(c_int), POINTER(c_int), c_void_p, c_size_t, c_void_p]),
    "qtx_lyapunov_refine": (c_int, [c_int, c_int64, QtxMat, QtxMat, QtxMat, QtxMat, c_void_p, c_void_p,
                                    c_void_p, c_size_t, c_void_p]),
    "qtx_copy_ranges": (c_int, [c_void_p, c_int64, c_void_p, c_int64, c_int64, POINTER(c_int64),
                                POINTER(c_int64), c_int, c_void_p]),
    "qtx_profile_enable": (c_int, [c_int]),
    "qtx_profile_reset": (c_int, []),
    "qtx_profile_read": (c_int, [c_int, POINTER(c_double), POINTER(c_double), POINTER(c_int64)]),
    "qtx_assemble_energies": (c_int, [c_int64, c_void_p, c_double, c_void_p, c_void_p]),
    "qtx_assemble_diag": (c_int, [c_int, c_int64, QtxMat, c_void_p, QtxMat, c_void_p]),
    "qtx_assemble_system": (c_int, [POINTER(QtxBT), c_void_p, c_void_p, POINTER(QtxBT), POINTER(QtxBT),
                                    POINTER(QtxBT), POINTER(QtxBT), c_int64, c_void_p]),
}

_lib = None


class QtxError(RuntimeError):
    """Error returned by libqtx_b200."""

    def __init__(self, status: int, message: str):
        super().__init__(f"libqtx_b200 status {status}: {message}")
        self.status = status


def load() -> ctypes.CDLL:
    """Loads the library (once) and binds the entry-point signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m quatrex_b200.build` "
            "(the CUDA library is the only implementation of this path)")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int) -> None:
    if status != QTX_OK:
        msg = load().qtx_last_error()
        raise QtxError(status, msg.decode() if msg else "")


def profile_read(kind: int = -1) -> tuple[float, float, int]:
    """(device ms, algorithmic work, launches) of the recorded launches."""
    ms, work, n = c_double(0.0), c_double(0.0), c_int64(0)
    check(load().qtx_profile_read(kind, ctypes.byref(ms), ctypes.byref(work), ctypes.byref(n)))
    return ms.value, work.value, n.value


def exported_symbols() -> list[str]:
    return list(SIGNATURES)
