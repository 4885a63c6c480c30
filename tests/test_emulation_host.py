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


# --- the arithmetic of the int8 emulation, restated in NumPy -----------------
import numpy as np  # noqa: E402


def _digits_bytes(X, S):
    """Balanced base-256 digits of int64 X (most significant first) as the
    bytes of (X + C) xor C, C = 0x80 in each of the S low bytes."""
    C = np.uint64(int("80" * S, 16))
    Z = (X.astype(np.uint64) + C) ^ C
    return [((Z >> np.uint64(8 * (S - 1 - p))) & np.uint64(0xFF)).astype(np.uint8).view(np.int8).astype(np.int64)
            for p in range(S)]


def _digits_reference(X, S):
    """The same digits by repeated sign-extended low bytes."""
    out, X = [], X.copy()
    for _ in range(S - 1):
        d = ((X & 0xFF) ^ 0x80) - 0x80
        out.append(d)
        X = (X - d) >> 8
    out.append(X)
    return out[::-1]


def test_digit_identity_matches_balanced_expansion():
    rng = np.random.default_rng(0)
    for S in range(3, 9):
        L = 8 * S - 2
        X = rng.integers(-(2 ** L), 2 ** L + 1, size=20000, dtype=np.int64)
        X[:4] = [0, 2 ** L, -(2 ** L), -1]
        a, b = _digits_bytes(X, S), _digits_reference(X, S)
        for p in range(S):
            assert np.array_equal(a[p], b[p])
            assert a[p].min() >= -128 and a[p].max() <= 127
        assert np.abs(a[0]).max() <= 65  # the leading digit
        recon = sum(a[p] * (256 ** (S - 1 - p)) for p in range(S))
        assert np.array_equal(recon, X)


def _emulated_product(A, B, S):
    """A @ B (complex) the way the kernels form it: per-row / per-column
    power-of-two scales, S digit planes of A' and B'', digit pairs with
    p + q < S summed exactly, combined in FP64."""
    M, K = A.shape
    N = B.shape[1]
    L = 8 * S - 2
    Ap = np.empty((M, 2 * K))
    Ap[:, 0::2], Ap[:, 1::2] = A.real, A.imag
    Bpp = np.empty((2 * N, 2 * K))
    Bpp[0::2, 0::2], Bpp[0::2, 1::2] = B.real.T, -B.imag.T
    Bpp[1::2, 0::2], Bpp[1::2, 1::2] = B.imag.T, B.real.T

    def scale_exp(rows):
        m = np.max(np.abs(rows), axis=1)
        return np.where(m > 0, np.frexp(m)[1], -1022)

    ea = scale_exp(Ap)
    eb = np.repeat(scale_exp(np.maximum(np.abs(Bpp[0::2]), np.abs(Bpp[1::2]))), 2)
    DA = _digits_bytes(np.rint(np.ldexp(Ap, (L - ea)[:, None])).astype(np.int64), S)
    DB = _digits_bytes(np.rint(np.ldexp(Bpp, (L - eb)[:, None])).astype(np.int64), S)
    T = np.zeros((M, 2 * N))
    for d in range(S):
        acc = sum(DA[p] @ DB[d - p].T for p in range(d + 1))
        assert np.abs(acc).max() < 2 ** 31  # exact int32 sums
        T = T * 256 + acc
    C = np.ldexp(T, ea[:, None] + eb[None, :] - 2 * L + 8 * (S - 1))
    return C[:, 0::2] + 1j * C[:, 1::2]


def test_truncated_pair_product_meets_the_stated_bound():
    rng = np.random.default_rng(1)
    for S in (4, 5, 6, 7):
        M, K, N = 24, 40, 20
        A = (rng.standard_normal((M, K)) + 1j * rng.standard_normal((M, K))) * np.exp(rng.uniform(-10, 10, (M, 1)))
        B = (rng.standard_normal((K, N)) + 1j * rng.standard_normal((K, N))) * np.exp(rng.uniform(-10, 10, (K, 1)))
        got = _emulated_product(A, B, S)
        ref = A @ B
        amax = np.max(np.maximum(np.abs(A.real), np.abs(A.imag)), axis=1)[:, None]
        bmax = np.max(np.maximum(np.abs(B.real), np.abs(B.imag)), axis=0)[None, :]
        bound = 2 * S * K * 2.0 ** (4 - 8 * S) * amax * bmax + (K + 4) * 2.0 ** -53 * (np.abs(A) @ np.abs(B))
        assert np.all(np.abs(got - ref) <= bound)
