"""The mixed-precision path: complex64 GEMM on tcgen05 with split-TF32
products and FP32 accumulation. Tolerance: max(5e-6, 5e-7 sqrt(K)) relative
to the complex128 product (FP32-level: the split recovers ~21 of FP32's 24
mantissa bits and the FP32 accumulation error grows like sqrt(K))."""

import ctypes

import numpy as np
import pytest
import torch

from quatrex_b200 import _native
from quatrex_b200._native import QtxMat

pytestmark = pytest.mark.gpu

TOL = 5e-6


def _mat(t):
    return QtxMat(t.data_ptr(), t.stride(-2), t.stride(0))


def _op(x, op):
    return x.conj().swapaxes(-2, -1) if op else x


@pytest.mark.parametrize("m,n,k", [(128, 64, 32), (1, 1, 1), (5, 3, 7), (130, 70, 40), (256, 256, 256),
                                   (512, 512, 512), (100, 200, 300)])
@pytest.mark.parametrize("op_a,op_b", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_cgemm_tc_matches_complex128(cuda_device, m, n, k, op_a, op_b):
    rng = np.random.default_rng(m + 7 * n + 13 * k + op_a + 2 * op_b)
    B = 3
    a = (rng.standard_normal((B, *((k, m) if op_a else (m, k)))) +
         1j * rng.standard_normal((B, *((k, m) if op_a else (m, k))))).astype(np.complex64)
    b = (rng.standard_normal((B, *((n, k) if op_b else (k, n)))) +
         1j * rng.standard_normal((B, *((n, k) if op_b else (k, n))))).astype(np.complex64)
    d = (rng.standard_normal((B, m, n)) + 1j * rng.standard_normal((B, m, n))).astype(np.complex64)
    ref = (0.5 - 2j) * (_op(a.astype(np.complex128), op_a) @ _op(b.astype(np.complex128), op_b)) + \
        (1.5 + 0.25j) * d.astype(np.complex128)
    A, Bt, D = (torch.from_numpy(x).to(cuda_device) for x in (a, b, d))
    C = torch.empty((B, m, n), dtype=torch.complex64, device=cuda_device)
    err = torch.zeros(1, dtype=torch.int32, device=cuda_device)
    lib = _native.load()
    _native.check(lib.qtx_cgemm_batched(m, n, k, B, 0.5, -2.0, _mat(A), op_a, _mat(Bt), op_b, 1.5, 0.25, _mat(D), 0,
                                        _mat(C), err.data_ptr(),
                                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    got = C.cpu().numpy().astype(np.complex128)
    rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert rel < max(TOL, 5e-7 * np.sqrt(k)), rel


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def cfg0_pair(cuda_device):
    from quatrex_b200 import EnergyPointSolver, synthetic

    dev = synthetic.cfg0()
    out = {}
    for prec in ("fp64", "mixed"):
        s = EnergyPointSolver(dev.h_diag, dev.coupling, eta=dev.eta, sr_tol=1e-12, per_energy=False, precision=prec)
        r = s.solve(dev.energies, dev.fermi_left(), dev.fermi_right())
        torch.cuda.synchronize()
        out[prec] = dict(T=r.transmission.cpu().numpy(), density=r.density.cpu().numpy(),
                         current=r.current.cpu().numpy(),
                         xr=r.blocks["xr_diag"].cpu().numpy().astype(np.complex128),
                         xl=r.blocks["xl_diag"].cpu().numpy().astype(np.complex128))
    return dev, out


def test_mixed_energy_point_errors_vs_fp64(cfg0_pair):
    """Errors of the mixed path against the FP64 path (itself at the oracle's
    1e-10 gate). Stated tolerances: G^R diagonal blocks 1e-3, density 1e-3,
    transmission 1e-3 (FP32-level products; the eta = 1e-4 recursion amplifies
    rounding, see the accuracy study in the design notes)."""
    _, out = cfg0_pair
    f, m = out["fp64"], out["mixed"]
    errs = {
        "transmission": float(np.max(np.abs(m["T"] - f["T"]) / np.abs(f["T"]))),
        "density": _rel(m["density"], f["density"]),
        "xr_diag": _rel(m["xr"], f["xr"]),
        "xl_diag": _rel(m["xl"], f["xl"]),
        "current": _rel(m["current"], f["current"]),
    }
    print("mixed vs fp64 (cfg0):", errs)
    assert errs["transmission"] < 1e-3 and errs["density"] < 1e-3 and errs["xr_diag"] < 1e-3, errs


@pytest.mark.parametrize("symmetric", [False, True])
def test_rgf_plugin_mixed_precision(cuda_device, symmetric):
    """RGF(precision="mixed") through the qttools-style interface: complex128
    containers in and out, split-TF32 solve inside; within the mixed path's
    stated accuracy of the FP64 plugin path on a well-conditioned system."""
    import scipy.sparse as sps

    from quatrex_b200 import RGF, DSDBCOO, synthetic

    bs = np.array([8, 16, 12, 16])
    dense = synthetic.random_bt_dense(bs, seed=5) + 4.0 * np.eye(bs.sum())
    bl = sps.coo_matrix(dense)
    bl = sps.coo_matrix(bl - bl.conj().T)
    bg = sps.coo_matrix(1j * dense)
    bg = sps.coo_matrix(bg - bg.conj().T)

    def dev(m):
        x = DSDBCOO.from_sparray(m, bs, (6,))
        return DSDBCOO(x.data.to(cuda_device), x.rows, x.cols, x.block_sizes, x.global_stack_shape)

    out = {}
    for prec in ("fp64", "mixed"):
        A, Bl, Bg = dev(sps.coo_matrix(dense)), dev(bl), dev(bg)
        Xl, Xg, Xr = (DSDBCOO.zeros_like(A) for _ in range(3))
        for X in (Xl, Xg):
            X.data.fill_(5.0 + 1.0j)
            X.symmetry = symmetric
        cur = RGF(max_batch_size=4, precision=prec).selected_solve(A, Bl, Bg, out=(Xl, Xg, Xr),
                                                                   return_retarded=True, return_current=True)
        out[prec] = [X.data.cpu().numpy() for X in (Xl, Xg, Xr)] + [cur.cpu().numpy()]
    for a, b in zip(out["mixed"], out["fp64"]):
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-4
    if symmetric:  # lower blocks untouched in both paths
        np.testing.assert_array_equal(out["mixed"][0] == 5.0 + 1.0j, out["fp64"][0] == 5.0 + 1.0j)
    with pytest.raises(ValueError):
        RGF(precision="half")
