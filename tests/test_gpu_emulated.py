"""The int8 tensor-core emulation of the complex128 GEMM (csrc/zgemm_oz.cu)
against NumPy complex128, and the FP64 drivers run on it.

Tolerances: every element obeys the kernel's stated bound
|err_ij| <= 2 S k 2^(4-8S) max_l|op(A)_il| max_l|op(B)_lj| (k complex), and the error
relative to (|op(A)||op(B)|)_ij stays below the per-slice-count figure in
REL (measured ~3e-10 / 1e-12 / 7e-15 at S = 5 / 6 / 7 on operands whose rows
and columns span 2^+-29)."""

import numpy as np
import pytest
import torch

from quatrex_b200 import _native
from quatrex_b200.emulation import gemm_path, status, workspace_bytes, zgemm_emulated

pytestmark = pytest.mark.gpu

REL = {4: 5e-7, 5: 2e-9, 6: 1e-11, 7: 1e-13, 8: 1e-13}


def _rand(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def _op(x, op):
    return x.conj().swapaxes(-2, -1) if op else x


def _check(got, a, b, op_a, op_b, slices, extra=0.0):
    A, B = _op(a, op_a), _op(b, op_b)
    ref = A @ B
    k = A.shape[-1]
    absprod = np.abs(A) @ np.abs(B)
    amax = np.max(np.maximum(np.abs(A.real), np.abs(A.imag)), axis=-1)[..., :, None]
    bmax = np.max(np.maximum(np.abs(B.real), np.abs(B.imag)), axis=-2)[..., None, :]
    # the stated bound plus FP64 rounding of the kernel's sum and of NumPy's
    bound = 2 * slices * k * 2.0 ** (4 - 8 * slices) * amax * bmax + (k + 4) * 2.0 ** -53 * absprod + extra
    err = np.abs(got - ref)
    assert np.all(err <= bound + 1e-300), float(np.max(err / (bound + 1e-300)))
    rel = np.max(err / np.maximum(absprod, 1e-300))
    assert rel < REL[slices], rel
    return rel


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (2, 3, 5), (17, 33, 9), (64, 64, 64), (100, 70, 130),
                                   (256, 256, 256), (65, 129, 257), (128, 32, 512)])
@pytest.mark.parametrize("op_a,op_b", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("slices", [5, 6])  # 48- and 64-column tiles
def test_emulated_zgemm_matches_numpy(cuda_device, m, n, k, op_a, op_b, slices):
    rng = np.random.default_rng(7 * m + 3 * n + k + 11 * op_a + 5 * op_b)
    B = 3
    a = _rand(rng, B, *((k, m) if op_a else (m, k)))
    b = _rand(rng, B, *((n, k) if op_b else (k, n)))
    C = zgemm_emulated(torch.from_numpy(a).to(cuda_device), torch.from_numpy(b).to(cuda_device),
                       op_a=op_a, op_b=op_b, slices=slices)
    _check(C.cpu().numpy(), a, b, op_a, op_b, slices)
    assert status() == 0


@pytest.mark.parametrize("slices", [4, 5, 6, 7, 8])
def test_emulated_accuracy_per_slice_count_wide_range(cuda_device, slices):
    """Rows of A and columns of B spanning 2^+-29: the per-row / per-column
    scales keep every element within the bound."""
    rng = np.random.default_rng(slices)
    B, m, n, k = 2, 96, 80, 200
    a = _rand(rng, B, m, k) * np.exp(rng.uniform(-20, 20, (B, m, 1)))
    b = _rand(rng, B, k, n) * np.exp(rng.uniform(-20, 20, (B, k, 1))) * np.exp(rng.uniform(-5, 5, (B, 1, n)))
    C = zgemm_emulated(torch.from_numpy(a).to(cuda_device), torch.from_numpy(b).to(cuda_device), slices=slices)
    _check(C.cpu().numpy(), a, b, 0, 0, slices)


def test_emulated_epilogue_alpha_beta_and_transposed_addend(cuda_device):
    rng = np.random.default_rng(3)
    B, m, n, k = 4, 70, 90, 110
    a, b, d = _rand(rng, B, m, k), _rand(rng, B, k, n), _rand(rng, B, n, m)
    C = zgemm_emulated(torch.from_numpy(a).to(cuda_device), torch.from_numpy(b).to(cuda_device),
                       alpha=0.5 - 2j, beta=1.5 + 0.25j, d=torch.from_numpy(d).to(cuda_device), op_d=1,
                       slices=7)
    ref = (0.5 - 2j) * (a @ b) + (1.5 + 0.25j) * _op(d, 1)
    err = np.linalg.norm(C.cpu().numpy() - ref) / np.linalg.norm(ref)
    assert err < 1e-13, err


def test_emulated_zero_rows_and_columns(cuda_device):
    rng = np.random.default_rng(4)
    a, b = _rand(rng, 2, 40, 50), _rand(rng, 2, 50, 60)
    a[:, 5, :] = 0.0
    a[1] = 0.0
    b[:, :, 7] = 0.0
    C = zgemm_emulated(torch.from_numpy(a).to(cuda_device), torch.from_numpy(b).to(cuda_device), slices=6)
    got = C.cpu().numpy()
    assert np.all(got[:, 5, :] == 0) and np.all(got[1] == 0) and np.all(got[:, :, 7] == 0)
    _check(got, a, b, 0, 0, 6)


def test_emulated_batch_chunks_match_whole_batch(cuda_device):
    """A workspace for 3 entries makes the call run the batch of 10 in chunks."""
    rng = np.random.default_rng(5)
    B, m, n, k = 10, 64, 96, 128
    a, b = _rand(rng, B, m, k), _rand(rng, B, k, n)
    ta, tb = torch.from_numpy(a).to(cuda_device), torch.from_numpy(b).to(cuda_device)
    full = zgemm_emulated(ta, tb, slices=6)
    small = torch.empty(workspace_bytes(m, n, k, 3, 6), dtype=torch.uint8, device=cuda_device)
    chunked = zgemm_emulated(ta, tb, slices=6, workspace=small)
    assert torch.equal(full, chunked)
    tiny = torch.empty(1024, dtype=torch.uint8, device=cuda_device)
    with pytest.raises(_native.QtxError):
        zgemm_emulated(ta, tb, slices=6, workspace=tiny)


def test_emulated_is_deterministic(cuda_device):
    rng = np.random.default_rng(6)
    ta = torch.from_numpy(_rand(rng, 5, 200, 150)).to(cuda_device)
    tb = torch.from_numpy(_rand(rng, 5, 150, 220)).to(cuda_device)
    assert torch.equal(zgemm_emulated(ta, tb), zgemm_emulated(ta, tb))


@pytest.mark.parametrize("bs", [np.array([48] * 6), np.array([3, 64, 17, 64])], ids=["const", "uneven"])
def test_selected_inv_on_emulated_path(cuda_device, bs):
    import scipy.sparse as sps

    from quatrex_b200 import DSDBCOO, RGF, synthetic

    dense = synthetic.random_bt_dense(bs, seed=int(bs.sum()))
    mask = dense.astype(bool)
    ref = np.linalg.inv(dense) * mask
    a = DSDBCOO.from_sparray(sps.coo_matrix(dense), bs, (4,))
    a = DSDBCOO(a.data.to(cuda_device), a.rows, a.cols, a.block_sizes, a.global_stack_shape)
    x = RGF(max_batch_size=4, precision="emulated", slices=7).selected_inv(a)
    assert status() == 0
    # an explicit fp64 solver ignores the thread's GEMM path
    with gemm_path(3):
        x64 = RGF(max_batch_size=4).selected_inv(a)
    got64 = x64.to_dense().cpu().numpy() * mask
    assert np.linalg.norm(got64 - ref) / np.linalg.norm(ref) < 1e-13
    got = x.to_dense().cpu().numpy() * mask
    err = np.linalg.norm(got - np.broadcast_to(ref, got.shape)) / np.linalg.norm(np.broadcast_to(ref, got.shape))
    assert err < 1e-11, err


@pytest.mark.parametrize("slices,tol", [(6, 1e-7), (7, 1e-9)])
def test_energy_point_solver_emulated_matches_fp64(cuda_device, slices, tol):
    from quatrex_b200 import EnergyPointSolver, synthetic

    dev = synthetic.make_device(num_blocks=8, block_size=64, energies=np.linspace(-1.5, 1.5, 6), seed=3)
    kw = dict(device=cuda_device, eta=dev.eta, device_loop=True)
    args = (dev.energies, dev.fermi_left(), dev.fermi_right())
    ref = EnergyPointSolver(dev.h_diag, dev.coupling, **kw).solve(*args)
    emu = EnergyPointSolver(dev.h_diag, dev.coupling, precision="emulated", slices=slices, **kw)
    got = emu.solve(*args)
    assert status() == 0
    T0, T1 = ref.transmission.cpu().numpy(), got.transmission.cpu().numpy()
    assert np.max(np.abs(T1 - T0) / np.maximum(np.abs(T0), 1e-300)) < tol
    d0, d1 = ref.density.cpu().numpy(), got.density.cpu().numpy()
    assert np.max(np.abs(d1 - d0)) / np.max(np.abs(d0)) < tol
    # the graph-captured pipeline reproduces the eager emulated run
    g = emu.solve_graph(*args)
    assert np.max(np.abs(g.transmission.cpu().numpy() - T1) / np.maximum(np.abs(T1), 1e-300)) < tol


def test_emulated_broadcast_operands(cuda_device):
    """Operands with batch stride 0 (one matrix for every entry) are split once."""
    rng = np.random.default_rng(8)
    B, m, n, k = 6, 80, 72, 96
    a1, b1 = _rand(rng, 1, m, k), _rand(rng, 1, k, n)
    a, b = _rand(rng, B, m, k), _rand(rng, B, k, n)
    ta1 = torch.from_numpy(a1).to(cuda_device).expand(B, m, k)
    tb1 = torch.from_numpy(b1).to(cuda_device).expand(B, k, n)
    ta, tb = torch.from_numpy(a).to(cuda_device), torch.from_numpy(b).to(cuda_device)
    for x, y, xa, ya in ((ta1, tb, np.broadcast_to(a1, a.shape), b), (ta, tb1, a, np.broadcast_to(b1, b.shape)),
                         (ta1, tb1, np.broadcast_to(a1, a.shape), np.broadcast_to(b1, b.shape))):
        assert x.stride(0) == 0 or y.stride(0) == 0
        C = zgemm_emulated(x, y, slices=6)
        _check(C.cpu().numpy(), xa, ya, 0, 0, 6)
    # conjugate-transposed broadcast operands
    C = zgemm_emulated(torch.from_numpy(a1.conj().swapaxes(-1, -2).copy()).to(cuda_device).expand(B, k, m), tb,
                       op_a=1, slices=7)
    _check(C.cpu().numpy(), np.broadcast_to(a1, a.shape), b, 0, 0, 7)


def test_emulated_non_finite_inputs_give_nan(cuda_device):
    """A row of op(A) or a column of op(B) holding Inf / NaN makes its output
    row / column NaN; everything else is unaffected."""
    rng = np.random.default_rng(9)
    a, b = _rand(rng, 2, 40, 50), _rand(rng, 2, 50, 60)
    a[0, 3, 7] = np.inf
    b[1, 11, 5] = complex(0.0, np.nan)
    C = zgemm_emulated(torch.from_numpy(a).to(cuda_device), torch.from_numpy(b).to(cuda_device), slices=6)
    got = C.cpu().numpy()
    bad = np.zeros(got.shape, dtype=bool)
    bad[0, 3, :] = True
    bad[1, :, 5] = True
    assert np.all(np.isnan(got[bad]))
    assert np.all(np.isfinite(got[~bad]))
    ok_a, ok_b = a.copy(), b.copy()
    ok_a[0, 3, 7] = 0.0
    ok_b[1, 11, 5] = 0.0
    ref = ok_a @ ok_b
    scale = np.abs(ok_a) @ np.abs(ok_b)
    assert np.max(np.abs(got - ref)[~bad] / scale[~bad]) < REL[6]


def test_sancho_rubio_and_contact_on_emulated_path(cuda_device):
    """The boundary-condition drivers bind the plane scratch from their own
    workspace under gemm_path(); at 7 planes they agree with FP64 DMMA."""
    from quatrex_b200 import SanchoRubio, contact_self_energy, synthetic

    dev = synthetic.make_device(num_blocks=4, block_size=64, energies=np.linspace(-1.0, 1.0, 5), seed=2)
    d, u, l = dev.system_blocks()
    a_ii, a_ij, a_ji = (torch.from_numpy(np.ascontiguousarray(x)).to(cuda_device) for x in (d[0], u[0], l[0]))
    f = torch.from_numpy(dev.fermi_left()).to(cuda_device)
    sr = SanchoRubio(convergence_tol=1e-12, per_energy=True)
    g64 = sr(a_ii, a_ij, a_ji, "left")
    s64 = contact_self_energy(a_ij, a_ji, g64, f)
    with gemm_path(7):
        g7 = sr(a_ii, a_ij, a_ji, "left")
        s7 = contact_self_energy(a_ij, a_ji, g7, f)
    assert status() == 0
    rel = float(torch.linalg.norm(g7 - g64) / torch.linalg.norm(g64))
    assert rel < 1e-8, rel
    for x7, x64 in zip(s7, s64):
        assert float(torch.linalg.norm(x7 - x64) / torch.linalg.norm(x64)) < 1e-8
