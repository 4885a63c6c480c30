"""RGF.selected_inv / selected_solve through the qttools-style interface.

Mirrors the reference suites tests/qttools/greens_function_solver/
test_selected_inv.py:37-69 and test_selected_solve.py:37-117 (dense inverse
on the selected pattern, block layouts x stack shapes x batching x out),
with the CPU oracle as a second, tighter check (FP64: 1e-12 relative)."""

import numpy as np
import pytest
import scipy.sparse as sps
import torch

from oracle import negf_oracle as o
from quatrex_b200 import RGF, DSDBCOO, OBCBlocks, synthetic

pytestmark = pytest.mark.gpu

BLOCK_SIZES = [np.array([2] * 10), np.array([2] * 3 + [4] * 2 + [2] * 3), np.array([3, 64, 17, 64])]
STACKS = [(10,), (7, 2), (9, 2, 4)]
RTOL_ORACLE = 1e-12


def _bt_mask(dense):
    return dense.astype(bool)


def _dev(m, device):
    return DSDBCOO(m.data.to(device), m.rows, m.cols, m.block_sizes, m.global_stack_shape)


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("bs", BLOCK_SIZES, ids=["const", "mixed", "uneven"])
@pytest.mark.parametrize("stack", STACKS, ids=["1D", "2D", "3D"])
@pytest.mark.parametrize("max_batch_size", [1, 2, 100])
@pytest.mark.parametrize("out", [True, False])
@pytest.mark.parametrize("host", [False, True], ids=["device", "host"])
def test_selected_inv(cuda_device, bs, stack, max_batch_size, out, host):
    dense = synthetic.random_bt_dense(bs, seed=int(bs.sum()))
    mask = _bt_mask(dense)
    ref = np.linalg.inv(dense) * mask
    a = DSDBCOO.from_sparray(sps.coo_matrix(dense), bs, stack)
    if not host:
        a = _dev(a, cuda_device)
    solver = RGF(max_batch_size=max_batch_size)
    if out:
        x = DSDBCOO.zeros_like(a)
        assert solver.selected_inv(a, out=x) is None
    else:
        x = solver.selected_inv(a)
    got = x.to_dense().cpu().numpy()
    assert x.data.device == a.data.device
    np.testing.assert_allclose(np.broadcast_to(ref, got.shape), got * mask)
    assert _rel(got * mask, np.broadcast_to(ref, got.shape)) < RTOL_ORACLE * 10


@pytest.mark.parametrize("bs", BLOCK_SIZES, ids=["const", "mixed", "uneven"])
@pytest.mark.parametrize("stack", STACKS, ids=["1D", "2D", "3D"])
@pytest.mark.parametrize("max_batch_size", [1, 2, 100])
@pytest.mark.parametrize("out", [True, False])
@pytest.mark.parametrize("return_retarded", [True, False])
def test_selected_solve(cuda_device, bs, stack, max_batch_size, out, return_retarded):
    dense = synthetic.random_bt_dense(bs, seed=int(bs.sum()) + 1)
    coo_a = sps.coo_matrix(dense)
    bl = sps.coo_matrix(dense)
    bl = sps.coo_matrix(bl + -bl.conj().T)
    bg = sps.coo_matrix(1j * dense)
    bg = sps.coo_matrix(bg + -bg.conj().T)
    ref_r = np.linalg.inv(dense)
    ref_l = ref_r @ bl.toarray() @ ref_r.conj().T
    ref_g = ref_r @ bg.toarray() @ ref_r.conj().T
    A = _dev(DSDBCOO.from_sparray(coo_a, bs, stack), cuda_device)
    Bl = _dev(DSDBCOO.from_sparray(bl, bs, stack), cuda_device)
    Bg = _dev(DSDBCOO.from_sparray(bg, bs, stack), cuda_device)
    solver = RGF(max_batch_size=max_batch_size)
    if out:
        Xr, Xl, Xg = DSDBCOO.zeros_like(A), DSDBCOO.zeros_like(A), DSDBCOO.zeros_like(A)
        assert solver.selected_solve(A, Bl, Bg, out=[Xl, Xg, Xr], return_retarded=return_retarded) is None
    elif return_retarded:
        Xl, Xg, Xr = solver.selected_solve(A, Bl, Bg, return_retarded=True)
    else:
        Xl, Xg = solver.selected_solve(A, Bl, Bg)
    if return_retarded:
        xr = Xr.to_dense().cpu().numpy()
        m = xr.astype(bool)
        np.testing.assert_allclose(np.broadcast_to(ref_r, xr.shape) * m, xr * m)
    for X, ref in ((Xl, ref_l), (Xg, ref_g)):
        x = X.to_dense().cpu().numpy()
        m = x.astype(bool)
        np.testing.assert_allclose(np.broadcast_to(ref, x.shape) * m, x * m)
        assert _rel(x * m, np.broadcast_to(ref, x.shape) * m) < 1e-11


def test_selected_solve_out_length_error(cuda_device):
    bs = np.array([2] * 4)
    dense = synthetic.random_bt_dense(bs, seed=3)
    A = _dev(DSDBCOO.from_sparray(sps.coo_matrix(dense), bs, (2,)), cuda_device)
    with pytest.raises(ValueError, match="Invalid number of output matrices"):
        RGF().selected_solve(A, A, A, out=[DSDBCOO.zeros_like(A), DSDBCOO.zeros_like(A)], return_retarded=True)


@pytest.mark.parametrize("tag", ["const", "mixed"])
def test_golden_bt_small(cuda_device, golden, tag):
    g = golden("bt_small")
    bs = g[f"{tag}_block_sizes"]
    dense = g[f"{tag}_a"]
    mask = dense != 0
    A = _dev(DSDBCOO.from_sparray(sps.coo_matrix(dense), bs, (4,)), cuda_device)
    x = RGF(max_batch_size=2).selected_inv(A).to_dense().cpu().numpy()
    np.testing.assert_allclose(x[0] * mask, g[f"{tag}_inv"], rtol=0, atol=1e-13)
    Bl = _dev(DSDBCOO.from_sparray(sps.coo_matrix(g[f"{tag}_sigma_lesser"]), bs, (4,)), cuda_device)
    Bg = _dev(DSDBCOO.from_sparray(sps.coo_matrix(g[f"{tag}_sigma_greater"]), bs, (4,)), cuda_device)
    xl, xg, xr = RGF().selected_solve(A, Bl, Bg, return_retarded=True)
    for X, key in ((xl, "xl"), (xg, "xg"), (xr, "xr")):
        got = X.to_dense().cpu().numpy()[0]
        ref = g[f"{tag}_{key}"]
        m = ref != 0
        np.testing.assert_allclose(got * m, ref, rtol=0, atol=1e-12 * np.abs(ref).max())


def test_current_matches_oracle(cuda_device):
    """return_current (no reference test exists) against the oracle."""
    bs = np.array([3, 5, 4, 6])
    dense = synthetic.random_bt_dense(bs, seed=11)
    bl = sps.coo_matrix(dense)
    bl = sps.coo_matrix(bl - bl.conj().T)
    bg = sps.coo_matrix(2j * dense)
    bg = sps.coo_matrix(bg - bg.conj().T)
    stack = (5,)
    A = _dev(DSDBCOO.from_sparray(sps.coo_matrix(dense), bs, stack), cuda_device)
    Bl = _dev(DSDBCOO.from_sparray(bl, bs, stack), cuda_device)
    Bg = _dev(DSDBCOO.from_sparray(bg, bs, stack), cuda_device)
    rng = np.random.default_rng(0)
    ob = OBCBlocks(4)
    obr = [None] * 4
    obl = [None] * 4
    obg = [None] * 4
    for idx in (0, -1):
        b = bs[idx]
        s = (rng.standard_normal((5, b, b)) + 1j * rng.standard_normal((5, b, b))) * 0.1
        gam = 1j * (s - s.conj().swapaxes(-2, -1))
        obr[idx], obl[idx], obg[idx] = s, 0.3j * gam, -0.7j * gam
        ob.retarded[idx] = torch.from_numpy(s).to(cuda_device)
        ob.lesser[idx] = torch.from_numpy(obl[idx]).to(cuda_device)
        ob.greater[idx] = torch.from_numpy(obg[idx]).to(cuda_device)
    xl, xg, xr, cur = RGF().selected_solve(A, Bl, Bg, obc_blocks=ob, return_retarded=True, return_current=True)
    offs = np.concatenate(([0], np.cumsum(bs)))
    blocks = lambda d: ([np.broadcast_to(d[offs[i]:offs[i + 1], offs[i]:offs[i + 1]], (5, bs[i], bs[i])) for i in range(4)],  # noqa: E731
                        [np.broadcast_to(d[offs[i]:offs[i + 1], offs[i + 1]:offs[i + 2]], (5, bs[i], bs[i + 1])) for i in range(3)],
                        [np.broadcast_to(d[offs[i + 1]:offs[i + 2], offs[i]:offs[i + 1]], (5, bs[i + 1], bs[i])) for i in range(3)])
    d, u, lo = blocks(dense)
    sld, slu, sll = blocks(bl.toarray())
    sgd, sgu, sgl = blocks(bg.toarray())
    r = o.selected_solve(d, u, lo, sld, slu, sll, sgd, sgu, sgl, obr, obl, obg, return_current=True)
    c = cur.cpu().numpy()
    assert _rel(c, r["current"]) < 1e-11, _rel(c, r["current"])
    xld = xl.to_dense().cpu().numpy()
    for i in range(4):
        blk = xld[:, offs[i]:offs[i + 1], offs[i]:offs[i + 1]]
        m = blk.astype(bool)
        assert _rel(blk * m, r["xl_diag"][i] * m) < 1e-11


@pytest.mark.parametrize("pinned", [True, False], ids=["pinned", "pageable"])
@pytest.mark.parametrize("symmetric", [False, True], ids=["full", "symmetric"])
def test_selected_solve_host_pipelined(cuda_device, pinned, symmetric):
    """Host (CPU torch) containers with several batches take the pipelined
    path (upload of batch k+1 and write-back of batch k-1 overlap the solve
    of batch k); results equal the device-container path bit for bit."""
    bs = np.array([3, 64, 17, 64])
    dense = synthetic.random_bt_dense(bs, seed=23)
    bl = sps.coo_matrix(dense)
    bl = sps.coo_matrix(bl - bl.conj().T)
    bg = sps.coo_matrix(1j * dense)
    bg = sps.coo_matrix(bg - bg.conj().T)
    stack = (10,)

    def mk(m, dev):
        x = DSDBCOO.from_sparray(m, bs, stack)
        if dev:
            return _dev(x, cuda_device)
        d = x.data.clone()
        return DSDBCOO(d.pin_memory() if pinned else d, x.rows, x.cols, x.block_sizes, x.global_stack_shape)

    rng = np.random.default_rng(2)
    ob = OBCBlocks(4)
    s0 = (rng.standard_normal((10, 3, 3)) + 1j * rng.standard_normal((10, 3, 3))) * 0.1
    ob.retarded[0] = torch.from_numpy(s0).to(cuda_device)
    res = {}
    for dev in (True, False):
        A, Bl, Bg = mk(sps.coo_matrix(dense), dev), mk(bl, dev), mk(bg, dev)
        Xl, Xg, Xr = (DSDBCOO.zeros_like(A) for _ in range(3))
        if not dev:  # sentinel values where nothing may be written
            for X in (Xl, Xg, Xr):
                X.data.fill_(7.0 + 3.0j)
        if symmetric:
            Xl.symmetry = Xg.symmetry = True
        cur = RGF(max_batch_size=3).selected_solve(A, Bl, Bg, obc_blocks=ob, out=(Xl, Xg, Xr),
                                                   return_retarded=True, return_current=True)
        res[dev] = [X.data.cpu().numpy().copy() for X in (Xl, Xg, Xr)] + [torch.as_tensor(cur).cpu().numpy()]
    dev_r, host_r = res[True], res[False]
    np.testing.assert_array_equal(host_r[3], dev_r[3])  # current
    # written blocks equal; unwritten entries keep the sentinel on the host
    for k in range(3):
        written = dev_r[k] != 0
        np.testing.assert_array_equal(host_r[k][written], dev_r[k][written])
    assert (host_r[2][dev_r[2] == 0] == 7.0 + 3.0j).any()  # X^R off-diagonal blocks untouched
