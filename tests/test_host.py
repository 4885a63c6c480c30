"""Host-side logic: batching, block layouts, the torch DSDBCOO container and
the flop model (no GPU)."""

import numpy as np
import pytest
import scipy.sparse as sps
import torch

from oracle import negf_oracle as o
from quatrex_b200 import synthetic
from quatrex_b200._interop import BlockLayout
from quatrex_b200.datastructures import DSDBCOO
from quatrex_b200.negf import flops_per_energy
from quatrex_b200.utils import get_batches, get_section_sizes


@pytest.mark.parametrize("n,mb", [(10, 1), (10, 2), (10, 100), (7, 3), (1024, 148), (32, 32), (33, 8)])
def test_get_batches_matches_oracle(n, mb):
    s1, sl1 = get_batches(n, mb)
    s2, sl2 = o.get_batches(n, mb)
    assert s1 == s2 and np.array_equal(sl1, sl2)


def test_section_sizes_strategies():
    assert get_section_sizes(10, 3, "balanced") == ([4, 3, 3], 12)
    assert get_section_sizes(10, 3, "greedy") == ([4, 4, 2], 12)
    with pytest.raises(ValueError):
        get_section_sizes(10, 3, "fair")


@pytest.mark.parametrize("bs", [[2] * 10, [2, 2, 2, 4, 4, 2, 2, 2], [3, 5, 1]])
def test_dsdbcoo_roundtrip_and_layout(bs):
    dense = synthetic.random_bt_dense(bs, seed=1)
    m = DSDBCOO.from_sparray(sps.coo_matrix(dense), bs, (3, 2))
    assert m.data.shape == (3, 2, np.count_nonzero(dense))
    np.testing.assert_array_equal(m.to_dense()[1, 1].numpy(), dense)
    offs = np.concatenate(([0], np.cumsum(bs)))
    for i in range(len(bs)):
        for j in (i - 1, i, i + 1):
            if 0 <= j < len(bs):
                blk = m.blocks[i, j]
                np.testing.assert_array_equal(blk[2, 0].numpy(), dense[offs[i]:offs[i + 1], offs[j]:offs[j + 1]])
    # block writes hit only the pattern
    m2 = DSDBCOO.zeros_like(m)
    m2.blocks[0, 0] = torch.ones(bs[0], bs[0], dtype=torch.complex128)
    got = m2.to_dense()[0, 0].numpy()
    mask = dense[:bs[0], :bs[0]] != 0
    np.testing.assert_array_equal(got[:bs[0], :bs[0]], mask.astype(complex))
    np.testing.assert_array_equal(m.diagonal()[0, 0].numpy(), np.diagonal(dense))


def test_block_layout_dense_detection():
    bs = [4, 4, 4]
    pattern = np.zeros((12, 12))
    for i in range(3):
        for j in (i - 1, i, i + 1):
            if 0 <= j < 3:
                pattern[4 * i:4 * i + 4, 4 * j:4 * j + 4] = 1
    m = DSDBCOO.from_sparray(sps.coo_matrix(pattern + 0j), bs, (2,))
    lay = BlockLayout(m.rows, m.cols, bs)
    assert all(e.dense for e in lay.entries.values())
    dense = synthetic.random_bt_dense(bs, seed=2)
    m = DSDBCOO.from_sparray(sps.coo_matrix(dense), bs, (2,))
    lay = BlockLayout(m.rows, m.cols, bs)
    assert not all(e.dense for e in lay.entries.values() if e is not None)


def test_block_layout_rejects_unsorted():
    rows = np.array([0, 2, 1])
    cols = np.array([0, 2, 1])
    with pytest.raises(ValueError):
        BlockLayout(rows, cols, np.array([2, 1]))


def test_flop_model():
    f = flops_per_energy(32, 256, (20, 20))
    u = 8 * 256 ** 3
    assert f["solve"] == u * (32 + 4 + 33 * 31)
    assert f["current"] == u * (9 * 31 + 4)
    assert abs(f["solve"] / 1e9 - 142.1) < 0.1
    assert abs(f["current"] / 1e9 - 38.0) < 0.1
    assert f["sr"] == 2 * u * (11 * 20 + 1)


def test_w_solve_validates_block_counts():
    """The W solve rejects polarizations whose block structure does not match
    the Coulomb matrix before anything reaches the GPU (the constructor only
    needs the Coulomb blocks; checked without a device by a CPU-side stub)."""
    import numpy as np
    import pytest

    from quatrex_b200.screening import CoulombScreeningSolve

    s = CoulombScreeningSolve.__new__(CoulombScreeningSolve)
    s.num_small, s.b, s.nc, s.device = 6, 4, 3, "cpu"
    blocks = ([np.zeros((2, 4, 4))] * 6, [np.zeros((2, 4, 4))] * 5, [np.zeros((2, 4, 4))] * 4)
    with pytest.raises(ValueError, match="off-diagonal"):
        s.solve(blocks, blocks, blocks)
    bad = ([np.zeros((2, 4, 4))] * 6, [np.zeros((2, 4, 4))] * 5, [np.zeros((2, 4, 3))] * 5)
    with pytest.raises(ValueError, match="stacks"):
        s.solve(bad, bad, bad)
