"""The CPU oracle against golden vectors produced by the reference package
(tests/golden/make_golden.py). This pins the oracle before it is used as
the checker of the CUDA path."""

import numpy as np
import pytest
import scipy.sparse as sps

from oracle import negf_oracle as o
from quatrex_b200 import synthetic


def _blocks_of(dense, block_sizes):
    offs = np.concatenate(([0], np.cumsum(block_sizes)))
    n = len(block_sizes)
    d = [dense[None, offs[i]:offs[i + 1], offs[i]:offs[i + 1]] for i in range(n)]
    u = [dense[None, offs[i]:offs[i + 1], offs[i + 1]:offs[i + 2]] for i in range(n - 1)]
    lo = [dense[None, offs[i + 1]:offs[i + 2], offs[i]:offs[i + 1]] for i in range(n - 1)]
    return d, u, lo


def _assemble(diag, upper, lower, block_sizes):
    offs = np.concatenate(([0], np.cumsum(block_sizes)))
    n = len(block_sizes)
    out = np.zeros((diag[0].shape[0], offs[-1], offs[-1]), dtype=np.complex128)
    for i in range(n):
        out[:, offs[i]:offs[i + 1], offs[i]:offs[i + 1]] = diag[i]
        if i + 1 < n:
            out[:, offs[i]:offs[i + 1], offs[i + 1]:offs[i + 2]] = upper[i]
            out[:, offs[i + 1]:offs[i + 2], offs[i]:offs[i + 1]] = lower[i]
    return out


@pytest.mark.parametrize("tag", ["const", "mixed"])
def test_selected_inv_matches_reference(golden, tag):
    g = golden("bt_small")
    bs = g[f"{tag}_block_sizes"]
    d, u, lo = _blocks_of(g[f"{tag}_a"], bs)
    xd, xu, xl = o.selected_inv(d, u, lo)
    got = _assemble(xd, xu, xl, bs)[0]
    mask = g[f"{tag}_a"] != 0
    np.testing.assert_allclose(got * mask, g[f"{tag}_inv"] * mask, rtol=0, atol=1e-14)


@pytest.mark.parametrize("tag", ["const", "mixed"])
def test_selected_solve_matches_reference(golden, tag):
    g = golden("bt_small")
    bs = g[f"{tag}_block_sizes"]
    d, u, lo = _blocks_of(g[f"{tag}_a"], bs)
    sld, slu, sll = _blocks_of(g[f"{tag}_sigma_lesser"], bs)
    sgd, sgu, sgl = _blocks_of(g[f"{tag}_sigma_greater"], bs)
    r = o.selected_solve(d, u, lo, sld, slu, sll, sgd, sgu, sgl)
    mask = g[f"{tag}_a"] != 0
    for key, ref in (("xl", g[f"{tag}_xl"]), ("xg", g[f"{tag}_xg"])):
        got = _assemble(r[f"{key}_diag"], r[f"{key}_upper"], r[f"{key}_lower"], bs)[0]
        np.testing.assert_allclose(got * mask, ref * mask, rtol=0, atol=1e-13)
    zero_u = [np.zeros_like(x) for x in u]
    got = _assemble(r["xr_diag"], zero_u, [np.zeros_like(x) for x in lo], bs)[0]
    np.testing.assert_allclose(got * mask, g[f"{tag}_xr"], rtol=0, atol=1e-14)


@pytest.fixture(scope="module")
def cfg0_oracle():
    dev = synthetic.cfg0()
    diag, upper, lower = dev.system_blocks()
    return dev, o.energy_point_solve(diag, upper, lower, dev.fermi_left(), dev.fermi_right())


def test_synthetic_generator_pinned(golden):
    g = golden("cfg0")
    dev = synthetic.cfg0()
    np.testing.assert_array_equal(dev.energies, g["energies"])
    np.testing.assert_array_equal(dev.h_diag[0, :4, :4], g["h_corner"])
    np.testing.assert_array_equal(dev.coupling[:4, :4], g["t_corner"])
    chk = np.array([dev.h_diag.sum(), np.abs(dev.h_diag).sum(), dev.coupling.sum()])
    np.testing.assert_allclose(chk, g["h00_checksum"], rtol=1e-14)


def test_cfg0_energy_point_matches_reference(golden, cfg0_oracle):
    g = golden("cfg0")
    _, r = cfg0_oracle
    pick = g["pick"]

    def rel(a, b):
        return np.linalg.norm(a - b) / np.linalg.norm(b)

    assert rel(r["current"], g["current"]) < 1e-13
    assert rel(r["density"], g["density"]) < 1e-13
    assert rel(r["transmission"], g["transmission"]) < 1e-12
    for k, i in enumerate(g["pick_blocks"]):
        assert rel(r["xr_diag"][i][pick], g["xr_diag"][k]) < 1e-13
        assert rel(r["xl_diag"][i][pick], g["xl_diag"][k]) < 1e-13
    assert rel(r["xg_diag"][8][pick], g["xg_diag8"]) < 1e-13
    assert rel(r["xl_upper"][0][pick], g["xl_upper01"]) < 1e-13
    assert rel(r["xl_lower"][0][pick], g["xl_lower10"]) < 1e-13
    assert rel(r["sigma_left"][pick], g["sigma_left"]) < 1e-13
    assert rel(r["sigma_right"][pick], g["sigma_right"]) < 1e-13


def test_cfg0_selected_inv_with_obc_matches_reference(golden, cfg0_oracle):
    g = golden("cfg0")
    dev, r = cfg0_oracle
    diag, upper, lower = dev.system_blocks()
    n = dev.num_blocks
    obc = [None] * n
    obc[0], obc[-1] = r["sigma_left"], r["sigma_right"]
    xd, xu, _ = o.selected_inv(diag, upper, lower, obc)
    pick = g["pick"]
    np.testing.assert_allclose(xd[8][pick], g["inv_diag8"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(xu[0][pick], g["inv_upper01"], rtol=0, atol=1e-12)


def test_transmission_rgf_equals_dense_caroli(cfg0_oracle):
    dev, r = cfg0_oracle
    diag, upper, lower = dev.system_blocks(dev.energies[:3])
    n, b = dev.num_blocks, dev.block_size
    a = np.zeros((3, n * b, n * b), dtype=np.complex128)
    for i in range(n):
        a[:, i * b:(i + 1) * b, i * b:(i + 1) * b] = diag[i]
        if i + 1 < n:
            a[:, i * b:(i + 1) * b, (i + 1) * b:(i + 2) * b] = upper[i]
            a[:, (i + 1) * b:(i + 2) * b, i * b:(i + 1) * b] = lower[i]
    a[:, :b, :b] -= r["sigma_left"][:3]
    a[:, -b:, -b:] -= r["sigma_right"][:3]
    t = o.transmission_caroli_dense(a, r["sigma_left"][:3], r["sigma_right"][:3], b, b)
    np.testing.assert_allclose(r["transmission"][:3], t, rtol=1e-10)


def test_cfg1_sample_matches_reference(golden):
    g = golden("cfg1_sample")
    dev = synthetic.cfg1()
    e = g["energy_index"][:1]
    diag, upper, lower = dev.system_blocks(dev.energies[e])
    r = o.energy_point_solve(diag, upper, lower, dev.fermi_left(dev.energies[e]),
                             dev.fermi_right(dev.energies[e]))
    np.testing.assert_allclose(r["transmission"], g["transmission"][:1], rtol=1e-11)
    np.testing.assert_allclose(r["current"], g["current"][:1], rtol=0, atol=1e-12 * np.abs(g["current"]).max())
    np.testing.assert_allclose(r["density"], g["density"][:1], rtol=0, atol=1e-12 * np.abs(g["density"]).max())
    xr_fro = np.stack([np.linalg.norm(r["xr_diag"][i], axis=(-2, -1)) for i in range(dev.num_blocks)], -1)
    np.testing.assert_allclose(xr_fro, g["xr_fro"][:1], rtol=1e-12)


def test_sancho_rubio_max_iterations_warns():
    dev = synthetic.make_device(2, 8, np.array([0.1]), seed=3)
    diag, upper, lower = dev.system_blocks()
    with pytest.warns(RuntimeWarning):
        o.sancho_rubio(diag[0], upper[0], lower[0], max_iterations=1, convergence_tol=1e-8)


def test_get_batches_matches_reference_examples():
    assert o.get_section_sizes(10, 3, "balanced") == ([4, 3, 3], 12)
    assert o.get_section_sizes(10, 3, "greedy") == ([4, 4, 2], 12)
    sizes, slices = o.get_batches(10, 3)
    assert sizes == [4, 3, 3] and list(slices) == [0, 4, 7, 10]
    sizes, slices = o.get_batches(7, 100)
    assert sizes == [7]
