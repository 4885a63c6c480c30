"""The electron solve of an SCBA iteration: scattering self-energies in the
system matrix and in the selected solve (quatrex electron/solver.py:611-709
and :845-872), on the GPU against the oracle.

Tolerances: the one-pass assembly (qtx_assemble_system) against the oracle's
restatement of _assemble_system_matrix at 1e-14 (rounding of a few
additions); the energy point end to end at 1e-8 (the decimation noise floor
of the 24-wide leads, as for the potential test in test_gpu_negf.py).
"""

import ctypes

import numpy as np
import pytest
import torch

from oracle import negf_oracle as o
from quatrex_b200 import EnergyPointSolver, ScatteringSelfEnergy, _native, synthetic
from quatrex_b200._interop import mat
from quatrex_b200._native import QtxBT, QtxMat

pytestmark = pytest.mark.gpu


def _scattering(rng, n, b, ne, scale):
    """Random causal scattering self-energies with the reference's
    symmetries: Sigma^R Hermitian; Sigma^< = i P_<, Sigma^> = -i P_> with
    P = Q Q^H positive semidefinite and block-tridiagonal (Q block upper
    bidiagonal), so that (Sigma^> - Sigma^<) / 2 only broadens the levels."""
    def rand(*s):
        return (rng.standard_normal(s) + 1j * rng.standard_normal(s)) * scale

    def herm(x):
        return 0.5 * (x + x.conj().swapaxes(-2, -1))

    def h(x):
        return x.conj().swapaxes(-2, -1)

    out = {}
    d = [herm(rand(ne, b, b)) for _ in range(n)]
    u = [rand(ne, b, b) for _ in range(n - 1)]
    out["retarded"] = (d, u, [h(x) for x in u])
    for name, sign in (("lesser", 1.0), ("greater", -1.0)):
        qd = [rand(ne, b, b) for _ in range(n)]
        qu = [rand(ne, b, b) for _ in range(n - 1)]
        pd = [qd[i] @ h(qd[i]) + (qu[i] @ h(qu[i]) if i < n - 1 else 0) for i in range(n)]
        pu = [qu[i] @ h(qd[i + 1]) for i in range(n - 1)]
        out[name] = ([1j * sign * x for x in pd], [1j * sign * x for x in pu], [1j * sign * h(x) for x in pu])
    return out


def _dev(blocks, device):
    return tuple(torch.from_numpy(np.ascontiguousarray(np.stack(x))).to(device) for x in blocks)


@pytest.fixture(scope="module")
def case(cuda_device):
    rng = np.random.default_rng(17)
    dev = synthetic.make_device(6, 24, np.linspace(-1.4, 1.3, 5), seed=23)
    n, b, ne = dev.num_blocks, dev.block_size, dev.energies.size
    V = rng.uniform(-0.1, 0.1, n * b)
    sc = _scattering(rng, n, b, ne, 0.03)
    h_diag = [dev.h_diag[i] for i in range(n)]
    h_up = [dev.coupling] * (n - 1)
    h_lo = [dev.coupling.conj().T] * (n - 1)
    blocks = o.assemble_system(h_diag, h_up, h_lo, dev.energies, dev.eta, V, sc["retarded"], sc["lesser"],
                               sc["greater"])
    return dev, V, sc, (h_diag, h_up, h_lo), blocks


def test_assemble_system_matches_oracle(case, cuda_device):
    dev, V, sc, (h_diag, h_up, h_lo), (d_ref, u_ref, l_ref) = case
    lib = _native.load()
    n, b, ne = dev.num_blocks, dev.block_size, dev.energies.size
    keep = []

    def bt(diag, up, lo):
        bs = (ctypes.c_int32 * n)(*([b] * n))
        d = (QtxMat * n)(*diag)
        u = (QtxMat * (n - 1))(*up)
        lw = (QtxMat * (n - 1))(*lo)
        keep.extend([bs, d, u, lw])
        return QtxBT(n, bs, d, u, lw)

    def bcast(x):
        t = torch.from_numpy(np.ascontiguousarray(x)).to(cuda_device)
        keep.append(t)
        return QtxMat(t.data_ptr(), b, 0)

    def stk(blocks):
        ts = [torch.from_numpy(np.ascontiguousarray(x)).to(cuda_device) for x in blocks]
        keep.extend(ts)
        return [mat(t) for t in ts]

    H = bt([bcast(x) for x in h_diag], [bcast(x) for x in h_up], [bcast(x) for x in h_lo])
    S = {k: bt(stk(v[0]), stk(v[1]), stk(v[2])) for k, v in sc.items()}
    out = [torch.empty((ne, b, b), dtype=torch.complex128, device=cuda_device) for _ in range(3 * n - 2)]
    A = bt([mat(t) for t in out[:n]], [mat(t) for t in out[n:2 * n - 1]], [mat(t) for t in out[2 * n - 1:]])
    z = torch.from_numpy(dev.energies + 1j * dev.eta).to(cuda_device)
    v = torch.from_numpy(V).to(cuda_device)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _native.check(lib.qtx_assemble_system(ctypes.byref(H), v.data_ptr(), z.data_ptr(), ctypes.byref(S["retarded"]),
                                          ctypes.byref(S["lesser"]), ctypes.byref(S["greater"]), ctypes.byref(A),
                                          ne, stream))
    torch.cuda.synchronize()
    for got, ref in zip(out, d_ref + u_ref + l_ref):
        g = got.cpu().numpy()
        assert np.abs(g - ref).max() <= 1e-14 * np.abs(ref).max()


def test_energy_point_with_scattering_matches_oracle(case, cuda_device):
    dev, V, sc, _, (diag, upper, lower) = case
    solver = EnergyPointSolver(dev.h_diag, dev.coupling, eta=dev.eta, sr_tol=1e-12, per_energy=False,
                               potential=V.reshape(dev.num_blocks, dev.block_size))
    scatt = ScatteringSelfEnergy(*(_dev(sc[k], cuda_device) for k in ("retarded", "lesser", "greater")))
    r = solver.solve(dev.energies, dev.fermi_left(), dev.fermi_right(), scattering=scatt)
    ref = o.energy_point_solve(diag, upper, lower, dev.fermi_left(), dev.fermi_right(),
                               sigma_lesser=sc["lesser"], sigma_greater=sc["greater"])

    def rel(a, b_):
        return float(np.linalg.norm(a - b_) / np.linalg.norm(b_))

    errs = {
        "current": rel(r.current.cpu().numpy(), ref["current"]),
        "density": rel(r.density.cpu().numpy(), ref["density"]),
        "xl_diag2": rel(r.blocks["xl_diag"][2].cpu().numpy(), ref["xl_diag"][2]),
        "xg_upper1": rel(r.blocks["xg_upper"][1].cpu().numpy(), ref["xg_upper"][1]),
        "sigma_left": rel(r.sigma_left.cpu().numpy(), ref["sigma_left"]),
    }
    print("scattering energy point vs oracle:", errs)
    assert all(v < 1e-8 for v in errs.values()), errs
    # the scattering self-energies change the result (the test is not vacuous)
    plain = solver.solve(dev.energies, dev.fermi_left(), dev.fermi_right())
    assert rel(plain.density.cpu().numpy(), ref["density"]) > 1e-4
    with pytest.raises(ValueError):
        bad = ScatteringSelfEnergy(lesser=tuple(t[:, :2] for t in scatt.lesser))
        solver.solve(dev.energies, dev.fermi_left(), dev.fermi_right(), scattering=bad)
