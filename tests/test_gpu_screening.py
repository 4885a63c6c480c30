"""Screened-interaction (W) boundary conditions on the GPU against the
reference's own outputs (tests/golden/screening.npz): the Lyapunov doubling
solver (qtx_lyapunov_doubling), the memoizing LyapunovSystem and the contact
glue of the Coulomb-screening solve (coulomb_screening/solver.py:211-378).
Tolerance 1e-10 relative (FP64 GPU rounding through a few dozen products and
one decimation)."""

import numpy as np
import pytest
import torch

from quatrex_b200 import Doubling, LyapunovSystem, OBCSystem, SanchoRubio, screened_contact_obc, synthetic

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_doubling_and_lyapunov_system(cuda_device, golden):
    g = golden("screening")
    a, q = g["lyap_a"], g["lyap_q"]
    x = Doubling()(a, q, "test")
    assert isinstance(x, np.ndarray) and x.shape == q.shape
    assert _rel(x, g["lyap_x"]) < TOL
    xs, rel, ab = LyapunovSystem(Doubling(), memoization_mode="off")((a, q), "test")
    assert _rel(xs, g["lyap_system_x"]) < TOL
    assert rel.shape == q.shape[:-2]
    np.testing.assert_allclose(ab, g["lyap_system_abs"], rtol=1e-3, atol=1e-14)
    # device tensors in, device tensors out; memoized second call reuses the cache
    ad, qd = torch.from_numpy(a).to(cuda_device), torch.from_numpy(q).to(cuda_device)
    sys_ = LyapunovSystem(Doubling(), memoization_mode="force-after-first")
    x1, _, _ = sys_((ad, qd), "left")
    x2, _, _ = sys_((ad, qd), "left")
    assert isinstance(x2, torch.Tensor) and x2.is_cuda
    assert _rel(x2.cpu().numpy(), g["lyap_system_x"]) < 1e-8


def test_screened_contact_obc_matches_reference(cuda_device, golden):
    g = golden("screening")
    w = synthetic.screened_lead(16, 3, seed=4)
    obc = OBCSystem(SanchoRubio(max_iterations=100, convergence_tol=1e-12), memoization_mode="off")
    lyap = LyapunovSystem(Doubling(), memoization_mode="off")
    res = screened_contact_obc(w["p_retarded"], w["p_lesser"], w["p_greater"], w["v"], obc, lyap)
    for got, key in zip(res, ("obc_retarded", "obc_lesser", "obc_greater")):
        assert isinstance(got, np.ndarray)
        err = _rel(got, g[key])
        print(key, "rel error vs reference", err)
        assert err < TOL, key
