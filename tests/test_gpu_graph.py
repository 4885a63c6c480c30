"""Host-sync-free energy points and CUDA-graph replay: the device-side
Sancho-Rubio loop and a captured pipeline reproduce the eager FP64 results
(bit-for-bit for the graph replay of the same device-loop sequence)."""

import numpy as np
import pytest
import torch

from quatrex_b200 import EnergyPointSolver, synthetic

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_device_loop_matches_host_loop(cuda_device):
    dev = synthetic.make_device(8, 64, np.linspace(-1.5, 1.5, 12), seed=2)
    host = EnergyPointSolver(dev.h_diag, dev.coupling, eta=dev.eta, sr_tol=1e-12, per_energy=True)
    devl = EnergyPointSolver(dev.h_diag, dev.coupling, eta=dev.eta, sr_tol=1e-12, per_energy=True,
                             device_loop=True)
    a = host.solve(dev.energies, dev.fermi_left(), dev.fermi_right())
    ta, da = a.transmission.cpu().numpy().copy(), a.density.cpu().numpy().copy()
    b = devl.solve(dev.energies, dev.fermi_left(), dev.fermi_right())
    it, conv = devl.sr_status(dev.energies.size)
    assert conv and 5 < it < 100
    assert _rel(b.transmission.cpu().numpy(), ta) < 1e-12
    assert _rel(b.density.cpu().numpy(), da) < 1e-12


def test_graph_replay_matches_eager(cuda_device):
    dev = synthetic.make_device(6, 64, np.linspace(-2.0, 2.0, 24), seed=3)
    s = EnergyPointSolver(dev.h_diag, dev.coupling, eta=dev.eta, sr_tol=1e-12, per_energy=True,
                          device_loop=True)
    e1, e2 = dev.energies[:12], dev.energies[12:]
    fl, fr = dev.fermi_left(), dev.fermi_right()
    ref1 = s.solve(e1, fl[:12], fr[:12]).transmission.cpu().numpy().copy()
    ref2 = s.solve(e2, fl[12:], fr[12:]).transmission.cpu().numpy().copy()
    g1 = s.solve_graph(e1, fl[:12], fr[:12]).transmission.cpu().numpy().copy()
    g2 = s.solve_graph(e2, fl[12:], fr[12:]).transmission.cpu().numpy().copy()
    np.testing.assert_array_equal(g1, ref1)
    np.testing.assert_array_equal(g2, ref2)
