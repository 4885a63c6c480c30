"""Uneven device batch on the GPU: concurrent graph replays of several
devices reproduce each device solved alone."""

import numpy as np
import pytest
import torch

from quatrex_b200 import EnergyPointSolver, synthetic
from quatrex_b200.uneven import UnevenBatchRunner, jobs_from_devices

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("precision", ["fp64", "mixed", "emulated"])
def test_uneven_runner_matches_single_device(cuda_device, precision):
    devs = [synthetic.make_device(4, 32, np.linspace(-1.5, 1.5, 11), seed=5),
            synthetic.make_device(6, 48, np.linspace(-1.0, 1.2, 7), seed=6),
            synthetic.make_device(3, 64, np.linspace(-2.0, 2.0, 16), seed=7)]
    jobs = jobs_from_devices(devs)
    runner = UnevenBatchRunner(jobs, precision=precision, batches=[4, 8, 16], budget_bytes=8e9)
    res = runner.run()
    assert all(runner.sr_converged().values())
    for d, j in zip(devs, jobs):
        alone = EnergyPointSolver(d.h_diag, d.coupling, eta=d.eta, sr_tol=1e-12, per_energy=True,
                                  precision=precision)
        r = alone.solve(d.energies, d.fermi_left(), d.fermi_right())
        got = res[j.name]
        tol = {"fp64": 1e-10, "emulated": 1e-9, "mixed": 1e-5}[precision]
        assert _rel(got["transmission"].cpu().numpy(), r.transmission.cpu().numpy()) < tol
        assert _rel(got["density"].cpu().numpy(), r.density.cpu().numpy()) < tol
        assert _rel(got["current"].cpu().numpy(), r.current.cpu().numpy()) < 10 * tol


def test_uneven_runner_replays_are_deterministic(cuda_device):
    devs = [synthetic.make_device(3, 32, np.linspace(-1.0, 1.0, 9), seed=8),
            synthetic.make_device(5, 16, np.linspace(-0.5, 0.5, 5), seed=9)]
    runner = UnevenBatchRunner(jobs_from_devices(devs), batches=[4, 2], budget_bytes=4e9)
    a = {k: v["transmission"].cpu().numpy().copy() for k, v in runner.run().items()}
    runner.enqueue()
    torch.cuda.synchronize()
    b = {k: v["transmission"].cpu().numpy() for k, v in runner.results().items()}
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])


def test_uneven_runner_autotune(cuda_device):
    devs = [synthetic.make_device(4, 32, np.linspace(-1.5, 1.5, 12), seed=15),
            synthetic.make_device(3, 48, np.linspace(-1.0, 1.0, 9), seed=16)]
    jobs = jobs_from_devices(devs)
    runner = UnevenBatchRunner(jobs, batches=[8, 9], budget_bytes=4e9, autotune=True, max_trials=2)
    res = runner.run()
    assert set(runner.tuning) == {j.name for j in jobs}
    for j, cap in zip(jobs, (8, 9)):
        t = runner.tuning[j.name]
        assert 1 <= int(t["batch"]) <= cap and len(t["trials"]) >= 1
    for d, j in zip(devs, jobs):
        r = EnergyPointSolver(d.h_diag, d.coupling, eta=d.eta, sr_tol=1e-12, per_energy=True).solve(
            d.energies, d.fermi_left(), d.fermi_right())
        assert _rel(res[j.name]["transmission"].cpu().numpy(), r.transmission.cpu().numpy()) < 1e-10


def test_uneven_batch_as_one_graph(cuda_device):
    """The whole uneven schedule captured as one CUDA graph reproduces the
    stream-by-stream run bit for bit."""
    devs = [synthetic.make_device(3, 32, np.linspace(-1.0, 1.0, 7), seed=18),
            synthetic.make_device(4, 24, np.linspace(-0.8, 0.9, 5), seed=19)]
    runner = UnevenBatchRunner(jobs_from_devices(devs), batches=[4, 2], budget_bytes=4e9)
    ref = {k: v["transmission"].cpu().numpy().copy() for k, v in runner.run().items()}
    for st in runner.states:
        st.transmission.zero_()
    g = runner.capture_all()
    g.replay()
    torch.cuda.synchronize()
    for k, v in runner.results().items():
        np.testing.assert_array_equal(v["transmission"].cpu().numpy(), ref[k])
