"""Serving loop on the GPU: a request's results do not depend on the
traffic it is batched with, and warm starts reproduce cold solves."""

import numpy as np
import pytest

from quatrex_b200 import synthetic
from quatrex_b200.serving import EnergyServer, Request
from quatrex_b200.uneven import jobs_from_devices

pytestmark = pytest.mark.gpu


def _catalogue():
    devs = [synthetic.make_device(4, 32, np.linspace(-1.5, 1.5, 24), seed=31),
            synthetic.make_device(3, 48, np.linspace(-1.0, 1.0, 16), seed=32)]
    return jobs_from_devices(devs)


def _copy(r):
    return r.transmission.copy(), r.density.copy(), r.current.copy()


@pytest.mark.parametrize("precision", ["fp64", "mixed", "emulated"])
def test_alone_equals_mixed_traffic(cuda_device, precision):
    cat = _catalogue()
    probe = np.array([1, 4, 5, 9, 13, 20, 22])
    alone = EnergyServer(cat, precision=precision, warm_start=False, batches=[4, 4], budget_bytes=8e9)
    ref = _copy(alone.solve_now(Request(0, 0, probe)))
    del alone
    srv = EnergyServer(cat, precision=precision, warm_start=False, batches=[4, 4], budget_bytes=8e9)
    rng = np.random.default_rng(5)
    reqs = [Request(k + 1, int(k % 2), np.sort(rng.choice(24 if k % 2 == 0 else 16, 5, replace=False)),
                    arrival=0.002 * k) for k in range(6)]
    target = Request(99, 0, probe, arrival=0.005)
    stats = srv.run(reqs + [target])
    assert stats["requests"] == 7 and stats["latency"]["count"] == 7
    got = _copy(target)
    for a, b in zip(got, ref):
        np.testing.assert_array_equal(a, b)  # bit-identical whatever shares the batch


def test_warm_start_matches_cold(cuda_device):
    cat = _catalogue()
    srv = EnergyServer(cat, warm_start=True, batches=[4, 4], budget_bytes=8e9)
    first = _copy(srv.solve_now(Request(0, 0, np.arange(0, 24, 3))))
    again = srv.solve_now(Request(1, 0, np.arange(0, 24, 3)))
    assert again.warm_energies == 8 and srv.lanes[0].batches["warm"] >= 2
    # warm = the cached refined surface function plus one more fixed-point
    # step; it agrees with the cold Sancho-Rubio solve within the OBC noise
    # floor of the end-to-end parity tests
    for a, b in zip(_copy(again), first):
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-8
