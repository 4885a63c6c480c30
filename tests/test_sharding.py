"""Energy sharding on 2 gloo ranks (CPU): partition, all-gather of uneven
sections, and a sweep whose gathered result equals the single-rank one."""

import os
import socket
from types import SimpleNamespace

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from quatrex_b200.sharding import ShardedEnergySweep, energy_partition, gather_energies


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def fake_solve(energies, fl, fr):
    e = torch.as_tensor(energies, dtype=torch.float64)
    return SimpleNamespace(transmission=e ** 2, current=torch.stack([e + 1j * e, e * 2 + 0j], -1),
                           density=torch.outer(e, torch.arange(3, dtype=torch.float64)))


def _worker(rank, world, port, n, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        energies = np.linspace(-1, 1, n)
        res = ShardedEnergySweep(fake_solve, batch_size=2).run(energies, energies * 0, energies * 0)
        a, b = energy_partition(n, world)[rank]
        g = gather_energies(torch.arange(a, b, dtype=torch.float64)[:, None] * torch.ones(1, 2), n)
        q.put((rank, {k: v.numpy() for k, v in res.items()}, g.numpy()))
    finally:
        dist.destroy_process_group()


def test_partition_balanced():
    assert energy_partition(10, 3) == [(0, 4), (4, 7), (7, 10)]
    assert energy_partition(1024, 8)[-1] == (896, 1024)
    with pytest.raises(ValueError):
        energy_partition(2, 3)


@pytest.mark.parametrize("n", [7, 8])
def test_two_rank_sweep_matches_single_rank(n):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, n, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ref = fake_solve(np.linspace(-1, 1, n), None, None)
    for rank, res, g in out:
        np.testing.assert_allclose(res["transmission"], ref.transmission.numpy())
        np.testing.assert_allclose(res["current"], ref.current.numpy())
        np.testing.assert_allclose(res["density"], ref.density.numpy())
        np.testing.assert_array_equal(g[:, 0], np.arange(n))


def _agreement_worker(rank, world, port, passing, q):
    """OBCSystem's "auto" memoizer decision on 2 gloo ranks
    (boundary_system.py:280-296): the entries whose warm start passes the
    residual test are counted over the stack communicator, divided by its
    size, and compared with the agreement threshold; every rank takes the
    same decision. The native residual step is replaced by fixed residuals
    (host-side test of the control flow)."""
    import datetime

    import quatrex_b200.obc as obc_mod

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ok = torch.tensor(passing[rank])

        class Probe(obc_mod.OBCSystem):
            fresh = 0

            def _get_residuals(self, system, test_solution):
                rel = torch.where(ok, torch.full(ok.shape, 1e-3), torch.full(ok.shape, 0.9)).double()
                ab = torch.where(ok, torch.full(ok.shape, 1e-9), torch.full(ok.shape, 1.0)).double()
                return rel, ab, test_solution

            def _solve(self, system, contact):
                Probe.fresh += 1
                return system[0]

            def _fixed_point_step(self, system, solution):
                return solution

        class Dummy(obc_mod.OBCSolver):
            def __call__(self, a_ii, a_ij, a_ji, contact):
                return a_ii

        system = tuple(torch.zeros((len(passing[rank]), 2, 2), dtype=torch.complex128) for _ in range(3))
        m = Probe(Dummy(), memoization_mode="auto", num_ref_iterations=3, stack_comm=dist.group.WORLD)
        m._cache["left"] = system[0].clone()
        m._memoized_solve(system, "left")
        q.put((rank, Probe.fresh))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("passing,fresh", [
    # 4 passing entries over 2 ranks: 4 / 2 = 2 > 0.999 -> both ranks solve afresh
    (([True, True], [True, True]), 1),
    # 1 passing entry: 1 / 2 = 0.5 -> both ranks keep the refined warm start
    (([True, False], [False, False]), 0),
    # 2 passing entries, all on one rank: 2 / 2 = 1.0 > 0.999 -> both solve afresh
    (([True, True], [False, False]), 1),
])
def test_obc_memoizer_agreement_across_ranks(passing, fresh):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_agreement_worker, args=(r, 2, port, passing, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out == {0: fresh, 1: fresh}
