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
