"""Energy sharding with the real solver: two ranks on one GPU.

Each rank is its own process with its own CUDA context on cuda:0 and runs
``ShardedEnergySweep`` over ``EnergyPointSolver`` on its contiguous energy
section (the reference's stack distribution, ``dsdbsparse.py:185-199``);
the observables are gathered over gloo. The ranks' kernels never wait on
each other (no collective or flag on the device), so sharing one GPU is
safe. The gathered transmission, current and density must equal the
single-rank solve of the whole grid bit for bit: with per-energy
Sancho-Rubio convergence every energy's arithmetic is independent of the
batch it is solved in.
"""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

N_BLOCKS, BLOCK, N_E = 6, 48, 11


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _device():
    from quatrex_b200 import synthetic

    return synthetic.make_device(N_BLOCKS, BLOCK, np.linspace(-1.8, 1.8, N_E), seed=3)


def _solver(dev):
    from quatrex_b200 import EnergyPointSolver

    return EnergyPointSolver(dev.h_diag, dev.coupling, eta=dev.eta, sr_tol=1e-12, per_energy=True,
                             store_blocks=False)


def _worker(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist

    from quatrex_b200.sharding import ShardedEnergySweep

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        dev = _device()
        solver = _solver(dev)

        def solve_batch(e, fl, fr):
            r = solver.solve(e, fl, fr)
            torch.cuda.synchronize()
            # gloo gathers host tensors
            return type("R", (), {k: getattr(r, k).cpu() for k in ("transmission", "current", "density")})

        res = ShardedEnergySweep(solve_batch, batch_size=3).run(dev.energies, dev.fermi_left(), dev.fermi_right())
        q.put((rank, {k: v.numpy() for k, v in res.items()}))
    finally:
        dist.destroy_process_group()


def test_two_ranks_on_one_gpu_match_single_rank(cuda_device):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=600) for _ in procs)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    dev = _device()
    r = _solver(dev).solve(dev.energies, dev.fermi_left(), dev.fermi_right())
    ref = {k: getattr(r, k).cpu().numpy() for k in ("transmission", "current", "density")}
    for rank in (0, 1):
        for k in ref:
            np.testing.assert_array_equal(out[rank][k], ref[k], err_msg=f"rank {rank} {k}")
