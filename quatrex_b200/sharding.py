"""Energy sharding across GPUs (one process per GPU).

Energies are independent, so the stack is split into contiguous, balanced
sections per rank -- the reference's stack distribution
(``src/qttools/datastructures/dsdbsparse.py:185-199`` with
``get_section_sizes(..., strategy="balanced")``) -- and every rank solves
its own section with no communication. The per-energy observables
(transmission, current, density) are gathered afterwards with one
``all_gather`` per array (NCCL over NVLink on GPUs; gloo on CPU for tests).
Green's-function blocks stay sharded on their rank.
"""

from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist

from .utils import get_section_sizes


def energy_partition(num_energies: int, world_size: int) -> list[tuple[int, int]]:
    """Contiguous (start, stop) energy ranges of every rank."""
    if world_size > num_energies:
        raise ValueError(f"Number of ranks {world_size} exceeds the number of energies {num_energies}.")
    sizes, _ = get_section_sizes(num_energies, world_size, strategy="balanced")
    offs = np.concatenate(([0], np.cumsum(sizes)))
    return [(int(offs[r]), int(offs[r + 1])) for r in range(world_size)]


def gather_energies(local: torch.Tensor, num_energies: int, group=None) -> torch.Tensor:
    """Concatenates every rank's (n_r, ...) section into (num_energies, ...)
    on all ranks. Sections may differ by one element; they are padded to a
    common length for the collective and trimmed afterwards."""
    if not dist.is_available() or not dist.is_initialized():
        return local
    world = dist.get_world_size(group)
    parts = energy_partition(num_energies, world)
    longest = max(b - a for a, b in parts)
    pad = torch.zeros((longest,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    bufs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(bufs, pad, group=group)
    return torch.cat([bufs[r][: b - a] for r, (a, b) in enumerate(parts)], dim=0)


class ShardedEnergySweep:
    """Runs an energy grid on every rank's section and gathers observables.

    ``solve_batch(energies, f_left, f_right)`` must return an object with
    ``transmission`` (B,), ``current`` (B, N+1) and ``density`` (B, M)
    tensors (e.g. :meth:`quatrex_b200.EnergyPointSolver.solve`).
    """

    def __init__(self, solve_batch, batch_size: int, group=None):
        self.solve_batch = solve_batch
        self.batch_size = batch_size
        self.group = group

    def run(self, energies: np.ndarray, f_left: np.ndarray, f_right: np.ndarray) -> dict:
        world = dist.get_world_size(self.group) if dist.is_initialized() else 1
        rank = dist.get_rank(self.group) if dist.is_initialized() else 0
        a, b = energy_partition(energies.size, world)[rank]
        outs = {"transmission": [], "current": [], "density": []}
        for s in range(a, b, self.batch_size):
            e = slice(s, min(s + self.batch_size, b))
            r = self.solve_batch(energies[e], f_left[e], f_right[e])
            outs["transmission"].append(r.transmission.clone())
            outs["current"].append(r.current.clone())
            outs["density"].append(r.density.clone())
        return {k: gather_energies(torch.cat(v, 0), energies.size, self.group) for k, v in outs.items()}
