"""Serving loop for energy-point requests on one GPU: continuous batching,
HBM-budget admission and resident OBC warm starts.

A *request* asks for a set of energies of one device of a fixed catalogue
(the reference's unit of work per energy is ``ElectronSolver.solve``,
``src/quatrex/electron/solver.py:756-888``, with the ``OBCSystem`` memoizer
of ``qttools/boundary_conditions/obc/boundary_system.py:200-373`` keeping
surface Green's functions between calls). The server keeps one *lane* per
catalogue device resident on the GPU:

* a grid-bound :class:`~quatrex_b200.negf.EnergyPointSolver` (observables
  only) with two captured CUDA graphs of one batch size: *cold* (both-contact
  Sancho-Rubio) and *warm* (the lane's resident surface Green's functions of
  the requested grid points, then the OBCSystem fixed-point step);
* two streams (low and high priority) and pinned staging buffers for two
  batches in flight; a batch whose oldest request has at most the median
  remaining work of all active requests goes to the high-priority stream
  (shortest remaining work first across lanes), and a lane's batches stay
  ordered through an event chain;
* a queue of pending (request, energy) items, ordered by the requests'
  remaining work (shortest first). Whenever fewer than two batches are in
  flight the lane launches the next batch from the queue, items of
  different requests mixed (continuous batching): warm items (grid points
  already solved once) go together in a warm batch, the rest in a cold
  batch. One replay needs only the index vector as input.

Admission: at start-up every lane gets a batch size from
:func:`quatrex_b200.uneven.plan_batches` such that all lanes, their graphs,
workspaces and warm-start caches fit the HBM budget together; a catalogue
that does not fit at batch size 1 is refused.

Results of an energy do not depend on which other energies share its
batch: every kernel treats the batch entries independently, and the
Sancho-Rubio loop masks converged entries per energy.
"""

from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass

import numpy as np
import torch

from .negf import EnergyPointSolver
from .uneven import DeviceJob, plan_batches


@dataclass
class Request:
    """Energies ``grid_index`` (indices into the device's energy grid) of
    catalogue device ``device``; ``arrival`` in seconds from the start."""

    rid: int
    device: int
    grid_index: np.ndarray
    arrival: float = 0.0
    # filled by the server
    transmission: np.ndarray | None = None
    density: np.ndarray | None = None
    current: np.ndarray | None = None
    remaining: int = -1
    t_submit: float = float("nan")
    t_done: float = float("nan")
    warm_energies: int = 0

    @property
    def latency(self) -> float:
        return self.t_done - self.arrival


def poisson_requests(rate: float, duration: float, grid_sizes: list[int], energies: tuple[int, int] = (64, 512),
                     seed: int = 0) -> list[Request]:
    """Poisson arrivals at ``rate`` per second over ``duration`` seconds; each
    request picks a catalogue device uniformly and ``energies[0]`` to
    ``energies[1]`` distinct grid points of it (capped at the grid size),
    all from ``numpy.random.default_rng(seed)``."""
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        d = int(rng.integers(len(grid_sizes)))
        g = grid_sizes[d]
        n = int(rng.integers(min(energies[0], g), min(energies[1], g) + 1))
        idx = np.sort(rng.choice(g, size=n, replace=False))
        out.append(Request(len(out), d, idx, t))
    return out


def form_batch(pending: deque, cached: np.ndarray, B: int) -> tuple[list, bool]:
    """Next batch of a lane: up to B items from the FIFO ``pending`` (items
    are (request, position) pairs). If the oldest item's grid point is
    cached, the batch takes the oldest cached items (warm); otherwise the
    oldest uncached ones (cold). Taken items are removed from ``pending``."""
    if not pending:
        return [], False
    first = pending[0]
    warm = bool(cached[first[0].grid_index[first[1]]])
    take, keep = [], deque()
    while pending and len(take) < B:
        it = pending.popleft()
        if bool(cached[it[0].grid_index[it[1]]]) == warm:
            take.append(it)
        else:
            keep.append(it)
    keep.extend(pending)
    pending.clear()
    pending.extend(keep)
    return take, warm


def slowdown_stats(mixed: dict, alone: dict) -> dict:
    """Per-request latency in the mix divided by the same request's latency
    served alone on an idle server ({rid: seconds} each)."""
    r = np.array([mixed[k] / alone[k] for k in mixed if k in alone and alone[k] > 0])
    if r.size == 0:
        return {"count": 0}
    return {"count": int(r.size), "p50": float(np.percentile(r, 50)), "p99": float(np.percentile(r, 99)),
            "max": float(r.max())}


def order_pending(pending: deque) -> None:
    """Shortest remaining work first: reorders the (request, position) items
    by their request's remaining energies, in place. Stable, so each
    request's energies keep their order and equal requests keep FIFO order."""
    if len({r.rid for r, _ in pending}) > 1:
        ordered = sorted(pending, key=lambda it: it[0].remaining)
        pending.clear()
        pending.extend(ordered)


def latency_stats(latencies) -> dict:
    lat = np.asarray(latencies, dtype=np.float64)
    if lat.size == 0:
        return {"count": 0}
    return {"count": int(lat.size), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "max_s": float(lat.max())}


class _Lane:
    def __init__(self, k: int, job: DeviceJob, B: int, precision: str, device: torch.device, warm_start: bool):
        self.k, self.job, self.B = k, job, B
        self.solver = EnergyPointSolver(job.h_diag, job.coupling, eta=job.eta, sr_tol=1e-12, per_energy=True,
                                        device=device, precision=precision, device_loop=True, store_blocks=False)
        self.solver.bind_grid(job.energies, job.f_left, job.f_right)
        self.warm_start = warm_start
        if warm_start:
            self.solver.enable_obc_cache()
        self.stream = torch.cuda.Stream(device)
        # Two priorities for the shortest-remaining-work rule; a lane's
        # batches stay ordered through `last` whichever stream they use.
        lo, hi = torch.cuda.Stream.priority_range()
        self.streams = {False: torch.cuda.Stream(device, priority=lo), True: torch.cuda.Stream(device, priority=hi)}
        self.last = None
        self.urgent_batches = 0
        G = job.num_energies
        self.cached = np.zeros(G, dtype=bool)
        self.pending: deque = deque()
        self.inflight: deque = deque()
        N, b = job.num_blocks, job.block_size
        pin = dict(pin_memory=True)
        self.stage = [dict(idx=torch.zeros(B, dtype=torch.int64, **pin),
                           T=torch.zeros(B, dtype=torch.float64, **pin),
                           dens=torch.zeros((B, N * b), dtype=torch.float64, **pin),
                           cur=torch.zeros((B, N + 1), dtype=torch.complex128, **pin)) for _ in range(2)]
        self.free_slots = [0, 1]
        self.batches = {"cold": 0, "warm": 0}
        with torch.cuda.stream(self.stream):
            self.solver.set_indices(np.zeros(B, dtype=np.int64))
            # the warm graph first: its capture pass reads the (empty) cache
            # and writes slot 0, which the cold capture pass then recomputes
            self.graphs = {True: self.solver.capture(B, warm=True)} if warm_start else {}
            self.graphs[False] = self.solver.capture(B, warm=False)
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record()
            self.graphs[False].replay()
            t1.record()
        t1.synchronize()
        self.t_energy = t0.elapsed_time(t1) * 1e-3 / B  # seconds per energy of a full cold batch
        self.buf = self.solver._bufs[B]

    def launch(self, items: list, warm: bool, urgent: bool = False) -> None:
        slot = self.free_slots.pop()
        st = self.stage[slot]
        idx = np.array([r.grid_index[p] for r, p in items], dtype=np.int64)
        st["idx"][:idx.size] = torch.from_numpy(idx)
        st["idx"][idx.size:] = int(idx[-1])  # padding repeats the last energy
        stream = self.streams[urgent]
        with torch.cuda.stream(stream):
            if self.last is not None:
                stream.wait_event(self.last)
            self.buf["idx"].copy_(st["idx"], non_blocking=True)
            self.graphs[warm].replay()
            st["T"].copy_(self.buf["T"], non_blocking=True)
            st["dens"].copy_(self.buf["density"], non_blocking=True)
            st["cur"].copy_(self.buf["current"], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(stream)
        self.last = ev
        self.inflight.append((ev, slot, items, idx, warm))
        self.batches["warm" if warm else "cold"] += 1
        self.urgent_batches += int(urgent)

    def poll(self, now: float, done: list) -> None:
        while self.inflight and self.inflight[0][0].query():
            _, slot, items, idx, warm = self.inflight.popleft()
            st = self.stage[slot]
            for j, (r, p) in enumerate(items):
                r.transmission[p] = float(st["T"][j])
                r.density[p] = st["dens"][j].numpy()
                r.current[p] = st["cur"][j].numpy()
                r.warm_energies += int(warm)
                r.remaining -= 1
                if r.remaining == 0:
                    r.t_done = now
                    done.append(r)
            if self.warm_start:
                self.cached[idx] = True
            self.free_slots.append(slot)

    def remaining_cost(self, req: Request) -> float:
        return req.remaining * self.t_energy

    def try_launch(self, threshold: float = -1.0) -> bool:
        """Launches the next batch if a staging slot is free. The batch goes
        to the high-priority stream when its oldest request's remaining work
        is at most ``threshold`` seconds (shortest remaining work first
        across lanes)."""
        if not self.free_slots or not self.pending:
            return False
        order_pending(self.pending)
        head = self.pending[0][0]
        urgent = self.remaining_cost(head) <= threshold
        items, warm = form_batch(self.pending, self.cached, self.B)  # cached stays False without warm starts
        self.launch(items, warm, urgent)
        return True


class EnergyServer:
    """Serves energy-point requests for a catalogue of devices on one GPU.

    Parameters
    ----------
    catalogue : list of DeviceJob — each device with its energy grid.
    precision : "fp64" or "mixed".
    budget_bytes : HBM for all lanes together (solvers, graphs, caches).
    warm_start : keep each lane's surface Green's functions resident and
        serve already-solved grid points with the warm graph.
    batches : optional batch size per lane (default: planned).
    """

    def __init__(self, catalogue: list[DeviceJob], precision: str = "fp64", budget_bytes: float = 150e9,
                 warm_start: bool = True, batches: list[int] | None = None, device: torch.device | None = None):
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.catalogue = list(catalogue)
        num_sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        cache = sum(2 * j.num_energies * j.block_size ** 2 * 16 for j in self.catalogue) if warm_start else 0
        if batches is None:
            batches = plan_batches(self.catalogue, budget_bytes - cache, precision, num_sms)
        self.lanes = [_Lane(k, j, B, precision, self.device, warm_start)
                      for k, (j, B) in enumerate(zip(self.catalogue, batches))]
        torch.cuda.synchronize(self.device)
        self.done: list[Request] = []
        self.active: dict = {}  # rid -> request, submitted and not finished

    def submit(self, req: Request, now: float) -> None:
        lane = self.lanes[req.device]
        n = len(req.grid_index)
        N, b = lane.job.num_blocks, lane.job.block_size
        req.transmission = np.zeros(n)
        req.density = np.zeros((n, N * b))
        req.current = np.zeros((n, N + 1), dtype=np.complex128)
        req.remaining = n
        req.t_submit = now
        self.active[req.rid] = req
        lane.pending.extend((req, p) for p in range(n))

    def pump(self, now: float) -> bool:
        """Collects finished batches and launches new ones; True if anything
        happened."""
        busy = False
        for lane in self.lanes:
            before = len(self.done)
            lane.poll(now, self.done)
            for r in self.done[before:]:
                self.active.pop(r.rid, None)
            busy |= len(self.done) != before
        # Requests whose remaining work is at or below the median of the
        # active ones run on the high-priority streams.
        costs = [self.lanes[r.device].remaining_cost(r) for r in self.active.values()]
        threshold = float(np.median(costs)) if len(costs) > 1 else -1.0
        for lane in self.lanes:
            while lane.try_launch(threshold):
                busy = True
        return busy

    def idle(self) -> bool:
        return all(not ln.pending and not ln.inflight for ln in self.lanes)

    def run(self, requests: list[Request], time_scale: float = 1.0) -> dict:
        """Replays ``requests`` in real time (arrival times multiplied by
        ``time_scale``) until every request is done; returns statistics.
        Latency = completion - arrival, on the host clock."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        for r in reqs:
            r.arrival *= time_scale
        t0 = time.perf_counter()
        nxt = 0
        while nxt < len(reqs) or not self.idle():
            now = time.perf_counter() - t0
            while nxt < len(reqs) and reqs[nxt].arrival <= now:
                self.submit(reqs[nxt], now)
                nxt += 1
            if not self.pump(time.perf_counter() - t0):
                time.sleep(2e-4)
        wall = time.perf_counter() - t0
        energies = sum(len(r.grid_index) for r in reqs)
        warm = sum(r.warm_energies for r in reqs)
        return {"requests": len(reqs), "energies": energies, "wall_s": wall, "energies_per_s": energies / wall,
                "warm_fraction": warm / max(energies, 1), "latency": latency_stats([r.latency for r in reqs]),
                "lanes": [{"device": ln.k, "N": ln.job.num_blocks, "b": ln.job.block_size, "batch": ln.B,
                           "urgent": ln.urgent_batches, **ln.batches} for ln in self.lanes]}

    def solve_now(self, req: Request) -> Request:
        """Serves one request alone (submit, drain) — the reference point of
        the alone-versus-mixed check."""
        t0 = time.perf_counter()
        req.arrival = 0.0
        self.submit(req, 0.0)
        while not self.idle():
            if not self.pump(time.perf_counter() - t0):
                time.sleep(2e-4)
        return req
