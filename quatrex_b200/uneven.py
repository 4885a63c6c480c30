"""Uneven batches of devices on one GPU: HBM-budget admission, batch-size
autotuning and concurrent CUDA-graph replay.

The reference solves one device at a time: ``ElectronSolver.solve``
(``src/quatrex/electron/solver.py:756-888``) loops over its local energies in
batches of ``max_batch_size`` (``qttools/utils/solvers_utils.py:7-32``), and
every batch goes through the same RGF / OBC sequence. Here a set of devices
with different block counts N and block sizes b shares the GPU:

* :func:`plan_batches` gives every device a batch size under one HBM budget
  (water-filling on the estimated device time, with the per-energy
  footprint from :func:`quatrex_b200.negf.resident_bytes`);
* :class:`BatchTuner` times candidate batch sizes of one shape (one captured
  graph replay each) and caches the winner per (GPU, N, b, precision) behind
  a lock;
* :class:`UnevenBatchRunner` captures one CUDA graph per device (the whole
  energy-point pipeline, Sancho-Rubio with device-side convergence) and
  replays the batches of all devices on one stream per device, so small
  devices fill the SMs that large ones leave idle. Inside ``enqueue`` the
  host only enqueues: energies are staged on the device once, every replay
  reads its slice and its observables are copied to per-device result arrays
  on the same stream.
"""

from __future__ import annotations

import json
import math
import threading
from dataclasses import dataclass, field
from pathlib import Path
from typing import Callable

import numpy as np
import torch

from . import _native
from .negf import EnergyPointSolver, flops_per_energy, resident_bytes


@dataclass
class DeviceJob:
    """One device of the batch: Hamiltonian blocks, lead coupling and the
    energies (with lead occupations) to solve."""

    name: str
    h_diag: np.ndarray  # (N, b, b)
    coupling: np.ndarray  # (b, b), block (i, i+1) of H
    energies: np.ndarray
    f_left: np.ndarray
    f_right: np.ndarray
    eta: float = 1e-4

    @property
    def num_blocks(self) -> int:
        return int(self.h_diag.shape[0])

    @property
    def block_size(self) -> int:
        return int(self.h_diag.shape[-1])

    @property
    def num_energies(self) -> int:
        return int(np.asarray(self.energies).size)

    def flops(self, sr_iterations: float = 20.0) -> float:
        """Algorithmic flops of all its energy points."""
        f = flops_per_energy(self.num_blocks, self.block_size, (sr_iterations, sr_iterations))
        return f["total"] * self.num_energies


def jobs_from_devices(devices) -> list[DeviceJob]:
    """DeviceJobs from :class:`quatrex_b200.synthetic.Device` objects."""
    out = []
    for k, d in enumerate(devices):
        out.append(DeviceJob(f"dev{k}-N{d.num_blocks}-b{d.block_size}", np.asarray(d.h_diag),
                             np.asarray(d.coupling), np.asarray(d.energies), d.fermi_left(), d.fermi_right(),
                             d.eta))
    return out


# ---------------------------------------------------------------------------
# Planning


def batch_ladder(num_sms: int, max_batch: int) -> list[int]:
    """Candidate batch sizes: fractions and multiples of the SM count (one
    CTA per matrix in the small-block inversions), plus small powers of two."""
    c = {1, 2, 4, 8, 16, 32, 64}
    for f in (0.25, 0.5, 1, 2, 3, 4):
        c.add(max(1, int(round(num_sms * f))))
    return sorted(x for x in c if x <= max_batch)


def plan_batches(jobs: list[DeviceJob], budget_bytes: float, precision: str = "fp64", num_sms: int = 148,
                 bytes_fn: Callable | None = None, lib=None, store_blocks: bool = False) -> list[int]:
    """Batch size per job such that all jobs are resident at once within
    ``budget_bytes``.

    Every job starts at batch 1; then the job with the largest estimated
    device time moves up one rung of :func:`batch_ladder` while the total
    stays within the budget. The time model is work / (B-dependent
    occupancy): a batch of B matrices occupies min(1, B / num_sms) of the
    GPU. Raises ValueError when even batch 1 of every job does not fit.
    """
    if bytes_fn is None:
        lib = lib or _native.load()

        def bytes_fn(job, B):
            return resident_bytes(job.num_blocks, job.block_size, B, precision, lib, store_blocks)

    ladders = []
    for j in jobs:
        n = max(1, j.num_energies)
        lad = set(batch_ladder(num_sms, n))
        if n <= 4 * num_sms:
            lad.add(n)  # the whole job in one batch
        ladders.append(sorted(lad) or [1])
    rung = [0] * len(jobs)
    size = [bytes_fn(j, ladders[k][0]) for k, j in enumerate(jobs)]
    if sum(size) > budget_bytes:
        raise ValueError(f"the uneven batch does not fit the HBM budget even at batch size 1 "
                         f"({sum(size) / 1e9:.1f} GB > {budget_bytes / 1e9:.1f} GB)")

    def est(k):
        B = ladders[k][rung[k]]
        return jobs[k].flops() / min(1.0, B / num_sms)

    frozen = [False] * len(jobs)
    while not all(frozen):
        k = max((i for i in range(len(jobs)) if not frozen[i]), key=est)
        if rung[k] + 1 >= len(ladders[k]):
            frozen[k] = True
            continue
        nb = bytes_fn(jobs[k], ladders[k][rung[k] + 1])
        if sum(size) - size[k] + nb > budget_bytes:
            frozen[k] = True
            continue
        rung[k] += 1
        size[k] = nb
    return [ladders[k][rung[k]] for k in range(len(jobs))]


class BatchTuner:
    """Measured batch-size choice per shape, cached process-wide (and in an
    optional JSON file) under a lock.

    ``measure(B)`` returns seconds per batch of B energies; the tuner keeps
    the candidate with the most energies per second, skipping candidates
    that do not fit ``budget_bytes`` according to ``bytes_fn(B)``.
    """

    _lock = threading.Lock()
    _cache: dict = {}

    def __init__(self, cache_file: str | Path | None = None):
        self.cache_file = Path(cache_file) if cache_file else None
        if self.cache_file and self.cache_file.exists():
            with self._lock:
                for k, v in json.loads(self.cache_file.read_text()).items():
                    self._cache.setdefault(k, v)

    @staticmethod
    def key(gpu: str, N: int, b: int, precision: str) -> str:
        return f"{gpu}|N{N}|b{b}|{precision}"

    def lookup(self, key: str):
        with self._lock:
            return self._cache.get(key)

    def tune(self, key: str, candidates: list[int], measure: Callable[[int], float],
             bytes_fn: Callable[[int], float] | None = None, budget_bytes: float = math.inf) -> dict:
        hit = self.lookup(key)
        if hit is not None:
            return hit
        trials = {}
        for B in candidates:
            if bytes_fn is not None and bytes_fn(B) > budget_bytes:
                continue
            sec = float(measure(B))
            trials[B] = B / sec if sec > 0 else 0.0
        if not trials:
            raise ValueError(f"no batch size of {candidates} fits {budget_bytes / 1e9:.1f} GB for {key}")
        best = max(trials, key=trials.get)
        res = {"batch": int(best), "energies_per_s": trials[best], "trials": {str(k): v for k, v in trials.items()}}
        with self._lock:
            self._cache[key] = res
            if self.cache_file:
                self.cache_file.parent.mkdir(parents=True, exist_ok=True)
                self.cache_file.write_text(json.dumps(self._cache, indent=1, sort_keys=True))
        return res


# ---------------------------------------------------------------------------
# Execution


@dataclass
class JobState:
    job: DeviceJob
    batch: int
    solver: EnergyPointSolver
    stream: torch.cuda.Stream
    energies: torch.Tensor
    f_left: torch.Tensor
    f_right: torch.Tensor
    transmission: torch.Tensor
    density: torch.Tensor
    current: torch.Tensor
    graph: object = None
    batches: list = field(default_factory=list)


class UnevenBatchRunner:
    """Solves every energy point of several devices on one GPU.

    Parameters
    ----------
    jobs : list of DeviceJob
    precision : "fp64" or "mixed" (see EnergyPointSolver)
    budget_bytes : HBM the resident solvers may hold together.
    batches : optional batch size per job (default: :func:`plan_batches`).
    """

    def __init__(self, jobs: list[DeviceJob], precision: str = "fp64", budget_bytes: float = 150e9,
                 batches: list[int] | None = None, device: torch.device | None = None, sr_tol: float = 1e-12,
                 sr_max_iterations: int = 100, autotune: bool = False, tuner: BatchTuner | None = None,
                 max_trials: int = 3):
        self.jobs = list(jobs)
        self.precision = precision
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.budget = float(budget_bytes)
        num_sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        self.batches = list(batches) if batches is not None else plan_batches(self.jobs, self.budget, precision,
                                                                              num_sms)
        if len(self.batches) != len(self.jobs):
            raise ValueError("one batch size per job is required")
        self.sr_tol = sr_tol
        self.sr_max_iterations = sr_max_iterations
        self.states: list[JobState] = []
        self.autotune = autotune
        self.tuner = tuner or BatchTuner()
        self.max_trials = max_trials
        self.num_sms = num_sms
        self.tuning: dict = {}

    def _measure(self, job: DeviceJob, B: int) -> float:
        """Seconds of one captured-graph replay of B energies of ``job``."""
        dev = self.device
        s = EnergyPointSolver(job.h_diag, job.coupling, eta=job.eta, sr_tol=self.sr_tol,
                              sr_max_iterations=self.sr_max_iterations, per_energy=True, device=dev,
                              precision=self.precision, device_loop=True, store_blocks=False)
        idx = np.arange(B) % job.num_energies
        E = torch.as_tensor(np.asarray(job.energies, dtype=np.float64)[idx], device=dev)
        fl = torch.as_tensor(np.asarray(job.f_left, dtype=np.float64)[idx], device=dev)
        fr = torch.as_tensor(np.asarray(job.f_right, dtype=np.float64)[idx], device=dev)
        s.set_inputs_device(E, fl, fr)
        g = s.capture(B)  # runs the pipeline once eagerly, then captures
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record()
        g.replay()
        t1.record()
        torch.cuda.synchronize(dev)
        sec = t0.elapsed_time(t1) * 1e-3
        del g, s
        torch.cuda.empty_cache()
        return sec

    def tune(self) -> None:
        """Measured batch sizes: per (N, b) the largest ``max_trials`` rungs
        of the ladder up to the planned (budget-feasible) batch are timed and
        the one with the most energies per second is kept (cached per GPU
        and shape in the BatchTuner)."""
        gpu = torch.cuda.get_device_name(self.device)
        for k, job in enumerate(self.jobs):
            plan = self.batches[k]
            cands = [c for c in batch_ladder(self.num_sms, plan)]
            if plan not in cands:
                cands.append(plan)
            cands = sorted(set(cands))[-self.max_trials:]
            key = BatchTuner.key(gpu, job.num_blocks, job.block_size, self.precision)
            res = self.tuner.tune(key, cands, lambda B, j=job: self._measure(j, B))
            self.tuning[job.name] = res
            self.batches[k] = min(int(res["batch"]), plan)

    def prepare(self) -> None:
        """Allocates every solver and captures its graph (runs each pipeline
        once eagerly), after tuning the batch sizes if asked. Nothing here
        belongs in a timed region."""
        if self.autotune and not self.tuning:
            self.tune()
        dev = self.device
        for job, B in zip(self.jobs, self.batches):
            solver = EnergyPointSolver(job.h_diag, job.coupling, eta=job.eta, sr_tol=self.sr_tol,
                                       sr_max_iterations=self.sr_max_iterations, per_energy=True, device=dev,
                                       precision=self.precision, device_loop=True, store_blocks=False)
            n = job.num_energies
            nb = max(1, -(-n // B))
            pad = nb * B - n  # the last batch repeats the last energy; its extra results are dropped
            E = np.concatenate([np.asarray(job.energies, dtype=np.float64), np.repeat(job.energies[-1:], pad)])
            fl = np.concatenate([np.asarray(job.f_left, dtype=np.float64), np.repeat(job.f_left[-1:], pad)])
            fr = np.concatenate([np.asarray(job.f_right, dtype=np.float64), np.repeat(job.f_right[-1:], pad)])
            st = JobState(job, B, solver, torch.cuda.Stream(dev),
                          torch.as_tensor(E, device=dev), torch.as_tensor(fl, device=dev),
                          torch.as_tensor(fr, device=dev),
                          torch.zeros(n, dtype=torch.float64, device=dev),
                          torch.zeros((n, job.num_blocks * job.block_size), dtype=torch.float64, device=dev),
                          torch.zeros((n, job.num_blocks + 1), dtype=torch.complex128, device=dev))
            st.batches = [(k * B, min(n, (k + 1) * B)) for k in range(nb)]
            with torch.cuda.stream(st.stream):
                solver.set_inputs_device(st.energies[:B], st.f_left[:B], st.f_right[:B])
                st.graph = solver.capture(B)
            self.states.append(st)
        torch.cuda.synchronize(dev)

    def enqueue(self, nested: bool = True) -> None:
        """Enqueues every batch of every job, round-robin over the jobs, each
        job on its own stream. Returns without synchronising. ``nested=False``
        issues the pipelines' kernels instead of replaying the per-device
        graphs (used while capturing the whole schedule)."""
        cur = torch.cuda.current_stream(self.device)
        for st in self.states:
            st.stream.wait_stream(cur)
        rounds = max(len(st.batches) for st in self.states)
        for r in range(rounds):
            for st in self.states:
                if r >= len(st.batches):
                    continue
                lo, hi = st.batches[r]
                B = st.batch
                with torch.cuda.stream(st.stream):
                    st.solver.set_inputs_device(st.energies[lo:lo + B], st.f_left[lo:lo + B],
                                                st.f_right[lo:lo + B])
                    if nested:
                        st.graph.replay()
                    else:
                        st.solver._run(B, device_loop=True)
                    res = st.solver._result(B)
                    n = hi - lo
                    st.transmission[lo:hi].copy_(res.transmission[:n], non_blocking=True)
                    st.density[lo:hi].copy_(res.density[:n], non_blocking=True)
                    st.current[lo:hi].copy_(res.current[:n], non_blocking=True)
        for st in self.states:
            cur.wait_stream(st.stream)

    def capture_all(self) -> "torch.cuda.CUDAGraph":
        """The whole schedule of ``enqueue`` — every batch of every device on
        its own stream, with the input and output copies — captured as one
        CUDA graph, so that one launch solves the uneven batch. The
        pipelines' kernels are captured directly (a graph launch inside a
        capture is not accepted by the runtime here), in the same order as
        the per-device replays."""
        if not self.states:
            self.prepare()
        dev = self.device
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        torch.cuda.synchronize(dev)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side):
            self.enqueue(nested=False)
        self.all_graph = g
        return g

    def run(self) -> dict:
        """prepare() if needed, enqueue(), synchronise; returns per-job
        device results {name: {"transmission", "density", "current"}}."""
        if not self.states:
            self.prepare()
        self.enqueue()
        torch.cuda.synchronize(self.device)
        return self.results()

    def results(self) -> dict:
        return {st.job.name: {"transmission": st.transmission, "density": st.density, "current": st.current}
                for st in self.states}

    def sr_converged(self) -> dict:
        """Per job: did the last replay's Sancho-Rubio loop converge."""
        return {st.job.name: st.solver.sr_status(st.batch)[1] for st in self.states}

    def summary(self) -> list[dict]:
        return [{"name": st.job.name, "N": st.job.num_blocks, "b": st.job.block_size,
                 "energies": st.job.num_energies, "batch": st.batch, "replays": len(st.batches),
                 "resident_gb": st.solver.resident_bytes(st.batch) / 1e9} for st in self.states]
