"""Host logic of the uneven device batch: batch ladder, HBM-budget
planning, the autotuner cache and the per-energy footprint model."""

import threading

import numpy as np
import pytest

from quatrex_b200 import synthetic
from quatrex_b200.negf import resident_bytes
from quatrex_b200.uneven import BatchTuner, DeviceJob, batch_ladder, jobs_from_devices, plan_batches


def _job(N, b, n, name="j"):
    return DeviceJob(name, np.zeros((N, b, b), complex), np.zeros((b, b), complex), np.linspace(-1, 1, n),
                     np.zeros(n), np.zeros(n))


def test_batch_ladder_sm_multiples():
    lad = batch_ladder(148, 1000)
    assert lad == sorted(set(lad))
    for x in (37, 74, 148, 296, 444, 592):
        assert x in lad
    assert max(batch_ladder(148, 20)) <= 20


def test_plan_respects_budget_and_prefers_big_jobs():
    jobs = [_job(64, 768, 256, "big"), _job(8, 128, 256, "small"), _job(16, 384, 64, "mid")]
    per = lambda j, B: B * j.num_blocks * j.block_size ** 2 * 16 * 6.0  # noqa: E731
    budget = 60e9
    B = plan_batches(jobs, budget, bytes_fn=per)
    assert sum(per(j, b) for j, b in zip(jobs, B)) <= budget
    assert B[0] >= B[2] and all(b >= 1 for b in B)
    # a budget that does not even hold batch 1 of each job is refused
    with pytest.raises(ValueError):
        plan_batches(jobs, 1e6, bytes_fn=per)


def test_plan_caps_at_job_size():
    B = plan_batches([_job(4, 32, 5)], 1e12, bytes_fn=lambda j, b: b)
    assert B == [5]


def test_resident_bytes_model():
    # linear in the batch apart from constant terms; observables-only mode
    # drops exactly the output block stacks
    a1, a2, a4 = (resident_bytes(16, 128, B) for B in (1, 2, 4))
    assert a4 - a2 == pytest.approx(2 * (a2 - a1), rel=0.05)
    full, obs = resident_bytes(16, 128, 8), resident_bytes(16, 128, 8, store_blocks=False)
    assert full - obs == (3 * 16 + 4 * 15) * 8 * 128 * 128 * 16
    assert resident_bytes(16, 128, 8, "mixed") < full


def test_tuner_picks_fastest_and_caches(tmp_path):
    calls = []

    def measure(B):
        calls.append(B)
        return 1.0 + 0.02 * B if B <= 32 else 10.0  # best throughput at B = 32

    path = tmp_path / "tune.json"
    key = BatchTuner.key("test-gpu-a", 8, 64, "fp64")
    res = BatchTuner(path).tune(key, [8, 16, 32, 64], measure, bytes_fn=lambda B: B, budget_bytes=40)
    assert res["batch"] == 32 and calls == [8, 16, 32]  # 64 exceeds the budget
    again = BatchTuner(path).tune(key, [8], lambda B: 1 / 0)  # served from the cache
    assert again["batch"] == 32
    assert key in path.read_text()


def test_tuner_is_thread_safe():
    t = BatchTuner()
    out = []

    def work(k):
        out.append(t.tune(BatchTuner.key("test-gpu-b", k % 3, 1, "fp64"), [1, 2], lambda B: 1.0)["batch"])

    th = [threading.Thread(target=work, args=(k,)) for k in range(12)]
    for x in th:
        x.start()
    for x in th:
        x.join()
    assert out == [2] * 12


def test_uneven_shapes_and_jobs():
    shapes = synthetic.uneven_devices()
    assert len(shapes) == 8
    assert all(n in (8, 16, 32, 64) and b in (128, 256, 384, 512, 768) for n, b in shapes)
    devs = [synthetic.make_device(n, 8, np.linspace(-1, 1, 3), seed=k) for k, (n, _) in enumerate(shapes[:2])]
    jobs = jobs_from_devices(devs)
    assert jobs[0].num_blocks == shapes[0][0] and jobs[0].block_size == 8 and jobs[0].num_energies == 3
    assert jobs[0].flops() > 0
