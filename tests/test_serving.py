"""Host logic of the serving loop: seeded Poisson workload, batch
formation (continuous batching with warm/cold separation), latency
statistics."""

from collections import deque

import numpy as np

from quatrex_b200.serving import Request, form_batch, latency_stats, order_pending, poisson_requests, slowdown_stats


def test_poisson_workload_is_seeded_and_bounded():
    a = poisson_requests(50.0, 20.0, [100, 300, 40], (64, 512), seed=4)
    b = poisson_requests(50.0, 20.0, [100, 300, 40], (64, 512), seed=4)
    assert [(r.device, r.arrival, r.grid_index.tolist()) for r in a] == \
           [(r.device, r.arrival, r.grid_index.tolist()) for r in b]
    assert abs(len(a) - 1000) < 5 * np.sqrt(1000)  # Poisson count, 5 sigma
    arr = np.array([r.arrival for r in a])
    assert (np.diff(arr) > 0).all() and arr.max() <= 20.0
    for r in a:
        g = [100, 300, 40][r.device]
        idx = r.grid_index
        assert len(np.unique(idx)) == len(idx) and idx.min() >= 0 and idx.max() < g
        assert min(64, g) <= len(idx) <= min(512, g)
    assert {r.device for r in a} == {0, 1, 2}


def _items(req_idx_pairs):
    return deque((r, p) for r, p in req_idx_pairs)


def test_form_batch_mixes_requests_and_separates_warm_items():
    r1 = Request(0, 0, np.array([0, 1, 2, 3]))
    r2 = Request(1, 0, np.array([2, 5, 6]))
    cached = np.zeros(10, dtype=bool)
    pending = _items([(r1, p) for p in range(4)] + [(r2, p) for p in range(3)])
    take, warm = form_batch(pending, cached, 6)
    assert not warm and [(r.rid, p) for r, p in take] == [(0, 0), (0, 1), (0, 2), (0, 3), (1, 0), (1, 1)]
    assert [(r.rid, p) for r, p in pending] == [(1, 2)]
    # grid points 2 and 5 solved before: the head item decides, warm items go together
    cached[[2, 5]] = True
    pending = _items([(r2, 0), (r1, 0), (r2, 1), (r2, 2)])
    take, warm = form_batch(pending, cached, 4)
    assert warm and [(r.rid, p) for r, p in take] == [(1, 0), (1, 1)]
    assert [(r.rid, p) for r, p in pending] == [(0, 0), (1, 2)]  # order kept
    take, warm = form_batch(pending, cached, 4)
    assert not warm and len(take) == 2 and not pending
    assert form_batch(deque(), cached, 4) == ([], False)


def test_latency_stats():
    s = latency_stats(np.arange(1, 101, dtype=float))
    assert s["count"] == 100 and abs(s["p50_s"] - 50.5) < 1e-12 and abs(s["p99_s"] - 99.01) < 1e-9
    assert latency_stats([]) == {"count": 0}


def test_order_pending_shortest_remaining_first():
    big = Request(0, 0, np.arange(6))
    small = Request(1, 0, np.arange(2))
    mid = Request(2, 0, np.arange(4))
    big.remaining, small.remaining, mid.remaining = 6, 2, 4
    pending = deque([(big, p) for p in range(6)] + [(mid, p) for p in range(4)] + [(small, p) for p in range(2)])
    order_pending(pending)
    assert [(r.rid, p) for r, p in pending][:6] == [(1, 0), (1, 1), (2, 0), (2, 1), (2, 2), (2, 3)]
    assert [r.rid for r, _ in pending][6:] == [0] * 6
    single = deque([(big, 3), (big, 1)])
    order_pending(single)  # one request: order untouched
    assert [p for _, p in single] == [3, 1]


def test_slowdown_stats():
    s = slowdown_stats({1: 2.0, 2: 3.0, 3: 1.0}, {1: 1.0, 2: 1.0, 3: 2.0})
    assert s["count"] == 3 and s["max"] == 3.0 and abs(s["p50"] - 2.0) < 1e-12
    assert slowdown_stats({}, {}) == {"count": 0}
