"""Host logic of the serving loop (no GPU): the seeded request mix and the
latency / throughput summary."""
import math

import numpy as np

from lbflow_b200 import serve
from lbflow_b200.core import Storage


def test_request_mix_is_seeded_and_in_range():
    a = serve.make_requests(2000, rate=40.0, seed=7)
    b = serve.make_requests(2000, rate=40.0, seed=7)
    assert [(r.kind, r.side, r.porosity, r.storage, r.arrival) for r in a] == \
           [(r.kind, r.side, r.porosity, r.storage, r.arrival) for r in b]
    cav = [r for r in a if r.kind == "cavity"]
    ch = [r for r in a if r.kind == "channel"]
    assert 0.45 < len(cav) / len(a) < 0.55
    assert all(64 <= r.side <= 1024 for r in cav) and all(32 <= r.side <= 160 for r in ch)
    assert all(0.5 <= r.porosity <= 0.9 for r in ch)
    # log-uniform sides: log(side) has the mean of the uniform on [log lo, log hi]
    assert abs(np.mean([math.log(r.side) for r in cav]) - 0.5 * math.log(64 * 1024)) < 0.1
    assert 0.45 < np.mean([r.storage == Storage.F16DEV for r in a]) < 0.55
    gaps = np.diff([r.arrival for r in a])
    assert a[0].arrival == 0.0 and np.all(gaps >= 0)
    assert abs(gaps.mean() - 1 / 40.0) < 0.1 / 40.0     # Poisson arrivals at 40 per second


def test_all_at_once_and_summary():
    reqs = serve.make_requests(10, rate=float("inf"), seed=1)
    assert all(r.arrival == 0.0 for r in reqs)
    recs = [serve.Record(i, "cavity", 100, 0.0, 0.0, 0.1 * (i + 1), 50, 2) for i in range(10)]
    s = serve.summary(recs)
    assert s["solves"] == 10 and abs(s["seconds"] - 1.0) < 1e-12
    assert abs(s["solves_per_s"] - 10.0) < 1e-9
    assert abs(s["p50_s"] - 0.55) < 1e-9 and s["p99_s"] <= 1.0
    assert abs(s["mlups_all_nodes"] - 10 * 100 * 50 / 1e6) < 1e-12


def test_lanes_and_smallest_first():
    reqs = serve.make_requests(200, rate=float("inf"), seed=3)
    big = [r for r in reqs if serve.request_nodes(r) >= 1 << 19]
    assert big and all(serve.lane_of(r, 1 << 19) == 1 for r in big)
    assert all(serve.lane_of(r, 1 << 19) == 0 for r in reqs if r not in big)
    arr = serve._Arrivals(reqs)
    arr.arrive(0.0)
    order = [serve.request_nodes(arr.pop()) for _ in range(len(reqs))]
    assert order == sorted(order)                      # smallest work first
    assert arr.empty()
    timed = serve.make_requests(50, rate=10.0, seed=4)
    arr = serve._Arrivals(timed)
    arr.arrive(timed[10].arrival)
    assert len(arr.heap) == 11 and arr.next_arrival() == timed[11].arrival
