"""A serving loop over `Batch`: solve requests arrive, are admitted while the
device-memory budget allows, advance together, and leave with their fields.

Requests (the serving mix): Poisson arrivals at rate `rate` per second; half
(`cavity_frac`) are D2Q9 BGK lid-driven cavities with side log-uniform in
[64, 1024], the others D3Q19 TRT porous channels with side log-uniform in
[32, 160] and porosity uniform in [0.5, 0.9]; storage FP32 or FP16 deviation
(half each); every request stops after `max_steps` steps or when its velocity
residual drops below `tol_velocity` (checked every `residual_interval` steps,
with the rule of `Domain.run`).  Everything is generated from one seed.

`serve_batched` runs the requests through one `Batch`; `serve_lanes` through two
batches that advance independently (small requests on a high-priority stream,
smallest first); `serve_sequential` runs them one at a time with `Domain.run` in
arrival order (the same stop rule, so the same fields and step counts).  Both record per request the arrival, start and
finish times (finish = after the density and velocity fields reached the host).
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import cases
from .batch import Batch, BatchFull, estimate_bytes
from .core import Storage
from .domain import Domain


@dataclass
class Request:
    rid: int
    kind: str            # "cavity" (D2Q9) or "channel" (D3Q19)
    side: int
    porosity: float
    storage: Storage
    arrival: float       # seconds after the start of the run
    seed: int
    params: object = None
    est_bytes: int = 0


@dataclass
class Record:
    rid: int
    kind: str
    nodes: int
    arrival: float
    start: float
    finish: float
    steps: int
    status: int

    @property
    def latency(self) -> float:
        return self.finish - self.arrival


def make_requests(n: int = 4000, rate: float = 50.0, seed: int = 1234, cavity_frac: float = 0.5,
                  fp16_frac: float = 0.5, cavity_sides=(64, 1024), channel_sides=(32, 160),
                  porosity=(0.5, 0.9)) -> List[Request]:
    """The seeded serving mix; rate = inf puts every arrival at t = 0."""
    rng = np.random.default_rng(seed)
    gaps = np.zeros(n) if math.isinf(rate) else rng.exponential(1.0 / rate, n)
    arrivals = np.cumsum(gaps) - (gaps[0] if n else 0.0)
    reqs = []
    for i in range(n):
        cav = rng.random() < cavity_frac
        lo, hi = cavity_sides if cav else channel_sides
        side = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        por = float(rng.uniform(*porosity))
        st = Storage.F16DEV if rng.random() < fp16_frac else Storage.F32
        reqs.append(Request(i, "cavity" if cav else "channel", side, por, st, float(arrivals[i]),
                            int(rng.integers(0, 2**31 - 1))))
    return reqs


def build_params(r: Request):
    """momentum.Parameters of a request (geometry generated from its seed)."""
    if r.kind == "cavity":
        return cases.cavity_d2q9(r.side, 0.6, 0.1, r.storage)
    n = [r.side] * 3
    mask = cases.sphere_pack(n, r.porosity, 2.0, max(2.5, r.side / 16), r.seed, overlap=True)
    return cases.porous_channel_d3q19(n, mask=mask, force=1e-5, storage=r.storage)


def prepare(reqs: List[Request]) -> None:
    """Build every request's parameters and device-byte estimate (client side, untimed)."""
    for r in reqs:
        r.params = build_params(r)
        r.est_bytes = estimate_bytes(r.params)


def _now(t0):
    return time.perf_counter() - t0


def serve_batched(reqs: List[Request], max_steps: int = 2000, tol_velocity: float = 1e-6,
                  residual_interval: int = 50, budget_bytes: int = 0, chunks_per_poll: int = 1,
                  create_ms: float = 20.0) -> List[Record]:
    """Run the requests through one Batch; returns one Record per request.

    The batch runs on its own CUDA stream.  While a chunk runs, the host builds
    and initialises the domains of arrived requests on a second stream (for at
    most `create_ms` per chunk); they join the batch at the next chunk.
    Admission is by device-memory budget: a request waits until its byte
    estimate fits.
    """
    import threading
    from concurrent.futures import ThreadPoolExecutor

    import torch
    max_it = max_steps - 2     # the rule stops after step t > max_iterations: max_steps steps in all
    pending = sorted(reqs, key=lambda r: r.arrival)
    records: List[Record] = []
    live = {}
    ready = []                 # (request, initialised domain) waiting for admission
    s_batch, s_init = torch.cuda.Stream(), torch.cuda.Stream()
    # finished domains hand their fields to the host on worker threads, each with
    # its own stream, so that the copies of several results overlap each other
    # and the batch's next chunk
    lock = threading.Lock()
    local = threading.local()

    def collect(r, dom, start, status, t0):
        if not hasattr(local, "stream"):
            local.stream = torch.cuda.Stream()
        dom.moments(local.stream)
        rec = Record(r.rid, r.kind, int(np.prod(r.params.n[: r.params.dim])), r.arrival, start, _now(t0),
                     dom.time_step, status)
        dom.close()
        with lock:
            records.append(rec)
    host = {"create_s": 0.0, "step_enqueue_s": 0.0, "poll_wait_s": 0.0, "moments_tail_s": 0.0, "chunks": 0}
    pool = ThreadPoolExecutor(max_workers=4)
    futures = []
    with Batch(budget_bytes, residual_interval) as batch:
        budget = batch.info()["budget"]
        used = 0
        t0 = time.perf_counter()
        i = 0

        def create(limit_s):
            nonlocal i, used
            t_start = time.perf_counter()
            t_end = t_start + limit_s
            while i < len(pending) and pending[i].arrival <= _now(t0) and used + pending[i].est_bytes <= budget:
                r = pending[i]
                dom = Domain(r.params)
                dom.init(s_init)
                ready.append((r, dom))
                used += r.est_bytes
                i += 1
                if time.perf_counter() > t_end:
                    break
            s_init.synchronize()
            host["create_s"] += time.perf_counter() - t_start

        while i < len(pending) or live or ready:
            if not live and not ready:
                create(create_ms / 1e3)
                if not ready:
                    if i < len(pending):
                        time.sleep(max(0.0, min(pending[i].arrival - _now(t0), 0.01)))
                    continue
            for r, dom in ready:
                batch.admit(dom, max_it, tol_density=math.inf, tol_velocity=tol_velocity, tol_scalar=math.inf)
                live[dom.h.value] = (r, dom, _now(t0))
            ready.clear()
            t1 = time.perf_counter()
            batch.step(chunks_per_poll, s_batch)
            host["step_enqueue_s"] += time.perf_counter() - t1
            host["chunks"] += chunks_per_poll
            create(create_ms / 1e3)          # overlaps the chunk on the GPU
            t1 = time.perf_counter()
            done = batch.poll(wait=True)
            host["poll_wait_s"] += time.perf_counter() - t1
            for dom, status in done:
                r, _, start = live.pop(dom.h.value)
                futures.append(pool.submit(collect, r, dom, start, status, t0))   # the fields reach the host
                used -= r.est_bytes
        t1 = time.perf_counter()
        for f in futures:
            f.result()
        host["moments_tail_s"] = time.perf_counter() - t1
        pool.shutdown(wait=True)
    serve_batched.host_times = host
    return records


def request_nodes(r: Request) -> int:
    return int(r.side) ** (2 if r.kind == "cavity" else 3)


def lane_of(r: Request, large_nodes: int) -> int:
    """0: the small-request lane, 1: the large-request lane."""
    return 1 if request_nodes(r) >= large_nodes else 0


class _Arrivals:
    """Requests that have arrived and wait to be built, smallest work first
    (nodes x steps is the same step budget for all, so nodes decide)."""

    def __init__(self, reqs: List[Request]):
        import heapq
        self._heapq = heapq
        self.pending = sorted(reqs, key=lambda r: r.arrival)
        self.i = 0
        self.heap: list = []

    def arrive(self, now: float) -> None:
        while self.i < len(self.pending) and self.pending[self.i].arrival <= now:
            r = self.pending[self.i]
            self._heapq.heappush(self.heap, (request_nodes(r), r.rid, r))
            self.i += 1

    def peek(self):
        return self.heap[0][2] if self.heap else None

    def pop(self) -> Request:
        return self._heapq.heappop(self.heap)[2]

    def next_arrival(self):
        return self.pending[self.i].arrival if self.i < len(self.pending) else None

    def empty(self) -> bool:
        return not self.heap and self.i >= len(self.pending)


def serve_lanes(reqs: List[Request], max_steps: int = 2000, tol_velocity: float = 1e-6,
                residual_interval: int = 50, budget_bytes: int = 0, large_nodes: int = 1 << 19,
                create_ms: float = 5.0, keep: Optional[set] = None, large_slots: int = 1,
                small_cap_busy: int = 0) -> List[Record]:
    """Run the requests through two batches ("lanes") that advance independently.

    Small requests (fewer than `large_nodes` nodes) go to a lane on a high-priority
    CUDA stream: its chunks hold only small domains, so they are short, and when
    SMs free up the scheduler runs its blocks ahead of the other lane's.  Large
    requests go to a lane on a normal-priority stream, at most `large_slots` at a
    time (a large request fills the GPU alone; sharing it between several only
    delays all of them, which sets the tail latency).  Each lane runs one chunk
    at a time; the host polls both without blocking, admits new members at chunk
    boundaries and, between polls, builds the domains of arrived requests,
    smallest first, while the device-memory budget allows.  The stop rule, the
    fields and the step counts are those of `serve_batched` and `Domain.run`.
    `small_cap_busy` > 0 admits at most that many small requests while a large
    one runs (its share of the GPU sets the tail latency); 0: no cap.
    The velocity fields of the requests whose ids are in `keep` are kept in
    `serve_lanes.fields` (id -> (N, D) array).
    """
    import threading
    from concurrent.futures import ThreadPoolExecutor

    import torch
    max_it = max_steps - 2
    records: List[Record] = []
    lock = threading.Lock()
    local = threading.local()

    fields = {}

    def collect(r, dom, start, status, t0):
        if not hasattr(local, "stream"):
            local.stream = torch.cuda.Stream()
        _, u, _ = dom.moments(local.stream)
        rec = Record(r.rid, r.kind, int(np.prod(r.params.n[: r.params.dim])), r.arrival, start, _now(t0),
                     dom.time_step, status)
        dom.close()
        with lock:
            records.append(rec)
            if keep and r.rid in keep:
                fields[r.rid] = u

    arrivals = _Arrivals(reqs)
    s_init = torch.cuda.Stream()
    pool = ThreadPoolExecutor(max_workers=4)
    futures = []
    host = {"create_s": 0.0, "chunks": [0, 0], "idle_s": 0.0}
    b0 = Batch(budget_bytes, residual_interval)
    budget = b0.info()["budget"]
    b1 = Batch(budget, residual_interval)
    lanes = [{"batch": b0, "stream": torch.cuda.Stream(priority=-100), "ev": None, "live": {}, "ready": []},
             {"batch": b1, "stream": torch.cuda.Stream(priority=0), "ev": None, "live": {}, "ready": []}]
    used = 0
    t0 = time.perf_counter()
    try:
        while not arrivals.empty() or any(ln["live"] or ln["ready"] for ln in lanes):
            # build the domains of arrived requests (smallest first) while memory allows
            t1 = time.perf_counter()
            arrivals.arrive(_now(t0))
            built = 0
            while arrivals.peek() is not None and used + arrivals.peek().est_bytes <= budget:
                # smallest first: once the next one is large and the large lane has one
                # waiting, the rest wait too (they are no smaller)
                if lane_of(arrivals.peek(), large_nodes) == 1 and len(lanes[1]["ready"]) >= large_slots:
                    break
                r = arrivals.pop()
                dom = Domain(r.params)
                dom.init(s_init)
                lanes[lane_of(r, large_nodes)]["ready"].append((r, dom))
                used += r.est_bytes
                built += 1
                if time.perf_counter() - t1 > create_ms / 1e3:
                    break
            if built:
                s_init.synchronize()
            host["create_s"] += time.perf_counter() - t1
            progressed = False
            for li, ln in enumerate(lanes):
                if ln["ev"] is not None and not ln["ev"].query():
                    continue
                if ln["ev"] is not None:   # its chunk is complete: finished members leave
                    for dom, status in ln["batch"].poll(wait=False):
                        r, _, start = ln["live"].pop(dom.h.value)
                        futures.append(pool.submit(collect, r, dom, start, status, t0))
                        used -= r.est_bytes
                    ln["ev"] = None
                cap = large_slots if li == 1 else len(ln["ready"]) + len(ln["live"])
                if li == 0 and small_cap_busy > 0 and lanes[1]["live"]:
                    cap = small_cap_busy
                while ln["ready"] and len(ln["live"]) < cap:
                    r, dom = ln["ready"].pop(0)
                    ln["batch"].admit(dom, max_it, tol_density=math.inf, tol_velocity=tol_velocity,
                                      tol_scalar=math.inf)
                    ln["live"][dom.h.value] = (r, dom, _now(t0))
                if ln["live"]:
                    ln["batch"].step(1, ln["stream"])
                    ln["ev"] = torch.cuda.Event()
                    ln["ev"].record(ln["stream"])
                    host["chunks"][li] += 1
                    progressed = True
            if not progressed:
                t1 = time.perf_counter()
                nxt = arrivals.next_arrival()
                if not any(ln["live"] for ln in lanes) and nxt is not None and arrivals.peek() is None:
                    time.sleep(max(0.0, min(nxt - _now(t0), 0.01)))
                else:
                    time.sleep(0.0002)
                host["idle_s"] += time.perf_counter() - t1
        for f in futures:
            f.result()
    finally:
        pool.shutdown(wait=True)
        b0.close()
        b1.close()
    serve_lanes.host_times = host
    serve_lanes.fields = fields
    return records


def serve_sequential(reqs: List[Request], max_steps: int = 2000, tol_velocity: float = 1e-6,
                     residual_interval: int = 50, stream=None, plain: bool = False) -> List[Record]:
    """One solve at a time in arrival order with Domain.run (same stop rule).

    plain=True runs every solve with the dense single-domain sweep (the sparse
    fluid-only layout off), the plain kernel without any layout choice."""
    from . import _abi
    max_it = max_steps - 2
    records = []
    t0 = time.perf_counter()
    for r in sorted(reqs, key=lambda r: r.arrival):
        wait = r.arrival - _now(t0)
        if wait > 0:
            time.sleep(wait)
        start = _now(t0)
        with Domain(r.params) as dom:
            if plain:
                dom.set_option(_abi.LBF_OPT_SPARSE, 0)
            dom.init(stream)
            steps = dom.run(max_it, residual_interval, tol_density=math.inf, tol_velocity=tol_velocity,
                            tol_scalar=math.inf, stream=stream)
            dom.moments(stream)
            conv = steps <= max_it + 1
            records.append(Record(r.rid, r.kind, int(np.prod(r.params.n[: r.params.dim])), r.arrival, start,
                                  _now(t0), steps, 1 if conv else 2))
    return records


def summary(records: List[Record]) -> dict:
    if not records:
        return {"solves": 0}
    lat = np.array([r.latency for r in records])
    t_first = min(r.arrival for r in records)
    t_last = max(r.finish for r in records)
    lups = sum(r.nodes * r.steps for r in records)
    return {"solves": len(records), "seconds": t_last - t_first, "solves_per_s": len(records) / (t_last - t_first),
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "mlups_all_nodes": lups / (t_last - t_first) / 1e6,
            "converged": int(sum(r.status == 1 for r in records))}
