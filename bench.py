"""Benchmark: MLUPS and HBM-roofline fraction of the fused LB step, D3Q19 TRT
porous channel 256^3 (FP32 storage), the headline configuration.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--storage f32|f16dev|bf16dev|f64] [--n 256]

One step = one main_steps over the whole lattice (one fused kernel launch).
Inputs are resident in HBM (2 x 19 x 4 B x 11.7 M fluid nodes = 1.8 GB of
populations, far larger than the 126 MB L2, so no flush is needed between steps).
`e2e` is the same metric through lbf_solve with host buffers (node-type upload,
layout build, init, K steps and the FP64 moment download inside the timed
region), with the phase split of a second solve.  `accuracy` compares the engine
(the benchmarked storage, FP32 and FP16 deviations) after --acc-steps steps (100)
with the FP64 oracle on the same lattice; that oracle run, timed, is the
`cpu_baseline`.  `same_precision` is the FP64-storage figure.  Under torchrun each
rank advances its own part (z-slabs, or replicas with --decomp replicas); timing
is the max over ranks of CUDA-event time on the launching stream.

--impl reference times the CPU oracle (a restatement of the reference's Rust
step, OpenMP over all host cores) on the same geometry.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

STORAGE = {"f64": 0, "f32": 1, "f16dev": 2, "bf16dev": 3}
SBYTES = {"f64": 8, "f32": 4, "f16dev": 2, "bf16dev": 2}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--storage", default="f32", choices=list(STORAGE))
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--porosity", type=float, default=0.7, help="target fluid fraction (1.0 = empty channel)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the oracle run (CPU baseline and accuracy against the oracle)")
    ap.add_argument("--no-same-precision", action="store_true", help="skip the FP64-storage figure")
    ap.add_argument("--block", type=int, default=0, help="override the x block size")
    ap.add_argument("--sweep", default="auto", choices=["auto", "pipe", "stage", "plain", "sparse"],
                    help="auto: the library's default (the fluid-only sparse layout for porous lean lattices); "
                         "pipelined bulk-copy sweep, one-shot staged sweep, plain dense loads, or sparse")
    ap.add_argument("--stages", type=int, default=0, help="pipeline ring depth (0 = auto)")
    ap.add_argument("--compact", type=int, default=-1, help="1/0: force the fluid work-list sweep on/off")
    ap.add_argument("--streaming", default="auto", choices=["auto", "pull", "push", "inplace"],
                    help="streaming scheme of the sparse layout (auto: the library's default)")
    ap.add_argument("--sround", type=int, default=-1, help="16-bit storage: 1/0 stochastic rounding on/off")
    ap.add_argument("--autotune", action="store_true",
                    help="pick the sweep variant and block size by timing candidates first (untimed)")
    ap.add_argument("--workload", default="step", choices=["step", "serve", "batch", "accuracy", "c3", "c4"],
                    help="step: the fused step on one lattice (headline); serve: the serving mix; "
                         "c3: the D3Q27 central-moment Taylor-Green step (384^3, Re 1600); "
                         "c4: the coupled momentum + scalar step on the packed bed (192x192x384); "
                         "batch: batched vs single-domain sweeps and per-request host costs; "
                         "accuracy: FP32 / FP16 / BF16 storage against FP64 at full size (--case)")
    ap.add_argument("--case", default="c2", choices=["c2", "c3", "c4"],
                    help="accuracy: c2 porous channel 256^3 (5000 steps), c3 D3Q27 MRT Taylor-Green 384^3 "
                         "(10000 steps), c4 packed bed with scalar 192x192x384 (20000 steps)")
    ap.add_argument("--acc-steps", type=int, default=0, help="accuracy: override the number of steps")
    ap.add_argument("--acc-curve", default="",
                    help="accuracy c2: comma-separated steps; the storages run side by side and the velocity "
                         "error against FP64 is reported at each (with --acc-n for the lattice side)")
    ap.add_argument("--acc-n", type=int, default=256, help="accuracy c2 with --acc-curve: lattice side")
    ap.add_argument("--c4-collision", default="trt0.55", choices=["bgk0.6", "bgk0.8", "trt0.8", "trt0.55"],
                    help="accuracy c4: momentum collision (BGK tau 0.6 / 0.8, or TRT tau+ 0.8 / 0.55 magic 1/4)")
    ap.add_argument("--c4-u", type=float, default=0.01, help="accuracy c4: inlet velocity u_z")
    ap.add_argument("--scalars", type=int, default=1,
                    help="c4: adsorbing scalars advanced by the one momentum sweep (1..4); with more than one, "
                         "the same scalars as separate single-scalar domains are timed beside it")
    ap.add_argument("--c3-re", type=float, default=1600.0, help="accuracy c3: Reynolds number of the vortex")
    ap.add_argument("--c3-collision", default="central", choices=["central", "mrt"],
                    help="accuracy c3: central-moment collision (default) or the raw-moment MRT")
    ap.add_argument("--requests", type=int, default=4000, help="serve: number of requests")
    ap.add_argument("--rate", type=float, default=20.0, help="serve: Poisson arrivals per second (inf = all at t=0)")
    ap.add_argument("--serve-mode", default="lanes", choices=["lanes", "single"],
                    help="serve: two batches (small requests on a high-priority stream) or one batch")
    ap.add_argument("--max-steps", type=int, default=2000, help="serve: steps per request at most")
    ap.add_argument("--small-cap-busy", type=int, default=0,
                    help="serve (lanes): small requests admitted at most while a large one runs (0: no cap)")
    ap.add_argument("--chunk", type=int, default=50, help="serve: residual interval (steps per chunk)")
    ap.add_argument("--no-sequential", action="store_true", help="serve: skip the one-at-a-time baseline")
    ap.add_argument("--seq-plain", action="store_true",
                    help="serve: also run the one-at-a-time baseline with the plain dense sweep")
    ap.add_argument("--decomp", default="slab", choices=["slab", "replicas"],
                    help="N > 1: z-slabs of one n x n x (n N) channel with a halo exchange per step, "
                         "or independent replicas")
    return ap.parse_args()


def geometry(n: int, seed: int, porosity: float = 0.7) -> np.ndarray:
    from lbflow_b200.cases import sphere_pack
    if porosity >= 1.0:
        return np.zeros(n ** 3, dtype=np.uint8)
    cache = os.path.join(tempfile.gettempdir(), "lbflow_b200_cache")
    os.makedirs(cache, exist_ok=True)
    path = os.path.join(cache, f"spheres_{n}_{seed}_p{int(round(porosity * 100)):03d}_r4-10.npy")
    if os.path.exists(path):
        return np.load(path)
    mask = sphere_pack([n, n, n], porosity, 4.0, 10.0, seed)
    np.save(path, mask)
    return mask


def params_for(args, mask):
    from lbflow_b200 import cases
    from lbflow_b200.core import Storage
    return cases.porous_channel_d3q19([args.n] * 3, mask=mask, force=1e-6, storage=Storage(STORAGE[args.storage]))


def workload_name(args):
    return (f"D3Q19 TRT porous channel {args.n}^3 (tau+=0.8, magic 1/4, g_x=1e-6, spheres r in [4,10], "
            f"porosity {args.porosity:g}, periodic x, no-slip y/z)")


def config_of(args, n_fluid, world, sweep):
    return {"workload": workload_name(args), "storage": args.storage, "n_fluid": int(n_fluid),
            "l2": f"inputs larger than L2 (populations 2 x 19 x {SBYTES[args.storage]} B per fluid node, "
                  f"{2 * 19 * SBYTES[args.storage] * int(n_fluid) / 1e6:.0f} MB)",
            "parallelism": "replicas" if world > 1 else "single", "sweep": sweep}


class Clocks:
    """nvidia-smi sampler for the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.path = os.path.join(tempfile.gettempdir(), f"lbf_clocks_{os.getpid()}.csv")
        self.proc = None

    def _lines(self) -> int:
        try:
            with open(self.path) as fh:
                return sum(1 for _ in fh)
        except OSError:
            return 0

    def _wait_lines(self, n: int, limit_s: float) -> None:
        t_end = time.perf_counter() + limit_s
        while self._lines() < n and time.perf_counter() < t_end and self.proc.poll() is None:
            time.sleep(0.01)

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
            # the sampler is running (its first line written) when the timed region starts
            self._wait_lines(1, 3.0)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            # a timed region shorter than the sampling period still gets the sample
            # that follows it
            self._wait_lines(2, 0.5)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    smax.append(float(p[2]))
                except ValueError:
                    continue
                for k, nm in enumerate(names):
                    if p[5 + k].lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of the
# headline step kernel, from ncu.  Keyed by (sweep, storage, n).  Provenance of each
# figure is given beside it; None where no capture exists.
TRAFFIC_BYTES = {
    # k_step_sparse<D3Q19, TRT, FP32>: one launch captured at 160^3 (421,772,288 B,
    # 2,867,096 fluid nodes), scaled to 256^3 by the fluid nodes per launch
    # (11,743,596); the writes of a single captured launch are under-counted by the
    # stores still held in L2 when it ends (ncu flushes L2 before each replay).
    ("sparse", "f32", 256): 1727574994.0,
}


def traffic_of(sweep_key: str, storage: str, n: int):
    return TRAFFIC_BYTES.get((sweep_key, storage, n))


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def run_reference(args, rank, world):
    if rank != 0:
        return
    mask = geometry(args.n, args.seed, args.porosity)
    from lbflow_b200 import momentum as m
    from oracle import oracle as orc
    p = params_for(argparse.Namespace(**{**vars(args), "storage": "f64"}), mask)
    desc, keep = m.to_desc(p)
    od = orc.Domain(desc, keep=keep).init()
    warm = min(args.warmup, 2)
    od.step(warm)
    k = max(1, min(args.steps, 8))   # bounded sample: a few full-lattice steps
    t0 = time.perf_counter()
    od.step(k)
    dt = time.perf_counter() - t0
    mlups = od.num_fluid * k / dt / 1e6
    cores = orc.num_threads()
    sample = (f"oracle (FP64 CPU restatement of the reference step) on the {args.n}^3 lattice, {k} main_steps timed "
              f"after {warm} warm-up, {cores} OpenMP threads (the Rust reference cannot be built here)")
    line = {"impl": "reference", "metric": "MLUPS", "value": mlups, "unit": "MLUPS", "n_gpus": world,
            "steps": k, "warmup": warm, "ms_per_step": dt / k * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded sphere packing)",
            "config": config_of(args, od.num_fluid, world, "CPU oracle, FP64, OpenMP"),
            "cpu_baseline": {"value": mlups, "unit": "MLUPS", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": mlups, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def sweep_name(dom, _abi):
    if dom.get_option(_abi.LBF_OPT_SPARSE):
        sch = dom.get_option(_abi.LBF_OPT_STREAMING)
        return "sparse fluid-only layout, " + {_abi.LBF_STREAM_PULL: "pull (two buffers)",
                                               _abi.LBF_STREAM_PUSH: "push (two buffers)",
                                               _abi.LBF_STREAM_INPLACE: "in place (AA pattern, one buffer)"}[sch]
    return ("sparse fluid-only layout" if dom.get_option(_abi.LBF_OPT_SPARSE) else
            "pipelined bulk-copy" if dom.get_option(_abi.LBF_OPT_PIPE) else
            "one-shot staged" if dom.get_option(_abi.LBF_OPT_STAGE) else
            "compacted fluid work list" if dom.get_option(_abi.LBF_OPT_COMPACT) else "dense lattice")


def configure(dom, args, _abi, tuned=None):
    if tuned is not None:
        from lbflow_b200 import autotune
        autotune.apply(dom, tuned)
    if args.block:
        dom.set_option(_abi.LBF_OPT_BLOCK_X, args.block)
    if tuned is None and args.sweep != "auto":
        dom.set_option(_abi.LBF_OPT_PIPE, 1 if args.sweep == "pipe" else 0)
        dom.set_option(_abi.LBF_OPT_STAGE, 1 if args.sweep == "stage" else 0)
        dom.set_option(_abi.LBF_OPT_SPARSE, 1 if args.sweep == "sparse" else 0)
    if args.stages:
        dom.set_option(_abi.LBF_OPT_PIPE_STAGES, args.stages)
    if args.compact >= 0:
        dom.set_option(_abi.LBF_OPT_COMPACT, args.compact)
    if args.streaming != "auto":
        dom.set_option(_abi.LBF_OPT_STREAMING, {"pull": _abi.LBF_STREAM_PULL, "push": _abi.LBF_STREAM_PUSH,
                                                "inplace": _abi.LBF_STREAM_INPLACE}[args.streaming])
    if args.sround >= 0:
        dom.set_option(_abi.LBF_OPT_SROUND, args.sround)


def time_steps(dom, steps, warmup, stream, world):
    """CUDA-event time of `steps` steps after `warmup` untimed ones (max over ranks)."""
    import torch
    import torch.distributed as dist
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dom.step(warmup, 0, stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    start.record(stream)
    dom.step(steps, 0, stream)
    end.record(stream)
    torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    return ms


def measure_e2e(args, p, n_fluid, N, stream, world):
    """The same metric through lbf_solve (the C-ABI call with host buffers): node
    types uploaded, layout built, initialised, K steps, FP64 density and velocity
    downloaded, all inside the timed region; then the same sequence through the
    separate ABI calls, timed phase by phase."""
    import torch
    import torch.distributed as dist
    from lbflow_b200.domain import Domain, solve_arrays
    # the results land in page-locked host buffers, allocated before the timed
    # region (a serving caller keeps them): the library copies into them directly
    d = p.dim
    out = tuple(torch.empty(n, dtype=torch.float64, pin_memory=True).numpy() for n in (N, N * d))
    out = (out[0], out[1], None)
    # untimed warm-up solves (pool, pinned staging, module loads): for the first
    # seconds after process start, solves of the 256^3 case run slower (layout and
    # init up to 190 ms against 4 ms, one 20-step solve of 880 ms against 23 ms),
    # so the timed solves start after 4 s of warm-up solves (at least two, at most 200)
    w0, nw = time.perf_counter(), 0
    while nw < 2 or (time.perf_counter() - w0 < 4.0 and nw < 200):
        solve_arrays(p, args.steps, stream=stream, out=out)
        torch.cuda.synchronize()
        nw += 1
    if world > 1:
        # every rank runs the same number of warm-up solves (the MAX over ranks)
        t = torch.tensor([nw], device="cuda", dtype=torch.int64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        for _ in range(int(t.item()) - nw):
            solve_arrays(p, args.steps, stream=stream, out=out)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    reps = 3
    t0 = torch.cuda.Event(enable_timing=True); t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    wall0 = time.perf_counter()
    for _ in range(reps):
        solve_arrays(p, args.steps, stream=stream, out=out)
    t1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    e_sec = max(t0.elapsed_time(t1) / 1e3, wall) / reps
    if world > 1:
        t = torch.tensor([e_sec], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e_sec = float(t.item())
    # phase split of the same work (host clock, device synchronised after each phase)
    sync = torch.cuda.synchronize
    split = {}
    c0 = time.perf_counter()
    dom = Domain(p)
    sync(); c1 = time.perf_counter()
    dom.init(stream)
    sync(); c2 = time.perf_counter()
    dom.step(args.steps, 0, stream)
    sync(); c3 = time.perf_counter()
    dom.moments(stream, out=out)
    sync(); c4 = time.perf_counter()
    dom.close()
    sync(); c5 = time.perf_counter()
    split = {"create_ms": 1e3 * (c1 - c0), "layout_and_init_ms": 1e3 * (c2 - c1), "steps_ms": 1e3 * (c3 - c2),
             "download_ms": 1e3 * (c4 - c3), "destroy_ms": 1e3 * (c5 - c4)}
    return {"value": world * n_fluid * args.steps / e_sec / 1e6, "unit": "MLUPS",
            "h2d_bytes_per_step": N / args.steps, "d2h_bytes_per_step": N * (1 + 3) * 8 / args.steps,
            "ms_per_solve": 1e3 * e_sec,
            "split": split,
            "note": f"lbf_solve per solve of {args.steps} steps (mean of {reps} after {nw} untimed warm-up solves, 4 s "
                    "or more): "
                    f"node-type upload (N x 1 B), layout build, init, {args.steps} steps, FP64 density + velocity "
                    "download (N x 32 B) into page-locked host buffers; split measured on a further solve through "
                    "the separate calls"}


def accuracy_vs_oracle(args, mask, steps, storages, threads=0):
    """Engine fields after `steps` steps on the headline lattice, against the FP64
    oracle after the same steps: relative L2 over fluid nodes of velocity and
    density, exact node-class agreement.  The oracle's run is timed and returned
    as the CPU baseline (same lattice, all host threads)."""
    import torch
    from lbflow_b200 import _abi
    from lbflow_b200 import momentum as m
    from lbflow_b200.domain import Domain
    from oracle import oracle as orc
    if threads:
        orc.set_threads(threads)
    p64 = params_for(argparse.Namespace(**{**vars(args), "storage": "f64"}), mask)
    desc, keep = m.to_desc(p64)
    od = orc.Domain(desc, keep=keep).init()
    t0 = time.perf_counter()
    od.step(steps)
    dt = time.perf_counter() - t0
    ro, uo, _ = od.observe()
    cls_o, links_o = od.node_class()
    fl = (cls_o & _abi.LBF_CLASS_SOLID) == 0
    base = {"value": od.num_fluid * steps / dt / 1e6, "unit": "MLUPS", "cores": orc.num_threads(), "kind": "port",
            "sample": f"oracle (FP64 CPU restatement of the reference step) on the same {args.n}^3 lattice, "
                      f"{steps} main_steps from initialisation, {orc.num_threads()} OpenMP threads "
                      "(the Rust reference cannot be built here)"}
    del od

    def rel(a, b):
        nb = float(np.linalg.norm(b))
        return float(np.linalg.norm(a - b)) / (nb if nb > 0 else 1.0)

    acc = {"steps": steps, "reference": "oracle, FP64", "runs": {}}
    for st in storages:
        p = params_for(argparse.Namespace(**{**vars(args), "storage": st}), mask)
        with Domain(p) as d:
            d.init().step(steps)
            rg, ug, _ = d.moments()
            cls_g, links_g = d.node_class()
        torch.cuda.synchronize()
        acc["runs"][st] = {"u": rel(ug[fl], uo[fl]), "rho": rel(rg[fl], ro[fl]),
                           "mask_equal": bool(np.array_equal(cls_g, cls_o) and np.array_equal(links_g, links_o))}
    return acc, base


def same_precision(args, mask, stream):
    """FP64 storage (the reference's precision) on the same lattice: MLUPS and roofline."""
    from lbflow_b200 import _abi
    from lbflow_b200.domain import Domain
    p = params_for(argparse.Namespace(**{**vars(args), "storage": "f64"}), mask)
    n_fluid = int(np.count_nonzero(mask == 0))
    steps = max(20, min(args.steps, 200))
    with Domain(p) as d:
        configure(d, args, _abi)
        d.init(stream)
        ms = time_steps(d, steps, 3, stream, 1)
        sweep = sweep_name(d, _abi)
    per = ms / 1e3 / steps
    alg = n_fluid * 2 * 19 * 8 + mask.size
    peak, kind = peaks()
    return {"storage": "f64", "value": n_fluid / per / 1e6, "unit": "MLUPS", "steps": steps,
            "ms_per_step": 1e3 * per, "roofline_frac": alg / per / 1e9 / peak, "peak_source": kind,
            "algorithmic_bytes_per_launch": alg, "sweep": sweep}


def run_engine(args, rank, world, local_rank):
    import torch
    from lbflow_b200 import _abi
    from lbflow_b200.domain import Domain

    torch.cuda.set_device(local_rank)
    mask = geometry(args.n, args.seed, args.porosity)
    p = params_for(args, mask)
    n_fluid = int(np.count_nonzero(mask == 0))
    N = mask.size
    stream = torch.cuda.current_stream()
    tuned = None
    if args.autotune:
        from lbflow_b200 import autotune
        tuned = autotune.autotune(p, steps=20, cache=None)
    dom = Domain(p)
    configure(dom, args, _abi, tuned)
    dom.init(stream)
    sweep = sweep_name(dom, _abi)
    sweep_key = "sparse" if dom.get_option(_abi.LBF_OPT_SPARSE) else "dense"
    if tuned is not None:
        sweep += f" (autotuned: {tuned.get('sweep')}, block_x {tuned.get('block_x', 0)})"
    # the clock sampler starts before the warm-up so that its samples cover the timed steps
    with Clocks(local_rank) as clk:
        ms = time_steps(dom, args.steps, args.warmup, stream, world)
    clocks = clk.summary()
    dom.close()
    sec = ms / 1e3
    mlups = world * n_fluid * args.steps / sec / 1e6
    # roofline of the step kernel (one launch per step)
    s = SBYTES[args.storage]
    alg_bytes = n_fluid * 2 * 19 * s + N * 1   # read + write Q populations per fluid node + 1 B node type
    per_launch = sec / args.steps
    achieved = alg_bytes / per_launch / 1e9
    peak, peak_kind = peaks()
    traffic = traffic_of(sweep_key, args.storage, args.n)
    e2e = None if args.no_e2e else measure_e2e(args, p, n_fluid, N, stream, world)
    if rank != 0:
        return
    acc, base = (None, None)
    if not args.no_cpu_baseline:
        stores = [args.storage] + ([x for x in ("f32", "f16dev") if x != args.storage])
        acc, base = accuracy_vs_oracle(args, mask, args.acc_steps or 100, stores)
    same = None if args.storage == "f64" or args.no_same_precision else same_precision(args, mask, stream)
    line = {"metric": "MLUPS", "value": mlups, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.storage != "f64" else "f64",
            "data": "synthetic (seeded sphere packing)",
            "config": config_of(args, n_fluid, world, sweep),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": alg_bytes},
            "accuracy": acc, "same_precision": same,
            "cpu_baseline": base, "e2e": e2e, "gpu_launches": args.steps, "clocks": clocks}
    print(json.dumps(line), flush=True)


def run_c3(args, rank, world, local_rank):
    """The D3Q27 Taylor-Green vortex step (384^3 periodic, u0 = 0.05, Re = 1600, the
    central-moment collision, or --c3-collision mrt), FP32 / FP16-deviation / FP64
    storage: MLUPS and the roofline of the step kernel (read and write 27
    populations per node, every node fluid, plus 1 B of node type)."""
    import torch
    from lbflow_b200 import _abi, cases
    from lbflow_b200.core import Storage
    from lbflow_b200.domain import Domain
    torch.cuda.set_device(local_rank)
    st = {"f32": Storage.F32, "f64": Storage.F64, "f16dev": Storage.F16DEV, "bf16dev": Storage.BF16DEV}[args.storage]
    side = 384 if args.n == 256 else args.n
    p, nu = cases.tgv_d3q27(side, 0.05, args.c3_re, st, collision=args.c3_collision)
    stream = torch.cuda.current_stream()
    with Domain(p) as d:
        configure(d, args, _abi)
        d.init(stream)
        sweep = sweep_name(d, _abi)
        with Clocks(local_rank) as clk:
            ms = time_steps(d, args.steps, args.warmup, stream, world)
        clocks = clk.summary()
        inv = d.inventory()
    N = side ** 3
    sec = ms / 1e3
    alg = N * 2 * 27 * SBYTES[args.storage] + N
    peak, kind = peaks()
    achieved = alg / (sec / args.steps) / 1e9
    if rank != 0:
        return
    line = {"metric": "MLUPS", "value": world * N * args.steps / sec / 1e6, "unit": "MLUPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if st == Storage.F64 else "f32",
            "data": "synthetic (analytic initial field)",
            "config": {"workload": f"D3Q27 Taylor-Green vortex {side}^3 periodic, u0 0.05, Re {args.c3_re:g}, "
                                   f"{args.c3_collision} collision (tau {3 * nu + 0.5:.5f})",
                       "storage": args.storage, "sweep": sweep,
                       "l2": f"inputs larger than L2 (populations 2 x 27 x {SBYTES[args.storage]} B per node)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "peak_source": kind, "algorithmic_bytes_per_launch": alg},
            "finite_after_run": bool(np.all(np.isfinite(inv))), "gpu_launches": args.steps, "clocks": clocks}
    print(json.dumps(line), flush=True)


def run_c4(args, rank, world, local_rank):
    """The coupled D3Q19 momentum + passive-scalar step with Langmuir adsorption on
    the packed bed (192 x 192 x 384, porosity 0.6 of seeded overlapping spheres
    r in [4, 10], Zou-He inlet u_z = 0.04 with scalar C = 1, anti-bounce-back
    outlet with second-order scalar outflow, scalar tau 0.55, k_a 1e-3, k_d 1e-5,
    q_max 1; --c4-u and --c4-collision as in the accuracy run, whose defaults keep
    the flow finite: at u_z = 0.04 the reference's algorithm diverges on this bed),
    FP32 or FP64 storage: MFLUPS and the roofline of the step kernels.
    Algorithmic bytes per fluid update: 2 Q s for f and 2 Q s for g, plus q_ads and
    the previous scalar value read and written at each bounce-back node (4 s),
    plus 1 B of node type per node.  With --scalars K, K scalars (adsorption rates
    k_a 1e-3 (1 + i)) share the momentum sweep: 2 Q s (1 + K) per fluid update and
    4 s K per bounce-back node."""
    import torch
    from lbflow_b200 import _abi, cases
    from lbflow_b200.core import Storage
    from lbflow_b200.domain import Domain
    torch.cuda.set_device(local_rank)
    st = {"f32": Storage.F32, "f64": Storage.F64}[args.storage if args.storage in ("f32", "f64") else "f32"]
    side = 192 if args.n == 256 else args.n     # --n: a smaller bed of the same shape (n x n x 2n)
    n = [side, side, 2 * side]
    cache = os.path.join(tempfile.gettempdir(), "lbflow_b200_cache")
    os.makedirs(cache, exist_ok=True)
    path = os.path.join(cache, f"bed_{side}x{side}x{2 * side}_{args.seed}_p060.npy")
    if os.path.exists(path):
        mask = np.load(path)
    else:
        mask = cases.sphere_pack(n, 0.6, 4.0, 10.0, args.seed, overlap=True)
        np.save(path, mask)
    # 8 clear layers at the inlet and the outlet, as in the accuracy run of this bed
    mask = mask.reshape(n[2], n[1], n[0]).copy()
    mask[:8] = 0
    mask[-8:] = 0
    mask = mask.ravel()
    from lbflow_b200.core import BGK, TRT
    coll = {"bgk0.6": BGK(0.6), "bgk0.8": BGK(0.8), "trt0.8": TRT.from_magic(0.8, 0.25),
            "trt0.55": TRT.from_magic(0.55, 0.25)}[args.c4_collision]
    K = max(1, min(4, args.scalars))
    sps = []
    for i in range(K):
        mp, sp = cases.packed_bed_scalar(n, mask=mask, storage=st, u_in=args.c4_u, tau_g=0.55, collision=coll,
                                         ka=1e-3 * (1 + i))
        sps.append(sp)
    stream = torch.cuda.current_stream()
    separate_ms = None
    if K > 1:
        # the reference's cost model on this engine: one full domain per scalar
        separate_ms = 0.0
        for sp in sps:
            with Domain(mp, sp) as d1:
                configure(d1, args, _abi)
                d1.init(stream)
                separate_ms += time_steps(d1, args.steps, args.warmup, stream, world)
    with Domain(mp, sps) as d:
        configure(d, args, _abi)
        d.init(stream)
        cls, _ = d.node_class()
        fl = (cls & _abi.LBF_CLASS_SOLID) == 0
        n_fluid = int(np.count_nonzero(fl))
        n_bb = int(np.count_nonzero(fl & ((cls & _abi.LBF_CLASS_BOUNCE_BACK) != 0)))
        sweep = sweep_name(d, _abi)
        with Clocks(local_rank) as clk:
            ms = time_steps(d, args.steps, args.warmup, stream, world)
        clocks = clk.summary()
        inv = d.inventory()
        finite = bool(np.all(np.isfinite(inv)))
    sec = ms / 1e3
    s_b = 8 if st == Storage.F64 else 4
    alg = n_fluid * 2 * 19 * s_b * (1 + K) + n_bb * 4 * s_b * K + mask.size
    peak, kind = peaks()
    achieved = alg / (sec / args.steps) / 1e9
    if rank != 0:
        return
    line = {"metric": "MFLUPS", "value": world * n_fluid * args.steps / sec / 1e6, "unit": "MFLUPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if st == Storage.F64 else "f32",
            "data": "synthetic (seeded sphere packing)",
            "config": {"workload": f"coupled D3Q19 momentum + {K} D3Q19 scalar{'s' if K > 1 else ''} with Langmuir "
                                   f"adsorption, packed bed {side}x{side}x{2 * side}, porosity 0.6 (8 clear layers at "
                                   f"each end), Zou-He inlet u_z={args.c4_u:g}, momentum {args.c4_collision}, "
                                   "scalar tau 0.55",
                       "scalars": K,
                       "storage": "f64" if st == Storage.F64 else "f32", "n_fluid": n_fluid,
                       "bounce_back_nodes": n_bb, "sweep": sweep,
                       "l2": "inputs larger than L2 (f and g populations, 2 buffers each)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "peak_source": kind, "algorithmic_bytes_per_launch": alg},
            "finite_after_run": finite, "gpu_launches": args.steps * 2, "clocks": clocks}
    if separate_ms is not None:
        line["separate_domains"] = {"ms_per_step": separate_ms / args.steps,
                                    "note": f"the {K} scalars as {K} single-scalar domains, each with its own "
                                            "momentum sweep, timed one after another"}
    print(json.dumps(line), flush=True)


def run_serve(args, rank, world, local_rank):
    """The serving mix through the batches, and one solve at a time as the baseline;
    then the FP16-deviation requests of a sample are solved again in FP64 storage
    and compared (velocity, relative L2), so that the batched results are shown to
    be of the stated accuracy."""
    import math
    import torch
    from lbflow_b200 import serve
    from lbflow_b200.core import Storage
    from lbflow_b200.domain import Domain
    torch.cuda.set_device(local_rank)
    reqs = serve.make_requests(args.requests, args.rate, args.seed + rank)
    serve.prepare(reqs)
    warm = serve.make_requests(6, float("inf"), args.seed + 999)
    serve.prepare(warm)
    run = serve.serve_lanes if args.serve_mode == "lanes" else serve.serve_batched
    run(warm, max_steps=200, residual_interval=args.chunk)
    serve.serve_sequential(warm, max_steps=200, residual_interval=args.chunk)
    torch.cuda.synchronize()
    rng = np.random.default_rng(args.seed)
    f16 = [r.rid for r in reqs if r.storage == Storage.F16DEV]
    check = set(int(x) for x in rng.choice(f16, size=min(12, len(f16)), replace=False)) if f16 else set()
    with Clocks(local_rank) as clk:
        if args.serve_mode == "lanes":
            rb = serve.serve_lanes(reqs, max_steps=args.max_steps, residual_interval=args.chunk, keep=check,
                                   small_cap_busy=args.small_cap_busy)
        else:
            rb = serve.serve_batched(reqs, max_steps=args.max_steps, residual_interval=args.chunk)
    sb = serve.summary(rb)
    sb["host_times"] = getattr(run, "host_times", None)
    # accuracy of the FP16 half: the same requests in FP64 storage, same stop rule
    acc = []
    fields = getattr(serve.serve_lanes, "fields", {}) if args.serve_mode == "lanes" else {}
    for r in reqs:
        if r.rid not in fields:
            continue
        p64 = serve.build_params(r)
        p64.storage = Storage.F64
        with Domain(p64) as d:
            d.init().run(args.max_steps - 2, args.chunk, tol_density=math.inf, tol_velocity=1e-6, tol_scalar=math.inf)
            _, u64, _ = d.moments()
        u16 = fields[r.rid]
        acc.append({"rid": r.rid, "kind": r.kind, "side": r.side,
                    "rel_l2_velocity": float(np.linalg.norm(u16 - u64) / max(np.linalg.norm(u64), 1e-300))})
    ss = None
    if not args.no_sequential:
        ss = serve.summary(serve.serve_sequential(reqs, max_steps=args.max_steps, residual_interval=args.chunk))
    sp = None
    if args.seq_plain:
        sp = serve.summary(serve.serve_sequential(reqs, max_steps=args.max_steps, residual_interval=args.chunk,
                                                  plain=True))
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([sb["seconds"]], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        sb["seconds"] = float(t.item())
    if rank != 0:
        return
    line = {"metric": "solves/s", "value": world * sb["solves"] / sb["seconds"], "unit": "solves/s", "n_gpus": world,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded serving mix)",
            "config": {"workload": f"serving mix: {args.requests} requests, arrivals "
                                   f"{'all at t=0' if args.rate == float('inf') else f'Poisson {args.rate:g}/s'}, "
                                   "50% D2Q9 BGK cavities side log-U[64,1024], 50% D3Q19 TRT porous channels side "
                                   "log-U[32,160] porosity U[0.5,0.9], FP32 / FP16-deviation storage 50/50, "
                                   f"stop at {args.max_steps} steps or velocity residual < 1e-6 "
                                   f"(checked every {args.chunk} steps)",
                       "serving": ("two batches: small requests on a high-priority stream, smallest first; "
                                   "large requests (>= 2^19 nodes) on a normal-priority stream")
                       if args.serve_mode == "lanes" else "one batch",
                       "parallelism": "replicas" if world > 1 else "single"},
            "p50_s": sb.get("p50_s"), "p99_s": sb.get("p99_s"),
            "batched": sb, "sequential": ss, "fp16_vs_fp64": acc, "clocks": clk.summary()}
    if acc:
        line["fp16_vs_fp64_max_rel_l2_velocity"] = max(a["rel_l2_velocity"] for a in acc)
    if ss:
        line["speedup_vs_sequential"] = sb["solves_per_s"] / ss["solves_per_s"]
    if sp:
        line["sequential_plain"] = sp
        line["speedup_vs_sequential_plain"] = sb["solves_per_s"] / sp["solves_per_s"]
    print(json.dumps(line), flush=True)


def run_slabs(args, rank, world, local_rank):
    """Weak scaling over z-slabs: rank r owns an n^3 slab of an n x n x (n * world)
    channel (no-slip y and z walls at the ends, periodic x), exchanges its halo
    planes with its neighbours after every step (NCCL send/recv)."""
    import torch
    import torch.distributed as dist
    from lbflow_b200 import slab
    torch.cuda.set_device(local_rank)
    dist.barrier()        # the first collective of the group includes every rank
    own = geometry(args.n, args.seed + rank, args.porosity).reshape(args.n, args.n, args.n)
    p = params_for(args, own.ravel())
    p.n = [args.n, args.n, args.n * world]
    ex = slab.TorchExchange(rank, world, periodic=False)
    stream = torch.cuda.current_stream()
    t_e2e0 = time.perf_counter()
    sd = slab.SlabDomain(p, rank, world, ex, own_mask=own)
    sd.init()
    n_fluid = sd.n_fluid_own
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local_rank) as clk:
        sd.step(args.warmup)
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        start.record(stream)
        sd.step(args.steps)
        end.record(stream)
        torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    rho, u = sd.moments()                      # the fields reach the host
    e2e_sec = time.perf_counter() - t_e2e0
    t = torch.tensor([ms, e2e_sec, float(n_fluid)], device="cuda", dtype=torch.float64)
    tmax = t.clone()
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    tsum = t.clone()
    dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
    dist.barrier()
    sd.close()
    if rank != 0:
        return
    ms, e2e_sec, fluid_all = float(tmax[0]), float(tmax[1]), float(tsum[2])
    sec = ms / 1e3
    mlups = fluid_all * args.steps / sec / 1e6
    s_b = SBYTES[args.storage]
    alg_bytes = n_fluid * 2 * 19 * s_b + args.n ** 3
    peak, peak_kind = peaks()
    achieved = alg_bytes / (sec / args.steps) / 1e9
    halo = 2 * 5 * args.n * args.n * s_b
    line = {"metric": "MLUPS", "value": mlups, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.storage != "f64" else "f64",
            "data": "synthetic (seeded sphere packing per slab)",
            "config": {"workload": f"D3Q19 TRT porous channel {args.n}x{args.n}x{args.n * world} in z-slabs of "
                                   f"{args.n}^3 per GPU (tau+=0.8, magic 1/4, g_x=1e-6, spheres r in [4,10], "
                                   f"porosity {args.porosity:g}, periodic x, no-slip y/z)",
                       "storage": args.storage, "n_fluid": int(fluid_all), "parallelism": f"z-slabs x{world}",
                       "halo_bytes_per_step_per_gpu": 2 * halo,
                       "l2": f"inputs larger than L2 (populations 2 x 19 x {s_b} B per fluid node and GPU)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic_of("sparse", args.storage, args.n), "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "note": "per GPU, step kernels + halo exchange in the timed step; the exchange "
                                 "(pack, NCCL send/recv, unpack on a second stream) overlaps the interior sweep"},
            "cpu_baseline": None,
            "e2e": {"value": fluid_all * args.steps / e2e_sec / 1e6, "unit": "MLUPS",
                    "h2d_bytes_per_step": args.n ** 3 * world / args.steps,
                    "d2h_bytes_per_step": args.n ** 3 * 4 * 8 * world / args.steps,
                    "note": "SlabDomain: node-type upload, init, warm-up + K steps with halos, moments download"},
            # per step: boundary planes (2 launches), interior (1), 2 packs, one unpack per neighbour
            "gpu_launches": args.steps * (5 + sum(x is not None for x in slab.neighbours(0, world, False))),
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def run_accuracy(args, rank, world, local_rank):
    """Full-size runs of one configuration in every storage format, each compared
    with the FP64-storage run of the same engine (which matches the FP64 oracle to
    1e-11 relative L2 on the parity cases): relative L2 over fluid nodes of velocity
    and density at the final step, plus the case's physical observable (kinetic
    energy for the vortex, outlet concentration and FP64 inventories for the bed)."""
    import math
    import torch
    from lbflow_b200 import _abi, cases
    from lbflow_b200.core import Storage
    from lbflow_b200.domain import Domain
    torch.cuda.set_device(local_rank)

    def rel(a, b):
        nb = float(np.linalg.norm(b))
        return float(np.linalg.norm(a - b)) / (nb if nb > 0 else 1.0)

    out = {"workload": f"accuracy {args.case}", "n_gpus": 1, "runs": {}}
    if args.case == "c2" and args.acc_curve:
        # the storages side by side: velocity error against FP64 at each listed step
        n = args.acc_n
        mask = geometry(n, args.seed, 0.7)
        fl = mask == 0
        marks = sorted(int(x) for x in args.acc_curve.split(","))
        stores = [Storage.F64, Storage.F32, Storage.F16DEV, Storage.BF16DEV]
        doms = {}
        for st in stores:
            d = Domain(cases.porous_channel_d3q19([n] * 3, mask=mask, force=1e-6, storage=st))
            if args.sround >= 0:
                d.set_option(_abi.LBF_OPT_SROUND, args.sround)
            doms[st] = d.init()
        out["case"] = (f"C2 geometry on {n}^3 (D3Q19 TRT tau+ 0.8 magic 1/4, g_x 1e-6, spheres r in [4,10], "
                       f"porosity 0.7, seed {args.seed})")
        out["sround"] = None if args.sround < 0 else args.sround
        out["curve"] = []
        t = 0
        for mark in marks:
            for d in doms.values():
                d.step(mark - t)
            t = mark
            ref = doms[Storage.F64].moments()[1][fl]
            row = {"step": mark}
            for st in stores[1:]:
                row[st.name] = rel(doms[st].moments()[1][fl], ref)
            out["curve"].append(row)
        for d in doms.values():
            d.close()
        print(json.dumps(out), flush=True)
        return
    if args.case == "c2":
        steps = args.acc_steps or 5000
        mask = geometry(256, args.seed, 0.7)
        stores = [Storage.F64, Storage.F32, Storage.F16DEV, Storage.BF16DEV]
        mk = lambda st: cases.porous_channel_d3q19([256] * 3, mask=mask, force=1e-6, storage=st)  # noqa: E731
        sample = []
    elif args.case == "c3":
        steps = args.acc_steps or 10000
        stores = [Storage.F64, Storage.F32, Storage.F16DEV]
        mk = lambda st: cases.tgv_d3q27(384, 0.05, args.c3_re, st, collision=args.c3_collision)[0]  # noqa: E731
        out["c3_re"] = args.c3_re
        out["c3_collision"] = args.c3_collision
        sample = list(range(0, steps + 1, 500))
    else:
        steps = args.acc_steps or 40000
        stores = [Storage.F64, Storage.F32]
        n = [192, 192, 384]
        # porosity 0.6 is below the jamming limit of non-overlapping random spheres,
        # so spheres may overlap; 8 clear layers at the inlet and the outlet keep the
        # Zou-He inlet from feeding closed pockets
        mask = cases.sphere_pack(n, 0.6, 4.0, 10.0, args.seed, overlap=True).reshape(n[2], n[1], n[0])
        mask[:8] = 0
        mask[-8:] = 0
        mask = mask.ravel()
        from lbflow_b200.core import BGK, TRT
        coll = {"bgk0.6": BGK(0.6), "bgk0.8": BGK(0.8), "trt0.8": TRT.from_magic(0.8, 0.25),
                "trt0.55": TRT.from_magic(0.55, 0.25)}[args.c4_collision]
        mk = lambda st: cases.packed_bed_scalar(n, mask=mask, storage=st, collision=coll, u_in=args.c4_u)  # noqa: E731
        out["c4"] = {"collision": args.c4_collision, "u_in": args.c4_u, "buffer_layers": 8}
        sample = list(range(0, steps + 1, 2000))
    ref = None
    for st in stores:
        p = mk(st)
        scal = None
        if isinstance(p, tuple):
            p, scal = p
        curve = []
        t_run = 0.0
        with Domain(p, scal) as d:
            d.init()
            cls, _ = d.node_class()
            fl = (cls & _abi.LBF_CLASS_SOLID) == 0
            t = 0
            for target in (sample if sample else [steps]):
                if target > t:
                    torch.cuda.synchronize()
                    t0 = time.perf_counter()
                    d.step(target - t)
                    torch.cuda.synchronize()
                    t_run += time.perf_counter() - t0
                    t = target
                if sample:
                    rho, u, c = d.moments()
                    if args.case == "c3":
                        curve.append(float(0.5 * np.sum(rho * np.sum(u * u, axis=1)) / rho.size))
                    else:
                        pl = n[0] * n[1]
                        out_fl = fl[-pl:]
                        inv = d.inventory()
                        curve.append([float(np.mean(c[-pl:][out_fl])), *[float(x) for x in inv]])
            rho, u, c = d.moments()
        n_fluid = int(np.count_nonzero(fl))
        run = {"mflups": n_fluid * steps / t_run / 1e6 if t_run > 0 else None, "steps": steps}
        if ref is None:
            ref = (rho[fl], u[fl], None if c is None else c[fl], curve)
        else:
            run["rel_l2_velocity"] = rel(u[fl], ref[1])
            run["rel_l2_density"] = rel(rho[fl], ref[0])
            run["rel_l2_density_deviation"] = rel(rho[fl] - 1.0, ref[0] - 1.0)
            if c is not None:
                run["rel_l2_scalar"] = rel(c[fl], ref[2])
            if args.case == "c3":
                e, e0 = np.array(curve), np.array(ref[3])
                run["energy_max_rel_dev"] = float(np.max(np.abs(e - e0) / e0))
            elif args.case == "c4":
                a, b = np.array(curve), np.array(ref[3])
                run["outlet_c_max_abs_dev"] = float(np.max(np.abs(a[:, 0] - b[:, 0])))
                run["inventory_max_rel_dev"] = [float(np.max(np.abs(a[:, k] - b[:, k]) /
                                                             np.maximum(np.abs(b[:, k]), 1e-300)))
                                                for k in range(1, a.shape[1])]
        if curve:
            run["curve_steps"] = sample
            run["curve"] = curve
        out["runs"][st.name] = run
    if args.case == "c3":
        nu = 0.05 * (384 / (2 * math.pi)) / args.c3_re
        k2 = 3 * (2 * math.pi / 384) ** 2
        e = np.array(out["runs"]["F64"]["curve"])
        out["c3_early_decay_vs_exp(-2 nu k^2 t)"] = float(abs(e[1] / e[0] - math.exp(-2 * nu * k2 * 500)) /
                                                          (1 - math.exp(-2 * nu * k2 * 500)))
    print(json.dumps(out), flush=True)


def run_batch_probe(args, rank, world, local_rank):
    """Batched sweep vs single-domain sweep on one large domain and on many small
    ones, and the host cost of one request's lifecycle (create, init, moments, destroy)."""
    import math
    import torch
    from lbflow_b200 import _abi, cases, serve
    from lbflow_b200.batch import Batch
    from lbflow_b200.core import Storage
    from lbflow_b200.domain import Domain
    torch.cuda.set_device(local_rank)
    sync = torch.cuda.synchronize
    out = {"workload": "batch probe", "n_gpus": 1}
    n = 192
    mask = cases.sphere_pack([n] * 3, 0.7, 4.0, 10.0, args.seed)
    nf = int(np.count_nonzero(mask == 0))
    for st in (Storage.F32, Storage.F16DEV):
        p = cases.porous_channel_d3q19([n] * 3, mask=mask, force=1e-6, storage=st)
        with Domain(p) as d:
            d.init().step(10)
            sync()
            t = time.perf_counter()
            d.step(200)
            sync()
            out[f"single_{st.name}_mflups_{n}"] = nf * 200 / (time.perf_counter() - t) / 1e6
        with Batch(0, 50) as b:
            d = Domain(p).init()
            b.admit(d, 10**6, math.inf, 0.0, math.inf)
            b.step(1)
            b.poll(wait=True)
            sync()
            t = time.perf_counter()
            b.step(4)
            b.poll(wait=True)
            sync()
            out[f"batched_{st.name}_mflups_{n}"] = nf * 200 / (time.perf_counter() - t) / 1e6
            b.evict(d)
            d.close()
    doms = [Domain(cases.cavity_d2q9(64, 0.6, 0.1, Storage.F32)).init() for _ in range(64)]
    for d in doms:
        d.step(1)
    sync()
    t = time.perf_counter()
    for d in doms:
        d.step(100)
    sync()
    out["small_64x64sq_single_domain_steps_per_s"] = 64 * 100 / (time.perf_counter() - t)
    with Batch(0, 50) as b:
        for d in doms:
            b.admit(d, 10**6, math.inf, 0.0, math.inf)
        # one launch per step (the default), then a group's chunk in one cooperative launch
        for chunk, key in ((0, "small_64x64sq_batched_domain_steps_per_s"),
                           (1, "small_64x64sq_batched_chunk_launch_domain_steps_per_s")):
            b.set_option(_abi.LBF_BATCH_OPT_CHUNK_LAUNCH, chunk)
            b.step(1)
            b.poll(wait=True)
            sync()
            t = time.perf_counter()
            b.step(2)
            b.poll(wait=True)
            sync()
            out[key] = 64 * 100 / (time.perf_counter() - t)
        for d in doms:
            b.evict(d)
    for d in doms:
        d.close()
    reqs = serve.make_requests(40, float("inf"), 77)
    serve.prepare(reqs)
    tc = ti = tm = tx = 0.0
    for r in reqs:
        t = time.perf_counter(); d = Domain(r.params); tc += time.perf_counter() - t
        t = time.perf_counter(); d.init(); sync(); ti += time.perf_counter() - t
        d.step(10)
        sync()
        t = time.perf_counter(); d.moments(); tm += time.perf_counter() - t
        t = time.perf_counter(); d.close(); tx += time.perf_counter() - t
    out["request_ms"] = {"create": 1e3 * tc / 40, "init": 1e3 * ti / 40, "moments": 1e3 * tm / 40,
                         "destroy": 1e3 * tx / 40}
    if rank == 0:
        print(json.dumps(out), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and args.impl == "engine":
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    if args.impl == "reference":
        run_reference(args, rank, world)
    elif args.workload == "serve":
        run_serve(args, rank, world, local_rank)
    elif args.workload == "batch":
        run_batch_probe(args, rank, world, local_rank)
    elif args.workload == "c3":
        run_c3(args, rank, world, local_rank)
    elif args.workload == "c4":
        run_c4(args, rank, world, local_rank)
    elif args.workload == "accuracy":
        run_accuracy(args, rank, world, local_rank)
    elif world > 1 and args.decomp == "slab":
        run_slabs(args, rank, world, local_rank)
    else:
        run_engine(args, rank, world, local_rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
