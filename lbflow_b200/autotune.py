"""Autotuner for the step kernel's launch shape and sweep variant.

The best sweep depends on the lattice: the dense sweep with 256-thread blocks
suits large lattices, narrow rows want smaller blocks, FP64 porous media prefer
the compacted fluid work list, and the staged / pipelined bulk-copy sweeps win on
some row lengths.  `autotune(params)` times each candidate on a scratch domain
built from the same parameters (a few warm-up steps, then CUDA-event timing over
`steps` steps), returns the fastest option set, and caches it by the lattice's
key (velocity set, collision, storage, faces, scalar, size, solid fraction)
in a JSON file.  `apply(domain, options)` sets them on a domain before init.

Candidates (options of include/lbflow.h):
  dense sweep, LBF_OPT_BLOCK_X in {32, 64, 128, 256};
  staged rows (LBF_OPT_STAGE) where rows are 16-byte aligned and nx <= 512;
  pipelined rows (LBF_OPT_PIPE) on the lean path;
  compacted fluid work list (LBF_OPT_COMPACT) on the lean path;
  fluid-only population layout (LBF_OPT_SPARSE) on the lean path.
All candidates compute the same values (tests/test_autotune_gpu.py).
"""
from __future__ import annotations

import json
import os
import threading
from typing import Dict, List, Optional

import numpy as np

from . import _abi
from . import momentum as _m
from . import passive_scalar as _ps

_LOCK = threading.Lock()
DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "lbflow_b200", "autotune.json")


def tuning_key(params: _m.Parameters, scalar: Optional[_ps.Parameters] = None) -> str:
    """Cache key: what the kernel choice depends on."""
    desc, _ = _m.to_desc(params)
    n = [int(desc.n[a]) for a in range(3)]
    mask = params.node_types.generate(params.n[: params.dim])
    solid = 0.0 if mask is None else float(np.mean(np.asarray(mask) != 0))
    faces = "".join(str(int(desc.bc[f].kind)) for f in range(6))
    return (f"vs{desc.velocity_set}-c{desc.collision.kind}-s{desc.storage}-f{faces}-"
            f"sc{1 if scalar is not None else 0}-n{n[0]}x{n[1]}x{n[2]}-solid{round(solid, 2):.2f}")


def candidates(params: _m.Parameters, scalar: Optional[_ps.Parameters] = None) -> List[Dict[str, int]]:
    desc, _ = _m.to_desc(params)
    lean = scalar is None and all(int(desc.bc[f].kind) in (_abi.LBF_BC_NO_SLIP, _abi.LBF_BC_PERIODIC)
                                  for f in range(6))
    nx = int(desc.n[0])
    out = [{"sweep": "dense", "block_x": b} for b in (32, 64, 128, 256) if b <= max(32, 2 * nx)]
    esz = {0: 8, 1: 4, 2: 2, 3: 2}[int(desc.storage)]
    if nx <= 512 and (nx * esz) % 16 == 0:
        out.append({"sweep": "stage"})
    if lean and (nx * esz) % 16 == 0:
        out.append({"sweep": "pipe"})
    if lean:
        out.append({"sweep": "compact"})
        out.append({"sweep": "sparse"})
    return out


def apply(dom, opt: Dict) -> None:
    """Set a tuned option set on a domain (before lbf_domain_init)."""
    sweep = opt.get("sweep", "dense")
    dom.set_option(_abi.LBF_OPT_COMPACT, 1 if sweep == "compact" else 0)
    dom.set_option(_abi.LBF_OPT_STAGE, 1 if sweep == "stage" else 0)
    dom.set_option(_abi.LBF_OPT_PIPE, 1 if sweep == "pipe" else 0)
    dom.set_option(_abi.LBF_OPT_SPARSE, 1 if sweep == "sparse" else 0)
    dom.set_option(_abi.LBF_OPT_BLOCK_X, int(opt.get("block_x", 0)) if sweep == "dense" else 0)


def _load(path: str) -> dict:
    try:
        with open(path) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store(path: str, table: dict) -> None:
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as fh:
        json.dump(table, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def time_candidate(params, scalar, opt, steps: int = 20, warmup: int = 3) -> float:
    """Milliseconds per step of one candidate on a scratch domain."""
    import torch
    from .domain import Domain
    with Domain(params, scalar) as d:
        apply(d, opt)
        d.init()
        d.step(warmup)
        s = torch.cuda.current_stream()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(s)
        d.step(steps, 0, s)
        b.record(s)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / steps


def autotune(params: _m.Parameters, scalar: Optional[_ps.Parameters] = None, steps: int = 20,
             cache: Optional[str] = DEFAULT_CACHE, force: bool = False) -> Dict:
    """The fastest option set for this lattice (cached by tuning_key)."""
    key = tuning_key(params, scalar)
    with _LOCK:
        table = _load(cache) if cache else {}
        if not force and key in table:
            return dict(table[key]["best"], cached=True)
    timings = []
    for opt in candidates(params, scalar):
        try:
            timings.append((time_candidate(params, scalar, opt, steps), opt))
        except _abi.LbfError:
            continue   # a candidate the library refuses for this shape
    if not timings:
        return {"sweep": "dense", "block_x": 0}
    timings.sort(key=lambda x: x[0])
    best = timings[0][1]
    if cache:
        with _LOCK:
            table = _load(cache)
            table[key] = {"best": best, "ms_per_step": [[ms, o] for ms, o in timings]}
            _store(cache, table)
    return dict(best, cached=False, ms_per_step=timings[0][0])
