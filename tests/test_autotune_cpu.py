"""Autotuner host logic (no GPU): candidate sets, cache keys, cache round trip."""
import numpy as np

from lbflow_b200 import autotune, cases
from lbflow_b200.core import Storage


def test_candidates_and_key():
    mask = cases.sphere_pack([128, 16, 16], 0.7, 2.0, 3.0, seed=1)
    p = cases.porous_channel_d3q19([128, 16, 16], mask=mask, storage=Storage.F32)
    c = autotune.candidates(p)
    sweeps = [o["sweep"] for o in c]
    assert sweeps.count("dense") == 4 and {"stage", "pipe", "compact", "sparse"} <= set(sweeps)
    k1 = autotune.tuning_key(p)
    assert k1 == autotune.tuning_key(p) and "n128x16x16" in k1 and "s1" in k1
    cav = cases.cavity_d2q9(24, 0.6, 0.1, Storage.F64)      # explicit faces: no lean-only sweeps
    s2 = [o["sweep"] for o in autotune.candidates(cav)]
    assert "pipe" not in s2 and "compact" not in s2 and "sparse" not in s2


def test_cache_round_trip(tmp_path, monkeypatch):
    p = cases.cavity_d2q9(24, 0.6, 0.1, Storage.F32)
    calls = []

    def fake(params, scalar, opt, steps=20, warmup=3):
        calls.append(opt)
        return {"dense": 1.0 + 0.001 * opt.get("block_x", 0), "stage": 0.5}.get(opt["sweep"], 2.0)

    monkeypatch.setattr(autotune, "time_candidate", fake)
    path = str(tmp_path / "tune.json")
    best = autotune.autotune(p, cache=path)
    assert best["sweep"] == "stage" and not best["cached"]
    n = len(calls)
    again = autotune.autotune(p, cache=path)
    assert again["sweep"] == "stage" and again["cached"] and len(calls) == n
    assert np.isclose(best["ms_per_step"], 0.5)
