"""Autotuner on the GPU: every candidate computes the same fields, and the tuned
choice is one of them and is cached."""
import numpy as np
import pytest

from lbflow_b200 import autotune, cases
from lbflow_b200.core import Storage

pytestmark = pytest.mark.gpu


def test_autotune_porous_channel(tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from lbflow_b200.domain import Domain
    mask = cases.sphere_pack([64, 24, 20], 0.7, 2.0, 3.5, seed=2)
    p = cases.porous_channel_d3q19([64, 24, 20], mask=mask, force=1e-5, storage=Storage.F32)
    path = str(tmp_path / "tune.json")
    best = autotune.autotune(p, steps=10, cache=path)
    cands = autotune.candidates(p)
    assert {k: v for k, v in best.items() if k in ("sweep", "block_x")} in cands
    assert autotune.autotune(p, cache=path)["cached"]
    ref = None
    for opt in cands:
        with Domain(p) as d:
            autotune.apply(d, opt)
            d.init().step(50)
            rho, u, _ = d.moments()
        if ref is None:
            ref = (rho, u)
        else:
            assert np.allclose(rho, ref[0], rtol=1e-6, atol=1e-7), opt
            assert np.allclose(u, ref[1], rtol=1e-4, atol=1e-8), opt
