"""Reference-format inputs and restarts on the GPU, against the oracle.

- A 3-D map.xyz in the layout the reference reads (src/io.rs:121-143; written as
  aux/image_pre_processing.py:42-56 writes each slice) drives
  NodeTypes.FromBounceBackMapFile: node classes and link masks agree exactly
  with the oracle, and the fields after 120 steps agree to FP64 rounding.
- FromTimeStep restart (src/momentum/io.rs:358-394): `solve` writes data/<t>/
  from the GPU run; a second case starts from those files
  (InitialDensity/InitialVelocity::FromTimeStep(t), populations at the
  equilibrium of the read fields, time step counting from 0 again) and is
  compared with the oracle started from the same files.
"""
import os

import numpy as np
import pytest

from lbflow_b200 import _abi, cases
from lbflow_b200 import momentum as m
from lbflow_b200.core import Storage

pytestmark = pytest.mark.gpu

TOL64 = 1e-9


@pytest.fixture(scope="module")
def Domain():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from lbflow_b200.domain import Domain as D
    return D


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def oracle(params, steps):
    from oracle import oracle as orc
    desc, keep = m.to_desc(params)
    return orc.Domain(desc, keep=keep).init().step(steps)


def test_map_xyz_porous_channel(Domain, tmp_path, monkeypatch):
    n = [30, 18, 14]
    solid = cases.sphere_pack(n, 0.7, 1.5, 3.5, seed=21).reshape(n[2], n[1], n[0])
    os.makedirs(tmp_path / "pre_processing")
    with open(tmp_path / "pre_processing" / "map.xyz", "w") as fh:
        for z in range(n[2]):
            if z:
                fh.write("\n")
            for y in range(n[1] - 1, -1, -1):          # image row 0 = y = ny - 1
                fh.write(" ".join(str(int(v)) for v in solid[z, y]) + "\n")
    monkeypatch.chdir(tmp_path)
    p = cases.porous_channel_d3q19(n, mask=solid.ravel(), force=1e-5, storage=Storage.F64)
    p.node_types = m.NodeTypes.FromBounceBackMapFile
    od = oracle(p, 120)
    with Domain(p) as d:
        cls_g, links_g = d.node_class()
        d.init().step(120)
        rg, ug, _ = d.moments()
    cls_o, links_o = od.node_class()
    assert np.array_equal(cls_g, cls_o) and np.array_equal(links_g, links_o)
    assert np.array_equal((cls_g & _abi.LBF_CLASS_SOLID) != 0, solid.ravel() == 1)
    ro, uo, _ = od.observe()
    fl = solid.ravel() == 0
    assert rel(rg[fl], ro[fl]) <= TOL64 and rel(ug[fl], uo[fl]) <= TOL64


@pytest.mark.parametrize("storage", [Storage.F64, Storage.F32])
def test_from_time_step_restart(Domain, tmp_path, monkeypatch, storage):
    from lbflow_b200.solver import solve
    monkeypatch.chdir(tmp_path)
    first = cases.cavity_d2q9(40, 0.6, 0.1, storage)
    solve(first, write_data=150, max_iterations=299, verbose=False)   # writes data/0, 150, 300
    assert os.path.exists(os.path.join("data", "300", "density.csv"))
    # the written step matches the oracle at t = 300
    ro, uo, _ = oracle(cases.cavity_d2q9(40, 0.6, 0.1, Storage.F64), 300).observe()
    from lbflow_b200 import io
    rf = io.read_scalar_csv(os.path.join("data", "300", "density.csv"))
    uf = io.read_vector_csv(os.path.join("data", "300", "velocity.csv"))
    tol = 1e-8 if storage == Storage.F64 else 1e-4     # {:.8e} text; FP32 deviations
    assert rel(rf, ro) <= tol and rel(uf, uo) <= tol
    # restart from the files
    again = cases.cavity_d2q9(40, 0.6, 0.1, storage)
    again.initial_density = m.InitialDensity.FromTimeStep(300)
    again.initial_velocity = m.InitialVelocity.FromTimeStep(300)
    ref = cases.cavity_d2q9(40, 0.6, 0.1, Storage.F64)
    ref.initial_density = m.InitialDensity.FromTimeStep(300)
    ref.initial_velocity = m.InitialVelocity.FromTimeStep(300)
    od = oracle(ref, 200)
    with Domain(again) as d:
        d.init()
        r0, u0, _ = d.moments()                        # before the first step: the files' fields
        d.step(200)
        assert d.time_step == 200
        rg, ug, _ = d.moments()
    assert rel(r0, rf) <= (1e-15 if storage == Storage.F64 else 1e-7)
    ro2, uo2, _ = od.observe()
    tol_u = TOL64 if storage == Storage.F64 else 1e-4
    assert rel(rg, ro2) <= tol_u and rel(ug, uo2) <= tol_u
