"""The central-moment collision (D2Q9, D3Q27) on the GPU against the oracle's
restatement of the same definition (no reference counterpart exists), plus the
physics it must reproduce:
- parity: FP64 storage to 1e-9, FP32 deviation storage to 1e-4 relative L2, in
  the dense and the sparse layouts, with a body force and with walls;
- the Taylor-Green vortex decays at 2 nu k^2 per step with nu = (tau - 1/2) / 3
  (low Reynolds number), as with BGK at the same tau;
- at tau = 0.5057 (the Re = 1600 vortex on 384^3 has this tau) a vortex with the
  same tau stays finite and loses energy over 2,000 steps on 96^3, in FP32 and
  FP64.
"""
import math

import numpy as np
import pytest

from lbflow_b200 import _abi, cases
from lbflow_b200 import momentum as m
from lbflow_b200.core import BGK, BoundaryFace, CentralMoment, Storage, VelocitySet

pytestmark = pytest.mark.gpu

W, E, S, N, B, T = (BoundaryFace.West, BoundaryFace.East, BoundaryFace.South, BoundaryFace.North,
                    BoundaryFace.Bottom, BoundaryFace.Top)


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


def _oracle(p, steps):
    from oracle import oracle as orc
    desc, keep = m.to_desc(p)
    return orc.Domain(desc, keep=keep).init().step(steps)


def _channel(vs, storage, porous):
    d = vs.d
    n = [24, 14] if d == 2 else [16, 12, 10]
    mask = None
    if porous:
        rng = np.random.default_rng(9)
        mask = (rng.random(int(np.prod(n))) < 0.15).astype(np.uint8)
    faces = [W, E, S, N, B, T][: 2 * d]
    bcs = [(f, m.Periodic if i < 2 else m.NoSlip) for i, f in enumerate(faces)]
    return m.Parameters(n=n, collision_operator=CentralMoment(0.62, 1.1, (1.0, 1.2, 0.9, 1.0)), velocity_set=vs,
                        force=[2e-5, 0.0] + ([1e-5] if d == 3 else []), storage=storage,
                        initial_velocity=m.InitialVelocity.Uniform([0.0] * d), boundary_conditions=bcs,
                        node_types=m.NodeTypes.FromArray(mask) if porous else m.NodeTypes.OnlyFluidNodes)


@pytest.mark.parametrize("vs", [VelocitySet.D2Q9, VelocitySet.D3Q27])
@pytest.mark.parametrize("storage", [Storage.F64, Storage.F32])
@pytest.mark.parametrize("porous", [False, True])
def test_central_matches_oracle(Domain, vs, storage, porous):
    p = _channel(vs, storage, porous)
    steps = 150
    ro, uo, _ = _oracle(_channel(vs, Storage.F64, porous), steps).observe()
    with Domain(p) as d:
        d.init().step(steps)
        assert d.get_option(_abi.LBF_OPT_SPARSE) == (1 if porous else 0)
        rg, ug, _ = d.moments()
        cls, _ = d.node_class()
    fl = (cls & _abi.LBF_CLASS_SOLID) == 0
    tol = 1e-9 if storage == Storage.F64 else 1e-4
    assert rel(ug[fl], uo[fl]) <= tol and rel(rg[fl], ro[fl]) <= tol


def test_central_tgv_matches_oracle(Domain):
    p, _ = cases.tgv_d3q27(24, 0.05, 100.0, Storage.F64, collision="central")
    ro, uo, _ = _oracle(p, 60).observe()
    with Domain(p) as d:
        d.init().step(60)
        rg, ug, _ = d.moments()
    assert rel(ug, uo) <= 1e-9 and rel(rg, ro) <= 1e-9


def test_central_tgv_viscous_decay(Domain):
    """Shear viscosity (tau - 1/2) / 3: after the start-up transient the vortex
    energy decays at 2 nu k^2 per step, as with BGK at the same tau."""
    n, u0, tau = 32, 0.005, 0.6
    nu = (tau - 0.5) / 3
    re = u0 * (n / (2 * math.pi)) / nu
    k2 = 3 * (2 * math.pi / n) ** 2

    def rate(p):
        with Domain(p) as d:
            d.init().step(100)
            r, u, _ = d.moments()
            e1 = np.sum(r * np.sum(u * u, axis=1))
            d.step(200)
            r, u, _ = d.moments()
            e2 = np.sum(r * np.sum(u * u, axis=1))
        return -math.log(e2 / e1) / 200
    p, nu_p = cases.tgv_d3q27(n, u0, re, Storage.F64, collision="central")
    assert abs(nu_p - nu) < 1e-12
    pb = m.Parameters(n=[n] * 3, collision_operator=BGK(tau), velocity_set=VelocitySet.D3Q27,
                      initial_velocity=p.initial_velocity, boundary_conditions=p.boundary_conditions)
    r_cm, r_bgk = rate(p), rate(pb)
    assert abs(r_cm - 2 * nu * k2) / (2 * nu * k2) < 0.02
    assert abs(r_cm - r_bgk) / r_bgk < 0.005


@pytest.mark.parametrize("storage", [Storage.F64, Storage.F32])
def test_central_stable_at_tau_05057(Domain, storage):
    # tau of the Re = 1600 vortex on 384^3 (u0 = 0.05): nu = u0 n / (2 pi Re), tau = 3 nu + 1/2
    nu384 = 0.05 * 384 / (2 * math.pi) / 1600
    n = 96
    re = 0.05 * n / (2 * math.pi) / nu384        # same tau on the smaller lattice
    p, nu = cases.tgv_d3q27(n, 0.05, re, storage, collision="central")
    assert abs(3 * nu + 0.5 - (3 * nu384 + 0.5)) < 1e-12
    with Domain(p) as d:
        d.init().step(2000)
        r, u, _ = d.moments()
    assert np.all(np.isfinite(u)) and np.all(np.isfinite(r))
    e = 0.5 * np.sum(r * np.sum(u * u, axis=1)) / r.size
    assert 0 < e < 0.05 ** 2 / 8                    # below the initial mean energy u0^2 / 8


def test_central_refused_for_d3q19(Domain):
    p = m.Parameters(n=[8, 8, 8], collision_operator=CentralMoment(0.6), velocity_set=VelocitySet.D3Q19,
                     boundary_conditions=[(f, m.Periodic) for f in (W, E, S, N, B, T)])
    with pytest.raises(_abi.LbfError) as ei:
        Domain(p)
    assert ei.value.status == _abi.LBF_EUNSUPPORTED
