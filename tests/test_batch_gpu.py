"""Batches (lbf_batch_*): a domain computes the same fields and stops at the same
step alone (Domain.run) and in a mixed batch.

The mix covers every batched kernel shape: D2Q9 with explicit faces (Zou-He
lid, anti-bounce-back outlet), D3Q19 lean porous channels (FP64, FP32, FP16
deviation storage), D3Q27 MRT; some domains converge, others run to
max_iterations.  Tolerance: relative L2 over fluid nodes 1e-12 for FP64
storage, 1e-5 for FP32 / FP16 (the batched and single-domain sweeps are
different kernels around the same per-node code); step counts must be equal.
"""
import math

import numpy as np
import pytest

from lbflow_b200 import _abi, cases
from lbflow_b200 import momentum as m
from lbflow_b200.core import BGK, BoundaryFace, Storage, VelocitySet

pytestmark = pytest.mark.gpu

W, E, S, N = BoundaryFace.West, BoundaryFace.East, BoundaryFace.South, BoundaryFace.North
K = 10
MAX_IT = 600


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from lbflow_b200.batch import Batch, BatchFull
    from lbflow_b200.domain import Domain
    return Domain, Batch, BatchFull


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def _channel_d2q9():
    n = [40, 18]
    mask = np.zeros(n[0] * n[1], np.uint8).reshape(n[1], n[0])
    mask[6:11, 14:19] = 1
    return m.Parameters(n=n, collision_operator=BGK(0.7), velocity_set=VelocitySet.D2Q9,
                        boundary_conditions=[(W, m.ZouHe(None, [0.05, 0.0])), (E, m.AntiBounceBack(1.0)),
                                             (S, m.NoSlip), (N, m.NoSlip)],
                        node_types=m.NodeTypes.FromArray(mask.ravel()))


def _mix():
    out = [
        (cases.cavity_d2q9(12, 0.8, 0.01, Storage.F64), 1e-12),   # converges before MAX_IT
        (cases.cavity_d2q9(20, 0.6, 0.1, Storage.F32), 1e-5),
        (_channel_d2q9(), 1e-12),
        (cases.porous_channel_d3q19([16, 12, 10], mask=cases.sphere_pack([16, 12, 10], 0.7, 1.5, 2.5, 3),
                                    force=1e-5, storage=Storage.F64), 1e-12),
        (cases.porous_channel_d3q19([20, 16, 12], mask=cases.sphere_pack([20, 16, 12], 0.75, 1.5, 3.0, 5),
                                    force=1e-5, storage=Storage.F32), 1e-5),
        (cases.porous_channel_d3q19([24, 12, 12], mask=cases.sphere_pack([24, 12, 12], 0.8, 1.5, 2.5, 7),
                                    force=1e-5, storage=Storage.F16DEV), 1e-5),
        (cases.tgv_d3q27(12, 0.05, 20.0, Storage.F64)[0], 1e-12),
    ]
    return out


def _alone(Domain, p, tol=1e-7):
    with Domain(p) as d:
        d.init()
        steps = d.run(MAX_IT, K, tol, tol, tol)
        rho, u, _ = d.moments()
        cls, _ = d.node_class()
    return steps, rho, u, (cls & _abi.LBF_CLASS_SOLID) == 0


def _drain(batch, live):
    got = {}
    for _ in range(10 * MAX_IT):
        if not live:
            break
        batch.step(1)
        for dom, status in batch.poll(wait=True):
            key = live.pop(dom.h.value)
            rho, u, _ = dom.moments()
            got[key] = (dom.time_step, rho, u, status)
            dom.close()
    assert not live
    return got


def test_batch_mix_matches_alone(env):
    Domain, Batch, _ = env
    mix = _mix()
    alone = [_alone(Domain, p) for p, _ in mix]
    assert alone[0][0] < MAX_IT and alone[1][0] == MAX_IT + 2
    with Batch(0, K) as batch:
        live = {}
        for i, (p, _) in enumerate(mix):
            d = Domain(p).init()
            batch.admit(d, MAX_IT, 1e-7, 1e-7, 1e-7)
            live[d.h.value] = i
        got = _drain(batch, live)
    for i, (p, tol) in enumerate(mix):
        steps, rho, u, fl = alone[i]
        gs, gr, gu, status = got[i]
        assert gs == steps, (i, gs, steps)
        assert status == (1 if steps <= MAX_IT + 1 else 2)
        assert rel(gr[fl], rho[fl]) <= tol and rel(gu[fl], u[fl]) <= tol, i


def test_batch_late_admission_and_phase(env):
    """Domains admitted after 7 standalone steps, and while others run, end where
    a standalone run from t = 0 ends."""
    Domain, Batch, _ = env
    p1 = cases.cavity_d2q9(12, 0.8, 0.01, Storage.F64)
    p2 = cases.cavity_d2q9(16, 0.7, 0.05, Storage.F64)
    a1, a2 = _alone(Domain, p1), _alone(Domain, p2)
    with Batch(0, K) as batch:
        d1 = Domain(p1).init()
        batch.admit(d1, MAX_IT, 1e-7, 1e-7, 1e-7)
        live = {d1.h.value: 1}
        batch.step(3)
        assert batch.poll(wait=True) == []
        d2 = Domain(p2).init()
        d2.step(7, K)
        batch.admit(d2, MAX_IT, 1e-7, 1e-7, 1e-7)
        live[d2.h.value] = 2
        got = _drain(batch, live)
    for key, a in ((1, a1), (2, a2)):
        gs, gr, gu, _ = got[key]
        assert gs == a[0]
        assert rel(gr[a[3]], a[1][a[3]]) <= 1e-12 and rel(gu[a[3]], a[2][a[3]]) <= 1e-12


def test_batch_budget_and_state(env):
    Domain, Batch, BatchFull = env
    from lbflow_b200.batch import estimate_bytes
    p = cases.cavity_d2q9(32, 0.6, 0.1, Storage.F32)
    with Domain(p) as d:
        d.init()
        assert estimate_bytes(p) >= d.device_bytes
        with Batch(d.device_bytes // 2, K) as small:
            with pytest.raises(BatchFull):
                small.admit(d, 100)
        with Batch(0, K) as batch:
            batch.admit(d, 100)
            with pytest.raises(_abi.LbfError) as ei:
                d.step(1)
            assert ei.value.status == _abi.LBF_ESTATE
            batch.step(2)
            batch.evict(d)
            t = d.time_step
            assert t == 21            # one phase-alignment step + 2 chunks of 10
            d.step(5)                 # standalone again
            assert d.time_step == 26


def test_batch_many_small_domains(env):
    """40 small domains of two configurations in one batch, all to max_iterations."""
    Domain, Batch, _ = env
    ps_ = [cases.cavity_d2q9(8 + (i % 7), 0.6, 0.1, Storage.F32) for i in range(20)]
    ps_ += [cases.porous_channel_d3q19([8 + i % 5, 8, 8], mask=np.zeros((8 + i % 5) * 64, np.uint8), force=1e-5,
                                       storage=Storage.F32) for i in range(20)]
    with Batch(0, 20) as batch:
        live = {}
        for i, p in enumerate(ps_):
            d = Domain(p).init()
            batch.admit(d, 98, math.inf, 1e-12, math.inf)
            live[d.h.value] = i
        got = {}
        while live:
            batch.step(2)
            for dom, status in batch.poll(wait=True):
                got[live.pop(dom.h.value)] = (dom.time_step, status, dom.moments()[0])
                dom.close()
    for i, p in enumerate(ps_):
        with Domain(p) as d:
            d.init()
            d.step(100)
            rho = d.moments()[0]
        assert got[i][0] == 100 and got[i][1] == 2
        assert rel(got[i][2], rho) <= 1e-5


def test_batch_large_members_run_their_own_sweep(env):
    """Members above SOLO_UNITS (2^19 nodes, or fluid nodes in the sparse layout)
    run the single-domain sweep inside the chunk graph, gated by their batch state;
    small members share the batched launches.  Same fields and steps as alone."""
    Domain, Batch, _ = env
    mask = cases.sphere_pack([96, 96, 96], 0.7, 3.0, 6.0, seed=4)
    mix = [
        (cases.porous_channel_d3q19([96, 96, 96], mask=mask, force=1e-5, storage=Storage.F32), 1e-5),  # sparse, solo
        (cases.cavity_d2q9(768, 0.6, 0.1, Storage.F32), 1e-5),                                        # dense faces, solo
        (cases.cavity_d2q9(12, 0.8, 0.01, Storage.F64), 1e-12),                                       # small, converges
        (cases.cavity_d2q9(40, 0.6, 0.1, Storage.F32), 1e-5),                                         # small
    ]
    max_it = 300
    alone = []
    for p, _ in mix:
        with Domain(p) as d:
            d.init()
            steps = d.run(max_it, K, 1e-7, 1e-7, 1e-7)
            rho, u, _ = d.moments()
            cls, _ = d.node_class()
        alone.append((steps, rho, u, (cls & _abi.LBF_CLASS_SOLID) == 0))
    with Batch(0, K) as batch:
        live = {}
        for i, (p, _) in enumerate(mix):
            d = Domain(p).init()
            batch.admit(d, max_it, 1e-7, 1e-7, 1e-7)
            live[d.h.value] = i
        got = {}
        for _ in range(200):
            if not live:
                break
            batch.step(2)
            for dom, status in batch.poll(wait=True):
                rho, u, _ = dom.moments()
                got[live.pop(dom.h.value)] = (dom.time_step, rho, u)
                dom.close()
    assert not live
    for i, (p, tol) in enumerate(mix):
        steps, rho, u, fl = alone[i]
        gs, gr, gu = got[i]
        assert gs == steps, (i, gs, steps)
        assert rel(gr[fl], rho[fl]) <= tol and rel(gu[fl], u[fl]) <= tol, i


def _scalar_mix():
    """Members the batched kernels do not cover, which run their own sweep in the
    chunk graph: a D2Q9 channel with a scalar (dense layout), a packed bed with
    two scalars (sparse layout, outflow face pass), a D3Q27 central-moment vortex;
    plus a small lean cavity in a batched launch beside them."""
    from lbflow_b200 import passive_scalar as ps
    from lbflow_b200.core import TRT
    ch = _channel_d2q9()
    s_ch = ps.Parameters(scalar_name="c", collision_operator=BGK(0.6), velocity_set=VelocitySet.D2Q9,
                         initial_scalar_value=ps.InitialScalarValue.Uniform(0.0),
                         boundary_conditions=[(W, ps.AntiBounceBack(1.0)), (E, ps.AntiBBNoFlux),
                                              (S, ps.BBNoFlux), (N, ps.BBNoFlux)],
                         inner_boundary_condition=ps.InnerBounceBack)
    n = [14, 12, 24]
    bed, s0 = cases.packed_bed_scalar(n, mask=cases.sphere_pack(n, 0.7, 1.5, 2.5, seed=4), storage=Storage.F32,
                                      ka=1e-2)
    s1 = ps.Parameters(scalar_name="tracer", collision_operator=TRT.from_magic(0.7), velocity_set=VelocitySet.D3Q19,
                       initial_scalar_value=ps.InitialScalarValue.Uniform(0.1),
                       boundary_conditions=[(W, ps.BBNoFlux), (E, ps.BBNoFlux), (S, ps.BBNoFlux), (N, ps.BBNoFlux),
                                            (BoundaryFace.Bottom, ps.AntiBounceBack(0.5)),
                                            (BoundaryFace.Top, ps.SecondOrderNoFlux(unknown_populations_only=False))],
                       inner_boundary_condition=ps.InnerBounceBack)
    return [(ch, [s_ch], 1e-12), (bed, [s0, s1], 1e-5),
            (cases.tgv_d3q27(12, 0.05, 20.0, Storage.F64, collision="central")[0], None, 1e-12),
            (cases.cavity_d2q9(20, 0.6, 0.1, Storage.F32), None, 1e-5)]


def test_batch_scalar_and_central_domains_match_alone(env):
    Domain, Batch, _ = env
    mix = _scalar_mix()
    max_it = 200
    alone = []
    for p, sps, _ in mix:
        with Domain(p, sps) as d:
            d.init()
            steps = d.run(max_it, K, 1e-7, 1e-7, 1e-7)
            rho, u, _ = d.moments()
            cs = [d.scalar(i) for i in range(d.num_scalars)]
            res, _ = d.residuals()
            cls, _ = d.node_class()
        alone.append((steps, rho, u, cs, res, (cls & _abi.LBF_CLASS_SOLID) == 0))
    with Batch(0, K) as batch:
        live = {}
        for i, (p, sps, _) in enumerate(mix):
            d = Domain(p, sps).init()
            batch.admit(d, max_it, 1e-7, 1e-7, 1e-7)
            live[d.h.value] = (i, d)
        got = {}
        for _ in range(200):
            if not live:
                break
            batch.step(2)
            for dom, status in batch.poll(wait=True):
                i, d = live.pop(dom.h.value)
                rho, u, _ = d.moments()
                got[i] = (d.time_step, rho, u, [d.scalar(j) for j in range(d.num_scalars)], d.residuals()[0])
                d.close()
    assert not live
    for i, (p, sps, tol) in enumerate(mix):
        steps, rho, u, cs, res, fl = alone[i]
        gs, gr, gu, gc, gres = got[i]
        assert gs == steps, (i, gs, steps)
        assert rel(gr[fl], rho[fl]) <= tol and rel(gu[fl], u[fl]) <= tol, i
        assert len(gc) == len(cs) and len(gres) == len(res)
        for a, b in zip(gc, cs):
            assert rel(a[fl], b[fl]) <= tol, i
        assert np.allclose(gres, res, rtol=1e-9, atol=0), i


def test_batch_scalar_domain_needs_even_interval(env):
    Domain, Batch, _ = env
    p, sps, _ = _scalar_mix()[0]
    with Batch(0, 5) as batch, Domain(p, sps) as d:
        d.init()
        with pytest.raises(RuntimeError, match="EUNSUPPORTED"):
            batch.admit(d, 100)


def test_batch_chunk_launch_equals_step_launches(env):
    """A group's chunk in one cooperative launch (grid barriers between the steps)
    and one launch per step give the same bits and the same stop steps, for dense
    and sparse groups, with domains joining late."""
    Domain, Batch, _ = env
    mix = [p for p, _ in _mix()]
    got = []
    for chunk in (1, 0):
        with Batch(0, K) as batch:
            batch.set_option(_abi.LBF_BATCH_OPT_CHUNK_LAUNCH, chunk)
            live = {}
            for i, p in enumerate(mix):
                d = Domain(p).init()
                if i % 2:
                    d.step(3)          # joins at another phase
                batch.admit(d, MAX_IT, 1e-7, 1e-7, 1e-7)
                live[d.h.value] = i
            got.append(_drain(batch, live))
    a, b = got
    for i in range(len(mix)):
        assert a[i][0] == b[i][0] and a[i][3] == b[i][3], i
        assert np.array_equal(a[i][1], b[i][1]) and np.array_equal(a[i][2], b[i][2]), i
