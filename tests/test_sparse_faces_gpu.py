"""The sparse (fluid-only) layout with explicit face BCs and the passive scalar.

Each case runs in the sparse layout (LBF_OPT_SPARSE 1) and in the dense layout
(LBF_OPT_SPARSE 0) and is compared with the FP64 oracle: node classes exactly,
moments, scalar and adsorbed amount to 1e-9 relative L2 in FP64 storage (1e-3 /
1e-4 in FP32); the two layouts agree with each other to 1e-12 (FP64).  The cases
cover Zou-He velocity and pressure faces, anti-bounce-back and moving-wall faces,
the scalar's anti-bounce-back, no-flux and extrapolation-outflow faces, both
inner scalar rules (with a per-node initial scalar for the anti-bounce-back
one), Langmuir adsorption, residuals, inventories and a checkpoint resume.
"""
import numpy as np
import pytest

from lbflow_b200 import _abi, cases
from lbflow_b200 import momentum as m
from lbflow_b200 import passive_scalar as ps
from lbflow_b200.core import BGK, TRT, BoundaryFace, Storage, VelocitySet

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


def _bed(storage):
    mask = cases.sphere_pack([14, 12, 24], 0.7, 1.5, 2.5, seed=4)
    return cases.packed_bed_scalar([14, 12, 24], mask=mask, storage=storage, ka=1e-2)


def _channel_d2q9(inner, c_field=False):
    n = [40, 18]
    rng = np.random.default_rng(3)
    mask = (rng.random(n[0] * n[1]) < 0.12).astype(np.uint8).reshape(n[1], n[0])
    mask[:, :2] = 0
    mask[:, -3:] = 0
    mp = m.Parameters(n=n, collision_operator=BGK(0.7), velocity_set=VelocitySet.D2Q9,
                      boundary_conditions=[(W, m.ZouHe(None, [0.04, 0.0])), (E, m.AntiBounceBack(1.0)),
                                           (S, m.NoSlip), (N, m.BounceBack(1.0, [0.02, 0.0]))],
                      node_types=m.NodeTypes.FromArray(mask.ravel()))
    init = (ps.InitialScalarValue.FromArray(0.1 + 0.3 * rng.random(n[0] * n[1])) if c_field
            else ps.InitialScalarValue.Uniform(0.2))
    sp = ps.Parameters(scalar_name="c", collision_operator=BGK(0.55), velocity_set=VelocitySet.D2Q9,
                       initial_scalar_value=init,
                       boundary_conditions=[(W, ps.AntiBounceBack(1.0)),
                                            (E, ps.SecondOrderNoFlux(unknown_populations_only=True)),
                                            (S, ps.BBNoFlux), (N, ps.AntiBBNoFlux)],
                       inner_boundary_condition=inner,
                       adsorption_parameters=ps.AdsorptionParameters(ps.Langmuir(1e-2, 1e-4, 1.0), 0.1))
    return mp, sp


def _duct(vs, coll, storage):
    n = [18, 10, 9]
    mask = cases.sphere_pack(n, 0.8, 1.5, 2.0, seed=12)
    mask.reshape(n[2], n[1], n[0])[:, :, :2] = 0
    mask.reshape(n[2], n[1], n[0])[:, :, -2:] = 0
    return m.Parameters(n=n, collision_operator=coll, velocity_set=vs, storage=storage,
                        initial_velocity=m.InitialVelocity.Uniform([0, 0, 0]),
                        boundary_conditions=[(W, m.ZouHe(None, [0.03, 0.0, 0.0])), (E, m.ZouHe(1.0, [None, 0.0, 0.0])),
                                             (S, m.NoSlip), (N, m.NoSlip), (B, m.BounceBack(1.0, [0.01, 0.0, 0.0])),
                                             (T, m.NoSlip)],
                        node_types=m.NodeTypes.FromArray(mask))


CASES = {
    "bed_scalar_f64": (lambda: _bed(Storage.F64), 160, Storage.F64),
    "bed_scalar_f32": (lambda: _bed(Storage.F32), 160, Storage.F32),
    "channel_d2q9_inner_bb": (lambda: _channel_d2q9(ps.InnerBounceBack), 300, Storage.F64),
    "channel_d2q9_inner_anti_bb_field": (lambda: _channel_d2q9(ps.InnerAntiBounceBack, c_field=True), 300,
                                         Storage.F64),
    "duct_d3q19_trt": (lambda: (_duct(VelocitySet.D3Q19, TRT(1.25, 0.75), Storage.F64), None), 200, Storage.F64),
    "duct_d3q27_bgk_f32": (lambda: (_duct(VelocitySet.D3Q27, BGK(0.7), Storage.F32), None), 200, Storage.F32),
}


def _run(Domain, mp, sp, steps, sparse):
    with Domain(mp, sp) as d:
        d.set_option(_abi.LBF_OPT_SPARSE, 1 if sparse else 0)
        d.init()
        assert d.get_option(_abi.LBF_OPT_SPARSE) == (1 if sparse else 0)
        assert d.get_option(_abi.LBF_OPT_STREAMING) == _abi.LBF_STREAM_PULL
        d.step(steps - 1, residual_interval=1).step(1, residual_interval=1)
        rho, u, c = d.moments()
        res, t = d.residuals()
        inv = d.inventory()
        q = d.q_ads() if sp is not None else None
        cls, links = d.node_class()
    return rho, u, c, q, res, t, inv, cls, links


@pytest.mark.parametrize("name", list(CASES))
def test_sparse_faces_match_oracle_and_dense(Domain, name):
    from oracle import oracle as orc
    make, steps, storage = CASES[name]
    mp, sp = make()
    desc, keep = m.to_desc(mp)
    sdesc = None
    if sp is not None:
        sdesc, k2 = ps.to_desc(sp, mp.n[: mp.dim])
        keep += k2
    od = orc.Domain(desc, sdesc, keep=keep).init().step(steps)
    ro, uo, co = od.observe()
    sp_ = _run(Domain, mp, sp, steps, True)
    dn_ = _run(Domain, mp, sp, steps, False)
    cls_o, links_o = od.node_class()
    fl = (cls_o & _abi.LBF_CLASS_SOLID) == 0
    tol_u, tol_r = (1e-9, 1e-9) if storage == Storage.F64 else (1e-3, 1e-4)
    for rho, u, c, q, res, t, inv, cls, links in (sp_, dn_):
        assert np.array_equal(cls, cls_o) and np.array_equal(links, links_o)
        assert rel(u[fl], uo[fl]) <= tol_u and rel(rho[fl], ro[fl]) <= tol_r
        if sp is not None:
            assert rel(c[fl], co[fl]) <= tol_u
            assert rel(q, od.q_ads()) <= max(tol_u, 1e-12) * 10
        assert t == steps - 1
    # the two layouts: same per-node arithmetic
    lt = 1e-12 if storage == Storage.F64 else 1e-6
    assert rel(sp_[1][fl], dn_[1][fl]) <= lt and rel(sp_[0], dn_[0]) <= lt
    if sp is not None:
        assert rel(sp_[2], dn_[2]) <= lt and rel(sp_[3], dn_[3]) <= lt
    assert np.allclose(sp_[4], dn_[4], rtol=1e-6, atol=1e-18)
    assert np.allclose(sp_[6], dn_[6], rtol=1e-9 if storage == Storage.F64 else 1e-5)
    if storage == Storage.F64:
        assert np.allclose(sp_[4], od.residuals(), rtol=1e-6, atol=1e-18)


def test_sparse_scalar_checkpoint_resume(Domain, tmp_path):
    mp, sp = _bed(Storage.F32)
    path = str(tmp_path / "bed.ckpt")
    with Domain(mp, sp) as a:
        a.init().step(41, residual_interval=5)
        assert a.get_option(_abi.LBF_OPT_SPARSE) == 1
        a.save(path)
        a.step(20, residual_interval=5)
        ra, ua, ca = a.moments()
        qa = a.q_ads()
    with Domain(mp, sp) as b:
        b.init().load(path)
        b.step(20, residual_interval=5)
        rb, ub, cb = b.moments()
        assert np.array_equal(ra, rb) and np.array_equal(ua, ub) and np.array_equal(ca, cb)
        assert np.array_equal(qa, b.q_ads())


def test_sparse_faces_smaller_footprint(Domain):
    mp, sp = _bed(Storage.F32)
    with Domain(mp, sp) as a, Domain(mp, sp) as b:
        b.set_option(_abi.LBF_OPT_SPARSE, 0)
        a.init()
        b.init()
        assert a.device_bytes < b.device_bytes


@pytest.mark.parametrize("storage", [Storage.F64, Storage.F32])
def test_outflow_face_pass_overlap_same_bits(Domain, storage):
    """Steps without residuals run the top-face outflow pass of step t beside the
    lower planes of step t + 1 (a side stream); steps with residuals run in order.
    Both give the same bits, for one scalar and for two with different outflows."""
    mp, sp = _bed(storage)
    tracer = ps.Parameters(scalar_name="tracer", collision_operator=TRT.from_magic(0.7),
                           initial_scalar_value=ps.InitialScalarValue.Uniform(0.1), velocity_set=VelocitySet.D3Q19,
                           boundary_conditions=[(W, ps.BBNoFlux), (E, ps.BBNoFlux), (S, ps.BBNoFlux), (N, ps.BBNoFlux),
                                                (B, ps.AntiBounceBack(0.5)), (T, ps.ZerothOrderNoFlux(False))],
                           inner_boundary_condition=ps.InnerBounceBack)
    for sps in ([sp], [sp, tracer]):
        got = []
        for k in (0, 1):
            with Domain(mp, sps) as d:
                d.init().step(75, residual_interval=k)
                rho, u, _ = d.moments()
                got.append((rho, u, [d.scalar(i) for i in range(len(sps))], [d.q_ads(i) for i in range(len(sps))]))
        (r0, u0, c0, q0), (r1, u1, c1, q1) = got
        assert np.array_equal(r0, r1) and np.array_equal(u0, u1)
        for a, b in zip(c0 + q0, c1 + q1):
            assert np.array_equal(a, b)
