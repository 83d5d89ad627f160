"""Several passive scalars in one domain (passive_scalar::LatticeVec,
src/passive_scalar/lattice.rs:353-430): one momentum sweep advances every scalar.

The oracle advances the momentum lattice once per scalar domain, and each of
those runs is compared with the matching scalar of the multi-scalar domain:
node classes exactly, moments and scalars to 1e-9 relative L2 in FP64 storage
(1e-3 / 1e-4 in FP32).  The multi-scalar domain also equals, bit for bit, the
single-scalar engine domains of its scalars (the per-node arithmetic is the
same), in the sparse and the dense layouts.  Residuals list every scalar.
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


def _bed_scalars(n, storage):
    """The packed bed with three scalars of different set-ups: the adsorbing
    solute of the bed, a passive tracer (no adsorption, TRT), and a solute
    entering at another concentration with a zeroth-order outflow."""
    mask = cases.sphere_pack(n, 0.7, 1.5, 2.5, seed=4)
    mp, s0 = cases.packed_bed_scalar(n, mask=mask, storage=storage, ka=1e-2)
    walls = [(W, ps.BBNoFlux), (E, ps.BBNoFlux), (S, ps.BBNoFlux), (N, ps.BBNoFlux)]
    s1 = ps.Parameters(scalar_name="tracer", collision_operator=TRT.from_magic(0.7),
                       initial_scalar_value=ps.InitialScalarValue.Uniform(0.1), velocity_set=VelocitySet.D3Q19,
                       boundary_conditions=walls + [(B, ps.AntiBounceBack(0.5)),
                                                    (T, ps.SecondOrderNoFlux(unknown_populations_only=False))],
                       inner_boundary_condition=ps.InnerBounceBack)
    s2 = ps.Parameters(scalar_name="solute2", collision_operator=BGK(0.6),
                       initial_scalar_value=ps.InitialScalarValue.Uniform(0.0), velocity_set=VelocitySet.D3Q19,
                       boundary_conditions=walls + [(B, ps.AntiBounceBack(2.0)), (T, ps.ZerothOrderNoFlux(False))],
                       inner_boundary_condition=ps.InnerBounceBack,
                       adsorption_parameters=ps.AdsorptionParameters(ps.Langmuir(5e-3, 1e-4, 0.5), 0.05))
    return mp, [s0, s1, s2]


def _channel_d2q9_scalars():
    """A D2Q9 channel whose two scalars differ in inner rule, collision, faces and
    initial field; the second has an extrapolation outflow on E, the first an
    anti-bounce-back no-flux face there."""
    n = [40, 18]
    rng = np.random.default_rng(3)
    mask = (rng.random(n[0] * n[1]) < 0.12).astype(np.uint8).reshape(n[1], n[0])
    mask[:, :2] = 0
    mask[:, -3:] = 0
    mp = m.Parameters(n=n, collision_operator=BGK(0.7), velocity_set=VelocitySet.D2Q9,
                      boundary_conditions=[(W, m.ZouHe(None, [0.04, 0.0])), (E, m.AntiBounceBack(1.0)),
                                           (S, m.NoSlip), (N, m.BounceBack(1.0, [0.02, 0.0]))],
                      node_types=m.NodeTypes.FromArray(mask.ravel()))
    s0 = ps.Parameters(scalar_name="a", collision_operator=BGK(0.55), velocity_set=VelocitySet.D2Q9,
                       initial_scalar_value=ps.InitialScalarValue.FromArray(0.1 + 0.3 * rng.random(n[0] * n[1])),
                       boundary_conditions=[(W, ps.AntiBounceBack(1.0)), (E, ps.AntiBBNoFlux),
                                            (S, ps.BBNoFlux), (N, ps.AntiBBNoFlux)],
                       inner_boundary_condition=ps.InnerAntiBounceBack,
                       adsorption_parameters=ps.AdsorptionParameters(ps.Langmuir(1e-2, 1e-4, 1.0), 0.1))
    s1 = ps.Parameters(scalar_name="b", collision_operator=TRT.from_magic(0.8),
                       velocity_set=VelocitySet.D2Q9, initial_scalar_value=ps.InitialScalarValue.Uniform(0.4),
                       boundary_conditions=[(W, ps.AntiBounceBack(0.0)),
                                            (E, ps.SecondOrderNoFlux(unknown_populations_only=True)),
                                            (S, ps.BBNoFlux), (N, ps.BBNoFlux)],
                       inner_boundary_condition=ps.InnerBounceBack)
    return mp, [s0, s1]


def _run(Domain, mp, sps, steps, sparse):
    with Domain(mp, sps) as d:
        d.set_option(_abi.LBF_OPT_SPARSE, 1 if sparse else 0)
        d.init()
        assert d.num_scalars == len(sps)
        d.step(steps - 1, residual_interval=1).step(1, residual_interval=1)
        rho, u, c0 = d.moments()
        cs = [d.scalar(i) for i in range(len(sps))]
        assert np.array_equal(cs[0], c0)
        qs = [d.q_ads(i) for i in range(len(sps))]
        res, t = d.residuals()
        cls, links = d.node_class()
    return rho, u, cs, qs, res, t, cls, links


def _single(Domain, mp, sp, steps, sparse):
    with Domain(mp, sp) as d:
        d.set_option(_abi.LBF_OPT_SPARSE, 1 if sparse else 0)
        d.init()
        d.step(steps - 1, residual_interval=1).step(1, residual_interval=1)
        rho, u, c = d.moments()
        res, _ = d.residuals()
        return rho, u, c, d.q_ads(), res


CASES = {
    "bed3_f64": (lambda: _bed_scalars([14, 12, 24], Storage.F64), 150, Storage.F64, True),
    "bed3_f32": (lambda: _bed_scalars([14, 12, 24], Storage.F32), 150, Storage.F32, True),
    "channel2_d2q9_dense": (_channel_d2q9_scalars, 250, Storage.F64, False),
    "channel2_d2q9_sparse": (_channel_d2q9_scalars, 250, Storage.F64, True),
}


@pytest.mark.parametrize("name", list(CASES))
def test_scalars_in_one_sweep_match_oracle_and_single_domains(Domain, name):
    from oracle import oracle as orc
    make, steps, storage, sparse = CASES[name]
    mp, sps = make()
    desc, keep = m.to_desc(mp)
    got = _run(Domain, mp, sps, steps, sparse)
    rho, u, cs, qs, res, t, cls, links = got
    assert t == steps - 1 and len(res) == 1 + mp.dim + len(sps)
    tol_u, tol_r = (1e-9, 1e-9) if storage == Storage.F64 else (1e-3, 1e-4)
    for i, sp in enumerate(sps):
        sdesc, k2 = ps.to_desc(sp, mp.n[: mp.dim])
        od = orc.Domain(desc, sdesc, keep=keep + k2).init().step(steps)
        ro, uo, co = od.observe()
        cls_o, links_o = od.node_class()
        fl = (cls_o & _abi.LBF_CLASS_SOLID) == 0
        assert np.array_equal(cls, cls_o) and np.array_equal(links, links_o)
        assert rel(u[fl], uo[fl]) <= tol_u and rel(rho[fl], ro[fl]) <= tol_r
        assert rel(cs[i][fl], co[fl]) <= tol_u, (i, rel(cs[i][fl], co[fl]))
        assert rel(qs[i], od.q_ads()) <= max(tol_u, 1e-12) * 10
        # the same scalar alone in its own engine domain: the same bits
        rs, us, c1, q1, res1 = _single(Domain, mp, sp, steps, sparse)
        assert np.array_equal(rs, rho) and np.array_equal(us, u)
        assert np.array_equal(c1, cs[i]) and np.array_equal(q1, qs[i])
        # residuals: the same per-node terms; their per-block sums group nodes
        # differently when the domains' outflow face passes differ (a node of an
        # outflow face of any scalar is updated by the face pass)
        assert np.allclose(res1[: 1 + mp.dim], res[: 1 + mp.dim], rtol=1e-12, atol=0)
        assert np.isclose(res1[1 + mp.dim], res[1 + mp.dim + i], rtol=1e-12, atol=0)
        if storage == Storage.F64:
            assert np.allclose(res[1 + mp.dim + i], od.residuals()[1 + mp.dim], rtol=1e-6, atol=1e-18)


def test_scalars_checkpoint_resume(Domain, tmp_path):
    mp, sps = _bed_scalars([14, 12, 24], Storage.F32)
    path = str(tmp_path / "bed3.ckpt")
    with Domain(mp, sps) as a:
        a.init().step(37, residual_interval=5)
        a.save(path)
        a.step(20, residual_interval=5)
        ra, ua, _ = a.moments()
        ca = [a.scalar(i) for i in range(3)]
        qa = [a.q_ads(i) for i in range(3)]
    with Domain(mp, sps) as b:
        b.init().load(path)
        b.step(20, residual_interval=5)
        rb, ub, _ = b.moments()
        assert np.array_equal(ra, rb) and np.array_equal(ua, ub)
        for i in range(3):
            assert np.array_equal(ca[i], b.scalar(i)) and np.array_equal(qa[i], b.q_ads(i))
    # a checkpoint of three scalars does not load into a domain of one
    with Domain(mp, sps[:1]) as c:
        c.init()
        with pytest.raises(RuntimeError, match="EINVAL"):
            c.load(path)


def test_scalar_limit_and_index(Domain):
    mp, sps = _bed_scalars([14, 12, 24], Storage.F64)
    with pytest.raises(ValueError):
        Domain(mp, sps + sps)
    with Domain(mp, sps[:2]) as d:
        d.init()
        with pytest.raises(RuntimeError, match="EINVAL"):
            d.scalar(2)
