"""The streaming schemes of the sparse layout: pull (two buffers), push (two
buffers) and in place (AA pattern, one buffer).

All three move the same values and run the same arithmetic, so the fields,
residuals and inventories must agree bit for bit after even and odd step
counts, for every velocity set, collision and storage format; the in-place
layout holds one population buffer instead of two.  A checkpoint taken at an odd
time step resumes exactly, and a batch of push or in-place domains gives the
fields of each domain run alone.
"""
import math

import numpy as np
import pytest

from lbflow_b200 import _abi, cases
from lbflow_b200 import momentum as m
from lbflow_b200.core import BGK, MRT, TRT, BoundaryFace, Storage, VelocitySet

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


def _case(vs, coll, storage):
    rng = np.random.default_rng(17)
    if vs == VelocitySet.D2Q9:
        n = [37, 29]
        bcs = [(W, m.Periodic), (E, m.Periodic), (S, m.NoSlip), (N, m.NoSlip)]
    else:
        n = [27, 19, 15]
        bcs = [(W, m.Periodic), (E, m.Periodic), (S, m.NoSlip), (N, m.NoSlip), (B, m.Periodic), (T, m.Periodic)]
    mask = (rng.random(int(np.prod(n))) < 0.2).astype(np.uint8)
    q = vs.q
    if coll == "bgk":
        op = BGK(0.7)
    elif coll == "trt":
        op = TRT.from_magic(0.8, 0.25)
    else:
        rates = [1.0] * q
        rates[4 if vs == VelocitySet.D3Q27 else 1] = 1.1
        op = MRT(rates)
    force = [2e-5, -1e-5] + ([5e-6] if vs.d == 3 else [])
    return m.Parameters(n=n, collision_operator=op, velocity_set=vs, force=force,
                        initial_density=m.InitialDensity.Uniform(1.0),
                        initial_velocity=m.InitialVelocity.Uniform([0.0] * vs.d),
                        boundary_conditions=bcs, node_types=m.NodeTypes.FromArray(mask), storage=storage)


CASES = [(VelocitySet.D2Q9, "bgk", Storage.F64), (VelocitySet.D2Q9, "mrt", Storage.F32),
         (VelocitySet.D3Q19, "trt", Storage.F32), (VelocitySet.D3Q19, "trt", Storage.F16DEV),
         (VelocitySet.D3Q19, "bgk", Storage.BF16DEV), (VelocitySet.D3Q19, "mrt", Storage.F64),
         (VelocitySet.D3Q27, "trt", Storage.F32), (VelocitySet.D3Q27, "mrt", Storage.F32)]


def _schemed(Domain, p, scheme):
    d = Domain(p)
    d.set_option(_abi.LBF_OPT_STREAMING, scheme)
    d.init()
    assert d.get_option(_abi.LBF_OPT_SPARSE) == 1 and d.get_option(_abi.LBF_OPT_STREAMING) == scheme
    return d


@pytest.mark.parametrize("vs,coll,storage", CASES)
def test_streaming_schemes_agree(Domain, vs, coll, storage):
    p = _case(vs, coll, storage)
    doms = [_schemed(Domain, p, s) for s in (_abi.LBF_STREAM_PULL, _abi.LBF_STREAM_PUSH, _abi.LBF_STREAM_INPLACE)]
    try:
        assert doms[2].device_bytes < doms[0].device_bytes
        for steps in (1, 1, 6, 13):          # odd and even time steps
            out = []
            for d in doms:
                d.step(steps, residual_interval=3)
                out.append((*d.moments()[:2], d.residuals()[0], d.inventory()))
            for o in out[1:]:
                for a, b in zip(out[0], o):
                    assert np.array_equal(a, b), doms[0].time_step
    finally:
        for d in doms:
            d.close()


def test_inplace_run_stops_like_two_buffer(Domain):
    p = cases.porous_channel_d3q19([24, 16, 12], mask=cases.sphere_pack([24, 16, 12], 0.75, 1.5, 3.0, seed=5),
                                   force=1e-6, storage=Storage.F64)
    doms = [_schemed(Domain, p, s) for s in (_abi.LBF_STREAM_PULL, _abi.LBF_STREAM_PUSH, _abi.LBF_STREAM_INPLACE)]
    try:
        steps = [d.run(301, residual_interval=7) for d in doms]
        assert steps[0] == steps[1] == steps[2]
        assert np.array_equal(doms[0].moments()[1], doms[1].moments()[1])
        assert np.array_equal(doms[0].moments()[1], doms[2].moments()[1])
    finally:
        for d in doms:
            d.close()


@pytest.mark.parametrize("scheme", [1, 2])
def test_checkpoint_at_odd_step(Domain, tmp_path, scheme):
    p = _case(VelocitySet.D3Q19, "trt", Storage.F32)
    path = str(tmp_path / "s.ckpt")
    with Domain(p) as a:
        a.set_option(_abi.LBF_OPT_STREAMING, scheme)
        a.init().step(23, residual_interval=4)
        a.save(path)
        a.step(10, residual_interval=4)
        ra, ua, _ = a.moments()
    with Domain(p) as b:
        b.set_option(_abi.LBF_OPT_STREAMING, scheme)
        b.init().load(path)
        assert b.time_step == 23
        b.step(10, residual_interval=4)
        rb, ub, _ = b.moments()
    assert np.array_equal(ra, rb) and np.array_equal(ua, ub)


@pytest.mark.parametrize("scheme", [1, 2])
def test_batch_matches_alone(Domain, scheme):
    """In-place domains in a batch (k even and odd, so that the members' step
    parities differ within a launch) stop where they stop alone, with the same
    fields (1e-12 FP64, 1e-5 FP32 / FP16: other kernels around the same per-node code)."""
    from lbflow_b200.batch import Batch
    ps = [(_case(VelocitySet.D3Q19, "trt", Storage.F32), 1e-5), (_case(VelocitySet.D2Q9, "bgk", Storage.F64), 1e-12),
          (_case(VelocitySet.D3Q19, "trt", Storage.F16DEV), 1e-5), (_case(VelocitySet.D3Q27, "mrt", Storage.F32), 1e-5)]
    for k in (10, 7):
        alone = []
        for p, _ in ps:
            with _schemed(Domain, p, scheme) as d:
                steps = d.run(120, k, 1e-7, 1e-7, 1e-7)
                alone.append((steps, d.time_step, *d.moments()[:2]))
        with Batch(0, k) as bt:
            doms = []
            for (p, _), late in zip(ps, (0, 3, 0, 5)):
                d = _schemed(Domain, p, scheme)
                if late:
                    d.step(late, residual_interval=k)   # joins at another time step
                doms.append(d)
                bt.admit(d, 120, 1e-7, 1e-7, 1e-7)
            done = {}
            for _ in range(200):
                if len(done) == len(doms):
                    break
                bt.step(1)
                for d, stt in bt.poll(wait=True):
                    done[id(d)] = stt
            assert len(done) == len(doms)
            for d, (p, tol), (steps, t_alone, ra, ua) in zip(doms, ps, alone):
                assert d.time_step == t_alone
                rb, ub, _ = d.moments()
                nb = np.linalg.norm(ua)
                assert np.linalg.norm(ub - ua) <= tol * nb and np.linalg.norm(rb - ra) <= tol * np.linalg.norm(ra)
                d.close()
