"""Checkpoints (lbf_domain_save / lbf_domain_load): a run resumed from a
checkpoint continues bit for bit, and a checkpoint refuses a domain of another
lattice, storage or layout."""
import numpy as np
import pytest

from lbflow_b200 import _abi, cases
from lbflow_b200.core import Storage

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def Domain():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from lbflow_b200.domain import Domain as D
    return D


def _cases():
    mask = cases.sphere_pack([32, 20, 16], 0.7, 1.5, 3.0, seed=3)
    bed = cases.sphere_pack([12, 12, 24], 0.75, 1.5, 2.5, seed=4)
    return {
        "porous_sparse_f32": (cases.porous_channel_d3q19([32, 20, 16], mask=mask, force=1e-5, storage=Storage.F32),
                              None),
        "packed_bed_scalar_f64": cases.packed_bed_scalar([12, 12, 24], mask=bed, storage=Storage.F64, ka=1e-2),
        "cavity_f16": (cases.cavity_d2q9(24, 0.6, 0.1, Storage.F16DEV), None),
    }


@pytest.mark.parametrize("name", ["porous_sparse_f32", "packed_bed_scalar_f64", "cavity_f16"])
def test_resume_is_bit_exact(Domain, name, tmp_path):
    p, sp = _cases()[name]
    path = str(tmp_path / "state.ckpt")
    with Domain(p, sp) as a:
        a.init().step(81, residual_interval=5)
        a.save(path)
        a.step(37, residual_interval=5)
        ra, ua, ca = a.moments()
        res_a, t_a = a.residuals()
        qa = a.q_ads() if sp is not None else None
        ta = a.time_step
    with Domain(p, sp) as b:
        b.init().load(path)
        assert b.time_step == 81
        b.step(37, residual_interval=5)
        rb, ub, cb = b.moments()
        res_b, t_b = b.residuals()
        assert b.time_step == ta and t_b == t_a
        assert np.array_equal(ra, rb) and np.array_equal(ua, ub)
        assert np.array_equal(res_a, res_b)
        if sp is not None:
            assert np.array_equal(ca, cb) and np.array_equal(qa, b.q_ads())


def test_checkpoint_refuses_other_storage(Domain, tmp_path):
    p = cases.cavity_d2q9(24, 0.6, 0.1, Storage.F32)
    q = cases.cavity_d2q9(24, 0.6, 0.1, Storage.F64)
    path = str(tmp_path / "state.ckpt")
    with Domain(p) as a:
        a.init().step(10)
        a.save(path)
    with Domain(q) as b:
        b.init()
        with pytest.raises(_abi.LbfError) as ei:
            b.load(path)
        assert ei.value.status == _abi.LBF_EINVAL


@pytest.mark.parametrize("damage", ["truncated", "section_count", "other_lattice"])
def test_rejected_checkpoint_leaves_domain_unchanged(Domain, damage, tmp_path):
    """A checkpoint that is refused (truncated, with a wrong section count, or of
    another lattice) leaves the time step, the residuals and the fields as they
    were, so that the next step reads the right population buffer."""
    p = cases.cavity_d2q9(24, 0.6, 0.1, Storage.F32)
    path = str(tmp_path / "state.ckpt")
    with Domain(p) as a:
        a.init().step(17, residual_interval=4)   # odd time step: the other buffer parity
        a.save(path)
    buf = np.fromfile(path, dtype=np.uint8)
    if damage == "truncated":
        buf = buf[: buf.size - 64]
    elif damage == "section_count":
        # CkptHeader: magic[8], vs q st d (4 x i32), N Np nlist (3 x i64), sparse scalar ads nsec (4 x i32)
        off = 8 + 16 + 24 + 12
        buf = buf.copy()
        buf[off:off + 4] = np.frombuffer(np.int32(3).tobytes(), np.uint8)
    else:
        with Domain(cases.cavity_d2q9(20, 0.6, 0.1, Storage.F32)) as other:
            other.init().step(5)
            other.save(path)
        buf = np.fromfile(path, dtype=np.uint8)
    buf.tofile(path)
    with Domain(p) as b, Domain(p) as ref:
        b.init().step(10, residual_interval=4)
        ref.init().step(10, residual_interval=4)
        with pytest.raises(_abi.LbfError) as ei:
            b.load(path)
        assert ei.value.status == _abi.LBF_EINVAL
        assert b.time_step == 10
        assert np.array_equal(b.residuals()[0], ref.residuals()[0])
        b.step(9, residual_interval=4)
        ref.step(9, residual_interval=4)
        rb, ub, _ = b.moments()
        rr, ur, _ = ref.moments()
        assert np.array_equal(rb, rr) and np.array_equal(ub, ur)
        assert np.array_equal(b.residuals()[0], ref.residuals()[0])
