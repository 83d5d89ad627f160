"""Bounded waits: a step whose wait on its bulk copies gives up reports
LBF_ETIMEOUT and leaves the device usable.

The staged sweep (LBF_OPT_STAGE) waits on an mbarrier for the bulk copies of its
source rows.  LBF_OPT_WAIT_LIMIT 0 makes that wait give up at its first check,
so the timeout path runs without any real hang: each block records the error,
waits (with the default limit) for its copies to land, and returns.  The host
reads the flag at the next synchronising call.  Re-initialising the domain
clears the flag, and the same domain then computes the same fields as a fresh
one.
"""
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


def test_wait_limit_timeout_is_reported_and_recoverable(Domain):
    p = cases.cavity_d2q9(32, 0.6, 0.1, Storage.F32)
    with Domain(p) as d, Domain(p) as ref:
        d.set_option(_abi.LBF_OPT_STAGE, 1)
        assert d.get_option(_abi.LBF_OPT_STAGE) == 1          # the shape allows staging
        d.set_option(_abi.LBF_OPT_WAIT_LIMIT, 0)
        d.init().step(3, residual_interval=1)                 # steps 1 and 2 are staged
        with pytest.raises(_abi.LbfError) as ei:
            d.residuals()
        assert ei.value.status == _abi.LBF_ETIMEOUT
        with pytest.raises(_abi.LbfError) as ei:
            d.moments()
        assert ei.value.status == _abi.LBF_ETIMEOUT
        # the device context is intact: restore the limit, re-initialise, run
        d.set_option(_abi.LBF_OPT_WAIT_LIMIT, -1)
        d.init().step(50, residual_interval=1)
        ref.init().step(50, residual_interval=1)
        r1, u1, _ = d.moments()
        r2, u2, _ = ref.moments()
        assert np.array_equal(r1, r2) and np.array_equal(u1, u2)
        assert np.array_equal(d.residuals()[0], ref.residuals()[0])


def test_wait_limit_option_validation(Domain):
    p = cases.cavity_d2q9(16, 0.6, 0.1, Storage.F32)
    with Domain(p) as d:
        with pytest.raises(_abi.LbfError) as ei:
            d.set_option(_abi.LBF_OPT_WAIT_LIMIT, -2)
        assert ei.value.status == _abi.LBF_EINVAL
        d.set_option(_abi.LBF_OPT_WAIT_LIMIT, 123)
        assert d.get_option(_abi.LBF_OPT_WAIT_LIMIT) == 123
