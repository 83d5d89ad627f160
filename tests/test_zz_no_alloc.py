"""lbf_inventory_noalloc: the fluid-node FP64 sums without any device allocation.

This entry point is for callers that cannot allocate device memory when they
need the sums: an application whose HBM is already reserved by its own caching
allocator (an allocation behind its back breaks its accounting) or by lattices
sized to fill it (an allocation would fail).  The test prepares the input arrays
itself (with torch, as such a caller would have them), calls the entry point
twice through the C ABI, and checks both results against lbf_domain_inventory,
which computes the same sums with library-allocated scratch.  The file is named
so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from lbflow_b200 import _abi, cases
from lbflow_b200.core import Storage

pytestmark = pytest.mark.gpu


def _dev(torch, a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def test_inventory_noalloc_matches_domain_inventory():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from lbflow_b200.domain import Domain

    lib = _abi.load()
    mp, sp = cases.packed_bed_scalar([16, 14, 24], porosity=0.75, rmin=1.5, rmax=3.0, seed=21,
                                     storage=Storage.F64, ka=1e-2)
    with Domain(mp, sp) as dom:
        dom.init().step(120)
        expected = dom.inventory()
        rho, u, c = dom.moments()
        q = dom.q_ads()
        cls, _ = dom.node_class()
    n, d = rho.size, u.shape[1]

    d_rho = _dev(torch, rho, torch.float64)
    d_u = _dev(torch, u.ravel(), torch.float64)
    d_c = _dev(torch, c, torch.float64)
    d_q = _dev(torch, q, torch.float64)
    d_cls = _dev(torch, cls.view(np.int32), torch.int32)
    out = torch.full((3 + d,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()

    for call in range(2):   # the scratch array keeps the previous call's sums; each call clears it
        out.fill_(float("nan"))
        st = lib.lbf_inventory_noalloc(C.c_void_p(d_rho.data_ptr()), C.c_void_p(d_u.data_ptr()),
                                       C.c_void_p(d_c.data_ptr()), C.c_void_p(d_q.data_ptr()),
                                       C.c_void_p(d_cls.data_ptr()), n, d, C.c_void_p(out.data_ptr()),
                                       C.c_void_p(stream.cuda_stream))
        assert st == _abi.LBF_OK, lib.lbf_last_error().decode()
        got = out.cpu().numpy()
        assert np.allclose(got, expected, rtol=1e-12, atol=1e-12), (call, got, expected)

    # sizes beyond the stated limits are refused with an error, not run
    st = lib.lbf_inventory_noalloc(C.c_void_p(d_rho.data_ptr()), C.c_void_p(d_u.data_ptr()), None, None,
                                   C.c_void_p(d_cls.data_ptr()), 1 << 31, d, C.c_void_p(out.data_ptr()), None)
    assert st == _abi.LBF_EINVAL and "LBF_NOALLOC_MAX_NODES" in lib.lbf_last_error().decode()
    st = lib.lbf_inventory_noalloc(C.c_void_p(d_rho.data_ptr()), C.c_void_p(d_u.data_ptr()), None, None,
                                   C.c_void_p(d_cls.data_ptr()), n, 4, C.c_void_p(out.data_ptr()), None)
    assert st == _abi.LBF_EINVAL
