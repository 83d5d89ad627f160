"""The z-slab decomposition of the CUDA engine, emulated on one GPU.

R slab domains (R = 2, 3) of one lattice live in one process; after every step
each packs its leaving populations (lbf_domain_halo_pack), the buffers are
handed to the neighbours by device copies, and each unpacks into its ghost
planes (lbf_domain_halo_unpack).  Only ordinary launches on one stream are
involved; no kernel waits on another.  The owned planes must match the whole
lattice run as one domain: relative L2 over fluid nodes 1e-12 (FP64 storage),
1e-6 (FP32).  Lean porous slabs run the sparse sweep (fluid slots of the owned
planes, halos over each plane's fluid slots); the case with explicit x faces runs
the dense sweep.  The multi-process exchange of the same buffers (TorchExchange) is
covered on the CPU by tests/test_slab_cpu.py.
"""
import os
import sys

import numpy as np
import pytest

from lbflow_b200 import _abi
from lbflow_b200.core import Storage

pytestmark = pytest.mark.gpu
sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "helpers"))


class _Ring:
    """down / up neighbours only; the test moves the buffers itself."""

    def __init__(self, rank, world, periodic):
        from lbflow_b200 import slab
        self.down, self.up = slab.neighbours(rank, world, periodic)


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


@pytest.mark.parametrize("split", [False, True], ids=["step", "split"])
@pytest.mark.parametrize("name,world,storage,tol", [("walls", 2, Storage.F64, 1e-12), ("walls", 3, Storage.F32, 1e-6),
                                                    ("periodic", 2, Storage.F64, 1e-12),
                                                    ("periodic", 3, Storage.F64, 1e-12),
                                                    ("d3q27", 2, Storage.F64, 1e-12), ("d3q27", 3, Storage.F16DEV, 1e-6)])
def test_slabs_match_whole_lattice_gpu(name, world, storage, tol, split):
    """split: every step in two parts (lbf_domain_step_part), the halos packed,
    moved and unpacked between part 0 (boundary planes) and part 1 (interior)."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import ctypes as C
    from lbflow_b200 import slab
    from lbflow_b200.domain import Domain
    from slab_cases import case
    p = case(name)
    p.storage = storage
    steps = 60
    periodic = slab.z_periodic(p)
    slabs = [slab.SlabDomain(p, r, world, _Ring(r, world, periodic)) for r in range(world)]
    for s in slabs:
        s.init()
        # lean porous slabs run the sparse fluid-only sweep over their owned planes,
        # the others (explicit x faces) the dense sweep
        assert s.dom.get_option(_abi.LBF_OPT_SPARSE) == (0 if name == "periodic" else 1)
    lib = _abi.load()
    for _ in range(steps):
        for s in slabs:
            if split:
                _abi.check(lib.lbf_domain_step_part(s.dom.h, 0, 0, None))
            else:
                s.dom.step(1)
        for s in slabs:
            lib.lbf_domain_halo_pack(s.dom.h, _abi.LBF_BOTTOM, C.c_void_p(s.bufs[0].data_ptr()), None)
            lib.lbf_domain_halo_pack(s.dom.h, _abi.LBF_TOP, C.c_void_p(s.bufs[1].data_ptr()), None)
        for s in slabs:
            d, u = s.exchange.down, s.exchange.up
            if d is not None:
                s.bufs[2].copy_(slabs[d].bufs[1])     # lower neighbour's top plane -> my bottom ghost
                _abi.check(lib.lbf_domain_halo_unpack(s.dom.h, _abi.LBF_BOTTOM, C.c_void_p(s.bufs[2].data_ptr()), None))
            if u is not None:
                s.bufs[3].copy_(slabs[u].bufs[0])     # upper neighbour's bottom plane -> my top ghost
                _abi.check(lib.lbf_domain_halo_unpack(s.dom.h, _abi.LBF_TOP, C.c_void_p(s.bufs[3].data_ptr()), None))
        if split:
            for s in slabs:
                _abi.check(lib.lbf_domain_step_part(s.dom.h, 1, 0, None))
    torch.cuda.synchronize()
    with Domain(p) as whole:
        whole.init().step(steps)
        rho, u, _ = whole.moments()
        cls, _ = whole.node_class()
    fluid = (cls & _abi.LBF_CLASS_SOLID) == 0
    plane = p.n[0] * p.n[1]
    for s in slabs:
        r_s, u_s = s.moments()
        sl = slice(s.z0 * plane, s.z1 * plane)
        fl = fluid[sl]
        assert rel(r_s[fl], rho[sl][fl]) <= tol, s.rank
        assert rel(u_s[fl], u[sl][fl]) <= tol, s.rank
        s.close()


def test_split_step_order_and_residuals_gpu():
    """Parts alternate; other steps wait for part 1; a split step gives the same
    residuals as a whole step (up to summation order)."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from lbflow_b200 import slab
    from slab_cases import case
    p = case("walls")

    class _NoExchange:
        down = up = None

        def __call__(self, *a):
            pass

    a = slab.SlabDomain(p, 0, 1, _NoExchange()).init()
    b = slab.SlabDomain(p, 0, 1, _NoExchange()).init()
    lib = _abi.load()
    with pytest.raises(_abi.LbfError):
        _abi.check(lib.lbf_domain_step_part(a.dom.h, 1, 1, None))
    _abi.check(lib.lbf_domain_step_part(a.dom.h, 0, 1, None))
    with pytest.raises(_abi.LbfError):
        a.dom.step(1)
    with pytest.raises(_abi.LbfError):
        _abi.check(lib.lbf_domain_step_part(a.dom.h, 0, 1, None))
    _abi.check(lib.lbf_domain_step_part(a.dom.h, 1, 1, None))
    a.step(9, residual_interval=1, overlap=True)
    b.step(10, residual_interval=1, overlap=False)
    torch.cuda.synchronize()
    assert a.time_step == b.time_step == 10
    ra, rb = np.array(a.dom.residuals()[0]), np.array(b.dom.residuals()[0])
    np.testing.assert_allclose(ra, rb, rtol=1e-10, atol=1e-300)
    r_a, u_a = a.moments()
    r_b, u_b = b.moments()
    assert np.array_equal(r_a, r_b) and np.array_equal(u_a, u_b)
    a.close()
    b.close()
