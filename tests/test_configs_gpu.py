"""Parity at the benchmark configurations' stated sizes, engine vs the FP64 oracle.

- C1 exactly as stated: D2Q9 BGK lid-driven cavity 128 x 128, tau = 0.6, NoSlip
  on W/E/S, Zou-He velocity lid u = (0.1, 0) on N, rho = 1 and u = 0 at
  equilibrium, 20,000 steps, face order W, E, S, N (the declaration order of
  FACES_2D, src/lib.rs:27; the reference's HashMap order is unspecified).
  Reference passes: src/momentum/lattice.rs:431-441, Zou-He
  src/velocity_set/d2q9.rs:165-245.
- FP16 / BF16 deviation storage against the FP64 oracle on a D3Q19 TRT porous
  channel of 64^3 for 1,000 steps (the C2 geometry and parameters at a size the
  oracle finishes in seconds).  The bound is 1e-3 relative L2 in velocity.

Errors are relative L2 over fluid nodes, ||a - b|| / ||b||; node classes and
link masks must agree exactly.
"""
import numpy as np
import pytest

from lbflow_b200 import _abi, cases
from lbflow_b200 import momentum as m
from lbflow_b200.core import Storage

pytestmark = pytest.mark.gpu

# C1 bounds: FP64 storage differs from the oracle only by FMA contraction and
# summation order; FP32 deviation storage by its rounding over 20,000 steps.
C1_TOL = {Storage.F64: (1e-9, 1e-9), Storage.F32: (2e-4, 1e-6)}   # (velocity, density)
DEV_TOL_U = 1e-3      # deviation storage: velocity
DEV_TOL_RHO = 1e-4    # deviation storage: density


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


_ORACLE = {}


def oracle_fields(params, steps, key):
    """Oracle moments after `steps` main_steps (cached per configuration)."""
    if key not in _ORACLE:
        from oracle import oracle as orc
        desc, keep = m.to_desc(params)
        od = orc.Domain(desc, keep=keep).init().step(steps)
        rho, u, _ = od.observe()
        cls, links = od.node_class()
        _ORACLE[key] = (rho, u, cls, links)
    return _ORACLE[key]


@pytest.mark.parametrize("storage", [Storage.F64, Storage.F32])
def test_c1_cavity_128_20000_steps(Domain, storage):
    steps = 20000
    p = cases.cavity_d2q9(128, 0.6, 0.1, storage)
    ro, uo, cls_o, links_o = oracle_fields(cases.cavity_d2q9(128, 0.6, 0.1, Storage.F64), steps, "c1")
    with Domain(p) as d:
        d.init().step(steps)
        assert d.time_step == steps
        rg, ug, _ = d.moments()
        cls_g, links_g = d.node_class()
    assert np.array_equal(cls_g, cls_o) and np.array_equal(links_g, links_o)
    fl = (cls_o & _abi.LBF_CLASS_SOLID) == 0
    tol_u, tol_r = C1_TOL[storage]
    eu, er = rel(ug[fl], uo[fl]), rel(rg[fl], ro[fl])
    print(f"C1 {storage.name}: rel L2 u {eu:.3e} rho {er:.3e}")
    assert eu <= tol_u, f"velocity rel L2 {eu:.3e}"
    assert er <= tol_r, f"density rel L2 {er:.3e}"
    # the flow is developed: the lid drives a vortex of order u_lid / 10
    assert np.max(np.abs(uo[fl])) > 0.05


def _porous64(storage):
    mask = cases.sphere_pack([64, 64, 64], 0.7, 4.0, 10.0, seed=1234)
    return cases.porous_channel_d3q19([64] * 3, mask=mask, force=1e-6, storage=storage), mask


def _deviation_errors(Domain, storage, steps=1000):
    p, mask = _porous64(storage)
    ro, uo, cls_o, _ = oracle_fields(_porous64(Storage.F64)[0], steps, "porous64")
    with Domain(p) as d:
        d.init().step(steps)
        rg, ug, _ = d.moments()
        cls_g, _ = d.node_class()
    assert np.array_equal(cls_g, cls_o)
    fl = mask == 0
    return rel(ug[fl], uo[fl]), rel(rg[fl], ro[fl])


@pytest.mark.parametrize("storage", [Storage.F32, Storage.F16DEV])
def test_deviation_storage_vs_oracle_64cubed(Domain, storage):
    """FP32 and FP16-deviation storage meet the 1e-3 velocity bound against the FP64 oracle."""
    eu, er = _deviation_errors(Domain, storage)
    print(f"porous 64^3 x 1000 {storage.name}: rel L2 u {eu:.3e} rho {er:.3e}")
    assert eu <= DEV_TOL_U, f"velocity rel L2 {eu:.3e}"
    assert er <= DEV_TOL_RHO, f"density rel L2 {er:.3e}"


@pytest.mark.xfail(strict=True, reason="BF16 deviations keep 8 significant bits: the velocity error "
                                       "exceeds the 1e-3 bound")
def test_bf16_deviation_storage_fails_the_bound(Domain):
    eu, _ = _deviation_errors(Domain, Storage.BF16DEV)
    print(f"porous 64^3 x 1000 BF16DEV: rel L2 u {eu:.3e}")
    assert eu <= DEV_TOL_U


def test_bf16_deviation_storage_regression(Domain):
    """BF16 misses the 1e-3 bound; this pins how far, so that a regression shows."""
    eu, er = _deviation_errors(Domain, Storage.BF16DEV)
    assert eu <= 3e-2 and er <= 1e-3
