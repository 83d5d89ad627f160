"""The central-moment collision (D2Q9, D3Q27) as restated in the oracle.

The reference has no D3Q27 collision (src/velocity_set.rs:168), so the engine
defines this one; these checks pin the definition itself:
- mass and momentum are conserved;
- with every rate 1 the output is the product-form equilibrium, whose 1-D
  factor has moments (1, u, 1/3 + u^2): phi(0) = 2/3 - u^2, phi(+-1) = (1/3 + u^2 +- u)/2;
- the product-form equilibrium is a fixed point for any rates;
- a non-equilibrium shear moment decays by exactly (1 - 1/tau);
- a velocity shifted by F/(2 rho) gains exactly F of momentum (order-1 reflection).
"""
import itertools

import numpy as np
import pytest

from oracle import oracle as orc
from lbflow_b200 import _abi


def _tables(vs):
    t = orc.tables(vs)
    return t["c"][:, : t["d"]], t["q"], t["d"]


def _product_eq(c, rho, u):
    def phi(ci, ua):
        return 2.0 / 3.0 - ua * ua if ci == 0 else (1.0 / 3.0 + ua * ua + ci * ua) / 2.0
    return np.array([rho * np.prod([phi(ci[a], u[a]) for a in range(len(u))]) for ci in c])


@pytest.mark.parametrize("vs", [_abi.LBF_D2Q9, _abi.LBF_D3Q27])
def test_central_conserves_and_equilibrium(vs):
    c, q, d = _tables(vs)
    rng = np.random.default_rng(vs)
    for _ in range(20):
        rho = 1.0 + 0.05 * rng.standard_normal()
        u = 0.05 * rng.standard_normal(d)
        feq = _product_eq(c, rho, u)
        f = feq * (1.0 + 0.02 * rng.standard_normal(q))
        rho_f = f.sum()
        u_f = (f[:, None] * c).sum(0) / rho_f
        tau = rng.uniform(0.5005, 1.5)
        rates = rng.uniform(0.3, 1.9, 5)
        out = orc.central(vs, rho_f, u_f, f, tau, rates)
        assert abs(out.sum() - rho_f) < 1e-14
        assert np.allclose((out[:, None] * c).sum(0), (f[:, None] * c).sum(0), atol=1e-15)
        # every rate 1: the product-form equilibrium of the node's moments
        full = orc.central(vs, rho_f, u_f, f, 1.0, np.ones(5))
        assert np.allclose(full, _product_eq(c, rho_f, u_f), atol=1e-15)
        # the equilibrium is a fixed point
        assert np.allclose(orc.central(vs, rho, u, feq, tau, rates), feq, atol=1e-15)


@pytest.mark.parametrize("vs", [_abi.LBF_D2Q9, _abi.LBF_D3Q27])
def test_central_shear_rate_and_force(vs):
    c, q, d = _tables(vs)
    rho, u = 1.0, np.zeros(d)
    feq = _product_eq(c, rho, u)
    # add a pure xy shear: delta f = eps * c_x c_y (zero mass, momentum, trace)
    eps = 1e-3
    f = feq + eps * c[:, 0] * c[:, 1]
    tau = 0.7
    out = orc.central(vs, rho, u, f, tau, np.ones(5))
    pxy = lambda g: (g * c[:, 0] * c[:, 1]).sum()  # noqa: E731
    assert abs(pxy(out) - (1.0 - 1.0 / tau) * pxy(f)) < 1e-15
    # force: u = (j + F/2) / rho; the post-collision momentum is j + F
    F = np.array([2e-4, -1e-4, 3e-4][:d])
    f = feq.copy()
    j = (f[:, None] * c).sum(0)
    out = orc.central(vs, rho, (j + 0.5 * F) / rho, f, tau, np.ones(5))
    assert np.allclose((out[:, None] * c).sum(0), j + F, atol=1e-16)
