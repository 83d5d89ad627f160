"""3-D Zou-He on the oracle (CPU): D3Q19 and D3Q27 velocity and pressure faces.

The reference has no 3-D Zou-He (src/velocity_set.rs:134-135 returns None for
D3Q19; D3Q27 is a placeholder), so these are the engine's own definitions,
checked by what a Zou-He closure must satisfy:

- after the closure, the node's moments are the prescribed ones: rho and all of
  u for a velocity face; rho and the tangential u for a pressure face;
- only the unknown populations (c.n = +1, n the inward normal) change;
- D3Q19 reproduces Hecht & Harting's form N_t = S_t / 2 - rho u_t / 3 written
  out independently here;
- on a D3Q27 duct with a velocity inlet and a pressure outlet the steady mass
  flux is the same through every cross-section.
"""
import numpy as np
import pytest

from lbflow_b200 import momentum as m
from lbflow_b200.core import BGK, BoundaryFace, VelocitySet
from oracle import oracle as orc

OUTWARD = np.array([[-1, 0, 0], [1, 0, 0], [0, -1, 0], [0, 1, 0], [0, 0, -1], [0, 0, 1]])
VS3 = [(VelocitySet.D3Q19, "D3Q19"), (VelocitySet.D3Q27, "D3Q27")]


def _state(t, rng):
    """Near-equilibrium populations at rho ~ 1, |u| ~ 0.03, with a perturbation."""
    u = rng.uniform(-0.03, 0.03, 3)
    f = orc.equilibrium(int(t["id"]), 1.0 + rng.uniform(-0.02, 0.02), u)
    return f * (1.0 + rng.uniform(-0.01, 0.01, f.size))


def _moments(t, f):
    rho = f.sum()
    return rho, (t["c"].T @ f) / rho


@pytest.fixture(scope="module", params=VS3, ids=[n for _, n in VS3])
def lat(request):
    vs = int(request.param[0])
    t = orc.tables(vs)
    t["id"] = vs
    return t


@pytest.mark.parametrize("face", range(6))
@pytest.mark.parametrize("mode", ["velocity", "pressure"])
def test_closure_sets_the_prescribed_moments(lat, face, mode):
    rng = np.random.default_rng(100 + face)
    ax = face // 2
    n_in = -OUTWARD[face]
    cn = lat["c"] @ n_in
    for _ in range(5):
        f0 = _state(lat, rng)
        u_w = rng.uniform(-0.04, 0.04, 3)
        if mode == "velocity":
            f = orc.zou_he(lat["id"], face, f0, None, list(u_w))
        else:
            rho_w = 1.0 + rng.uniform(-0.01, 0.01)
            vel = [None if a == ax else float(u_w[a]) for a in range(3)]
            f = orc.zou_he(lat["id"], face, f0, rho_w, vel)
        assert np.array_equal(f[cn != 1], f0[cn != 1])
        rho, u = _moments(lat, f)
        tang = [a for a in range(3) if a != ax]
        if mode == "velocity":
            np.testing.assert_allclose(u, u_w, rtol=0, atol=1e-14)
        else:
            assert abs(rho - rho_w) <= 1e-14
            np.testing.assert_allclose(u[tang], u_w[tang], rtol=0, atol=1e-14)


def _hecht_harting_d3q19(t, face, f, u):
    """Hecht & Harting (2010) velocity face for D3Q19, written out on its own."""
    n_in = -OUTWARD[face]
    ax = face // 2
    cn = t["c"] @ n_in
    rho = (f[cn == 0].sum() + 2.0 * f[cn == -1].sum()) / (1.0 - n_in[ax] * u[ax])
    out = f.copy()
    N = np.zeros(3)
    for a in range(3):
        if a != ax:
            N[a] = 0.5 * np.dot(f[cn == 0], t["c"][cn == 0, a]) - rho * u[a] / 3.0
    for i in np.nonzero(cn == 1)[0]:
        ct = sum(t["c"][i, a] * N[a] for a in range(3) if a != ax)
        out[i] = f[t["q_bar"][i]] + 6.0 * t["w"][i] * rho * np.dot(t["c"][i], u) - ct
    return out


@pytest.mark.parametrize("face", range(6))
def test_d3q19_is_hecht_harting(face):
    t = orc.tables(int(VelocitySet.D3Q19))
    t["id"] = int(VelocitySet.D3Q19)
    rng = np.random.default_rng(7 + face)
    f0 = _state(t, rng)
    u = rng.uniform(-0.04, 0.04, 3)
    got = orc.zou_he(t["id"], face, f0, None, list(u))
    np.testing.assert_allclose(got, _hecht_harting_d3q19(t, face, f0, u), rtol=1e-14, atol=1e-16)


def test_wrong_zou_he_input_is_refused():
    t = orc.tables(int(VelocitySet.D3Q27))
    f0 = t["w"].copy()
    with pytest.raises(ValueError):
        orc.zou_he(int(VelocitySet.D3Q27), 4, f0, 1.0, [0.0, 0.0, 0.03])   # both rho and u_n
    with pytest.raises(ValueError):
        orc.zou_he(int(VelocitySet.D3Q27), 4, f0, None, [None, 0.0, 0.03])  # a tangential u missing


def test_d3q27_duct_mass_flux_is_uniform():
    """D3Q27 BGK duct: Zou-He velocity inlet (bottom), Zou-He pressure outlet (top),
    no-slip side walls.  At steady state sum(rho u_z) over every interior z-plane
    is the same."""
    W, E, S, N, B, T = (BoundaryFace.West, BoundaryFace.East, BoundaryFace.South, BoundaryFace.North,
                        BoundaryFace.Bottom, BoundaryFace.Top)
    n = [6, 6, 14]
    p = m.Parameters(n=n, collision_operator=BGK(0.8), velocity_set=VelocitySet.D3Q27,
                     initial_velocity=m.InitialVelocity.Uniform([0, 0, 0]),
                     boundary_conditions=[(W, m.NoSlip), (E, m.NoSlip), (S, m.NoSlip), (N, m.NoSlip),
                                          (B, m.ZouHe(None, [0.0, 0.0, 0.02])),
                                          (T, m.ZouHe(1.0, [0.0, 0.0, None]))])
    desc, keep = m.to_desc(p)
    od = orc.Domain(desc, keep=keep).init().step(9000)
    rho, u, _ = od.observe()
    rho = rho.reshape(n[2], n[1], n[0])
    uz = u.reshape(n[2], n[1], n[0], 3)[..., 2]
    flux = (rho * uz)[2:-2].sum(axis=(1, 2))
    assert flux.min() > 0
    assert (flux.max() - flux.min()) / flux.mean() < 1e-9, flux
    # the outlet keeps its prescribed density
    assert np.abs(rho[-1, 1:-1, 1:-1] - 1.0).max() < 1e-12
