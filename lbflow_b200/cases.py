"""Seeded synthetic cases with the shapes of the benchmark configurations.

No public dataset is involved: every geometry and initial field is generated
here from a seed.

- lid-driven cavity, D2Q9 BGK (NoSlip W/E/S, Zou-He velocity lid on N);
- porous channel, D3Q19 TRT: random non-overlapping spheres (radius uniform in
  [rmin, rmax]) placed until the fluid fraction drops to the target porosity,
  periodic in x, no-slip walls in y and z, body force along x;
- Taylor-Green vortex, D3Q27 MRT, fully periodic;
- packed bed with a passive scalar and Langmuir adsorption, D3Q19.
"""
from __future__ import annotations

import math
from typing import Optional, Sequence, Tuple

import numpy as np

from . import momentum as m
from . import passive_scalar as ps
from .core import BGK, MRT, TRT, BoundaryFace, CentralMoment, Compat, Storage, VelocitySet

W, E, S, N, B, T = (BoundaryFace.West, BoundaryFace.East, BoundaryFace.South, BoundaryFace.North,
                    BoundaryFace.Bottom, BoundaryFace.Top)


def sphere_pack(n: Sequence[int], porosity: float, rmin: float, rmax: float, seed: int = 1234,
                max_attempts: int = 2_000_000, overlap: bool = False) -> np.ndarray:
    """uint8 solid mask (node order x + nx*(y + ny*z)) of random spheres.

    Centres are uniform over the box, radii uniform in [rmin, rmax]; unless
    `overlap`, a sphere is rejected if it overlaps an accepted one (centre
    distance <= r1 + r2).  A node is solid when its centre (i + 0.5) lies within
    a sphere.  Spheres are added until the fluid fraction is <= `porosity`.
    Random sequential addition without overlap jams near 38 % solid, so
    porosities below about 0.65 need `overlap=True`.
    """
    nx, ny, nz = (int(v) for v in n)
    rng = np.random.default_rng(seed)
    solid = np.zeros((nz, ny, nx), dtype=np.uint8)
    target_solid = (1.0 - porosity) * nx * ny * nz
    n_solid = 0
    cell = 2.0 * rmax
    grid: dict = {}
    centres = []
    attempts = 0
    while n_solid < target_solid and attempts < max_attempts:
        attempts += 1
        c = rng.uniform((0.0, 0.0, 0.0), (nx, ny, nz))
        r = rng.uniform(rmin, rmax)
        key = tuple((c // cell).astype(int))
        ok = True
        for dx in ((-1, 0, 1) if not overlap else ()):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for j in grid.get((key[0] + dx, key[1] + dy, key[2] + dz), ()):
                        cj, rj = centres[j]
                        if np.sum((cj - c) ** 2) <= (r + rj) ** 2:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if not ok:
            continue
        grid.setdefault(key, []).append(len(centres))
        centres.append((c, r))
        lo = np.maximum(np.floor(c - r - 0.5).astype(int), 0)
        hi = np.minimum(np.ceil(c + r + 0.5).astype(int), (nx, ny, nz))
        xs = np.arange(lo[0], hi[0]) + 0.5
        ys = np.arange(lo[1], hi[1]) + 0.5
        zs = np.arange(lo[2], hi[2]) + 0.5
        d2 = ((zs[:, None, None] - c[2]) ** 2 + (ys[None, :, None] - c[1]) ** 2 + (xs[None, None, :] - c[0]) ** 2)
        inside = d2 <= r * r
        sub = solid[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]]
        n_solid += int(np.count_nonzero(inside & (sub == 0)))
        sub[inside] = 1
    return solid.ravel()


def cavity_d2q9(n: int = 128, tau: float = 0.6, u_lid: float = 0.1, storage: Storage = Storage.F64,
                lid_bounce_back: bool = False) -> m.Parameters:
    """D2Q9 BGK lid-driven cavity: NoSlip W/E/S, Zou-He velocity lid (or moving-wall BB) on N."""
    lid = m.BounceBack(1.0, [u_lid, 0.0]) if lid_bounce_back else m.ZouHe(None, [u_lid, 0.0])
    return m.Parameters(n=[n, n], collision_operator=BGK(tau), velocity_set=VelocitySet.D2Q9,
                        initial_density=m.InitialDensity.Uniform(1.0),
                        initial_velocity=m.InitialVelocity.Uniform([0.0, 0.0]),
                        boundary_conditions=[(W, m.NoSlip), (E, m.NoSlip), (S, m.NoSlip), (N, lid)],
                        storage=storage)


def porous_channel_d3q19(n: Sequence[int] = (256, 256, 256), porosity: float = 0.7, rmin: float = 4.0,
                         rmax: float = 10.0, seed: int = 1234, tau_plus: float = 0.8, magic: float = 0.25,
                         force: float = 1e-6, storage: Storage = Storage.F32,
                         mask: Optional[np.ndarray] = None, compat: Compat = Compat.REFERENCE) -> m.Parameters:
    """D3Q19 TRT porous channel: periodic x, NoSlip y/z walls, body force g_x."""
    if mask is None:
        mask = sphere_pack(n, porosity, rmin, rmax, seed)
    return m.Parameters(n=list(n), collision_operator=TRT.from_magic(tau_plus, magic), force=[force, 0.0, 0.0],
                        velocity_set=VelocitySet.D3Q19, initial_density=m.InitialDensity.Uniform(1.0),
                        initial_velocity=m.InitialVelocity.Uniform([0.0, 0.0, 0.0]),
                        boundary_conditions=[(W, m.Periodic), (E, m.Periodic), (S, m.NoSlip), (N, m.NoSlip),
                                             (B, m.NoSlip), (T, m.NoSlip)],
                        node_types=m.NodeTypes.FromArray(mask), storage=storage, compat=compat)


def tgv_rates(tau: float, q: int = 27, other: float = 1.0) -> list:
    """MRT rates for the D3Q27 basis: shear moments (rows 5-9) relax at 1/tau, bulk (row 4)
    and the higher moments at `other`; conserved rows at 1."""
    s = [1.0] * 4 + [other] + [1.0 / tau] * 5 + [other] * (q - 10)
    return s


def tgv_d3q27(n: int = 384, u0: float = 0.05, re: float = 1600.0, storage: Storage = Storage.F32,
              other_rate: float = 1.0, collision: str = "mrt") -> Tuple[m.Parameters, float]:
    """Taylor-Green vortex: u = u0 (sin x cos y cos z, -cos x sin y cos z, 0), rho = 1,
    x = 2 pi (i + 1/2) / n, nu = u0 (n / 2 pi) / Re; returns (params, nu).
    collision: "mrt" (raw-moment MRT on the engine's D3Q27 basis) or "central"
    (central moments, higher orders relaxed with `other_rate`)."""
    nu = u0 * (n / (2.0 * math.pi)) / re
    tau = 3.0 * nu + 0.5
    i = (np.arange(n) + 0.5) * 2.0 * math.pi / n
    z, y, x = np.meshgrid(i, i, i, indexing="ij")
    u = np.zeros((n, n, n, 3))
    u[..., 0] = u0 * np.sin(x) * np.cos(y) * np.cos(z)
    u[..., 1] = -u0 * np.cos(x) * np.sin(y) * np.cos(z)
    op = (CentralMoment(tau, other_rate, (other_rate,) * 4) if collision == "central"
          else MRT(tgv_rates(tau, 27, other_rate)))
    p = m.Parameters(n=[n, n, n], collision_operator=op,
                     velocity_set=VelocitySet.D3Q27, initial_density=m.InitialDensity.Uniform(1.0),
                     initial_velocity=m.InitialVelocity.FromArray(u.reshape(-1, 3)),
                     boundary_conditions=[(f, m.Periodic) for f in (W, E, S, N, B, T)], storage=storage)
    return p, nu


def packed_bed_scalar(n: Sequence[int] = (192, 192, 384), porosity: float = 0.6, rmin: float = 4.0,
                      rmax: float = 10.0, seed: int = 1234, u_in: float = 0.04, tau: float = 0.6,
                      tau_g: float = 0.55, ka: float = 1e-3, kd: float = 1e-5, q_max: float = 1.0,
                      storage: Storage = Storage.F32, zou_he_inlet: bool = True,
                      mask: Optional[np.ndarray] = None, collision=None) -> Tuple[m.Parameters, ps.Parameters]:
    """Coupled D3Q19 flow + scalar with Langmuir adsorption through a sphere packing.

    Inlet z = 0 (Bottom): Zou-He velocity u_z (engine extension) or, for the
    reference-expressible variant, a moving-wall BounceBack with the same
    velocity; scalar Dirichlet C = 1.  Outlet z = nz-1 (Top): AntiBounceBack
    density 1; scalar second-order extrapolation outflow (all populations).  Side
    walls: NoSlip, scalar BBNoFlux.
    """
    if mask is None:
        mask = sphere_pack(n, porosity, rmin, rmax, seed)
    inlet = m.ZouHe(None, [0.0, 0.0, u_in]) if zou_he_inlet else m.BounceBack(1.0, [0.0, 0.0, u_in])
    mp = m.Parameters(n=list(n), collision_operator=collision or BGK(tau), velocity_set=VelocitySet.D3Q19,
                      initial_density=m.InitialDensity.Uniform(1.0),
                      initial_velocity=m.InitialVelocity.Uniform([0.0, 0.0, 0.0]),
                      boundary_conditions=[(W, m.NoSlip), (E, m.NoSlip), (S, m.NoSlip), (N, m.NoSlip),
                                           (B, inlet), (T, m.AntiBounceBack(1.0))],
                      node_types=m.NodeTypes.FromArray(mask), storage=storage)
    sp = ps.Parameters(scalar_name="concentration", collision_operator=BGK(tau_g),
                       initial_scalar_value=ps.InitialScalarValue.Uniform(0.0), velocity_set=VelocitySet.D3Q19,
                       boundary_conditions=[(W, ps.BBNoFlux), (E, ps.BBNoFlux), (S, ps.BBNoFlux),
                                            (N, ps.BBNoFlux), (B, ps.AntiBounceBack(1.0)),
                                            (T, ps.SecondOrderNoFlux(unknown_populations_only=False))],
                       inner_boundary_condition=ps.InnerBounceBack,
                       adsorption_parameters=ps.AdsorptionParameters(ps.Langmuir(ka, kd, q_max), 0.0))
    return mp, sp
