"""`momentum` module: Parameters and boundary conditions of the flow lattice.

Mirrors momentum::Parameters (src/momentum.rs:22-37),
momentum::bc::BoundaryCondition (src/momentum/bc.rs:12-26) and the
InitialDensity / InitialVelocity / NodeTypes enums of src/momentum/io.rs:358-411.
`to_desc` turns a Parameters value into the C-ABI lbf_domain_desc.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence, Tuple, Union

import numpy as np

from . import _abi
from .core import (BGK, BoundaryFace, CollisionOperator, Compat, FACES_2D, FACES_3D, Storage,
                   VelocitySet)


# ---------------------------------------------------------------- boundary conditions
class BoundaryCondition:
    kind: int = -1

    def fill(self, d: _abi.BcDesc, dim: int) -> None:
        d.kind = self.kind


@dataclass(frozen=True)
class _NoSlip(BoundaryCondition):
    kind: int = _abi.LBF_BC_NO_SLIP


@dataclass(frozen=True)
class _Periodic(BoundaryCondition):
    kind: int = _abi.LBF_BC_PERIODIC


NoSlip = _NoSlip()
Periodic = _Periodic()


@dataclass(frozen=True)
class BounceBack(BoundaryCondition):
    """Moving-wall bounce-back (src/momentum/bc.rs:62-84)."""
    density: float = 1.0
    velocity: Sequence[float] = (0.0, 0.0, 0.0)
    kind: int = _abi.LBF_BC_BOUNCE_BACK

    def fill(self, d, dim):
        d.kind = self.kind
        d.density = float(self.density)
        d.has_density = 1
        for a, v in enumerate(list(self.velocity)[:3]):
            d.velocity[a] = float(v)
            d.has_velocity[a] = 1


@dataclass(frozen=True)
class AntiBounceBack(BoundaryCondition):
    """Pressure boundary by anti-bounce-back (src/momentum/bc.rs:86-117)."""
    density: float = 1.0
    kind: int = _abi.LBF_BC_ANTI_BOUNCE_BACK

    def fill(self, d, dim):
        d.kind = self.kind
        d.density = float(self.density)
        d.has_density = 1


@dataclass(frozen=True)
class ZouHe(BoundaryCondition):
    """ZouHe { density: Option<f64>, velocity: Vec<Option<f64>> } (src/momentum/bc.rs:21-24).

    D2Q9 follows src/velocity_set/d2q9.rs:165-245; D3Q19 and D3Q27 are an
    extension of this engine (the reference has no 3-D Zou-He).
    """
    density: Optional[float] = None
    velocity: Sequence[Optional[float]] = (None, None, None)
    kind: int = _abi.LBF_BC_ZOU_HE

    def fill(self, d, dim):
        d.kind = self.kind
        d.has_density = int(self.density is not None)
        d.density = 0.0 if self.density is None else float(self.density)
        for a, v in enumerate(list(self.velocity)[:3]):
            d.has_velocity[a] = int(v is not None)
            d.velocity[a] = 0.0 if v is None else float(v)


# ---------------------------------------------------------------- initial fields
class InitialDensity:
    """InitialDensity::{Uniform, FromFile, FromTimeStep} (src/momentum/io.rs:358-374)."""

    def __init__(self, kind: str, value=None):
        self.kind, self.value = kind, value

    @staticmethod
    def Uniform(value: float) -> "InitialDensity":
        return InitialDensity("uniform", float(value))

    @staticmethod
    def FromFile(path: str) -> "InitialDensity":
        return InitialDensity("file", path)

    @staticmethod
    def FromTimeStep(t: int) -> "InitialDensity":
        return InitialDensity("time_step", int(t))

    @staticmethod
    def FromArray(values) -> "InitialDensity":
        """Extension: a per-node array (length N, node order x + nx*(y + ny*z))."""
        return InitialDensity("array", np.ascontiguousarray(values, dtype=np.float64).ravel())

    def generate(self, n: Sequence[int]):
        """None for uniform values, else the per-node array."""
        from . import io
        if self.kind == "uniform":
            return None
        if self.kind == "file":
            return io.read_scalar_csv(self.value)
        if self.kind == "time_step":
            return io.read_scalar_csv(os.path.join(io.DATA_PATH, str(self.value), io.DENSITY_FILE))
        return self.value


class InitialVelocity:
    """InitialVelocity::{Uniform, FromFile, FromTimeStep} (src/momentum/io.rs:376-394)."""

    def __init__(self, kind: str, value=None):
        self.kind, self.value = kind, value

    @staticmethod
    def Uniform(value: Sequence[float]) -> "InitialVelocity":
        return InitialVelocity("uniform", [float(v) for v in value])

    @staticmethod
    def FromFile(path: str) -> "InitialVelocity":
        return InitialVelocity("file", path)

    @staticmethod
    def FromTimeStep(t: int) -> "InitialVelocity":
        return InitialVelocity("time_step", int(t))

    @staticmethod
    def FromArray(values) -> "InitialVelocity":
        """Extension: per-node velocities, shape (N, D)."""
        return InitialVelocity("array", np.ascontiguousarray(values, dtype=np.float64))

    def generate(self, n: Sequence[int]):
        from . import io
        if self.kind == "uniform":
            return None
        if self.kind == "file":
            return io.read_vector_csv(self.value)
        if self.kind == "time_step":
            return io.read_vector_csv(os.path.join(io.DATA_PATH, str(self.value), io.VELOCITY_FILE))
        return self.value


class NodeTypes:
    """NodeTypes::{OnlyFluidNodes, FromBounceBackMapFile} (src/momentum/io.rs:396-411)."""

    def __init__(self, kind: str, value=None):
        self.kind, self.value = kind, value

    def generate(self, n: Sequence[int]) -> Optional[np.ndarray]:
        """None for all-fluid, else a uint8 mask (0 fluid, 1 solid) of length N."""
        from . import io
        if self.kind == "fluid":
            return None
        if self.kind == "map":
            mask = io.read_bounce_back_map(os.path.join(io.PRE_PROCESSING_PATH, io.BOUNCE_BACK_MAP_FILE))
        else:
            mask = np.ascontiguousarray(self.value, dtype=np.uint8).ravel()
        if mask.size != int(np.prod(n)):
            raise ValueError(f"Number of nodes ({int(np.prod(n))}) does not match the length of node "
                             f"types ({mask.size})")
        return mask

    @staticmethod
    def FromArray(mask) -> "NodeTypes":
        """Extension: a uint8 mask in node order (0 fluid, 1 solid)."""
        return NodeTypes("array", mask)


NodeTypes.OnlyFluidNodes = NodeTypes("fluid")
NodeTypes.FromBounceBackMapFile = NodeTypes("map")
OnlyFluidNodes = NodeTypes.OnlyFluidNodes
FromBounceBackMapFile = NodeTypes.FromBounceBackMapFile


# ---------------------------------------------------------------- Parameters
@dataclass
class Parameters:
    """momentum::Parameters (src/momentum.rs:22-69); defaults as Parameters::default.

    `force` is a constant body-force vector (the reference's closure
    `Fn(&Node) -> Vec<f64>` evaluated to a constant).  `storage`, `compat`
    and `face_order` are engine options with no reference counterpart.
    """
    n: List[int] = field(default_factory=lambda: [10, 10])
    collision_operator: CollisionOperator = field(default_factory=lambda: BGK(0.5))
    force: Optional[Sequence[float]] = None
    delta_x: float = 0.01
    delta_t: float = 0.01
    physical_density: float = 998.0
    reference_pressure: float = 101325.0
    initial_density: InitialDensity = field(default_factory=lambda: InitialDensity.Uniform(1.0))
    initial_velocity: InitialVelocity = field(default_factory=lambda: InitialVelocity.Uniform([0.0, 0.0]))
    velocity_set: VelocitySet = VelocitySet.D2Q9
    boundary_conditions: List[Tuple[BoundaryFace, BoundaryCondition]] = field(default_factory=lambda: [
        (BoundaryFace.West, NoSlip), (BoundaryFace.East, NoSlip), (BoundaryFace.South, NoSlip),
        (BoundaryFace.North, BounceBack(density=1.0, velocity=[0.1, 0.0]))])
    node_types: NodeTypes = field(default_factory=lambda: NodeTypes.OnlyFluidNodes)
    post_functions: Optional[list] = None
    storage: Storage = Storage.F64
    compat: Compat = Compat.REFERENCE
    face_order: Optional[Sequence[BoundaryFace]] = None

    @property
    def dim(self) -> int:
        return VelocitySet(self.velocity_set).d

    @property
    def num_nodes(self) -> int:
        return int(np.prod(self.n[: self.dim]))


def to_desc(p: Parameters):
    """Build the lbf_domain_desc for `p`; returns (desc, keepalive arrays)."""
    vs = VelocitySet(p.velocity_set)
    dim = vs.d
    if len(p.n) < dim:
        raise ValueError(f"n must have {dim} entries")
    desc = _abi.DomainDesc()
    desc.velocity_set = int(vs)
    desc.storage = int(p.storage)
    desc.compat = int(p.compat)
    for a in range(3):
        desc.n[a] = int(p.n[a]) if a < dim else 1
    desc.collision = p.collision_operator.to_desc()
    if p.force is not None:
        desc.has_force = 1
        for a, v in enumerate(list(p.force)[:3]):
            desc.force[a] = float(v)
    faces = FACES_2D if dim == 2 else FACES_3D
    given = dict(p.boundary_conditions)
    for f in faces:
        if f not in given:
            raise ValueError("Boundary faces not found")   # lattice.rs:238-245 panics
        given[f].fill(desc.bc[int(f)], dim)
    for f in range(6):
        if f >= len(faces):
            desc.bc[f].kind = _abi.LBF_BC_PERIODIC
    if p.face_order is not None:
        order = [int(f) for f in p.face_order]
        for i, f in enumerate(order):
            desc.face_order[i] = f
    keep = []
    n = [int(x) for x in p.n[:dim]]
    N = int(np.prod(n))
    mask = p.node_types.generate(n)
    if mask is not None:
        mask = np.ascontiguousarray(mask, dtype=np.uint8)
        keep.append(mask)
        desc.node_type = mask.ctypes.data
    rho = p.initial_density.generate(n)
    if rho is None:
        desc.initial_density = float(p.initial_density.value)
    else:
        rho = np.ascontiguousarray(rho, dtype=np.float64).ravel()
        if rho.size != N:
            raise ValueError("initial density field has the wrong length")
        keep.append(rho)
        desc.initial_density_field = rho.ctypes.data
    u = p.initial_velocity.generate(n)
    if u is None:
        for a, v in enumerate(list(p.initial_velocity.value)[:3]):
            desc.initial_velocity[a] = float(v)
    else:
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(N, dim)
        keep.append(u)
        desc.initial_velocity_field = u.ctypes.data
    return desc, keep
