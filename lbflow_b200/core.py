"""Core enums and collision operators, mirroring the reference's public types.

BoundaryFace, NodeType, CollisionOperator (src/lib.rs:17-42) and VelocitySet
(src/velocity_set.rs:19-25), with the same discriminants, which are also the
values of the C ABI enums in include/lbflow.h.
"""
from __future__ import annotations

import enum
from dataclasses import dataclass, field
from typing import List, Tuple

from . import _abi


class BoundaryFace(enum.IntEnum):
    West = _abi.LBF_WEST
    East = _abi.LBF_EAST
    South = _abi.LBF_SOUTH
    North = _abi.LBF_NORTH
    Bottom = _abi.LBF_BOTTOM
    Top = _abi.LBF_TOP


FACES_2D = [BoundaryFace.West, BoundaryFace.East, BoundaryFace.South, BoundaryFace.North]
FACES_3D = FACES_2D + [BoundaryFace.Bottom, BoundaryFace.Top]


class NodeType(enum.IntEnum):
    Fluid = 0
    Solid = 1


class VelocitySet(enum.IntEnum):
    D2Q5 = _abi.LBF_D2Q5
    D2Q9 = _abi.LBF_D2Q9
    D3Q15 = _abi.LBF_D3Q15
    D3Q19 = _abi.LBF_D3Q19
    D3Q27 = _abi.LBF_D3Q27

    @property
    def d(self) -> int:
        return 2 if self in (VelocitySet.D2Q5, VelocitySet.D2Q9) else 3

    @property
    def q(self) -> int:
        return {0: 5, 1: 9, 2: 15, 3: 19, 4: 27}[int(self)]


class Storage(enum.IntEnum):
    """Population storage on the device (compute is FP64 for F64, FP32 otherwise)."""
    F64 = _abi.LBF_STORE_F64
    F32 = _abi.LBF_STORE_F32
    F16DEV = _abi.LBF_STORE_F16DEV
    BF16DEV = _abi.LBF_STORE_BF16DEV


class Compat(enum.IntEnum):
    REFERENCE = _abi.LBF_COMPAT_REFERENCE
    PHYSICS = _abi.LBF_COMPAT_PHYSICS


class CollisionOperator:
    """CollisionOperator::{BGK, TRT, MRT} (src/lib.rs:37-42)."""

    def to_desc(self) -> _abi.CollisionDesc:
        raise NotImplementedError


@dataclass(frozen=True)
class BGK(CollisionOperator):
    tau: float

    def to_desc(self):
        d = _abi.CollisionDesc()
        d.kind = _abi.LBF_BGK
        d.tau = float(self.tau)
        return d


@dataclass(frozen=True)
class TRT(CollisionOperator):
    """TRT(omega_plus, omega_minus): relaxation *rates* (src/kernel.rs:44-65)."""
    omega_plus: float
    omega_minus: float

    @staticmethod
    def from_magic(tau_plus: float, magic: float = 0.25) -> "TRT":
        """Rates from tau_plus and the magic parameter (tau+ - 1/2)(tau- - 1/2)."""
        tau_minus = 0.5 + magic / (tau_plus - 0.5)
        return TRT(1.0 / tau_plus, 1.0 / tau_minus)

    def to_desc(self):
        d = _abi.CollisionDesc()
        d.kind = _abi.LBF_TRT
        d.omega_plus = float(self.omega_plus)
        d.omega_minus = float(self.omega_minus)
        return d


@dataclass(frozen=True)
class MRT(CollisionOperator):
    """MRT(relaxation_vector): one rate per moment, length Q (src/kernel.rs:67-120)."""
    relaxation_vector: List[float] = field(default_factory=list)

    def to_desc(self):
        d = _abi.CollisionDesc()
        d.kind = _abi.LBF_MRT
        if len(self.relaxation_vector) > 27:
            raise ValueError("relaxation vector longer than 27")
        for i, s in enumerate(self.relaxation_vector):
            d.relaxation[i] = float(s)
        return d


@dataclass(frozen=True)
class CentralMoment(CollisionOperator):
    """Central-moment collision of the tensor-product sets D2Q9 and D3Q27 (engine
    extension; the reference has no D3Q27 collision): shear relaxation 1/tau,
    the trace of the second-order moments at `bulk`, third to sixth orders at
    `higher` (four rates; 1 relaxes them fully to the equilibrium)."""
    tau: float
    bulk: float = 1.0
    higher: Tuple[float, float, float, float] = (1.0, 1.0, 1.0, 1.0)

    def to_desc(self):
        d = _abi.CollisionDesc()
        d.kind = _abi.LBF_CENTRAL
        d.tau = float(self.tau)
        d.relaxation[0] = float(self.bulk)
        for i, w in enumerate(self.higher):
            d.relaxation[1 + i] = float(w)
        return d


def collision_from_desc(d: _abi.CollisionDesc, q: int) -> CollisionOperator:
    if d.kind == _abi.LBF_BGK:
        return BGK(d.tau)
    if d.kind == _abi.LBF_TRT:
        return TRT(d.omega_plus, d.omega_minus)
    if d.kind == _abi.LBF_CENTRAL:
        return CentralMoment(d.tau, d.relaxation[0], tuple(d.relaxation[1 + i] for i in range(4)))
    return MRT([d.relaxation[i] for i in range(q)])
