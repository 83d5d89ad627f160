"""`passive_scalar` module: Parameters, boundary conditions and adsorption.

Mirrors passive_scalar::Parameters (src/passive_scalar.rs:16-25),
passive_scalar::bc::{BoundaryCondition, InnerBoundaryCondition}
(src/passive_scalar/bc.rs:9-35), adsorption::{AdsorptionModel::Langmuir,
Parameters} (src/passive_scalar/adsorption.rs:4-28) and InitialScalarValue
(src/passive_scalar/io.rs:154-171).
"""
from __future__ import annotations

import enum
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _abi
from .core import BGK, BoundaryFace, CollisionOperator, FACES_2D, FACES_3D, VelocitySet


class BoundaryCondition:
    kind: int = -1

    def fill(self, d: _abi.ScalarBcDesc) -> None:
        d.kind = self.kind


@dataclass(frozen=True)
class AntiBounceBack(BoundaryCondition):
    """Dirichlet value by anti-bounce-back (src/passive_scalar/bc.rs:107-136)."""
    scalar_value: float = 0.0
    kind: int = _abi.LBF_SBC_ANTI_BOUNCE_BACK

    def fill(self, d):
        d.kind = self.kind
        d.scalar_value = float(self.scalar_value)


@dataclass(frozen=True)
class _Flagless(BoundaryCondition):
    kind: int = -1


AntiBBNoFlux = _Flagless(kind=_abi.LBF_SBC_ANTI_BB_NO_FLUX)
BBNoFlux = _Flagless(kind=_abi.LBF_SBC_BB_NO_FLUX)
Periodic = _Flagless(kind=_abi.LBF_SBC_PERIODIC)


@dataclass(frozen=True)
class ZerothOrderNoFlux(BoundaryCondition):
    unknown_populations_only: bool = False
    kind: int = _abi.LBF_SBC_ZEROTH_ORDER_NO_FLUX

    def fill(self, d):
        d.kind = self.kind
        d.unknown_populations_only = int(bool(self.unknown_populations_only))


@dataclass(frozen=True)
class SecondOrderNoFlux(BoundaryCondition):
    unknown_populations_only: bool = True
    kind: int = _abi.LBF_SBC_SECOND_ORDER_NO_FLUX

    def fill(self, d):
        d.kind = self.kind
        d.unknown_populations_only = int(bool(self.unknown_populations_only))


class InnerBoundaryCondition(enum.IntEnum):
    InnerAntiBounceBack = _abi.LBF_INNER_ANTI_BOUNCE_BACK
    InnerBounceBack = _abi.LBF_INNER_BOUNCE_BACK


InnerAntiBounceBack = InnerBoundaryCondition.InnerAntiBounceBack
InnerBounceBack = InnerBoundaryCondition.InnerBounceBack


@dataclass(frozen=True)
class Langmuir:
    """AdsorptionModel::Langmuir: r = k_a C (q_max - q) - k_d q."""
    adsorption_rate: float
    desorption_rate: float
    q_max: float


@dataclass(frozen=True)
class AdsorptionParameters:
    """adsorption::Parameters::new(adsorption_model, initial_q_ads)."""
    adsorption_model: Langmuir
    initial_q_ads: float = 0.0


class InitialScalarValue:
    def __init__(self, kind: str, value=None):
        self.kind, self.value = kind, value

    @staticmethod
    def Uniform(value: float) -> "InitialScalarValue":
        return InitialScalarValue("uniform", float(value))

    @staticmethod
    def FromFile(path: str) -> "InitialScalarValue":
        return InitialScalarValue("file", path)

    @staticmethod
    def FromTimeStep(t: int) -> "InitialScalarValue":
        return InitialScalarValue("time_step", int(t))

    @staticmethod
    def FromArray(values) -> "InitialScalarValue":
        return InitialScalarValue("array", np.ascontiguousarray(values, dtype=np.float64).ravel())

    def generate(self, n, scalar_name: str):
        from . import io
        if self.kind == "uniform":
            return None
        if self.kind == "file":
            return io.read_scalar_csv(self.value)
        if self.kind == "time_step":
            return io.read_scalar_csv(os.path.join(io.DATA_PATH, str(self.value), f"{scalar_name}.csv"))
        return self.value


@dataclass
class Parameters:
    """passive_scalar::Parameters.  `source_value` is a constant (the reference's closure)."""
    scalar_name: str = "scalar"
    collision_operator: CollisionOperator = field(default_factory=lambda: BGK(0.5))
    source_value: Optional[float] = None
    initial_scalar_value: InitialScalarValue = field(default_factory=lambda: InitialScalarValue.Uniform(0.0))
    velocity_set: VelocitySet = VelocitySet.D2Q9
    boundary_conditions: List[Tuple[BoundaryFace, BoundaryCondition]] = field(default_factory=list)
    inner_boundary_condition: InnerBoundaryCondition = InnerBoundaryCondition.InnerBounceBack
    adsorption_parameters: Optional[AdsorptionParameters] = None


def to_desc(p: Parameters, n: Sequence[int]):
    vs = VelocitySet(p.velocity_set)
    d = _abi.ScalarDesc()
    d.velocity_set = int(vs)
    d.inner_boundary_condition = int(p.inner_boundary_condition)
    d.collision = p.collision_operator.to_desc()
    if p.source_value is not None:
        d.has_source = 1
        d.source_value = float(p.source_value)
    keep = []
    init = p.initial_scalar_value.generate(n, p.scalar_name)
    if init is None:
        d.initial_scalar_value = float(p.initial_scalar_value.value)
    else:
        arr = np.ascontiguousarray(init, dtype=np.float64).ravel()
        if arr.size != int(np.prod(n)):
            raise ValueError("initial scalar field has the wrong length")
        keep.append(arr)
        d.initial_scalar_field = arr.ctypes.data
    faces = FACES_2D if vs.d == 2 else FACES_3D
    given = dict(p.boundary_conditions)
    for f in faces:
        if f not in given:
            raise ValueError("Boundary faces not found")
        given[f].fill(d.bc[int(f)])
    for f in range(len(faces), 6):
        d.bc[f].kind = _abi.LBF_SBC_PERIODIC
    if p.adsorption_parameters is not None:
        a = p.adsorption_parameters
        d.has_adsorption = 1
        d.adsorption_rate = float(a.adsorption_model.adsorption_rate)
        d.desorption_rate = float(a.adsorption_model.desorption_rate)
        d.q_max = float(a.adsorption_model.q_max)
        d.initial_q_ads = float(a.initial_q_ads)
    return d, keep
