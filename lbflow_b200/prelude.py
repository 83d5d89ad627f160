"""`from lbflow_b200.prelude import *` -- the names of the reference's prelude
(src/prelude.rs:1-15)."""
from . import momentum, passive_scalar  # noqa: F401
from . import momentum as m  # noqa: F401
from . import passive_scalar as ps  # noqa: F401
from .core import BGK, MRT, TRT, BoundaryFace, CollisionOperator, NodeType, VelocitySet  # noqa: F401
from .core import CentralMoment, Compat, Storage  # noqa: F401
from .momentum import InitialDensity, InitialVelocity, NodeTypes  # noqa: F401
from .momentum import FromBounceBackMapFile, OnlyFluidNodes  # noqa: F401
from .passive_scalar import AdsorptionParameters, InitialScalarValue, Langmuir  # noqa: F401

West, East, South, North, Bottom, Top = (BoundaryFace.West, BoundaryFace.East, BoundaryFace.South,
                                         BoundaryFace.North, BoundaryFace.Bottom, BoundaryFace.Top)
Fluid, Solid = NodeType.Fluid, NodeType.Solid
D2Q5, D2Q9, D3Q15, D3Q19, D3Q27 = (VelocitySet.D2Q5, VelocitySet.D2Q9, VelocitySet.D3Q15,
                                   VelocitySet.D3Q19, VelocitySet.D3Q27)
