"""lbflow_b200 -- a B200-native lattice Boltzmann engine with lbflow's API.

The hot path (fused collide-and-stream over D2Q9/D3Q19/D3Q27 with BGK/TRT/MRT,
bounce-back, Zou-He and face boundaries, and the coupled passive scalar with
Langmuir adsorption) runs as hand-written sm_100a CUDA kernels in
liblbflow_b200.so, behind the C ABI of include/lbflow.h.  This package is the
host side: the reference's parameter types (`momentum`, `passive_scalar`), the
`solve` driver with the reference's file outputs, the `post` tools (VTK files,
chunk unification), and ctypes bindings.
"""
from . import _abi, core, io, momentum, passive_scalar, post  # noqa: F401
from .core import (BGK, MRT, TRT, BoundaryFace, CentralMoment, CollisionOperator, Compat, NodeType,  # noqa: F401
                   Storage, VelocitySet)

__all__ = ["momentum", "passive_scalar", "io", "post", "core", "BGK", "TRT", "MRT", "BoundaryFace",
           "NodeType", "VelocitySet", "Storage", "Compat", "solve", "Domain"]


def __getattr__(name):
    # Heavy pieces load the CUDA library; import them lazily.
    if name == "Domain":
        from .domain import Domain
        return Domain
    if name == "solve":
        from .solver import solve
        return solve
    raise AttributeError(name)
