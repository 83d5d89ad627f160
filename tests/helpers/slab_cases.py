"""Small global lattices for the z-slab decomposition tests."""
from lbflow_b200 import cases
from lbflow_b200 import momentum as m
from lbflow_b200.core import BGK, BoundaryFace, Storage, VelocitySet


def case(name: str) -> m.Parameters:
    if name == "walls":          # D3Q19 TRT porous channel, no-slip y and z walls, periodic x
        mask = cases.sphere_pack([10, 8, 13], 0.75, 1.2, 2.2, seed=11)
        return cases.porous_channel_d3q19([10, 8, 13], mask=mask, force=1e-5, storage=Storage.F64)
    if name == "d3q27":          # D3Q27 BGK porous medium, periodic in x and z, no-slip y, body force
        mask = cases.sphere_pack([9, 8, 12], 0.8, 1.2, 2.0, seed=3)
        F = BoundaryFace
        return m.Parameters(n=[9, 8, 12], collision_operator=BGK(0.8), velocity_set=VelocitySet.D3Q27,
                            force=[1e-5, 0.0, 2e-6], initial_density=m.InitialDensity.Uniform(1.0),
                            initial_velocity=m.InitialVelocity.Uniform([0.0, 0.0, 0.0]),
                            boundary_conditions=[(F.West, m.Periodic), (F.East, m.Periodic), (F.South, m.NoSlip),
                                                 (F.North, m.NoSlip), (F.Bottom, m.Periodic), (F.Top, m.Periodic)],
                            node_types=m.NodeTypes.FromArray(mask), storage=Storage.F64)
    if name == "periodic":       # D3Q19 BGK, periodic z, Zou-He / anti-bounce-back in x, no-slip y
        mask = cases.sphere_pack([12, 8, 11], 0.8, 1.2, 2.0, seed=5)
        F = BoundaryFace
        return m.Parameters(n=[12, 8, 11], collision_operator=BGK(0.7), velocity_set=VelocitySet.D3Q19,
                            initial_density=m.InitialDensity.Uniform(1.0),
                            initial_velocity=m.InitialVelocity.Uniform([0.0, 0.0, 0.0]),
                            boundary_conditions=[(F.West, m.ZouHe(None, [0.03, 0.0, 0.0])),
                                                 (F.East, m.AntiBounceBack(1.0)), (F.South, m.NoSlip),
                                                 (F.North, m.NoSlip), (F.Bottom, m.Periodic), (F.Top, m.Periodic)],
                            node_types=m.NodeTypes.FromArray(mask), storage=Storage.F64)
    raise KeyError(name)
