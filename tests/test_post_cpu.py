"""The `post vtk` and `post unify` tools (lbflow_b200/post.py) on cases written
here on the CPU: the VTK text is compared line by line with the layout of
src/momentum/post/vtk.rs:89-205 and src/passive_scalar/post/vtk.rs:27-40
(legacy ASCII structured grid, Rust {:.4e} points and {:.8e} values), and a
case written in chunks (num_threads > 1) unifies to the single-file output."""
import os

import numpy as np

from lbflow_b200 import io, post
from lbflow_b200 import momentum as m
from lbflow_b200 import passive_scalar as ps
from lbflow_b200.core import BGK, MRT, TRT, VelocitySet


def _case(tmp_path, n, dim, steps=(0, 50), threads=1, scalars=("c",)):
    root = str(tmp_path / "data")
    N = int(np.prod(n))
    solid = np.zeros(N, np.uint8)
    solid[1] = 1
    io.write_coordinates(n, solid, 0.01, root=root)
    fields = {}
    for t in steps:
        rho = 1.0 + 0.25 * np.arange(N) / N + 1e-3 * t
        u = np.linspace(-0.02, 0.03, N * dim).reshape(N, dim) * (1 + t)
        sc = {s: np.full(N, 0.5 + 0.1 * i) + 1e-4 * t for i, s in enumerate(scalars)}
        io.write_step_data(t, rho, u, sc, num_threads=threads, root=root)
        fields[t] = (rho, u, sc)
    return solid, fields


def test_vtk_layout_2d_with_physical_data_and_scalar(tmp_path):
    n = [2, 2]
    solid, fields = _case(tmp_path, n, 2)
    mp = m.Parameters(n=n, collision_operator=BGK(0.8), velocity_set=VelocitySet.D2Q9)
    sp = ps.Parameters(scalar_name="c", velocity_set=VelocitySet.D2Q9)
    paths = post.post_vtk(mp, sp, case_dir=str(tmp_path), case_name="cav", physical_data=True)
    vtk = str(tmp_path / "post_processing" / "vtk_files")
    assert sorted(os.path.basename(p) for p in paths) == ["cav_node_type.vtk", "cav_output_00000000.vtk",
                                                           "cav_output_00000050.vtk"]
    head = ["# vtk DataFile Version 3.0", "lbflow simulation data", "ASCII", "DATASET STRUCTURED_GRID",
            "DIMENSIONS 2 2 1", "POINTS 4 float",
            "5.0000e-3 5.0000e-3 0.0000e0", "1.5000e-2 5.0000e-3 0.0000e0",
            "5.0000e-3 1.5000e-2 0.0000e0", "1.5000e-2 1.5000e-2 0.0000e0", "POINT_DATA 4"]
    nt = open(os.path.join(vtk, "cav_node_type.vtk")).read().split("\n")
    assert nt == head + ["SCALARS node_type float 1", "LOOKUP_TABLE default", "0", "1", "0", "0", ""]
    out = open(os.path.join(vtk, "cav_output_00000000.vtk")).read().split("\n")
    rho, u, sc = fields[0]
    want = head + ["SCALARS density float 1", "LOOKUP_TABLE default",
                   "1.00000000e0", "1.06250000e0", "1.12500000e0", "1.18750000e0",
                   "VECTORS velocity float"]
    want += [f"{io.rust_e8(a)} {io.rust_e8(b)} 0.00000000e0" for a, b in u]
    # p = p_ref + cs^2 (rho - 1) rho_phys (dx/dt)^2 = 101325 + (rho - 1) 998 / 3; u_phys = u dx/dt
    want += ["SCALARS physical_pressure float 1", "LOOKUP_TABLE default",
             "1.01325000e5", "1.01345792e5", "1.01366583e5", "1.01387375e5", "VECTORS physical_velocity float"]
    want += [f"{io.rust_e8(a)} {io.rust_e8(b)} 0.00000000e0" for a, b in u]
    want += ["SCALARS c float 1", "LOOKUP_TABLE default"] + ["5.00000000e-1"] * 4 + [""]
    assert out == want


def test_vtk_3d_several_scalars(tmp_path):
    n = [3, 2, 2]
    _, fields = _case(tmp_path, n, 3, scalars=("a", "b"))
    mp = m.Parameters(n=n, collision_operator=TRT.from_magic(0.7), velocity_set=VelocitySet.D3Q19)
    sps = [ps.Parameters(scalar_name=s, velocity_set=VelocitySet.D3Q19) for s in ("a", "b")]
    post.post_vtk(mp, sps, case_dir=str(tmp_path), case_name="bed", node_type=False)
    text = open(str(tmp_path / "post_processing" / "vtk_files" / "bed_output_00000050.vtk")).read()
    lines = text.split("\n")
    assert lines[4] == "DIMENSIONS 3 2 2" and lines[5] == "POINTS 12 float"
    assert lines[6] == "5.0000e-3 5.0000e-3 5.0000e-3" and lines[17] == "2.5000e-2 1.5000e-2 1.5000e-2"
    rho, u, sc = fields[50]
    i = lines.index("SCALARS density float 1")
    assert [float(x) for x in lines[i + 2:i + 14]] == [float(io.rust_e8(v)) for v in rho]
    j = lines.index("VECTORS velocity float")
    got = np.array([[float(x) for x in s.split(" ")] for s in lines[j + 1:j + 13]])
    assert np.array_equal(got, np.array([[float(io.rust_e8(v)) for v in row] for row in u]))
    assert "physical_pressure" not in text
    for name in ("a", "b"):
        k = lines.index(f"SCALARS {name} float 1")
        assert lines[k + 1] == "LOOKUP_TABLE default"
        assert [float(x) for x in lines[k + 2:k + 14]] == [float(io.rust_e8(v)) for v in sc[name]]
    assert lines.index("SCALARS a float 1") < lines.index("SCALARS b float 1")


def test_unify_chunks_equals_single_file(tmp_path):
    n = [5, 4]
    a, b = tmp_path / "one", tmp_path / "chunks"
    _case(a, n, 2, threads=1)
    _case(b, n, 2, threads=3)
    step = b / "data" / "50"
    assert (step / "density_0.csv").exists() and not (step / "density.csv").exists()
    mp = m.Parameters(n=n, velocity_set=VelocitySet.D2Q9)
    sp = ps.Parameters(scalar_name="c", velocity_set=VelocitySet.D2Q9)
    post.post_unify(mp, sp, case_dir=str(b), keep=True)
    for t in (0, 50):
        for f in ("density.csv", "velocity.csv", "c.csv"):
            assert (b / "data" / str(t) / f).read_text() == (a / "data" / str(t) / f).read_text()
    assert (step / "density_0.csv").exists()            # keep
    post.post_unify(mp, sp, case_dir=str(b), keep=False)
    assert not (step / "density_0.csv").exists() and not (step / "c_2.csv").exists()


def test_conversion_factors():
    mp = m.Parameters(n=[4, 4], collision_operator=BGK(0.8), delta_x=0.002, delta_t=0.001,
                      physical_density=1000.0, reference_pressure=0.0)
    cf = post.ConversionFactor.from_params(mp)
    assert cf.velocity_conversion_factor == 2.0
    assert cf.pressure_conversion_factor == 4000.0
    assert np.isclose(cf.shear_viscosity, (0.8 - 0.5) / 3)
    assert np.isclose(cf.physical_shear_viscosity, (0.8 - 0.5) / 3 * 0.004)
    s = [1.0] * 9
    s[7], s[1] = 1 / 0.9, 1 / 0.7
    cf2 = post.ConversionFactor.from_params(m.Parameters(n=[4, 4], collision_operator=MRT(s)))
    assert np.isclose(cf2.shear_viscosity, (0.9 - 0.5) / 3)
    assert np.isclose(cf2.bulk_viscosity, (0.7 - 0.5) / 3 - (0.9 - 0.5) / 9)
