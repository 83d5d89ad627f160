"""The reference driver (`lbflow_b200.solver.solve`) against the oracle.

solve() runs the loop of src/momentum.rs:262-293 / src/passive_scalar.rs:136-177
on the GPU and writes the reference's files.  These tests read the files back
and compare them with the oracle stepped on the CPU:
  data/<t>/density.csv, velocity.csv, <scalar>.csv at every output step,
  data/residuals.csv (one line per step, stop at the same step),
  data/coordinates.csv, post_processing/<file> of compute_mean_density.
FP64 storage; the 9 significant digits of the text are compared with a relative
tolerance of 5e-8 against the oracle's FP64 values.
"""
import os

import numpy as np
import pytest

from lbflow_b200 import _abi, cases, io
from lbflow_b200 import momentum as m
from lbflow_b200 import passive_scalar as ps
from lbflow_b200.core import BGK, BoundaryFace, Storage, VelocitySet

pytestmark = pytest.mark.gpu

W, E, S, N = BoundaryFace.West, BoundaryFace.East, BoundaryFace.South, BoundaryFace.North
TXT = 5e-8   # {:.8e} text holds 9 significant digits


@pytest.fixture(scope="module")
def solver():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from lbflow_b200 import solver as s
    return s


def _close(a, b, tol=TXT):
    a, b = np.asarray(a), np.asarray(b)
    return np.all(np.abs(a - b) <= tol * np.maximum(np.abs(b), 1e-12) + 1e-15)


def _read_chunks(step, prefix, reader):
    files = sorted((f for f in os.listdir(step) if f.startswith(prefix + "_")),
                   key=lambda f: int(f[len(prefix) + 1:-4]))
    return np.concatenate([reader(str(step / f)) for f in files])


def _oracle(params, scalars=()):
    from oracle import oracle as orc
    desc, keep = m.to_desc(params)
    doms = []
    for sp in scalars or [None]:
        sdesc = None
        if sp is not None:
            sdesc, k2 = ps.to_desc(sp, params.n[: params.dim])
            keep = keep + k2
        doms.append(orc.Domain(desc, sdesc, keep=keep).init())
    return doms


def test_solve_cavity_outputs_match_oracle(solver, tmp_path):
    p = cases.cavity_d2q9(16, 0.6, 0.1, Storage.F64)
    p.post_functions = [solver.PostFunction("mean_density.csv", 7, solver.compute_mean_density)]
    res = solver.solve(p, write_data=40, max_iterations=100, num_threads=3, case_dir=str(tmp_path), verbose=False)
    assert res.time_steps == 102          # stops after t = 101 > max_iterations
    assert res.data_steps == [0, 40, 80]
    od = _oracle(p)[0]
    data = tmp_path / "data"
    lines = (data / "residuals.csv").read_text().strip().split("\n")
    assert lines[0] == "time_step,density,velocity_x,velocity_y"
    assert len(lines) == 1 + 102
    post = (tmp_path / "post_processing" / "mean_density.csv").read_text().strip().split("\n")
    assert post[0] == "time_step,mean_density"
    post_rows = {int(r.split(",")[0]): float(r.split(",")[1]) for r in post[1:]}
    assert sorted(post_rows) == list(range(0, 102, 7))
    for t in range(102):
        if t in (0, 40, 80):
            rho, u, _ = od.observe()
            # par_chunks(256 / 3 = 85): four chunk files per field (85, 85, 85, 1 lines)
            assert len(os.listdir(data / str(t))) == 8
            rho_f = _read_chunks(data / str(t), "density", io.read_scalar_csv)
            u_f = _read_chunks(data / str(t), "velocity", io.read_vector_csv)
            assert _close(rho_f, rho) and _close(u_f, u)
        if t in post_rows:
            rho, _, _ = od.observe()
            cls, _ = od.node_class()
            fl = (cls & _abi.LBF_CLASS_SOLID) == 0
            assert _close(post_rows[t], rho[fl].mean())
        od.step(1)
        r = od.residuals()
        row = lines[1 + t].split(",")
        assert int(row[0]) == t
        assert np.allclose([float(x) for x in row[1:]], r, rtol=1e-6, atol=1e-15)
    coords = (data / "coordinates.csv").read_text().split("\n")
    assert coords[0] == "i,j,x,y,node_type" and coords[1] == "0,0,5.00000000e-3,5.00000000e-3,fluid"


def test_solve_stops_where_oracle_run_stops(solver, tmp_path):
    p = cases.cavity_d2q9(12, 0.8, 0.01, Storage.F64)
    od = _oracle(p)[0]
    steps = od.run(max_iterations=3000)
    res = solver.solve(p, write_data=100000, max_iterations=3000, case_dir=str(tmp_path), verbose=False)
    assert res.time_steps == steps < 3000
    assert np.all(res.residuals[:1] <= 1e-7)


def test_solve_two_scalars_match_oracle(solver, tmp_path):
    n = [24, 12]
    mask = np.zeros(n[0] * n[1], np.uint8).reshape(n[1], n[0])
    mask[4:8, 9:13] = 1
    mp = m.Parameters(n=n, collision_operator=BGK(0.7), velocity_set=VelocitySet.D2Q9,
                      boundary_conditions=[(W, m.ZouHe(None, [0.04, 0.0])), (E, m.AntiBounceBack(1.0)),
                                           (S, m.NoSlip), (N, m.NoSlip)],
                      node_types=m.NodeTypes.FromArray(mask.ravel()))

    def scalar(name, c_in, ads):
        return ps.Parameters(scalar_name=name, collision_operator=BGK(0.55), velocity_set=VelocitySet.D2Q9,
                             initial_scalar_value=ps.InitialScalarValue.Uniform(0.0),
                             boundary_conditions=[(W, ps.AntiBounceBack(c_in)), (E, ps.AntiBBNoFlux),
                                                  (S, ps.BBNoFlux), (N, ps.BBNoFlux)],
                             inner_boundary_condition=ps.InnerBounceBack,
                             adsorption_parameters=ps.AdsorptionParameters(ps.Langmuir(1e-2, 1e-4, 1.0), 0.0)
                             if ads else None)

    sps = [scalar("tracer", 1.0, False), scalar("solute", 0.5, True)]
    res = solver.solve(mp, sps, write_data=30, max_iterations=60, case_dir=str(tmp_path), verbose=False)
    assert res.time_steps == 62
    ods = _oracle(mp, sps)
    data = tmp_path / "data"
    lines = (data / "residuals.csv").read_text().strip().split("\n")
    assert lines[0] == "time_step,density,velocity_x,velocity_y,tracer,solute"
    for t in range(62):
        if t % 30 == 0:
            rho, u, c0 = ods[0].observe()
            c1 = ods[1].observe()[2]
            assert _close(io.read_scalar_csv(str(data / str(t) / "density.csv")), rho)
            assert _close(io.read_vector_csv(str(data / str(t) / "velocity.csv")), u)
            assert _close(io.read_scalar_csv(str(data / str(t) / "tracer.csv")), c0)
            assert _close(io.read_scalar_csv(str(data / str(t) / "solute.csv")), c1)
        for od in ods:
            od.step(1)
        r0, r1 = ods[0].residuals(), ods[1].residuals()
        want = list(r0[:3]) + [r0[3], r1[3]]
        got = [float(x) for x in lines[1 + t].split(",")[1:]]
        assert np.allclose(got, want, rtol=1e-6, atol=1e-15), t
