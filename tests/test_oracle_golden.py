"""Pin the CPU oracle to the reference's own tables and unit-test answers.

Every expected value comes from tests/golden/reference_golden.json, which
tests/golden/make_golden.py extracted from the reference sources.  The tests
mirror the reference tests they are named after (src/momentum/node.rs,
src/momentum/lattice.rs, src/momentum/bc.rs, src/velocity_set*.rs).
"""
import numpy as np
import pytest

from lbflow_b200 import _abi
from lbflow_b200 import momentum as m
from lbflow_b200.core import BGK, BoundaryFace, VelocitySet
from oracle import oracle as orc

VS_IDS = {"d2q9": _abi.LBF_D2Q9, "d3q19": _abi.LBF_D3Q19, "d3q27": _abi.LBF_D3Q27}
FACE_NAMES = ["West", "East", "South", "North", "Bottom", "Top"]


@pytest.mark.parametrize("name", ["d2q9", "d3q19", "d3q27"])
def test_velocity_set_tables_match_reference(golden, name):
    ref = golden["velocity_sets"][name]
    t = orc.tables(VS_IDS[name])
    q = t["q"]
    assert q == len(ref["c"])
    assert t["c"][:, :t["d"]].tolist() == ref["c"]
    assert t["w"].tolist() == ref["w"]            # exact: same rational literals
    assert t["q_bar"].tolist() == ref["q_bar"]
    nf = len(ref["q_faces"])
    for f in range(nf):
        qf = [i for i in t["q_faces"][f] if i >= 0]
        assert qf == ref["q_faces"][f], FACE_NAMES[f]
    normals = golden["face_normal_directions"][name]
    for f in range(nf):
        assert t["face_normal"][f] == normals[FACE_NAMES[f]]


@pytest.mark.parametrize("name", ["d2q9", "d3q19"])
def test_mrt_matrices_match_reference(golden, name):
    ref = golden["velocity_sets"][name]
    t = orc.tables(VS_IDS[name])
    assert np.array_equal(t["mrt"], np.array(ref["mrt"]))
    # M^-1 = M^T diag(1/|row|^2): the same rationals, correctly rounded
    assert np.array_equal(t["mrt_inverse"], np.array(ref["mrt_inverse"]))


def test_d3q27_mrt_basis_is_orthogonal_and_inverts():
    t = orc.tables(_abi.LBF_D3Q27)
    M, Mi = t["mrt"], t["mrt_inverse"]
    G = M @ M.T
    assert np.allclose(G - np.diag(np.diag(G)), 0.0, atol=1e-12)
    assert np.allclose(M @ Mi, np.eye(27), atol=1e-13)
    assert np.allclose(M[0], 1.0)
    assert np.allclose(M[1:4], t["c"].T)       # rows 1-3 are the momenta


def test_equilibrium_d2q9(golden):
    k = golden["kats"]["equilibrium_d2q9"]        # node.rs test_compute_equilibrium_d2q9
    rho = float(np.sum(k["f"]))
    out = orc.equilibrium(_abi.LBF_D2Q9, rho, [0.0, 0.0])
    assert np.allclose(out, k["target"], atol=1e-12, rtol=0)


def test_bgk_d2q9(golden):
    k = golden["kats"]["bgk_d2q9"]                # node.rs test_compute_bgk_collision_d2q9
    out = orc.bgk(_abi.LBF_D2Q9, k["f"], k["f_eq"], k["tau"])
    assert np.allclose(out, k["target"], atol=1e-12, rtol=0)


def _default_lattice(dim):
    """Lattice::_test_default (src/momentum/lattice.rs:209-213, src/momentum.rs:71-100)."""
    if dim == 2:
        p = m.Parameters()
    else:
        p = m.Parameters(n=[10, 10, 10], velocity_set=VelocitySet.D3Q19,
                         initial_velocity=m.InitialVelocity.Uniform([0, 0, 0]),
                         boundary_conditions=[(BoundaryFace.West, m.NoSlip), (BoundaryFace.East, m.NoSlip),
                                              (BoundaryFace.South, m.NoSlip),
                                              (BoundaryFace.North, m.BounceBack(1.0, [0.1, 0.0, 0.0])),
                                              (BoundaryFace.Bottom, m.NoSlip), (BoundaryFace.Top, m.NoSlip)])
    desc, keep = m.to_desc(p)
    return orc.Domain(desc, keep=keep)


def _idx(node, n):
    return node[0] + n[0] * (node[1] + (n[1] * node[2] if len(node) > 2 else 0))


@pytest.mark.parametrize("case", [1, 2])
def test_streaming_d2q9(golden, case):
    k = golden["kats"][f"streaming_d2q9_case_{case}"]   # node.rs test_compute_streaming_d2q9_case_*
    dom = _default_lattice(2)
    n = k["n"]
    node = _idx(k["node"], n)
    fs = dom.get("f_star").reshape(-1, 9)
    for i, vals in k["neighbor_f_star"].items():
        fs[dom.neighbor(node, int(i))] = vals
    dom.set("f_star", fs)
    dom.run_pass(3)
    f = dom.get("f").reshape(-1, 9)[node]
    assert np.allclose(f, k["target"], atol=0, rtol=0)


@pytest.mark.parametrize("name", ["neighbor_d2q9_inner_node", "neighbor_d2q9_edge_node",
                                  "neighbor_d3q19_inner_node", "neighbor_d3q19_edge_node"])
def test_neighbors(golden, name):
    k = golden["kats"][name]
    dom = _default_lattice(k["dim"])
    n = k["n"]
    node = _idx(k["node"], n)
    for i, target in k["neighbors"].items():
        assert dom.neighbor(node, int(i)) == _idx(target, n)
    if "chain" in k:
        (a, b), target = k["chain"]
        assert dom.neighbor(dom.neighbor(node, a), b) == _idx(target, n)


def test_node_index_layout(golden):
    k = golden["kats"]["node_index_d2q9"]       # lattice.rs test_get_node_d2q9_several_nodes
    for i, xy in k["nodes"].items():
        assert _idx(xy, k["n"]) == int(i)


def test_face_membership(golden):
    k = golden["kats"]["faces_d2q9"]            # lattice.rs test_get_boundary_nodes_by_face_*
    dom = _default_lattice(2)
    cls, _ = dom.node_class()
    n = k["n"]
    for f, face in enumerate(["west", "east", "south", "north"]):
        bit = 1 << (_abi.LBF_CLASS_FACE_SHIFT + f)
        for xy in k["faces"][face]["contains"]:
            assert cls[_idx(xy, n)] & bit
        for xy in k["faces"][face]["does_not_contain"]:
            assert not cls[_idx(xy, n)] & bit
    start = _idx(k["faces"]["north"]["contains_chain"]["from"], n)
    nb = dom.neighbor(dom.neighbor(start, 2), 2)
    assert cls[nb] & (1 << (_abi.LBF_CLASS_FACE_SHIFT + 3))


def _one_node_moments(vs, f):
    dim = VelocitySet(vs).d
    p = m.Parameters(n=[1] * dim, velocity_set=vs,
                     initial_velocity=m.InitialVelocity.Uniform([0.0] * dim),
                     boundary_conditions=[(face, m.Periodic) for face in list(BoundaryFace)[:2 * dim]])
    desc, keep = m.to_desc(p)
    dom = orc.Domain(desc, keep=keep)
    dom.set("f", f)
    dom.run_pass(0)
    return dom.get("density")[0], dom.get("velocity")


def test_density_kats(golden):
    for case in golden["kats"]["density_d2q9"]:
        rho, _ = _one_node_moments(VelocitySet.D2Q9, case["f"])
        assert abs(rho - case["density"]) < 1e-12
    for case in golden["kats"]["density_d3q19"]:
        rho, _ = _one_node_moments(VelocitySet.D3Q19, case["f"])
        assert abs(rho - case["density"]) < 1e-12


def test_velocity_kats(golden):
    k = golden["kats"]
    rho, u = _one_node_moments(VelocitySet.D2Q9, k["velocity_d2q9_implicit"]["f"])
    # the reference test holds density at its value (1.0) from Node::test_default
    assert np.allclose(u * rho, k["velocity_d2q9_implicit"]["target"], atol=1e-12)
    rho, u = _one_node_moments(VelocitySet.D3Q19, k["velocity_d3q19_implicit"]["f"])
    assert np.allclose(u * rho, k["velocity_d3q19_implicit"]["target"], atol=1e-12)
    for key, vs in (("velocity_d2q9_explicit", VelocitySet.D2Q9), ("velocity_d3q19_explicit", VelocitySet.D3Q19)):
        rho, u = _one_node_moments(vs, k[key]["f"])
        assert np.allclose(u * rho / k[key]["density"], k[key]["target"], atol=1e-12)
    for key, vs in (("velocity_computation_d2q9", VelocitySet.D2Q9), ("velocity_computation_d3q27", VelocitySet.D3Q27)):
        rho, u = _one_node_moments(vs, k[key]["f"])
        for case in k[key]["cases"]:
            assert np.allclose(u * rho / case["density"], case["target"], atol=1e-12)


@pytest.mark.parametrize("face", ["west", "east", "south", "north"])
def test_no_slip_d2q9(golden, face):
    k = golden["kats"]["no_slip_d2q9"][face]      # bc.rs test_compute_no_slip_bc_d2q9_*
    f_id = ["west", "east", "south", "north"].index(face)
    bcs = [(BoundaryFace(i), m.NoSlip if i == f_id else m.Periodic) for i in range(4)]
    p = m.Parameters(n=[10, 10], boundary_conditions=bcs)
    desc, keep = m.to_desc(p)
    dom = orc.Domain(desc, keep=keep)
    node = _idx({"west": [0, 5], "east": [9, 5], "south": [5, 0], "north": [5, 9]}[face], [10, 10])
    f = dom.get("f").reshape(-1, 9); f[node] = k["f"]; dom.set("f", f)
    fs = dom.get("f_star").reshape(-1, 9); fs[node] = k["f_star"]; dom.set("f_star", fs)
    dom.run_pass(5)
    assert dom.get("f").reshape(-1, 9)[node].tolist() == k["target"]


def test_node_residuals(golden):
    k = golden["kats"]["node_residuals"]          # node.rs test_compute_node_residuals
    p = m.Parameters(n=[1, 1], boundary_conditions=[(BoundaryFace(i), m.Periodic) for i in range(4)])
    desc, keep = m.to_desc(p)
    dom = orc.Domain(desc, keep=keep)
    dom.set("density", [k["density"]])
    dom.set("velocity", k["velocity"])
    dom.run_pass(6)
    r = dom.residuals()
    assert abs(r[0] - abs(k["target_density"])) < 1e-12
    assert np.allclose(r[1:3], np.abs(k["target_velocity"]), atol=1e-12)
