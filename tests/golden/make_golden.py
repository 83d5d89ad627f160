"""Generate tests/golden/reference_golden.json from the reference's Rust sources.

The reference (gilberto-ribeiro/lbflow) cannot be compiled here, so its tables
and its unit-test known answers are read as text: velocity-set tables from
src/velocity_set/*.rs and the expected values of the #[cfg(test)] functions in
src/momentum/node.rs, src/momentum/lattice.rs, src/momentum/bc.rs,
src/velocity_set.rs, src/velocity_set/d2q9.rs and src/velocity_set/d3q27.rs.

Run from the repository root:  python tests/golden/make_golden.py REFERENCE_ROOT
(REFERENCE_ROOT: a checkout of the reference; required).
The JSON it writes is committed; tests read only the JSON.
"""
from __future__ import annotations

import ast
import json
import operator
import os
import re
import sys

if __name__ == "__main__" and len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_golden.py REFERENCE_ROOT")
REF = sys.argv[1] if len(sys.argv) > 1 else ""
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_golden.json")


def read(rel):
    with open(os.path.join(REF, rel)) as fh:
        return fh.read()


_OPS = {ast.Add: operator.add, ast.Sub: operator.sub, ast.Mult: operator.mul, ast.Div: operator.truediv}


def num(expr: str) -> float:
    """Evaluate a Rust float literal expression such as `-5.0 / 399.0`."""
    def ev(n):
        if isinstance(n, ast.Expression):
            return ev(n.body)
        if isinstance(n, ast.Constant):
            return float(n.value)
        if isinstance(n, ast.UnaryOp) and isinstance(n.op, ast.USub):
            return -ev(n.operand)
        if isinstance(n, ast.BinOp) and type(n.op) in _OPS:
            return _OPS[type(n.op)](ev(n.left), ev(n.right))
        raise ValueError(expr)
    return ev(ast.parse(expr.strip(), mode="eval"))


def const_block(src: str, name: str) -> str:
    i = src.index(f"const {name}")
    j = src.index("= ", i) + 2
    depth, k = 0, j
    while True:
        ch = src[k]
        if ch == "[":
            depth += 1
        elif ch == "]":
            depth -= 1
            if depth == 0:
                return src[j:k + 1]
        k += 1


def parse_list(text: str):
    """Nested [..] list of numeric expressions -> nested Python lists."""
    text = text.strip()
    m = re.fullmatch(r"\[\s*\[(.*)\]\s*;\s*(\w+)\s*\]", text, re.S)
    if m:   # [[1.0; Q]; Q] repetition form
        return ("repeat", m.group(1), m.group(2))
    out, stack, tok = [], [], ""
    cur = out
    for ch in text:
        if ch == "[":
            new = []
            stack.append(cur)
            cur.append(new)
            cur = new
        elif ch in ",]":
            if tok.strip():
                cur.append(num(tok))
            tok = ""
            if ch == "]":
                cur = stack.pop()
        else:
            tok += ch
    return out[0]


def velocity_set(name: str) -> dict:
    src = read(f"src/velocity_set/{name}.rs")
    res = {
        "c": [[int(x) for x in row] for row in parse_list(const_block(src, "C:"))],
        "w": parse_list(const_block(src, "W:")),
        "q_bar": [int(x) for x in parse_list(const_block(src, "Q_BAR:"))],
    }
    faces = ["WEST", "EAST", "SOUTH", "NORTH"] + (["BOTTOM", "TOP"] if name.startswith("d3") else [])
    res["q_faces"] = [[int(x) for x in parse_list(const_block(src, f"Q_{f}:"))] for f in faces]
    for key, const in (("mrt", "MRT_MATRIX:"), ("mrt_inverse", "MRT_INVERSE_MATRIX:")):
        if f"const {const}" in src:
            val = parse_list(const_block(src, const))
            if isinstance(val, tuple):
                continue   # placeholder [[1.0; Q]; Q] (d3q27.rs:86)
            res[key] = val
    return res


def face_normals() -> dict:
    src = read("src/velocity_set.rs")
    out = {}
    for name, vs in (("D2Q9", "d2q9"), ("D3Q15", "d3q15"), ("D3Q19", "d3q19"), ("D3Q27", "d3q27")):
        i = src.index(f"{name} => Parameters")
        j = src.index("face_normal_directions", i)
        k = src.index("])", j)
        pairs = re.findall(r"\((\w+),\s*(\d+)\)", src[j:k])
        out[vs] = {face: int(v) for face, v in pairs}
    return out


def test_body(src: str, fn: str) -> str:
    i = src.index(f"fn {fn}()")
    j = src.index("\n    }\n", i)
    return src[i:j]


def arrays(body: str):
    """All `vec![..]` / `[..]` numeric literals of a test body, in order."""
    out = []
    for m in re.finditer(r"(?:vec!)?\[([-0-9.,\s]+)\]", body):
        items = [x for x in m.group(1).split(",") if x.strip()]
        try:
            out.append([num(x) for x in items])
        except ValueError:
            pass
    return out


def kats() -> dict:
    node = read("src/momentum/node.rs")
    lat = read("src/momentum/lattice.rs")
    bc = read("src/momentum/bc.rs")
    k = {}
    # src/momentum/node.rs tests
    b = test_body(node, "test_compute_equilibrium_d2q9")
    k["equilibrium_d2q9"] = {"f": [0.1] * 9, "target": arrays(b)[-1]}
    b = test_body(node, "test_compute_bgk_collision_d2q9")
    a = arrays(b)
    k["bgk_d2q9"] = {"f": [0.1] * 9, "f_eq": a[0], "tau": float(re.search(r"let tau = ([0-9.]+);", b).group(1)),
                     "target": a[-1]}
    for case in (1, 2):
        b = test_body(node, f"test_compute_streaming_d2q9_case_{case}")
        nb = re.findall(r"get_neighbor_node\((\d)\)\s*\.set_f_star\((?:vec!\[([-0-9.,\s]+)\]|vec!\[([0-9.]+);\s*9\])\)", b)
        fstar = {}
        for i, full, rep in nb:
            fstar[int(i)] = [num(x) for x in full.split(",")] if full else [num(rep)] * 9
        target = re.search(r"assert_eq!\(\s*node.get_f\(\),\s*vec!\[([^\]]+)\]", b).group(1)
        tgt = [num(x) for x in target.split(";")[0].split(",")] if ";" not in target else [num(target.split(";")[0])] * 9
        k[f"streaming_d2q9_case_{case}"] = {"node": [3, 7], "n": [10, 10], "neighbor_f_star": fstar, "target": tgt}
    for dim, fn in ((2, "test_get_neighbor_node_d2q9_inner_node"), (2, "test_get_neighbor_node_d2q9_edge_node"),
                    (3, "test_get_neighbor_node_d3q19_inner_node"), (3, "test_get_neighbor_node_d3q19_edge_node")):
        b = test_body(node, fn)
        start = [int(x) for x in re.search(r"_get_node_by_index\(&vec!\[([0-9,\s]+)\]\)", b).group(1).split(",")]
        pairs = re.findall(r"node.get_neighbor_node\((\d+)\).get_index\(\),\s*&vec!\[([0-9,\s]+)\]", b)
        k[fn.replace("test_get_neighbor_node_", "neighbor_")] = {
            "dim": dim, "n": [10] * dim, "node": start,
            "neighbors": {int(i): [int(x) for x in v.split(",")] for i, v in pairs}}
    b = test_body(node, "test_get_neighbor_node_d2q9_edge_node")
    two = re.search(r"get_neighbor_node\((\d)\)\.get_neighbor_node\((\d)\)\.get_index\(\),\s*&vec!\[([0-9,\s]+)\]", b)
    k["neighbor_d2q9_edge_node"]["chain"] = [[int(two.group(1)), int(two.group(2))],
                                             [int(x) for x in two.group(3).split(",")]]
    b = test_body(node, "test_compute_density_d2q9")
    k["density_d2q9"] = [{"f": [0.1] * 9, "density": 0.9},
                         {"f": [0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7, 0.8, 0.9], "density": 4.5}]
    assert "0.9).abs()" in b and "4.5).abs()" in b
    b = test_body(node, "test_compute_density_d3q19")
    assert "1.9).abs()" in b
    k["density_d3q19"] = [{"f": [0.1] * 19, "density": 1.9}]
    b = test_body(node, "test_compute_velocity_d2q9_implicit_computation")
    a = arrays(b)
    k["velocity_d2q9_implicit"] = {"f": a[0], "target": a[-1]}
    b = test_body(node, "test_compute_velocity_d3q19_implicit_computation")
    a = arrays(b)
    k["velocity_d3q19_implicit"] = {"f": a[0], "target": a[-1]}
    b = test_body(node, "test_compute_velocity_d2q9_explicit_computation")
    a = arrays(b)
    k["velocity_d2q9_explicit"] = {"f": a[0], "density": float(re.search(r"set_density\(([0-9.]+)\)", b).group(1)),
                                   "target": a[-1]}
    b = test_body(node, "test_compute_velocity_d3q19_explicit_computation")
    a = arrays(b)
    k["velocity_d3q19_explicit"] = {"f": a[0], "density": float(re.search(r"set_density\(([0-9.]+)\)", b).group(1)),
                                    "target": a[-1]}
    b = test_body(node, "test_compute_node_residuals")
    k["node_residuals"] = {"density": float(re.search(r"set_density\(([0-9.]+)\)", b).group(1)),
                           "velocity": arrays(b)[0], "shallow_density": 1.0, "shallow_velocity": [0.0, 0.0],
                           "target_density": float(re.search(r"- \(([-0-9.]+)\)\)\.abs", b).group(1)),
                           "target_velocity": arrays(b)[-1]}
    # src/velocity_set/{d2q9,d3q27}.rs velocity_computation tests
    for vs in ("d2q9", "d3q27"):
        b = test_body(read(f"src/velocity_set/{vs}.rs"), f"test_velocity_computation_{vs}")
        a = arrays(b)
        dens = [float(x) for x in re.findall(r"let density = ([0-9.]+);", b)]
        k[f"velocity_computation_{vs}"] = {"f": a[0], "cases": [{"density": dens[0], "target": a[1]},
                                                                  {"density": dens[1], "target": a[2]}]}
    # src/momentum/lattice.rs tests: index layout and face membership (10x10 lattice)
    b = test_body(lat, "test_get_node_d2q9_several_nodes")
    k["node_index_d2q9"] = {"n": [10, 10], "nodes": {int(i): [int(x) for x in v.split(",")] for i, v in
                                                     re.findall(r"_get_node\((\d+)\).get_index\(\),\s*&vec!\[([0-9,\s]+)\]", b)}}
    faces = {}
    for face in ("west", "east", "south", "north"):
        b = test_body(lat, f"test_get_boundary_nodes_by_face_d2q9_{face}_face_contains")
        faces[face] = {"contains": [[int(x) for x in v.split(",")] for v in re.findall(r"contains\(&&vec!\[([0-9,\s]+)\]\)", b)],
                       "does_not_contain": [[3, 7]]}
    b = test_body(lat, "test_get_boundary_nodes_by_face_d2q9_north_face_neighbor_node_contains")
    faces["north"]["contains_chain"] = {"from": [3, 7], "steps": [2, 2]}
    k["faces_d2q9"] = {"n": [10, 10], "faces": faces}
    # src/momentum/bc.rs NoSlip tests
    nos = {}
    for face in ("west", "east", "south", "north"):
        b = test_body(bc, f"test_compute_no_slip_bc_d2q9_{face}_face")
        a = arrays(b)
        nos[face] = {"f": a[-3], "f_star": a[-2], "target": a[-1]}
    k["no_slip_d2q9"] = nos
    return k


def lattice_defaults() -> dict:
    """Parameters::_test_default / Default (src/momentum.rs:39-100)."""
    src = read("src/momentum.rs")
    assert "n: vec![10, 10]" in src and "BounceBack {" in src
    return {"n2": [10, 10], "n3": [10, 10, 10], "north_bounce_back": {"density": 1.0, "velocity": [0.1, 0.0]}}


def main():
    out = {"source": "gilberto-ribeiro/lbflow (read as text by tests/golden/make_golden.py)",
           "velocity_sets": {vs: velocity_set(vs) for vs in ("d2q9", "d3q15", "d3q19", "d3q27")},
           "face_normal_directions": face_normals(),
           "kats": kats(),
           "defaults": lattice_defaults()}
    with open(OUT, "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
