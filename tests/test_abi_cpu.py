"""CPU-side checks of the C-ABI library: it loads, exports every symbol the
header declares, the descriptor layouts agree, and the velocity-set tables
compiled into the device code equal the reference's (golden) tables.  None of
these calls touch a GPU."""
import os
import re

import numpy as np
import pytest

from lbflow_b200 import _abi
from lbflow_b200.domain import tables
from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    with open(os.path.join(ROOT, "include", "lbflow.h")) as fh:
        src = fh.read()
    return sorted(set(re.findall(r"\b(lbf_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = _abi.load()
    names = header_functions()
    assert "lbf_domain_step" in names and len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) <= set(_abi.SIGNATURES), set(names) - set(_abi.SIGNATURES)


def test_header_constants_mirrored():
    with open(os.path.join(ROOT, "include", "lbflow.h")) as fh:
        src = fh.read()
    assert int(re.search(r"#define LBF_MAX_SCALARS (\d+)", src).group(1)) == _abi.LBF_MAX_SCALARS


def test_abi_version_and_layouts():
    lib = _abi.load()
    assert lib.lbf_abi_version() == 1
    import ctypes as C
    for which, st in enumerate((_abi.DomainDesc, _abi.ScalarDesc, _abi.BcDesc, _abi.CollisionDesc)):
        assert lib.lbf_sizeof(which) == C.sizeof(st)


@pytest.mark.parametrize("name,vs", [("d2q9", _abi.LBF_D2Q9), ("d3q19", _abi.LBF_D3Q19), ("d3q27", _abi.LBF_D3Q27)])
def test_device_tables_match_reference(golden, name, vs):
    ref = golden["velocity_sets"][name]
    t = tables(vs)
    assert t["c"][:, :t["d"]].tolist() == ref["c"]
    assert t["w"].tolist() == ref["w"]
    assert t["q_bar"].tolist() == ref["q_bar"]
    for f, qf in enumerate(ref["q_faces"]):
        assert [i for i in t["q_faces"][f] if i >= 0] == qf
    faces = ["West", "East", "South", "North", "Bottom", "Top"]
    for f in range(len(ref["q_faces"])):
        assert t["face_normal"][f] == golden["face_normal_directions"][name][faces[f]]
    if "mrt" in ref:
        assert np.array_equal(t["mrt"], np.array(ref["mrt"]))
        assert np.array_equal(t["mrt_inverse"], np.array(ref["mrt_inverse"]))


def test_d3q27_basis_matches_oracle():
    a, b = tables(_abi.LBF_D3Q27), orc.tables(_abi.LBF_D3Q27)
    assert np.allclose(a["mrt"], b["mrt"], atol=1e-14, rtol=0)
    assert np.allclose(a["mrt_inverse"], b["mrt_inverse"], atol=1e-14, rtol=0)


def test_unsupported_velocity_set_is_rejected():
    lib = _abi.load()
    assert lib.lbf_velocity_set_tables(_abi.LBF_D2Q5, None, None, None, None, None, None, None, None, None) \
        == _abi.LBF_EUNSUPPORTED
