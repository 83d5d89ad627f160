"""Output formats of the reference, written by the native formatter (host code, no GPU).

The reference writes `{:.8e}` CSV fields per node (src/momentum/io.rs:112-192,
src/passive_scalar/io.rs:76-108), the coordinates file (src/momentum/io.rs:194-224)
and, with --num-threads > 1, one chunk file per `par_chunks(N / threads)` chunk.
lbf_format_csv / lbf_format_coordinates must produce byte-identical text to the
pure-Python writers in lbflow_b200.io, which follow those sources line by line.
"""
import os

import numpy as np
import pytest

from lbflow_b200 import io


def _values(seed=3, n=20000):
    rng = np.random.default_rng(seed)
    v = np.concatenate([
        rng.normal(1.0, 1e-3, n // 4),                       # densities near 1
        rng.normal(0.0, 1e-2, n // 4),                       # velocities around 0
        np.exp(rng.uniform(-700, 700, n // 4)) * rng.choice([-1, 1], n // 4),
        rng.integers(-10**9, 10**9, n // 4).astype(float),
        [0.0, -0.0, 1.0, -1.0, 0.5, 1e-300, 5e-324, 1.7976931348623157e308, 9.999999995, 1.000000005,
         123456788.5, 2.5e-5, float("nan"), float("inf"), float("-inf")],
    ])
    return v


def test_rust_e8_edge_cases():
    assert io.rust_e8(1.0) == "1.00000000e0"
    assert io.rust_e8(-2.5e-5) == "-2.50000000e-5"
    assert io.rust_e8(0.0) == "0.00000000e0"
    assert io.rust_e8(1e100) == "1.00000000e100"
    assert io.rust_e8(float("nan")) == "NaN"
    assert io.rust_e8(float("-inf")) == "-inf"


@pytest.mark.parametrize("cols", [1, 2, 3])
def test_native_csv_matches_python(cols):
    v = _values()
    v = v[: (v.size // cols) * cols].reshape(-1, cols)
    got = bytes(io.format_rows_native(v, threads=4)).decode()
    want = "".join(",".join(io.rust_e8(float(x)) for x in row) + "\n" for row in v)
    assert got == want


def test_native_csv_single_thread_and_empty():
    v = _values(5, 400)[:400].reshape(-1, 2)
    assert bytes(io.format_rows_native(v, threads=1)) == bytes(io.format_rows_native(v, threads=7))
    assert bytes(io.format_rows_native(np.zeros((0, 3)))) == b""


@pytest.mark.parametrize("n", [[7, 5], [4, 3, 5]])
def test_native_coordinates_match_python(tmp_path, n):
    rng = np.random.default_rng(1)
    mask = (rng.random(int(np.prod(n))) < 0.3).astype(np.uint8)
    io.write_coordinates(n, mask, 0.01, root=str(tmp_path))
    want = open(os.path.join(tmp_path, io.COORDINATES_FILE)).read()
    header, body = want.split("\n", 1)
    assert header == ("i,j,x,y,node_type" if len(n) == 2 else "i,j,k,x,y,z,node_type")
    assert bytes(io.format_coordinates_native(n, mask, 0.01, threads=3)).decode() == body


@pytest.mark.parametrize("threads", [1, 3, 4])
def test_native_chunk_files_match_python(tmp_path, threads):
    rng = np.random.default_rng(2)
    rho = rng.normal(1.0, 1e-3, 103)
    u = rng.normal(0.0, 1e-2, (103, 2))
    a, b = tmp_path / "py", tmp_path / "native"
    a.mkdir(); b.mkdir()
    io.write_step_data(0, rho, u, {"C": rho * 0.5}, num_threads=threads, root=str(a))
    step = b / "0"
    step.mkdir()
    io.write_field_native(str(step), "density", "density", rho, threads)
    io.write_field_native(str(step), "velocity", "velocity_x,velocity_y", u, threads)
    io.write_field_native(str(step), "C", "C", rho * 0.5, threads)
    fa = sorted(os.listdir(a / "0"))
    assert fa == sorted(os.listdir(step))
    for f in fa:
        assert (a / "0" / f).read_bytes() == (step / f).read_bytes(), f
