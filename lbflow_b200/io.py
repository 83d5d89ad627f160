"""File formats of the reference: map.xyz masks, CSV fields and residuals.

- map.xyz (src/io.rs:60-143): whitespace-separated 0/1 tokens; blank lines
  separate z-slices; inside a slice the LAST line is y = 0 (lines are read in
  reverse), as written by aux/image_pre_processing.py:42-56 (image row 0 on top).
- data/<t>/density.csv, velocity.csv, <scalar>.csv (src/momentum/io.rs:112-192,
  src/passive_scalar/io.rs:76-108): a header line, then one `{:.8e}` value (or
  comma-separated vector) per node in node order.
- data/coordinates.csv (src/momentum/io.rs:194-224) and data/residuals.csv
  (src/io.rs:241-250, src/momentum/io.rs:52-72).
"""
from __future__ import annotations

import os
from typing import Optional, Sequence

import numpy as np

DATA_PATH = "./data"
PRE_PROCESSING_PATH = "./pre_processing"
POST_PROCESSING_PATH = "./post_processing"
VTK_PATH = "./post_processing/vtk_files"
COORDINATES_FILE = "coordinates.csv"
DENSITY_FILE = "density.csv"
VELOCITY_FILE = "velocity.csv"
RESIDUALS_FILE = "residuals.csv"
BOUNCE_BACK_MAP_FILE = "map.xyz"


def rust_e8(x: float) -> str:
    """Rust's `{:.8e}` formatting: 8 fraction digits, exponent without padding or '+'."""
    if x != x:
        return "NaN"
    if x in (float("inf"), float("-inf")):
        return "inf" if x > 0 else "-inf"
    s = f"{x:.8e}"
    mant, exp = s.split("e")
    return f"{mant}e{int(exp)}"


# ------------------------------------------------------------------ native text formatting
def format_rows_native(values: np.ndarray, threads: int = 0) -> memoryview:
    """`{:.8e}` CSV lines of a (rows, cols) FP64 array, formatted by lbf_format_csv
    on `threads` host threads (0 = all cores).  Same text as the pure-Python writers."""
    import ctypes as C
    from . import _abi
    lib = _abi.load()
    v = np.ascontiguousarray(values, dtype=np.float64)
    rows = v.shape[0]
    cols = 1 if v.ndim == 1 else v.shape[1]
    n = C.c_int64()
    cap = rows * (cols * 25 + 1)
    buf = np.empty(max(cap, 1), dtype=np.uint8)
    _abi.check(lib.lbf_format_csv(v.ctypes.data, rows, cols, buf.ctypes.data, cap, C.byref(n), threads))
    return memoryview(buf)[:n.value]


def format_coordinates_native(n: Sequence[int], node_type: Optional[np.ndarray], delta_x: float,
                              threads: int = 0) -> memoryview:
    import ctypes as C
    from . import _abi
    lib = _abi.load()
    d = len(n)
    nn = np.array(list(n) + [1] * (3 - d), dtype=np.int64)
    rows = int(np.prod(nn))
    nt = None if node_type is None else np.ascontiguousarray(node_type, dtype=np.uint8)
    cap = rows * (3 * 21 + 3 * 25 + 8)
    buf = np.empty(max(cap, 1), dtype=np.uint8)
    ln = C.c_int64()
    _abi.check(lib.lbf_format_coordinates(nn.ctypes.data_as(C.POINTER(C.c_int64)), d, float(delta_x), None if nt is None else nt.ctypes.data,
                                          buf.ctypes.data, cap, C.byref(ln), threads))
    return memoryview(buf)[:ln.value]


def _split_lines(text: memoryview, rows: int, parts: int) -> list:
    """Byte ranges of `parts` chunks of rows_per = rows // parts lines (the last ones
    may be shorter), matching rayon's par_chunks(rows / parts)."""
    if parts <= 1 or rows == 0:
        return [text]
    chunk = max(1, rows // parts)
    a = np.frombuffer(text, dtype=np.uint8)
    ends = np.flatnonzero(a == 10) + 1          # end offset of every line
    out, start = [], 0
    for r0 in range(0, rows, chunk):
        r1 = min(rows, r0 + chunk)
        stop = int(ends[r1 - 1])
        out.append(text[start:stop])
        start = stop
    return out


def write_field_native(step_path: str, prefix: str, header: str, values: np.ndarray, num_threads: int = 1,
                       format_threads: int = 0) -> None:
    """One field of an output step, as _write_chunks writes it, with native formatting."""
    text = format_rows_native(values, format_threads)
    rows = values.shape[0]
    parts = _split_lines(text, rows, num_threads)
    if num_threads <= 1:
        with open(os.path.join(step_path, f"{prefix}.csv"), "wb") as fh:
            fh.write((header + "\n").encode())
            fh.write(text)
        return
    for i, part in enumerate(parts):
        with open(os.path.join(step_path, f"{prefix}_{i}.csv"), "wb") as fh:
            fh.write((header + "\n").encode())
            fh.write(part)


def format_column(values: np.ndarray) -> list:
    return [rust_e8(float(v)) for v in values]


# ------------------------------------------------------------------ map.xyz
def parse_bounce_back_map(text: str) -> np.ndarray:
    """Tokens in node order, exactly as read_xyz_file (src/io.rs:121-143)."""
    out = []
    for slab in text.strip().split("\n\n"):
        lines = [ln.split() for ln in slab.strip().split("\n")]
        for ln in reversed(lines):
            out.extend(ln)
    bad = [t for t in out if t not in ("0", "1")]
    if bad:
        raise ValueError(f"Invalid node type: {bad[0]}")
    return np.array([int(t) for t in out], dtype=np.uint8)


def read_bounce_back_map(path: str) -> np.ndarray:
    with open(path) as fh:
        return parse_bounce_back_map(fh.read())


def format_bounce_back_map(mask: np.ndarray, n: Sequence[int]) -> str:
    """Inverse of parse_bounce_back_map for a mask in node order."""
    nx, ny = int(n[0]), int(n[1])
    nz = int(n[2]) if len(n) > 2 else 1
    m = np.asarray(mask, dtype=np.uint8).reshape(nz, ny, nx)
    slabs = []
    for z in range(nz):
        rows = [" ".join(str(int(v)) for v in m[z, y]) for y in range(ny - 1, -1, -1)]
        slabs.append("\n".join(rows))
    return "\n\n".join(slabs) + "\n"


def write_bounce_back_map(path: str, mask: np.ndarray, n: Sequence[int]) -> None:
    with open(path, "w") as fh:
        fh.write(format_bounce_back_map(mask, n))


# ------------------------------------------------------------------ CSV fields
def read_csv_rows(path: str) -> list:
    """read_csv_file (src/io.rs:145-155): drop the header line."""
    with open(path) as fh:
        lines = fh.read().strip().split("\n")
    return lines[1:]


def read_scalar_csv(path: str) -> np.ndarray:
    return np.array([float(s) for s in read_csv_rows(path)], dtype=np.float64)


def read_vector_csv(path: str) -> np.ndarray:
    return np.array([[float(v) for v in s.split(",")] for s in read_csv_rows(path)], dtype=np.float64)


def _write_chunks(step_path: str, prefix: str, header: str, lines: list, num_threads: int) -> None:
    if num_threads <= 1:
        with open(os.path.join(step_path, f"{prefix}.csv"), "w") as fh:
            fh.write(header + "\n")
            fh.write("\n".join(lines) + ("\n" if lines else ""))
        return
    # par_chunks(number_of_nodes / number_of_threads) (src/momentum/io.rs:126-141)
    chunk = max(1, len(lines) // num_threads)
    for i, start in enumerate(range(0, len(lines), chunk)):
        with open(os.path.join(step_path, f"{prefix}_{i}.csv"), "w") as fh:
            fh.write(header + "\n")
            part = lines[start:start + chunk]
            fh.write("\n".join(part) + ("\n" if part else ""))


def write_step_data(time_step: int, density: np.ndarray, velocity: np.ndarray,
                    scalars: Optional[dict] = None, num_threads: int = 1, root: str = DATA_PATH) -> str:
    """data/<t>/density.csv, velocity.csv and <scalar>.csv for every node."""
    step_path = os.path.join(root, str(time_step))
    os.makedirs(step_path, exist_ok=True)
    _write_chunks(step_path, "density", "density", format_column(density), num_threads)
    dim = velocity.shape[1]
    header = "velocity_x,velocity_y" + (",velocity_z" if dim == 3 else "")
    vel_lines = [",".join(rust_e8(float(v)) for v in row) for row in velocity]
    _write_chunks(step_path, "velocity", header, vel_lines, num_threads)
    for name, values in (scalars or {}).items():
        _write_chunks(step_path, name, name, format_column(values), num_threads)
    return step_path


def write_coordinates(n: Sequence[int], node_type: Optional[np.ndarray], delta_x: float,
                      root: str = DATA_PATH) -> None:
    dim = len(n)
    N = int(np.prod(n))
    idx = np.arange(N)
    cols = [idx % n[0], (idx // n[0]) % n[1]] + ([idx // (n[0] * n[1])] if dim == 3 else [])
    os.makedirs(root, exist_ok=True)
    with open(os.path.join(root, COORDINATES_FILE), "w") as fh:
        fh.write("i,j,x,y,node_type\n" if dim == 2 else "i,j,k,x,y,z,node_type\n")
        for k in range(N):
            ids = ",".join(str(int(c[k])) for c in cols)
            xyz = ",".join(rust_e8((int(c[k]) + 0.5) * delta_x) for c in cols)
            t = "solid" if node_type is not None and node_type[k] else "fluid"
            fh.write(f"{ids},{xyz},{t}\n")


def residuals_header(dim: int, scalar_names: Sequence[str] = ()) -> str:
    h = "time_step,density," + ",".join(f"velocity_{x}" for x in "xyz"[:dim])
    for s in scalar_names:
        h += f",{s}"
    return h


def residuals_line(time_step: int, res: Sequence[float]) -> str:
    return f"{time_step}," + ",".join(rust_e8(float(r)) for r in res)


def append_residuals(time_step: int, res: Sequence[float], dim: int, scalar_names=(), root: str = DATA_PATH):
    os.makedirs(root, exist_ok=True)
    path = os.path.join(root, RESIDUALS_FILE)
    with open(path, "a") as fh:
        if time_step == 0:
            fh.write(residuals_header(dim, scalar_names) + "\n")
        fh.write(residuals_line(time_step, res) + "\n")
