"""Post-processing of a finished case: VTK files and unification of chunked CSVs.

This is the reference's `post vtk` and `post unify` commands
(src/momentum/post/vtk.rs, src/passive_scalar/post/vtk.rs): they read what a
run wrote under data/ and write legacy-ASCII VTK structured grids under
post_processing/vtk_files/, or merge the chunk files that a run with
num_threads > 1 writes (data/<t>/<prefix>_<i>.csv) into one file per field.

File layout, as the reference writes it:

    # vtk DataFile Version 3.0
    lbflow simulation data
    ASCII
    DATASET STRUCTURED_GRID
    DIMENSIONS nx ny nz                 (nz = 1 in 2-D)
    POINTS N float                      (x y z per node, Rust {:.4e}; z = 0 in 2-D)
    POINT_DATA N
    SCALARS density float 1             (Rust {:.8e})
    LOOKUP_TABLE default
    VECTORS velocity float              (three components, z = 0 in 2-D)
    [SCALARS physical_pressure / VECTORS physical_velocity, with physical_data]
    [SCALARS <scalar name> float 1 + LOOKUP_TABLE default, one block per scalar]

The node-type file <case>_node_type.vtk holds the points and `SCALARS node_type`
(1 solid, 0 fluid).  Points come from data/coordinates.csv, parsed and printed
again at four digits, as the reference does.  Files for different time steps
are written by a pool of threads (the reference's rayon loop).
"""
from __future__ import annotations

import os
import re
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import io as _io
from . import momentum as _m
from . import passive_scalar as _ps
from .core import BGK, MRT, TRT, CentralMoment, VelocitySet

CS_2 = 1.0 / 3.0            # src/constants.rs:9 (DELTA_X = DELTA_T = 1)
LATTICE_DENSITY = 1.0       # src/constants.rs:7
DELTA_T = 1.0               # src/constants.rs:3


def rust_e(x: float, prec: int) -> str:
    """Rust's `{:.<prec>e}`: `prec` fraction digits, exponent without padding or '+'."""
    if x != x:
        return "NaN"
    if x in (float("inf"), float("-inf")):
        return "inf" if x > 0 else "-inf"
    mant, exp = f"{x:.{prec}e}".split("e")
    return f"{mant}e{int(exp)}"


def _format_column(values: np.ndarray, prec: int) -> List[str]:
    """Rust {:.<prec>e} of each value; a column with few distinct values (grid
    coordinates) is formatted once per distinct value."""
    v = np.asarray(values, dtype=np.float64)
    uniq, inv = np.unique(v, return_inverse=True)
    if uniq.size * 4 < v.size:
        txt = np.array([rust_e(float(x), prec) for x in uniq], dtype=object)
        return list(txt[inv])
    return [rust_e(float(x), prec) for x in v]


@dataclass
class ConversionFactor:
    """momentum::ConversionFactor (src/momentum.rs:135-245): lattice to physical units."""
    delta_x: float
    delta_t: float
    physical_density: float
    reference_pressure: float
    shear_viscosity: float
    bulk_viscosity: float

    @property
    def length_conversion_factor(self) -> float:
        return self.delta_x

    @property
    def time_conversion_factor(self) -> float:
        return self.delta_t

    @property
    def density_conversion_factor(self) -> float:
        return self.physical_density

    @property
    def velocity_conversion_factor(self) -> float:
        return self.delta_x / self.delta_t

    @property
    def pressure_conversion_factor(self) -> float:
        u = self.velocity_conversion_factor
        return self.density_conversion_factor * u * u

    @property
    def viscosity_conversion_factor(self) -> float:
        return self.delta_x * self.delta_x / self.delta_t

    @property
    def physical_shear_viscosity(self) -> float:
        return self.viscosity_conversion_factor * self.shear_viscosity

    @property
    def physical_bulk_viscosity(self) -> float:
        return self.viscosity_conversion_factor * self.bulk_viscosity

    @staticmethod
    def from_params(p: _m.Parameters) -> "ConversionFactor":
        """ConversionFactor::from (src/momentum.rs:155-244): the lattice viscosities
        of the collision operator."""
        c = p.collision_operator
        vs = VelocitySet(p.velocity_set)
        if isinstance(c, BGK) or isinstance(c, CentralMoment):
            nu = CS_2 * (c.tau - 0.5 * DELTA_T)
            zeta = 2.0 / 3.0 * nu
        elif isinstance(c, TRT):
            nu = CS_2 * (1.0 / (c.omega_plus * DELTA_T) - 0.5)
            zeta = 2.0 / 3.0 * nu
        elif isinstance(c, MRT):
            r = list(c.relaxation_vector)
            if vs == VelocitySet.D2Q9:
                nu = CS_2 * (1.0 / r[7] - 0.5)
                zeta = CS_2 * (1.0 / r[1] - 0.5) - nu / 3.0
            elif vs in (VelocitySet.D3Q15, VelocitySet.D3Q19, VelocitySet.D3Q27):
                nu = CS_2 * (1.0 / r[9] - 0.5 * DELTA_T)
                zeta = 2.0 / 3.0 * CS_2 * (1.0 / r[1] - 0.5 * DELTA_T)
            else:
                raise NotImplementedError("conversion factor for D2Q5 MRT (the reference's todo!)")
        else:
            raise TypeError(f"unknown collision operator {c!r}")
        return ConversionFactor(p.delta_x, p.delta_t, p.physical_density, p.reference_pressure, nu, zeta)

    def physical_pressure(self, density: np.ndarray) -> np.ndarray:
        """compute_physical_pressure (vtk.rs:247-255)."""
        return self.reference_pressure + CS_2 * (np.asarray(density) - LATTICE_DENSITY) * self.pressure_conversion_factor

    def physical_velocity(self, velocity: np.ndarray) -> np.ndarray:
        """compute_physical_velocity (vtk.rs:257-266)."""
        return np.asarray(velocity) * self.velocity_conversion_factor


# ------------------------------------------------------------------ reading a case
def read_coordinates_file(dim: int, case_dir: str = "."):
    """read_coordinates_file (vtk.rs:8-45): (indexes [N, D] int, coordinates [N, D],
    node_types [N] bool solid)."""
    rows = _io.read_csv_rows(os.path.join(case_dir, _io.DATA_PATH, _io.COORDINATES_FILE))
    idx = np.empty((len(rows), dim), dtype=np.int64)
    xyz = np.empty((len(rows), dim), dtype=np.float64)
    solid = np.empty(len(rows), dtype=bool)
    for k, line in enumerate(rows):
        items = line.split(",")
        idx[k] = [int(v) for v in items[:dim]]
        xyz[k] = [float(v) for v in items[dim:2 * dim]]
        t = items[-1]
        if t not in ("fluid", "solid"):
            raise ValueError("Value not expected: must be 'solid' ou 'fluid'.")
        solid[k] = t == "solid"
    return idx, xyz, solid


def collect_time_steps(case_dir: str = ".") -> List[int]:
    """collect_time_steps (src/io.rs:157-172): the numeric directories of data/, sorted."""
    root = os.path.join(case_dir, _io.DATA_PATH)
    steps = []
    for name in os.listdir(root):
        if os.path.isdir(os.path.join(root, name)) and name.isdigit():
            steps.append(int(name))
    return sorted(steps)


# ------------------------------------------------------------------ writing VTK
def _header(n: Sequence[int], points: str) -> str:
    N = int(np.prod(n))
    nn = list(n) + [1] * (3 - len(n))
    return ("# vtk DataFile Version 3.0\nlbflow simulation data\nASCII\nDATASET STRUCTURED_GRID\n"
            f"DIMENSIONS {nn[0]} {nn[1]} {nn[2]}\nPOINTS {N} float\n{points}")


def format_points(coordinates: np.ndarray) -> str:
    """The POINTS block: 'x y z' per node at Rust {:.4e} (z = 0 in 2-D)."""
    N, d = coordinates.shape
    cols = [_format_column(coordinates[:, a], 4) for a in range(d)]
    if d == 2:
        cols.append([rust_e(0.0, 4)] * N)
    return "".join(f"{a} {b} {c}\n" for a, b, c in zip(*cols))


def _vector_block(v: np.ndarray) -> str:
    N, d = v.shape
    cols = [[rust_e(float(x), 8) for x in v[:, a]] for a in range(d)]
    if d == 2:
        cols.append([rust_e(0.0, 8)] * N)
    return "".join(f"{a} {b} {c}\n" for a, b, c in zip(*cols))


def _scalar_block(name: str, values: np.ndarray) -> str:
    return (f"SCALARS {name} float 1\nLOOKUP_TABLE default\n" +
            "".join(rust_e(float(x), 8) + "\n" for x in np.asarray(values)))


def write_node_type_vtk(path: str, n: Sequence[int], points: str, solid: np.ndarray) -> None:
    """write_node_type_vtk (vtk.rs:89-130)."""
    N = int(np.prod(n))
    with open(path, "w") as fh:
        fh.write(_header(n, points))
        fh.write(f"POINT_DATA {N}\nSCALARS node_type float 1\nLOOKUP_TABLE default\n")
        fh.write("".join("1\n" if s else "0\n" for s in solid))


def write_momentum_vtk(path: str, cf: ConversionFactor, n: Sequence[int], points: str, density: np.ndarray,
                       velocity: np.ndarray, physical_data: bool) -> None:
    """write_momentum_vtk (vtk.rs:132-205)."""
    N = int(np.prod(n))
    with open(path, "w") as fh:
        fh.write(_header(n, points))
        fh.write(f"POINT_DATA {N}\n")
        fh.write(_scalar_block("density", density))
        fh.write("VECTORS velocity float\n" + _vector_block(velocity))
        if physical_data:
            fh.write(_scalar_block("physical_pressure", cf.physical_pressure(density)))
            fh.write("VECTORS physical_velocity float\n" + _vector_block(cf.physical_velocity(velocity)))


def append_passive_scalar_vtk(path: str, prefix: str, values: np.ndarray) -> None:
    """append_passive_scalar_vtk (src/passive_scalar/post/vtk.rs:27-40)."""
    with open(path, "a") as fh:
        fh.write(_scalar_block(prefix, values))


def _scalar_list(passive_scalar_params) -> list:
    if passive_scalar_params is None:
        return []
    if isinstance(passive_scalar_params, _ps.Parameters):
        return [passive_scalar_params]
    return list(passive_scalar_params)


def post_vtk(momentum_params: _m.Parameters, passive_scalar_params=None, *, case_dir: str = ".",
             case_name: Optional[str] = None, node_type: bool = True, physical_data: bool = False,
             freeze_momentum: bool = False, threads: int = 0, verbose: bool = False) -> List[str]:
    """`post vtk` (momentum/post/vtk.rs:207-229, passive_scalar/post/vtk.rs:150-215):
    <case>_node_type.vtk when `node_type`, then <case>_output_<t:08>.vtk for every
    time step under data/ with density and velocity (unless freeze_momentum), and
    each scalar appended.  `case_name` stands for the reference's executable name
    (default: the name of the case directory).  Returns the paths written."""
    dim = momentum_params.dim
    n = list(momentum_params.n)[:dim]
    name = case_name or os.path.basename(os.path.abspath(case_dir)) or "case"
    vtk_dir = os.path.join(case_dir, _io.VTK_PATH)
    os.makedirs(vtk_dir, exist_ok=True)
    _, coords, solid = read_coordinates_file(dim, case_dir)
    points = format_points(coords)
    written = []
    if node_type:
        p = os.path.join(vtk_dir, f"{name}_node_type.vtk")
        if verbose:
            print(f"Writing {os.path.basename(p)} for node types.\n")
        write_node_type_vtk(p, n, points, solid)
        written.append(p)
    cf = ConversionFactor.from_params(momentum_params)
    scalars = [sp.scalar_name for sp in _scalar_list(passive_scalar_params)]
    data = os.path.join(case_dir, _io.DATA_PATH)

    def one(t: int) -> str:
        p = os.path.join(vtk_dir, f"{name}_output_{t:08d}.vtk")
        step = os.path.join(data, str(t))
        if not freeze_momentum:
            if verbose:
                print(f"Writing {os.path.basename(p)} for time step {t}.")
            rho = _io.read_scalar_csv(os.path.join(step, _io.DENSITY_FILE))
            u = _io.read_vector_csv(os.path.join(step, _io.VELOCITY_FILE))
            write_momentum_vtk(p, cf, n, points, rho, u.reshape(len(rho), dim), physical_data)
        for s in scalars:
            append_passive_scalar_vtk(p, s, _io.read_scalar_csv(os.path.join(step, f"{s}.csv")))
        return p

    steps = collect_time_steps(case_dir)
    with ThreadPoolExecutor(max_workers=threads or min(8, os.cpu_count() or 1)) as ex:
        written += list(ex.map(one, steps))
    return written


# ------------------------------------------------------------------ unify
def unify_parallel_csv_files(directory: str, prefix: str, header: str, keep: bool) -> None:
    """unify_parallel_csv_files (src/io.rs:174-232): <prefix>_<i>.csv, i ascending,
    headers dropped, into <prefix>.csv under `header`; the chunks are deleted
    unless `keep`."""
    pat = re.compile(rf"^{re.escape(prefix)}_(\d+)\.csv$")
    parts = sorted((int(m.group(1)), f) for f in os.listdir(directory) if (m := pat.match(f)))
    lines = []
    for _, f in parts:
        lines += _io.read_csv_rows(os.path.join(directory, f))
    with open(os.path.join(directory, f"{prefix}.csv"), "w") as fh:
        fh.write(header + "\n")
        fh.write("".join(line + "\n" for line in lines))
    if not keep:
        for _, f in parts:
            os.remove(os.path.join(directory, f))


def post_unify(momentum_params: _m.Parameters, passive_scalar_params=None, *, case_dir: str = ".",
               keep: bool = False, freeze_momentum: bool = False) -> None:
    """`post unify` (momentum/post/vtk.rs:231-305, passive_scalar/post/vtk.rs:83-100)."""
    dim = momentum_params.dim
    data = os.path.join(case_dir, _io.DATA_PATH)
    scalars = [sp.scalar_name for sp in _scalar_list(passive_scalar_params)]
    for t in collect_time_steps(case_dir):
        step = os.path.join(data, str(t))
        if not freeze_momentum:
            unify_parallel_csv_files(step, "density", "density", keep)
            unify_parallel_csv_files(step, "velocity", ",".join(f"velocity_{x}" for x in "xyz"[:dim]), keep)
        for s in scalars:
            unify_parallel_csv_files(step, s, s, keep)
