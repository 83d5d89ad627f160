"""`solve`: the reference's driver loop with its file outputs, over the C ABI.

This is `lbflow::solve(momentum::Parameters, Option<Vec<passive_scalar::Parameters>>)`
(src/lib.rs:170-191), i.e. `momentum::run` (src/momentum.rs:262-293) or, with
scalars, `passive_scalar::run_vec` (src/passive_scalar.rs:136-177):

    case_setup; write_coordinates; initialize_nodes
    loop t = 0, 1, ...:
        main_steps                      (data/<t>/ written when t % write_data == 0)
        compute_lattice_residuals
        compute_post_processing        (post_processing/<file>, t % interval == 0)
        print + append residuals        (data/residuals.csv)
        stop if (t > 10 and all residuals <= 1e-7) or t > max_iterations

The step runs on the GPU (one fused kernel per main_steps).  The moments that
data/<t>/ holds are those of f_t, which the engine computes on demand before
step t runs ("observe"), so the files are the reference's.  Text formatting of
output steps runs on all host cores (lbf_format_csv) in a background thread
while the GPU keeps stepping.

The reference's CLI flags become keyword arguments: `write_data` (--write-data,
default 100), `max_iterations` (--max-iterations, default 100000) and
`num_threads` (--num-threads: the number of chunk files per field, as the
reference's parallel writer produces).  `freeze_momentum` is not supported by the
fused kernel (it always advances momentum) and raises.

Several scalars (`run_vec`, passive_scalar::LatticeVec) are attached to one
engine domain: each step advances the momentum populations once and every
scalar after them in the same sweep, as the reference advances one momentum
lattice and then each scalar lattice (src/passive_scalar.rs:136-177).
"""
from __future__ import annotations

import os
import sys
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence

import numpy as np

from . import _abi
from . import io as _io
from . import momentum as _m
from . import passive_scalar as _ps
from .domain import Domain

MIN_ITER = 10                     # src/constants.rs:15
TOLERANCE_DENSITY = 1e-7          # src/constants.rs:17
TOLERANCE_VELOCITY = 1e-7         # src/constants.rs:19
TOLERANCE_SCALAR_VALUE = 1e-7     # src/constants.rs:21
WRITE_DATA = 100                  # src/cli.rs:7
MAX_ITERATIONS = 100_000          # src/cli.rs:8


# ---------------------------------------------------------------- post-processing
@dataclass
class PostResult:
    """momentum::post::PostResult (src/momentum/post.rs:8-24)."""
    name: str
    label: str
    value: float
    unit: Optional[str] = None


@dataclass
class PostFunction:
    """momentum::post::PostFunction (src/momentum/post.rs:26-41): `function(lattice)` is
    evaluated every `interval` steps and appended to post_processing/<file_name>."""
    file_name: str
    interval: int
    function: Callable[["LatticeView"], List[PostResult]]


class LatticeView:
    """What a post function sees: the lattice at time step t (moments of f_t)."""

    def __init__(self, dom: Domain, time_step: int, num_fluid_nodes: int):
        self._dom = dom
        self.time_step = time_step
        self.num_fluid_nodes = num_fluid_nodes
        self.n = dom.n
        self.d = dom.d
        self._inv = None
        self._mom = None

    def inventory(self) -> np.ndarray:
        """FP64 sums over fluid nodes, reduced on the device: [sum rho, sum rho u_a, ...]."""
        if self._inv is None:
            self._inv = self._dom.inventory()
        return self._inv

    def moments(self):
        """(density[N], velocity[N, D], scalar[N] or None) of every node."""
        if self._mom is None:
            self._mom = self._dom.moments()
        return self._mom


def compute_mean_density(lattice: LatticeView) -> List[PostResult]:
    """momentum::post::compute_mean_density (src/momentum/post.rs:43-59)."""
    rho_mean = lattice.inventory()[0] / lattice.num_fluid_nodes
    return [PostResult("mean_density", "mean density", float(rho_mean), None)]


# ---------------------------------------------------------------- result
@dataclass
class SolveResult:
    time_steps: int                  # main_steps executed (last time step + 1)
    residuals: np.ndarray            # residuals of the last step: rho, u_a..., scalars...
    data_steps: List[int] = field(default_factory=list)
    wall_seconds: float = 0.0


def _case_directories(case_dir: str) -> dict:
    """crate::io::create_case_directories (src/io.rs:38-58)."""
    paths = {"data": os.path.join(case_dir, "data"), "pre": os.path.join(case_dir, "pre_processing"),
             "post": os.path.join(case_dir, "post_processing"),
             "vtk": os.path.join(case_dir, "post_processing", "vtk_files")}
    for p in paths.values():
        os.makedirs(p, exist_ok=True)
    return paths


def _print_header(dim: int, names: Sequence[str]) -> str:
    h = "\n" + f"{'time_step':>10} {'density':>16}" + "".join(f" {'velocity_' + x:>16}" for x in "xyz"[:dim])
    return h + "".join(f" {s:>16}" for s in names)


def _print_line(t: int, res: Sequence[float]) -> str:
    # Rust "{:>16.8e}": the {:.8e} text right-aligned in 16 columns
    return f"{t:>10}" + "".join(f" {_io.rust_e8(float(r)):>16}" for r in res)


def solve(momentum_params: _m.Parameters, passive_scalar_params: Optional[Sequence[_ps.Parameters]] = None, *,
          write_data: int = WRITE_DATA, max_iterations: int = MAX_ITERATIONS, num_threads: int = 1,
          case_dir: str = ".", verbose: bool = True, freeze_momentum: bool = False, format_threads: int = 0,
          stream=None) -> SolveResult:
    if freeze_momentum:
        raise NotImplementedError("freeze_momentum: the fused step always advances the momentum lattice")
    if passive_scalar_params is not None and len(passive_scalar_params) == 0:
        raise ValueError("Must provide at least one passive_scalar_parameters inside the vector.")
    if write_data < 1:
        raise ValueError("write_data must be >= 1")
    scalars = list(passive_scalar_params or [])
    names = [s.scalar_name for s in scalars]
    dim = momentum_params.dim
    paths = _case_directories(case_dir)
    wall0 = time.perf_counter()

    dom0 = Domain(momentum_params, scalars or None)
    writer = ThreadPoolExecutor(max_workers=1)
    pending = []
    try:
        cls, _ = dom0.node_class()
        solid = (cls & _abi.LBF_CLASS_SOLID) != 0
        num_fluid = int(np.count_nonzero(~solid))
        text = _io.format_coordinates_native(dom0.n, solid.astype(np.uint8), momentum_params.delta_x, format_threads)
        with open(os.path.join(paths["data"], _io.COORDINATES_FILE), "wb") as fh:
            fh.write(("i,j,x,y,node_type\n" if dim == 2 else "i,j,k,x,y,z,node_type\n").encode())
            fh.write(text)
        dom0.init(stream)

        post_functions = list(momentum_params.post_functions or [])
        res_path = os.path.join(paths["data"], _io.RESIDUALS_FILE)
        header = _print_header(dim, names)
        data_steps = []
        t = 0
        while True:
            # ---- main_steps(t): output of the moments of f_t --------------------
            if t % write_data == 0:
                rho, u, _ = dom0.moments(stream)
                fields = [("density", "density", rho),
                          ("velocity", ",".join(f"velocity_{x}" for x in "xyz"[:dim]), u)]
                for i, nm in enumerate(names):
                    fields.append((nm, nm, dom0.scalar(i, stream)))
                step_path = os.path.join(paths["data"], str(t))
                os.makedirs(step_path, exist_ok=True)
                for prefix, hdr, values in fields:
                    pending.append(writer.submit(_io.write_field_native, step_path, prefix, hdr, values,
                                                 num_threads, format_threads))
                data_steps.append(t)
            post_lines = []
            due = [pf for pf in post_functions if t % pf.interval == 0]
            if due:
                view = LatticeView(dom0, t, num_fluid)
                for pf in due:
                    post_lines.append((pf, pf.function(view)))
            dom0.step(1, 1, stream)
            # ---- residuals, post-processing, residual file, stop ---------------
            res = np.array(dom0.residuals()[0])
            for pf, results in post_lines:
                path = os.path.join(paths["post"], pf.file_name)
                with open(path, "a") as fh:
                    if t == 0:
                        fh.write("time_step" + "".join(f",{r.name}" for r in results) + "\n")
                    fh.write(f"{t}" + "".join(f",{_io.rust_e8(r.value)}" for r in results) + "\n")
            if verbose:
                if t % 100 == 0:
                    print(header + "\n", file=sys.stdout)
                print(_print_line(t, res), file=sys.stdout)
            with open(res_path, "a") as fh:
                if t == 0:
                    fh.write(_io.residuals_header(dim, names) + "\n")
                fh.write(_io.residuals_line(t, res) + "\n")
            if not np.all(np.isfinite(res)):
                raise FloatingPointError(f"non-finite residual at time step {t}")
            converged = (res[0] <= TOLERANCE_DENSITY and all(r <= TOLERANCE_VELOCITY for r in res[1:1 + dim])
                         and all(r <= TOLERANCE_SCALAR_VALUE for r in res[1 + dim:]))
            if (t > MIN_ITER and converged) or t > max_iterations:
                break
            t += 1
        for f in pending:
            f.result()
        return SolveResult(time_steps=t + 1, residuals=res, data_steps=data_steps,
                           wall_seconds=time.perf_counter() - wall0)
    finally:
        writer.shutdown(wait=True)
        dom0.close()
