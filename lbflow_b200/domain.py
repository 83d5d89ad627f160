"""`Domain`: one lattice on the GPU, driven through the C ABI of include/lbflow.h.

This replaces the reference's momentum::Lattice (+ passive_scalar::Lattice)
object graph: it is created from the same Parameters values, keeps the
populations resident on the device, and exposes the reference's passes as
calls (init / step / run / residuals / moments).  There is no CPU fallback:
creating a Domain loads liblbflow_b200.so or raises.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence, Union

import numpy as np

from . import _abi
from . import momentum as _m
from . import passive_scalar as _ps
from .core import VelocitySet


def _ptr(a: Optional[np.ndarray], ctype=C.c_double):
    return None if a is None else a.ctypes.data_as(C.POINTER(ctype))


def _stream_handle(stream) -> Optional[int]:
    """Accept None, an int handle, or a torch.cuda.Stream."""
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return int(stream.cuda_stream)


class Domain:
    """One lattice with up to LBF_MAX_SCALARS passive scalars.

    `scalar` is one passive_scalar.Parameters or a sequence of them (the
    reference's LatticeVec, src/passive_scalar/lattice.rs:353-430): one momentum
    sweep advances every scalar.  moments() reports scalar 0; scalar(i) and
    q_ads(i) the others; residuals() lists rho, u_a.., then every scalar.
    """

    def __init__(self, params: _m.Parameters,
                 scalar: Union[None, _ps.Parameters, Sequence[_ps.Parameters]] = None,
                 desc: Optional[_abi.DomainDesc] = None, scalar_desc: Optional[_abi.ScalarDesc] = None):
        self.lib = _abi.load()
        keep = []
        if desc is None:
            desc, keep = _m.to_desc(params)
        self.desc = desc
        vs = VelocitySet(desc.velocity_set)
        self.d, self.q = vs.d, vs.q
        self.n = tuple(int(desc.n[a]) for a in range(self.d))
        self.N = int(np.prod(self.n))
        h = C.c_void_p()
        _abi.check(self.lib.lbf_domain_create(C.byref(desc), C.byref(h)))
        self.h = h
        self.has_scalar = False
        self.scalar_name = None
        self.scalar_names = []
        scalars = [] if scalar is None else (list(scalar) if isinstance(scalar, (list, tuple)) else [scalar])
        if len(scalars) > _abi.LBF_MAX_SCALARS:
            self.close()
            raise ValueError(f"at most {_abi.LBF_MAX_SCALARS} scalars per domain")
        try:
            if scalar_desc is not None:
                _abi.check(self.lib.lbf_scalar_attach(self.h, C.byref(scalar_desc)))
                self.scalar_names.append(None)
            for sp in scalars:
                sd, k2 = _ps.to_desc(sp, self.n)
                keep += k2
                _abi.check(self.lib.lbf_scalar_attach(self.h, C.byref(sd)))
                self.scalar_names.append(sp.scalar_name)
            self.has_scalar = len(self.scalar_names) > 0
            self.scalar_name = self.scalar_names[0] if self.has_scalar else None
        except Exception:
            self.close()
            raise
        self._keep = keep   # the library copied them; kept only until here

    # -- lifecycle -----------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.lib.lbf_domain_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- passes ---------------------------------------------------------------
    def init(self, stream=None) -> "Domain":
        _abi.check(self.lib.lbf_domain_init(self.h, _stream_handle(stream)))
        return self

    def step(self, n: int = 1, residual_interval: int = 0, stream=None) -> "Domain":
        _abi.check(self.lib.lbf_domain_step(self.h, int(n), int(residual_interval), _stream_handle(stream)))
        return self

    def run(self, max_iterations: int, residual_interval: int = 1, tol_density: float = 1e-7,
            tol_velocity: float = 1e-7, tol_scalar: float = 1e-7, stream=None) -> int:
        steps = C.c_int64()
        _abi.check(self.lib.lbf_domain_run(self.h, int(max_iterations), int(residual_interval), tol_density,
                                           tol_velocity, tol_scalar, C.byref(steps), _stream_handle(stream)))
        return steps.value

    def set_option(self, option: int, value: int) -> "Domain":
        _abi.check(self.lib.lbf_domain_set_option(self.h, int(option), int(value)))
        return self

    def get_option(self, option: int) -> int:
        v = C.c_int64()
        _abi.check(self.lib.lbf_domain_get_option(self.h, int(option), C.byref(v)))
        return v.value

    @property
    def time_step(self) -> int:
        t = C.c_int64()
        _abi.check(self.lib.lbf_domain_time_step(self.h, C.byref(t)))
        return t.value

    @property
    def device_bytes(self) -> int:
        b = C.c_int64()
        _abi.check(self.lib.lbf_domain_device_bytes(self.h, C.byref(b)))
        return b.value

    @property
    def num_scalars(self) -> int:
        return len(self.scalar_names)

    def residuals(self):
        """([rho, u_a.., scalar_0, ..], time step they belong to)."""
        out = np.zeros(1 + 3 + _abi.LBF_MAX_SCALARS)
        t = C.c_int64()
        _abi.check(self.lib.lbf_domain_residuals(self.h, _ptr(out), C.byref(t)))
        return out[: 1 + self.d + self.num_scalars], t.value

    def moments(self, stream=None, out=None):
        """(density[N], velocity[N, D], scalar[N] or None) at the current time step.
        `out` = (rho, u, c) preallocated float64 arrays (any may be None) to fill;
        page-locked ones (e.g. numpy views of pinned tensors) download directly."""
        rho, u, c = _outputs(self.N, self.d, self.has_scalar, out)
        _abi.check(self.lib.lbf_domain_get_moments(self.h, _ptr(rho), _ptr(u), _ptr(c), _stream_handle(stream)))
        return rho, (u.reshape(self.N, self.d) if u is not None else None), c

    def scalar(self, index: int = 0, stream=None) -> np.ndarray:
        """Scalar `index` (attach order) at the current time step, [N]."""
        out = np.zeros(self.N)
        _abi.check(self.lib.lbf_domain_get_scalar(self.h, int(index), _ptr(out), _stream_handle(stream)))
        return out

    def q_ads(self, index: int = 0):
        out = np.zeros(self.N)
        _abi.check(self.lib.lbf_domain_get_q_ads_at(self.h, int(index), _ptr(out)))
        return out

    def inventory(self, stream=None):
        out = np.zeros(8)
        _abi.check(self.lib.lbf_domain_inventory(self.h, _ptr(out), _stream_handle(stream)))
        return out[: 3 + self.d]

    def save(self, path: str, stream=None) -> int:
        """Write a checkpoint of the carried state (lbf_domain_save); returns its bytes."""
        n = C.c_int64()
        _abi.check(self.lib.lbf_domain_checkpoint_bytes(self.h, C.byref(n)))
        buf = np.empty(n.value, dtype=np.uint8)
        _abi.check(self.lib.lbf_domain_save(self.h, buf.ctypes.data, n.value, _stream_handle(stream)))
        buf.tofile(path)
        return n.value

    def load(self, path: str, stream=None) -> "Domain":
        """Restore a checkpoint into this (initialised, same-descriptor) domain."""
        buf = np.fromfile(path, dtype=np.uint8)
        _abi.check(self.lib.lbf_domain_load(self.h, buf.ctypes.data, buf.size, _stream_handle(stream)))
        return self

    def node_class(self):
        cls = np.zeros(self.N, np.uint32)
        links = np.zeros(self.N, np.uint32)
        _abi.check(self.lib.lbf_domain_get_node_class(self.h, _ptr(cls, C.c_uint32), _ptr(links, C.c_uint32)))
        return cls, links


def tables(vs: int) -> dict:
    """Velocity-set tables as compiled into the device code (lbf_velocity_set_tables)."""
    lib = _abi.load()
    d, q = C.c_int32(), C.c_int32()
    c = np.zeros(81, np.int32); w = np.zeros(27); qb = np.zeros(27, np.int32)
    qf = np.zeros(54, np.int32); nrm = np.zeros(6, np.int32); M = np.zeros(729); Mi = np.zeros(729)
    i32 = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))  # noqa: E731
    _abi.check(lib.lbf_velocity_set_tables(vs, C.byref(d), C.byref(q), i32(c), _ptr(w), i32(qb), i32(qf), i32(nrm),
                                           _ptr(M), _ptr(Mi)))
    q = q.value
    return {"d": d.value, "q": q, "c": c[:3 * q].reshape(q, 3), "w": w[:q], "q_bar": qb[:q],
            "q_faces": qf.reshape(6, 9), "face_normal": nrm, "mrt": M[:q * q].reshape(q, q),
            "mrt_inverse": Mi[:q * q].reshape(q, q)}


def _outputs(N: int, d: int, has_scalar: bool, out):
    """Output arrays (rho[N], u[N*D], c[N] or None): the caller's, checked, or new."""
    if out is None:
        return np.zeros(N), np.zeros(N * d), (np.zeros(N) if has_scalar else None)
    rho, u, c = out
    for a, n in ((rho, N), (u, N * d), (c, N)):
        if a is not None and (a.dtype != np.float64 or a.size != n or not a.flags.c_contiguous):
            raise ValueError(f"output arrays must be contiguous float64 of {n} elements")
    return rho, (u.reshape(-1) if u is not None else None), (c if has_scalar else None)


def solve_arrays(params: _m.Parameters, nsteps: int, scalar: Optional[_ps.Parameters] = None, stream=None,
                 out=None):
    """lbf_solve: one call with host buffers (create, init, nsteps main_steps, moments).
    `out` = (rho, u, c) preallocated float64 arrays to fill, as in Domain.moments."""
    lib = _abi.load()
    desc, keep = _m.to_desc(params)
    vs = VelocitySet(desc.velocity_set)
    N = int(np.prod([desc.n[a] for a in range(vs.d)]))
    sdesc = None
    if scalar is not None:
        sdesc, k2 = _ps.to_desc(scalar, [desc.n[a] for a in range(vs.d)])
        keep += k2
    rho, u, c = _outputs(N, vs.d, scalar is not None, out)
    _abi.check(lib.lbf_solve(C.byref(desc), C.byref(sdesc) if sdesc is not None else None, int(nsteps),
                             _ptr(rho), _ptr(u), _ptr(c), _stream_handle(stream)))
    return rho, (u.reshape(N, vs.d) if u is not None else None), c
