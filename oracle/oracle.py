"""ctypes wrapper of the CPU oracle (oracle/liblbf_oracle.so) -- TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs as the
checker.  It takes the same descriptor structs as the product's C ABI
(include/lbflow.h), so a test builds one descriptor and feeds both.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from lbflow_b200 import _abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liblbf_oracle.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB):
        build()
    L = C.CDLL(_LIB)
    P, I32, I64, D = C.c_void_p, C.c_int, C.c_int64, C.c_double
    PD, PI = C.POINTER(C.c_double), C.POINTER(C.c_int)
    sig = {
        "orc_last_error": (C.c_char_p, []),
        "orc_num_threads": (I32, []),
        "orc_set_num_threads": (None, [I32]),
        "orc_velocity_set_tables": (I32, [I32, PI, PI, PI, PD, PI, PI, PI, PD, PD]),
        "orc_equilibrium": (I32, [I32, D, PD, PD]),
        "orc_bgk": (I32, [I32, PD, PD, D, PD]),
        "orc_trt": (I32, [I32, PD, PD, D, D, PD]),
        "orc_mrt": (I32, [I32, D, PD, PD, PD, PD, I32, PD]),
        "orc_momentum_source": (I32, [I32, PD, PD, D, PD]),
        "orc_central": (I32, [I32, D, PD, PD, D, PD, PD]),
        "orc_mrt_meq": (I32, [I32, D, PD, PD]),
        "orc_zou_he": (I32, [I32, I32, PD, I32, D, PI, PD]),
        "orc_create": (I32, [C.POINTER(_abi.DomainDesc), C.POINTER(P)]),
        "orc_scalar_attach": (I32, [P, C.POINTER(_abi.ScalarDesc)]),
        "orc_init": (I32, [P]),
        "orc_step": (I32, [P, I64]),
        "orc_run": (I32, [P, I64, D, D, D, C.POINTER(C.c_int64)]),
        "orc_observe": (I32, [P, PD, PD, PD]),
        "orc_residuals": (I32, [P, PD]),
        "orc_time_step": (I64, [P]),
        "orc_num_fluid": (I64, [P]),
        "orc_node_class": (I32, [P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
        "orc_get_q_ads": (I32, [P, PD]),
        "orc_inventory": (I32, [P, PD]),
        "orc_get_array": (I32, [P, I32, PD]),
        "orc_set_array": (I32, [P, I32, PD]),
        "orc_pass": (I32, [P, I32]),
        "orc_neighbor": (I64, [P, I64, I32]),
        "orc_destroy": (None, [P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _pd(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _pi(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _chk(st: int) -> None:
    if st != 0:
        raise RuntimeError(f"oracle: status {st}: {lib().orc_last_error().decode()}")


def set_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


def num_threads() -> int:
    return lib().orc_num_threads()


def tables(vs: int) -> dict:
    d, q = C.c_int(), C.c_int()
    c = np.zeros(27 * 3, np.int32); w = np.zeros(27); qbar = np.zeros(27, np.int32)
    qf = np.zeros(54, np.int32); nrm = np.zeros(6, np.int32)
    M = np.zeros(27 * 27); Mi = np.zeros(27 * 27)
    _chk(lib().orc_velocity_set_tables(vs, C.byref(d), C.byref(q), _pi(c), _pd(w), _pi(qbar),
                                       _pi(qf), _pi(nrm), _pd(M), _pd(Mi)))
    q = q.value
    return {"d": d.value, "q": q, "c": c[:3 * q].reshape(q, 3), "w": w[:q], "q_bar": qbar[:q],
            "q_faces": qf.reshape(6, 9), "face_normal": nrm, "mrt": M[:q * q].reshape(q, q),
            "mrt_inverse": Mi[:q * q].reshape(q, q)}


def equilibrium(vs, value, u):
    q = tables(vs)["q"]
    out = np.zeros(q); u = np.ascontiguousarray(u, float)
    _chk(lib().orc_equilibrium(vs, value, _pd(u), _pd(out)))
    return out


def bgk(vs, f, feq, tau):
    f = np.ascontiguousarray(f, float); feq = np.ascontiguousarray(feq, float); out = np.zeros_like(f)
    _chk(lib().orc_bgk(vs, _pd(f), _pd(feq), tau, _pd(out)))
    return out


def trt(vs, f, feq, op, om):
    f = np.ascontiguousarray(f, float); feq = np.ascontiguousarray(feq, float); out = np.zeros_like(f)
    _chk(lib().orc_trt(vs, _pd(f), _pd(feq), op, om, _pd(out)))
    return out


def mrt(vs, value, u, f, feq, relax, compat=0):
    f = np.ascontiguousarray(f, float); feq = np.ascontiguousarray(feq, float)
    u = np.ascontiguousarray(u, float); relax = np.ascontiguousarray(relax, float)
    out = np.zeros_like(f)
    _chk(lib().orc_mrt(vs, value, _pd(u), _pd(f), _pd(feq), _pd(relax), compat, _pd(out)))
    return out


def central(vs, rho, u, f, tau, rates=(1.0, 1.0, 1.0, 1.0, 1.0)):
    """Central-moment collision of one node (rates: bulk, 3rd..6th order)."""
    f = np.ascontiguousarray(f, float); u = np.ascontiguousarray(u, float)
    r = np.ascontiguousarray(rates, float); out = np.zeros_like(f)
    _chk(lib().orc_central(vs, rho, _pd(u), _pd(f), tau, _pd(r), _pd(out)))
    return out


def momentum_source(vs, u, force, tau):
    q = tables(vs)["q"]
    u = np.ascontiguousarray(u, float); F = np.ascontiguousarray(force, float); out = np.zeros(q)
    _chk(lib().orc_momentum_source(vs, _pd(u), _pd(F), tau, _pd(out)))
    return out


def mrt_meq(vs, rho, u):
    q = tables(vs)["q"]
    u = np.ascontiguousarray(u, float); out = np.zeros(q)
    _chk(lib().orc_mrt_meq(vs, rho, _pd(u), _pd(out)))
    return out


def zou_he(vs, face, f, density=None, velocity=(None, None, None)):
    f = np.array(f, float)
    hu = np.array([v is not None for v in list(velocity) + [None] * (3 - len(velocity))], np.int32)
    u = np.array([0.0 if v is None else v for v in list(velocity) + [None] * (3 - len(velocity))])
    st = lib().orc_zou_he(vs, face, _pd(f), int(density is not None), 0.0 if density is None else density,
                          _pi(hu), _pd(u))
    if st != 0:
        raise ValueError(lib().orc_last_error().decode())
    return f


class Domain:
    """One oracle lattice (momentum + optional scalar), driven pass by pass or step by step."""

    ARRAYS = {"f": 0, "f_eq": 1, "f_star": 2, "density": 3, "velocity": 4, "g": 5, "g_star": 6, "scalar": 7}

    def __init__(self, desc: _abi.DomainDesc, scalar: _abi.ScalarDesc | None = None, keep=()):
        self._keep = list(keep)
        self.desc = desc
        h = C.c_void_p()
        _chk(lib().orc_create(C.byref(desc), C.byref(h)))
        self.h = h
        vs = tables(desc.velocity_set)
        self.d, self.q = vs["d"], vs["q"]
        self.n = (desc.n[0], desc.n[1], desc.n[2] if self.d == 3 else 1)
        self.N = self.n[0] * self.n[1] * self.n[2]
        self.has_scalar = False
        if scalar is not None:
            _chk(lib().orc_scalar_attach(self.h, C.byref(scalar)))
            self.has_scalar = True
            self.qs = tables(scalar.velocity_set)["q"]

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def init(self):
        _chk(lib().orc_init(self.h))
        return self

    def step(self, n: int = 1):
        _chk(lib().orc_step(self.h, int(n)))
        return self

    def run(self, max_iterations: int, tol_density=1e-7, tol_velocity=1e-7, tol_scalar=1e-7) -> int:
        steps = C.c_int64()
        _chk(lib().orc_run(self.h, int(max_iterations), tol_density, tol_velocity, tol_scalar, C.byref(steps)))
        return steps.value

    @property
    def time_step(self) -> int:
        return lib().orc_time_step(self.h)

    @property
    def num_fluid(self) -> int:
        return lib().orc_num_fluid(self.h)

    def observe(self):
        rho = np.zeros(self.N); u = np.zeros(self.N * self.d)
        c = np.zeros(self.N) if self.has_scalar else None
        _chk(lib().orc_observe(self.h, _pd(rho), _pd(u), _pd(c) if c is not None else None))
        return rho, u.reshape(self.N, self.d), c

    def residuals(self):
        out = np.zeros(1 + self.d + (1 if self.has_scalar else 0))
        _chk(lib().orc_residuals(self.h, _pd(out)))
        return out

    def node_class(self):
        cls = np.zeros(self.N, np.uint32); links = np.zeros(self.N, np.uint32)
        _chk(lib().orc_node_class(self.h, cls.ctypes.data_as(C.POINTER(C.c_uint32)),
                                  links.ctypes.data_as(C.POINTER(C.c_uint32))))
        return cls, links

    def q_ads(self):
        out = np.zeros(self.N)
        _chk(lib().orc_get_q_ads(self.h, _pd(out)))
        return out

    def inventory(self):
        out = np.zeros(3 + self.d)
        _chk(lib().orc_inventory(self.h, _pd(out)))
        return out

    def _size(self, name):
        if name in ("f", "f_eq", "f_star"):
            return self.N * self.q
        if name in ("g", "g_star"):
            return self.N * self.qs
        if name == "velocity":
            return self.N * self.d
        return self.N

    def get(self, name):
        out = np.zeros(self._size(name))
        _chk(lib().orc_get_array(self.h, self.ARRAYS[name], _pd(out)))
        return out

    def set(self, name, values):
        a = np.ascontiguousarray(values, float).ravel()
        assert a.size == self._size(name)
        _chk(lib().orc_set_array(self.h, self.ARRAYS[name], _pd(a)))

    def run_pass(self, p: int):
        _chk(lib().orc_pass(self.h, p))

    def neighbor(self, idx: int, i: int) -> int:
        return lib().orc_neighbor(self.h, idx, i)
