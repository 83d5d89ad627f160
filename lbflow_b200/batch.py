"""`Batch`: many domains stepped together on one GPU (lbf_batch_* of include/lbflow.h).

The reference solves one case per process (`lbflow::solve`).  A serving loop
holds many small cases at once; stepping them one launch per domain and step
leaves most SMs idle, so a batch lays the domains of one kernel configuration
end to end in one launch per time step, runs chunks of `residual_interval`
steps as a replayed CUDA graph, and evaluates each domain's residuals and stop
rule on the device.  Each domain stops exactly where
`Domain.run(max_iterations, residual_interval, tol_*)` stops it, with the same
fields.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Optional, Tuple

from . import _abi
from . import momentum as _m
from . import passive_scalar as _ps
from .domain import Domain, _stream_handle

STATUS = {1: "converged", 2: "max_iterations", 3: "non-finite residual"}


class BatchFull(_abi.LbfError):
    """The domain does not fit the batch's device-memory budget."""


def estimate_bytes(params: _m.Parameters, scalar: Optional[_ps.Parameters] = None) -> int:
    """Upper bound of the device bytes of a domain built from these parameters
    (lbf_domain_estimate_bytes), for admission before any allocation."""
    lib = _abi.load()
    desc, keep = _m.to_desc(params)
    sdesc = None
    if scalar is not None:
        sdesc, k2 = _ps.to_desc(scalar, params.n[: params.dim])
        keep += k2
    b = C.c_int64()
    _abi.check(lib.lbf_domain_estimate_bytes(C.byref(desc), C.byref(sdesc) if sdesc is not None else None,
                                             C.byref(b)))
    return b.value


class Batch:
    def __init__(self, budget_bytes: int = 0, residual_interval: int = 50):
        self.lib = _abi.load()
        h = C.c_void_p()
        _abi.check(self.lib.lbf_batch_create(int(budget_bytes), int(residual_interval), C.byref(h)))
        self.h = h
        self.residual_interval = int(residual_interval)
        self._doms: Dict[int, Domain] = {}

    def close(self):
        if getattr(self, "h", None):
            self.lib.lbf_batch_destroy(self.h)
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

    def admit(self, dom: Domain, max_iterations: int, tol_density: float = 1e-7, tol_velocity: float = 1e-7,
              tol_scalar: float = 1e-7) -> None:
        st = self.lib.lbf_batch_admit(self.h, dom.h, int(max_iterations), float(tol_density), float(tol_velocity),
                                      float(tol_scalar))
        if st == _abi.LBF_ENOMEM:
            raise BatchFull(st, self.lib.lbf_last_error().decode())
        _abi.check(st)
        self._doms[dom.h.value] = dom

    def set_option(self, option: int, value: int) -> "Batch":
        """lbf_batch_set_option, e.g. LBF_BATCH_OPT_CHUNK_LAUNCH (1: a group's chunk
        in one cooperative launch; 0: one launch per step, the default)."""
        _abi.check(self.lib.lbf_batch_set_option(self.h, int(option), int(value)))
        return self

    def step(self, nchunks: int = 1, stream=None) -> "Batch":
        """Enqueue `nchunks` chunks of residual_interval steps (asynchronous)."""
        _abi.check(self.lib.lbf_batch_step(self.h, int(nchunks), _stream_handle(stream)))
        return self

    def poll(self, wait: bool = True, cap: int = 256) -> List[Tuple[Domain, int]]:
        """Domains that stopped, with their status (1 converged, 2 max_iterations,
        3 non-finite residual); they leave the batch and accept standalone calls again."""
        out: List[Tuple[Domain, int]] = []
        done = (C.c_void_p * cap)()
        status = (C.c_int32 * cap)()
        n = C.c_int32()
        while True:
            _abi.check(self.lib.lbf_batch_poll(self.h, done, status, cap, C.byref(n), 1 if wait else 0))
            for i in range(n.value):
                out.append((self._doms.pop(done[i]), int(status[i])))
            if n.value < cap:
                return out

    def evict(self, dom: Domain) -> None:
        _abi.check(self.lib.lbf_batch_evict(self.h, dom.h))
        self._doms.pop(dom.h.value, None)

    def info(self) -> dict:
        r, f, b, g = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        _abi.check(self.lib.lbf_batch_info(self.h, C.byref(r), C.byref(f), C.byref(b), C.byref(g)))
        return {"running": r.value, "finished": f.value, "bytes": b.value, "budget": g.value}

    def __len__(self) -> int:
        return self.info()["running"]
