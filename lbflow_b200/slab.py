"""Z-slab decomposition of one lattice over several GPUs (one process per GPU).

Rank r of R owns the z planes [z0, z1) of the global lattice (balanced split).
Its domain holds those planes plus one ghost plane below and above: local
lattice nx x ny x (z1 - z0 + 2), periodic in z, sweeping the owned planes
1 .. z1 - z0 (LBF_OPT_Z_BEGIN / LBF_OPT_Z_END).  A ghost plane is

  - the neighbour's boundary plane when the neighbour exists (an interior cut,
    or the wrap of a periodic z axis): after every step the leaving populations
    of each owned boundary plane (5 for D3Q19, 9 for D3Q27) are packed on the
    device, exchanged with the neighbours by NCCL send/recv, and unpacked into
    the ghost planes the next step pulls from;
  - solid nodes when the global z face is a no-slip wall: the link bits then
    bounce the populations back exactly as the reference's NoSlip face rule
    (src/momentum/bc.rs:119-129) does, the same folding the single-domain lean
    path uses.

Both z faces of the global lattice must be Periodic or both NoSlip; x and y
faces may carry any boundary condition.  Scalars are not decomposed.

Per rank and step: one fused step kernel over the owned planes, two pack
kernels, one grouped NCCL send/recv per neighbour, two unpack kernels.
Residuals combine over ranks as sqrt(sum over ranks of r_rank^2); inventories
sum.  The halo ordering (sends: down then up; receives: from up then from
down) matches in order per peer, which also holds when R = 2 and both
neighbours are the same rank.
"""
from __future__ import annotations

import copy
import ctypes as C
from typing import Optional, Sequence, Tuple

import numpy as np

from . import _abi
from . import momentum as _m
from .core import BoundaryFace, VelocitySet


def slab_bounds(nz: int, nranks: int, rank: int) -> Tuple[int, int]:
    """Planes [z0, z1) of `rank`: the first nz % nranks ranks get one extra plane."""
    base, extra = divmod(nz, nranks)
    z0 = rank * base + min(rank, extra)
    return z0, z0 + base + (1 if rank < extra else 0)


def z_periodic(params: _m.Parameters) -> bool:
    """True for periodic z faces, False for no-slip z walls; anything else raises."""
    kinds = {face: bc.kind for face, bc in params.boundary_conditions
             if face in (BoundaryFace.Bottom, BoundaryFace.Top)}
    b, t = kinds.get(BoundaryFace.Bottom), kinds.get(BoundaryFace.Top)
    per, ns = _abi.LBF_BC_PERIODIC, _abi.LBF_BC_NO_SLIP
    if b == per and t == per:
        return True
    if b == ns and t == ns:
        return False
    raise ValueError("a z-slab decomposition needs both z faces Periodic or both NoSlip")


def neighbours(rank: int, nranks: int, periodic: bool) -> Tuple[Optional[int], Optional[int]]:
    """(rank below, rank above); None where the slab touches a no-slip z wall."""
    down = rank - 1 if rank > 0 else (nranks - 1 if periodic else None)
    up = rank + 1 if rank < nranks - 1 else (0 if periodic else None)
    return down, up


def leaving_directions(vs: int, face: BoundaryFace) -> list:
    """Directions that leave through the bottom (c_z = -1) or top (c_z = +1) face."""
    from .domain import tables
    c = tables(int(vs))["c"]
    want = -1 if face == BoundaryFace.Bottom else 1
    return [i for i in range(len(c)) if int(c[i][2]) == want]


def local_mask(own: np.ndarray, below: Optional[np.ndarray], above: Optional[np.ndarray]) -> np.ndarray:
    """(nz_loc + 2, ny, nx) node types: ghost planes from the neighbours, or solid walls."""
    nzl, ny, nx = own.shape
    out = np.empty((nzl + 2, ny, nx), dtype=np.uint8)
    out[1:-1] = own
    out[0] = 1 if below is None else below
    out[-1] = 1 if above is None else above
    return out


def local_parameters(params: _m.Parameters, mask_local: np.ndarray) -> _m.Parameters:
    """The slab's own Parameters: local size, local node types, periodic z faces."""
    p = copy.copy(params)
    nzl2, ny, nx = mask_local.shape
    p.n = [nx, ny, nzl2]
    p.node_types = _m.NodeTypes.FromArray(mask_local.ravel())
    p.boundary_conditions = [(f, _m.Periodic if f in (BoundaryFace.Bottom, BoundaryFace.Top) else bc)
                             for f, bc in params.boundary_conditions]
    for attr, name in (("initial_density", "density"), ("initial_velocity", "velocity")):
        if getattr(params, attr).kind != "uniform":
            raise NotImplementedError(f"z slabs take a uniform initial {name}")
    return p


class TorchExchange:
    """Halo exchange over torch.distributed: NCCL (CUDA tensors, grouped send/recv)
    or gloo (CPU tensors)."""

    def __init__(self, rank: int, nranks: int, periodic: bool, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.down, self.up = neighbours(rank, nranks, periodic)
        self.grouped = dist.get_backend(group) == "nccl"

    def __call__(self, send_lo, send_hi, recv_lo, recv_hi) -> None:
        dist = self.dist
        plan = []
        if self.down is not None:
            plan.append((dist.isend, send_lo, self.down))
        if self.up is not None:
            plan.append((dist.isend, send_hi, self.up))
        if self.up is not None:
            plan.append((dist.irecv, recv_hi, self.up))
        if self.down is not None:
            plan.append((dist.irecv, recv_lo, self.down))
        if not plan:
            return
        if self.grouped:
            ops = [dist.P2POp(op, t, peer, self.group) for op, t, peer in plan]
            reqs = dist.batch_isend_irecv(ops)
        else:
            reqs = [op(t, peer, group=self.group) for op, t, peer in plan]
        for r in reqs:
            r.wait()


def exchange_masks(own: np.ndarray, exchange) -> Tuple[Optional[np.ndarray], Optional[np.ndarray]]:
    """Neighbour boundary planes of the node types (bottom plane goes down, top goes up)."""
    import torch
    dev = "cuda" if getattr(exchange, "grouped", False) else "cpu"
    lo = torch.from_numpy(np.ascontiguousarray(own[0])).to(dev)
    hi = torch.from_numpy(np.ascontiguousarray(own[-1])).to(dev)
    rlo, rhi = torch.empty_like(lo), torch.empty_like(hi)
    exchange(lo, hi, rlo, rhi)
    below = rlo.cpu().numpy() if exchange.down is not None else None
    above = rhi.cpu().numpy() if exchange.up is not None else None
    return below, above


class SlabDomain:
    """One rank's z-slab of a global lattice, stepped with its halo exchange.

    `own_mask` (nz_loc, ny, nx) gives this rank's node types; when None they are
    sliced from `params.node_types` of the whole lattice.  `exchange(send_lo,
    send_hi, recv_lo, recv_hi)` moves the halo buffers (TorchExchange for one
    process per GPU)."""

    def __init__(self, params: _m.Parameters, rank: int, nranks: int, exchange, own_mask=None, stream=None):
        import torch
        from .domain import Domain
        if VelocitySet(params.velocity_set).d != 3:
            raise ValueError("z slabs need a 3-D velocity set")
        self.periodic = z_periodic(params)
        if not self.periodic:
            # solid ghost planes act as no-slip walls applied before the other faces'
            # rules; that matches the reference only when the x and y faces are
            # periodic or no-slip too (their rules then commute with it)
            for f, bc in params.boundary_conditions:
                if bc.kind not in (_abi.LBF_BC_PERIODIC, _abi.LBF_BC_NO_SLIP):
                    raise ValueError("z walls in a z-slab decomposition need periodic or no-slip x and y faces")
        nx, ny, nz = params.n[:3]
        self.z0, self.z1 = slab_bounds(nz, nranks, rank)
        self.nzl = self.z1 - self.z0
        if self.nzl < 1:
            raise ValueError("more ranks than z planes")
        self.rank, self.nranks, self.exchange = rank, nranks, exchange
        if own_mask is None:
            full = params.node_types.generate(params.n[:3])
            full = np.zeros(nx * ny * nz, np.uint8) if full is None else np.asarray(full, np.uint8)
            full = full.reshape(nz, ny, nx)
            own = full[self.z0:self.z1]
            down, up = neighbours(rank, nranks, self.periodic)
            below = full[(self.z0 - 1) % nz] if down is not None else None
            above = full[self.z1 % nz] if up is not None else None
        else:
            own = np.asarray(own_mask, np.uint8).reshape(self.nzl, ny, nx)
            below, above = exchange_masks(own, exchange)
        self.mask = local_mask(own, below, above)
        self.params = local_parameters(params, self.mask)
        self.stream = stream
        self.dom = Domain(self.params)
        self.dom.set_option(_abi.LBF_OPT_Z_BEGIN, 1).set_option(_abi.LBF_OPT_Z_END, self.nzl + 1)
        # local plane 1 is global plane z0: nodes round (16-bit storage) as in the whole lattice
        self.dom.set_option(_abi.LBF_OPT_SEED_OFFSET, (self.z0 - 1) * nx * ny)
        nd, plane, nbytes = C.c_int32(), C.c_int64(), C.c_int64()
        _abi.check(self.dom.lib.lbf_domain_halo_info(self.dom.h, C.byref(nd), C.byref(plane), C.byref(nbytes)))
        self.halo_bytes = nbytes.value
        self.bufs = [torch.empty(self.halo_bytes, dtype=torch.uint8, device="cuda") for _ in range(4)]
        self.n_fluid_own = int(np.count_nonzero(own == 0))

    def _s(self):
        import torch
        return self.stream if self.stream is not None else torch.cuda.current_stream()

    def init(self) -> "SlabDomain":
        self.dom.init(self._s())
        return self

    def halo(self, stream=None) -> None:
        """Pack, exchange and unpack the halos on `stream` (default: the domain's)."""
        import torch
        st = stream if stream is not None else self._s()
        lib, h, s = self.dom.lib, self.dom.h, st.cuda_stream
        send_lo, send_hi, recv_lo, recv_hi = self.bufs
        _abi.check(lib.lbf_domain_halo_pack(h, _abi.LBF_BOTTOM, C.c_void_p(send_lo.data_ptr()), C.c_void_p(s)))
        _abi.check(lib.lbf_domain_halo_pack(h, _abi.LBF_TOP, C.c_void_p(send_hi.data_ptr()), C.c_void_p(s)))
        with torch.cuda.stream(st):   # the collective orders itself after the packs on this stream
            self.exchange(send_lo, send_hi, recv_lo, recv_hi)
        if self.exchange.down is not None:
            _abi.check(lib.lbf_domain_halo_unpack(h, _abi.LBF_BOTTOM, C.c_void_p(recv_lo.data_ptr()), C.c_void_p(s)))
        if self.exchange.up is not None:
            _abi.check(lib.lbf_domain_halo_unpack(h, _abi.LBF_TOP, C.c_void_p(recv_hi.data_ptr()), C.c_void_p(s)))

    def step(self, n: int = 1, residual_interval: int = 0, overlap: bool = True) -> "SlabDomain":
        """n steps with halo exchanges.  overlap: each step runs in two parts
        (lbf_domain_step_part): the boundary planes, then the interior planes on the
        domain's stream while the halos are packed, exchanged and unpacked on a
        second stream; the next step waits for the unpacks."""
        import torch
        if not overlap or self.nzl < 3:
            for _ in range(n):
                self.dom.step(1, residual_interval, self._s())
                self.halo()
            return self
        s = self._s()
        if not hasattr(self, "_comm"):
            self._comm = torch.cuda.Stream()
        c = self._comm
        lib, h = self.dom.lib, self.dom.h
        for _ in range(n):
            _abi.check(lib.lbf_domain_step_part(h, 0, residual_interval, C.c_void_p(s.cuda_stream)))
            c.wait_stream(s)
            self.halo(c)
            _abi.check(lib.lbf_domain_step_part(h, 1, residual_interval, C.c_void_p(s.cuda_stream)))
            s.wait_stream(c)
        return self

    @property
    def time_step(self) -> int:
        return self.dom.time_step

    def moments(self):
        """(density, velocity) of the owned planes, in global node order of the slab."""
        rho, u, _ = self.dom.moments(self._s())
        pl = self.params.n[0] * self.params.n[1]
        return rho[pl:pl * (self.nzl + 1)], u[pl:pl * (self.nzl + 1)]

    def close(self):
        self.dom.close()
