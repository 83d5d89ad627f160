"""One rank of the z-slab decomposition on the CPU (gloo), with the oracle as the
slab stepper.  Run by tests/test_slab_cpu.py as a separate process per rank:

    python tests/helpers/slab_worker.py RANK WORLD PORT CASE STEPS OUT.npz

The rank builds its slab exactly as lbflow_b200.slab does (slab_bounds,
neighbours, local_mask, local_parameters, leaving directions) and runs each
reference main_steps pass by pass: moments, equilibrium, collision; then the
halo exchange over gloo (TorchExchange) of the post-collision populations that
leave the owned boundary planes into the neighbours' ghost planes; then
streaming, inner bounce-back and face BCs.  It writes its owned planes'
density and velocity to OUT.npz.
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402
import torch  # noqa: E402
import torch.distributed as dist  # noqa: E402

from lbflow_b200 import momentum as m, slab  # noqa: E402
from lbflow_b200.core import BoundaryFace  # noqa: E402
from oracle import oracle as orc  # noqa: E402

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from slab_cases import case  # noqa: E402


def main():
    rank, world, port, name, steps, out = (int(sys.argv[1]), int(sys.argv[2]), sys.argv[3], sys.argv[4],
                                          int(sys.argv[5]), sys.argv[6])
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    orc.set_threads(1)
    p = case(name)
    nx, ny, nz = p.n
    periodic = slab.z_periodic(p)
    full = np.asarray(p.node_types.generate(p.n), np.uint8).reshape(nz, ny, nx)
    z0, z1 = slab.slab_bounds(nz, world, rank)
    down, up = slab.neighbours(rank, world, periodic)
    below = full[(z0 - 1) % nz] if down is not None else None
    above = full[z1 % nz] if up is not None else None
    lm = slab.local_mask(full[z0:z1], below, above)
    lp = slab.local_parameters(p, lm)
    desc, keep = m.to_desc(lp)
    od = orc.Domain(desc, keep=keep).init()
    q = od.q
    nzl = z1 - z0
    plane = nx * ny
    lo_dirs = slab.leaving_directions(int(p.velocity_set), BoundaryFace.Bottom)   # c_z = -1
    hi_dirs = slab.leaving_directions(int(p.velocity_set), BoundaryFace.Top)      # c_z = +1
    ex = slab.TorchExchange(rank, world, periodic)
    for _ in range(steps):
        for ps in (0, 1, 2):
            od.run_pass(ps)
        fs = od.get("f_star").reshape(nzl + 2, plane, q)
        send_lo = torch.from_numpy(np.ascontiguousarray(fs[1][:, lo_dirs]))
        send_hi = torch.from_numpy(np.ascontiguousarray(fs[nzl][:, hi_dirs]))
        recv_lo, recv_hi = torch.empty_like(send_hi), torch.empty_like(send_lo)
        ex(send_lo, send_hi, recv_lo, recv_hi)
        if down is not None:
            fs[0][:, hi_dirs] = recv_lo.numpy()         # entering from below: c_z = +1
        if up is not None:
            fs[nzl + 1][:, lo_dirs] = recv_hi.numpy()   # entering from above: c_z = -1
        od.set("f_star", fs.ravel())
        for ps in (3, 4, 5):
            od.run_pass(ps)
    rho, u, _ = od.observe()
    np.savez(out, rho=rho[plane:plane * (nzl + 1)], u=u[plane:plane * (nzl + 1)], z0=z0, z1=z1)
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
