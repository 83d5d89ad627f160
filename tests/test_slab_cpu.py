"""The z-slab decomposition on the CPU: world size 2 and 3 over gloo, each rank a
separate process stepping its slab with the oracle and exchanging halos with
lbflow_b200.slab.TorchExchange.  The owned planes must equal the same planes of
the whole lattice stepped by the oracle in one piece (identical arithmetic per
node, so the bound is 1e-14 relative).

Covers: slab bounds with uneven splits, ghost planes of no-slip z walls (solid)
and of a periodic z axis (wrap, including world size 2 where both neighbours
are the same rank), leaving / entering direction sets of D3Q19 and D3Q27, and the
send / receive ordering of the exchange.
"""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "helpers"))


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return str(s.getsockname()[1])


@pytest.mark.parametrize("name,world", [("walls", 2), ("walls", 3), ("periodic", 2), ("periodic", 3), ("d3q27", 2)])
def test_slabs_match_whole_lattice(tmp_path, name, world):
    from lbflow_b200 import momentum as m
    from oracle import oracle as orc
    from slab_cases import case
    steps = 40
    port = _port()
    env = dict(os.environ, OMP_NUM_THREADS="1")
    procs = [subprocess.Popen([sys.executable, os.path.join(HERE, "helpers", "slab_worker.py"), str(r), str(world),
                               port, name, str(steps), str(tmp_path / f"r{r}.npz")], env=env)
             for r in range(world)]
    try:
        for pr in procs:
            assert pr.wait(timeout=240) == 0
    finally:
        for pr in procs:
            if pr.poll() is None:
                pr.kill()
    p = case(name)
    desc, keep = m.to_desc(p)
    od = orc.Domain(desc, keep=keep).init().step(steps)
    rho, u, _ = od.observe()
    plane = p.n[0] * p.n[1]
    covered = 0
    for r in range(world):
        d = np.load(tmp_path / f"r{r}.npz")
        z0, z1 = int(d["z0"]), int(d["z1"])
        covered += z1 - z0
        sl = slice(z0 * plane, z1 * plane)
        fl = rho[sl] != 0
        assert np.allclose(d["rho"][fl], rho[sl][fl], rtol=1e-14, atol=0), r
        assert np.allclose(d["u"][fl], u[sl][fl], rtol=1e-12, atol=1e-17), r
    assert covered == p.n[2]
