"""The multi-rank plumbing of bench.py (barrier, max and sum over ranks) on
world size 2 with the gloo backend on CPU."""
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import os, sys
sys.path.insert(0, {root!r})
import bench
ws, rank, local = bench.dist_info()
d = bench.Dist(ws, rank, local, "gloo")
d.barrier()
m = d.max(float(rank + 1) * 1.5)
s = d.sum(float(rank + 1))
d.close()
print("RESULT", rank, m, s)
"""


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_ranks_reduce():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD.format(root=ROOT)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=180) for p in procs]
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, e[-2000:]
    res = sorted(l.split()[1:] for o, _ in outs for l in o.splitlines() if l.startswith("RESULT"))
    assert res == [["0", "3.0", "3.0"], ["1", "3.0", "3.0"]]
