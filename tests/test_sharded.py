"""Cell sharding's host logic on CPU: the cell ranges, and the exchanges and
step loop of sharded.py over 2 and 3 gloo ranks.  The step loop runs on a
stand-in shard whose head and tail are a small model coupled the way the
organoid's cells are (a sum over all cells, the cyclic index neighbours);
the sharded run must equal one rank holding every cell."""
import os
import socket
import subprocess
import sys

import pytest

from multicellular_phase_field_active_gel_organoids_b200.sharded import shard_bounds, shard_params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_shard_bounds():
    for ntot in (1, 2, 3, 7, 64, 65):
        for k in range(1, min(ntot, 9) + 1):
            b = shard_bounds(ntot, k)
            assert len(b) == k and b[0][0] == 0 and b[-1][1] == ntot
            assert all(b[i][1] == b[i + 1][0] for i in range(k - 1))
            sizes = [c1 - c0 for c0, c1 in b]
            assert min(sizes) >= 1 and max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)
    with pytest.raises(ValueError):
        shard_bounds(3, 4)
    with pytest.raises(ValueError):
        shard_bounds(3, 0)


def test_shard_params_keep_organoid_count():
    p = shard_params({"Ntot": 64, "N_current": 64, "dx": 1.0}, 16, 32)
    assert p["Ntot"] == 16 and p["N_current"] == 64 and p["dx"] == 1.0


CHILD = r"""
import os, sys
sys.path.insert(0, {root!r})
import torch
import torch.distributed as dist
from multicellular_phase_field_active_gel_organoids_b200.sharded import DistExchange, run_steps, shard_bounds

NTOT, P = {ntot}, 16
dist.init_process_group("gloo", init_method="env://", timeout=__import__("datetime").timedelta(seconds=60))
ex = DistExchange()
r, w = ex.rank, ex.world

# exchanges: planes tagged by their owner's cell index
first = torch.full((P,), 100.0 + r, dtype=torch.float64)
last = torch.full((P,), 200.0 + r, dtype=torch.float64)
lo = torch.zeros(P, dtype=torch.float64); hi = torch.zeros(P, dtype=torch.float64)
ex.halo(first, last, lo, hi)
assert torch.all(lo == 200.0 + (r - 1) % w) and torch.all(hi == 100.0 + (r + 1) % w), (r, lo[0], hi[0])
psi = torch.arange(P, dtype=torch.float64) * (r + 1)
ex.psi(psi)
assert torch.equal(psi, torch.arange(P, dtype=torch.float64) * sum(k + 1 for k in range(w)))

def init_cells():
    g = torch.Generator().manual_seed(5)
    return torch.rand((NTOT, P), generator=g, dtype=torch.float64)

class Shard:
    # cells c0..c1 of the stand-in model: head = the shard's partial sum of
    # x^2 in cell order; tail = each cell moved by psi and its cyclic index
    # neighbours (from lo / hi at the range ends)
    def __init__(self, c0, c1):
        self.x = init_cells()[c0:c1].clone()
        self.first, self.last = self.x[0], self.x[-1]
        self.lo = torch.zeros(P, dtype=torch.float64); self.hi = torch.zeros(P, dtype=torch.float64)
        self.psi_t = torch.zeros(P, dtype=torch.float64)
        self.steps = []
    def head(self, it):
        acc = torch.zeros(P, dtype=torch.float64)
        for c in range(self.x.shape[0]):
            acc = acc + self.x[c] * self.x[c]
        self.psi_t.copy_(acc)
    def tail(self, it):
        n = self.x.shape[0]
        old = self.x.clone()
        for c in range(n):
            a = self.lo if c == 0 else old[c - 1]
            b = self.hi if c == n - 1 else old[c + 1]
            self.x[c] = old[c] + 0.01 * (self.psi_t - old[c]) + 0.1 * (a - 2 * old[c] + b) + 1e-3 * it
        self.steps.append(it)

c0, c1 = shard_bounds(NTOT, w)[r]
sh = Shard(c0, c1)
run_steps(ex, sh, 3, 6)
assert sh.steps == [3, 4, 5, 6, 7, 8]
parts = [None] * w
dist.all_gather_object(parts, sh.x)
full = torch.cat(parts)

class Solo:
    def __init__(self):
        self.world, self.rank = 1, 0
    def halo(self, first, last, lo, hi):
        lo.copy_(last); hi.copy_(first)
    def psi(self, t):
        pass
ref = Shard(0, NTOT)
run_steps(Solo(), ref, 3, 6)
err = float((full - ref.x).abs().max() / ref.x.abs().max())
assert err < 1e-13, err
dist.destroy_process_group()
print("RESULT", r, w, err)
"""


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("world,ntot", [(2, 5), (3, 7), (3, 3)])
def test_gloo_sharded_steps_equal_one_rank(world, ntot):
    port = _free_port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD.format(root=ROOT, ntot=ntot)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=240) for p in procs]
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, e[-3000:]
    res = sorted(l.split()[1:3] for o, _ in outs for l in o.splitlines() if l.startswith("RESULT"))
    assert res == [[str(r), str(world)] for r in range(world)]
