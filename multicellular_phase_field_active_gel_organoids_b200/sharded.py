"""Cell sharding: one organoid's cells split by contiguous ranges over
fused-path contexts, one per GPU under torch.distributed (DistShard) or
several in one process on one GPU (LocalShards).

Cells couple only through psi = sum_n h(phi_n) (compute_psi_kernels,
useful_functions.cpp:305-322) and the index neighbours' phi that the class
map reads (create_turnover_rates_tensions, rho_functions.cpp:297-311, cyclic
over the organoid: cell 0's n1 is cell Ntot-1).  One step of a shard:
  1. halo: the neighbour planes (pfag_shard_enable) receive phi of the cell
     before the shard's first cell (from the previous shard) and of the cell
     after its last cell (from the next shard), as they stand at the start
     of the step;
  2. pfag_step_head: centroids, h(phi), the shard's partial psi;
  3. psi completed: the sum of the shards' partials, the same values on
     every shard (an all-reduce);
  4. pfag_step_tail: the rest of the step; lum and ECM are updated on every
     shard from the same psi, so they stay identical across shards.
psi is summed per shard in cell order and then over shards, so it differs
from the reference's single running sum over all cells by rounding only.
"""
from __future__ import annotations

import numpy as np

from . import capi


def shard_bounds(ntot: int, nshards: int) -> list[tuple[int, int]]:
    """Contiguous cell ranges [c0, c1), sizes differing by at most one, the
    larger ones first; every shard holds at least one cell."""
    if not 1 <= nshards <= ntot:
        raise ValueError(f"{nshards} shards for {ntot} cells: every shard needs a cell")
    q, r = divmod(ntot, nshards)
    out, c0 = [], 0
    for k in range(nshards):
        c1 = c0 + q + (1 if k < r else 0)
        out.append((c0, c1))
        c0 = c1
    return out


def shard_params(params: dict, c0: int, c1: int) -> dict:
    """A shard's parameter set: the organoid's, with Ntot = its cell count
    (N_current, which scales the reshaping deviation, stays the organoid's)."""
    p = dict(params)
    p["Ntot"] = int(c1 - c0)
    p["N_current"] = int(params["N_current"])
    return p


class _DeviceArray:
    """A context's device array seen through the CUDA array interface (no copy)."""

    def __init__(self, ptr: int, count: int, dtype):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": np.dtype(dtype).str,
                                         "data": (int(ptr), False), "version": 3, "strides": None}


class DistExchange:
    """The two exchanges of a sharded step over a torch.distributed group
    (NCCL between GPUs; gloo on the host in the tests).  Tensors are flat
    planes of the shard's precision."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def _peer(self, k: int) -> int:
        """Global rank of the group's k-th member (cyclic)."""
        k %= self.world
        return k if self.group is None else self.dist.get_global_rank(self.group, k)

    def halo(self, first, last, lo, hi) -> None:
        """lo <- `last` of the previous shard, hi <- `first` of the next one
        (cyclic; with one shard its own planes).  Two rounds of one send and
        one receive each, so messages between the same pair of ranks never
        need ordering."""
        if self.world == 1:
            lo.copy_(last)
            hi.copy_(first)
            return
        d = self.dist
        prev, nxt = self._peer(self.rank - 1), self._peer(self.rank + 1)
        for send, to, recv, frm, tag in ((last, nxt, lo, prev, 1), (first, prev, hi, nxt, 2)):
            ops = [d.P2POp(d.isend, send, to, self.group, tag), d.P2POp(d.irecv, recv, frm, self.group, tag)]
            for w in d.batch_isend_irecv(ops):
                w.wait()

    def psi(self, psi) -> None:
        """psi <- the sum of every shard's partial psi (in place)."""
        if self.world > 1:
            self.dist.all_reduce(psi, op=self.dist.ReduceOp.SUM, group=self.group)


def run_steps(ex, shard, it0: int, nsteps: int) -> None:
    """The sharded step loop: halo, head, psi, tail per step.  `shard` has
    the planes `first`, `last` (phi of its first and last cell), `lo`, `hi`
    (its neighbour planes), `psi_t` (its psi) and head(it) / tail(it)."""
    for k in range(nsteps):
        ex.halo(shard.first, shard.last, shard.lo, shard.hi)
        shard.head(it0 + k)
        ex.psi(shard.psi_t)
        shard.tail(it0 + k)


class DistShard:
    """This rank's shard of one organoid (fused path, the current CUDA
    device); the exchanges go through `exchange` (a DistExchange by default).
    `init` = the organoid's (phi, rho, lum, ECM); each rank uploads its cells."""

    def __init__(self, params: dict, init, precision: int = 32, exchange: DistExchange | None = None,
                 relax_cap: int | None = None):
        import torch
        self.torch = torch
        self.ex = exchange or DistExchange()
        ntot = int(params["Ntot"])
        self.bounds = shard_bounds(ntot, self.ex.world)
        self.c0, self.c1 = self.bounds[self.ex.rank]
        self.sim = capi.Simulation(shard_params(params, self.c0, self.c1), precision, capi.PATH_FUSED)
        if relax_cap:
            self.sim.set_relax_cap(relax_cap)
        phi, rho, lum, ecm = init
        dt = self.sim.dtype
        self.sim.upload(*(np.ascontiguousarray(a, dtype=dt) for a in (phi[self.c0:self.c1], rho[self.c0:self.c1],
                                                                        lum, ecm)))
        lo, hi = self.sim.shard_enable()
        N = self.sim.N
        plane = N * N
        w = np.dtype(dt).itemsize
        phi_p, _ = self.sim.device_field("phi")
        psi_p, _ = self.sim.device_field("psi")
        n = self.c1 - self.c0

        def view(ptr):
            return torch.as_tensor(_DeviceArray(ptr, plane, dt), device="cuda")
        self.first, self.last = view(phi_p), view(phi_p + (n - 1) * plane * w)
        self.lo, self.hi, self.psi_t = view(lo), view(hi), view(psi_p)
        self.stream = torch.cuda.ExternalStream(self.sim.stream())

    def head(self, it: int) -> None:
        self.sim.step_head(it)

    def tail(self, it: int) -> None:
        self.sim.step_tail(it)

    def step_async(self, it0: int, nsteps: int = 1) -> None:
        """Enqueue nsteps steps; the exchanges run on the context's stream."""
        with self.torch.cuda.stream(self.stream):
            run_steps(self.ex, self, it0, nsteps)

    def step(self, it0: int, nsteps: int = 1) -> None:
        self.step_async(it0, nsteps)
        self.sim.sync()

    def close(self):
        self.sim.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class LocalShards:
    """An organoid's cells split over `nshards` fused-path contexts in this
    process on the current GPU, exchanging by device copies (pfag_sum_planes)
    between the parts of each step: the sharded step on one GPU, e.g. to
    check it against the unsharded one."""

    def __init__(self, params: dict, init, nshards: int, precision: int = 64, relax_cap: int | None = None):
        ntot = int(params["Ntot"])
        self.bounds = shard_bounds(ntot, nshards)
        self.precision = precision
        self.sims = []
        try:
            phi, rho, lum, ecm = init
            for c0, c1 in self.bounds:
                s = capi.Simulation(shard_params(params, c0, c1), precision, capi.PATH_FUSED)
                self.sims.append(s)
                if relax_cap:
                    s.set_relax_cap(relax_cap)
                s.upload(*(np.ascontiguousarray(a, dtype=s.dtype) for a in (phi[c0:c1], rho[c0:c1], lum, ecm)))
            self.nb = [s.shard_enable() for s in self.sims]
        except Exception:
            self.close()
            raise
        s0 = self.sims[0]
        self.plane = s0.N * s0.N
        self.w = np.dtype(s0.dtype).itemsize

    def _phi_plane(self, k: int, cell: int) -> int:
        p, _ = self.sims[k].device_field("phi")
        return p + cell * self.plane * self.w

    def _halo(self) -> None:
        K = len(self.sims)
        for k, s in enumerate(self.sims):
            lo, hi = self.nb[k]
            prev, nxt = (k - 1) % K, (k + 1) % K
            last_prev = self._phi_plane(prev, self.sims[prev].ncells - 1)
            first_next = self._phi_plane(nxt, 0)
            capi.sum_planes(lo, [last_prev], self.plane, self.precision, s.stream())
            capi.sum_planes(hi, [first_next], self.plane, self.precision, s.stream())
        for s in self.sims:
            s.sync()

    def _psi(self) -> None:
        psis = [s.device_field("psi")[0] for s in self.sims]
        st = self.sims[0].stream()
        capi.sum_planes(psis[0], psis, self.plane, self.precision, st)      # in shard order
        for p in psis[1:]:
            capi.sum_planes(p, [psis[0]], self.plane, self.precision, st)
        self.sims[0].sync()

    def step(self, it0: int, nsteps: int = 1) -> None:
        for k in range(nsteps):
            self._halo()
            for s in self.sims:
                s.step_head(it0 + k)
            for s in self.sims:
                s.sync()
            self._psi()
            for s in self.sims:
                s.step_tail(it0 + k)
        for s in self.sims:
            s.sync()

    def download(self):
        """The organoid's (phi, rho, lum, ECM); lum and ECM from shard 0."""
        parts = [s.download() for s in self.sims]
        return (np.concatenate([p[0] for p in parts]), np.concatenate([p[1] for p in parts]),
                parts[0][2], parts[0][3])

    def fields(self, k: int):
        """Shard k's own (phi, rho, lum, ECM)."""
        return self.sims[k].download()

    def areas(self) -> np.ndarray:
        return np.concatenate([s.areas()[0] for s in self.sims])

    def centres(self):
        c = [s.centres() for s in self.sims]
        return np.concatenate([a for a, _ in c]), np.concatenate([b for _, b in c])

    def cell_iters(self) -> int:
        return sum(s.stats()["cell_iters_sum"] for s in self.sims)

    def close(self):
        for s in self.sims:
            s.close()
        self.sims = []

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
