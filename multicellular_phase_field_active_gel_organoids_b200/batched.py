"""Batched uneven sweep: many independent organoids advanced together.

The reference sweeps parameters by writing one folder and one batch job per
member (main_code/setup_simulation.py:206-312); every member is its own
process on its own GPU.  Here every member is a fused-path context on one
GPU, and after two warm-up steps a step of the whole sweep is ONE graph
launch (pfag_batch_*: the members' captured step graphs as child graphs of one
parent graph, no dependencies between members), so the GPU runs small
organoids side by side instead of one after another.

Members of the seeded uneven sweep (`sweep_members`): a grid of 256^2, 512^2
or 1024^2; a cell radius R ~ U(16, 32) (one radius per organoid: the
reference's parameter set has a single R, s0 and zone_size); a cell count
drawn log-uniform in [8, 128] and capped at what a hexagonal lattice of
spacing 2R holds inside the circle where every zone stays on the grid; cells
on that lattice, jittered by U(-3, 3); the active contractility (a_ort, hence
a_tan) and the cortex turnover rates (degradation and generation) times
U(0.5, 2) each.  Box bucketing: the FFT box M = 2 zone_size - 2 is 4R rounded
up to a multiple of 16 (64 .. 128 for R in 16 .. 32; the zone then covers the
cell with a margin of about R), so members share five box sizes and their
kernel instances (64 and 128 on the register FFTs, 80, 96 and 112 on the
Bluestein passes).  The autotuner (`autotune`) picks, per bucket of members
(box size, grid, cell-count class), the launch shapes of the persistent
relaxation kernel and the phi update (pfag_set_launch_shape), then whether the
lumen / ECM relaxation runs on TMA-staged tiles (pfag_set_lumen_tiles), by timing fresh
copies of up to eight of the bucket's members stepped together, and caches the
choice in a JSON file.
"""
from __future__ import annotations

import json
import math
import os
import time
from dataclasses import dataclass

import numpy as np

from . import capi
from .params import OrganoidConfig

GRIDS = (256, 512, 1024)


@dataclass
class Member:
    """One organoid of the sweep."""
    index: int
    N: int
    radius: float
    zone_size: int
    centres: np.ndarray          # (Ntot, 2) grid coordinates
    contract: float              # factor on a_ort (a_tan follows)
    turnover: float              # factor on the degradation and generation rates
    seed: int

    @property
    def ncells(self) -> int:
        return int(self.centres.shape[0])

    @property
    def box(self) -> int:
        return 2 * self.zone_size - 2

    @property
    def sites(self) -> int:
        return self.ncells * self.N * self.N

    def config(self, steps: int = 1000) -> OrganoidConfig:
        base = {}
        from .params import TEMPLATE_DEFAULTS as T
        for k in ("a_ort_apical", "a_ort_basal", "a_ort_lateral"):
            base[k] = T[k] * self.contract
        for k in ("degrate_apical", "degrate_lateral", "matgenrate_apical", "matgenrate_lateral"):
            base[k] = T[k] * self.turnover
        return OrganoidConfig(f"sweep{self.index}", self.N, self.centres, self.radius, self.zone_size,
                              self.seed, steps, overrides=base)

    def bucket(self) -> str:
        cls = "s" if self.ncells <= 16 else ("m" if self.ncells <= 48 else "l")
        return f"M{self.box}_N{self.N}_{cls}"

    def env_radius(self) -> float:
        cc = self.centres.mean(axis=0)
        return float(np.sqrt(((self.centres - cc) ** 2).sum(axis=1)).max() + self.radius + 2.0)


def box_for_radius(radius: float) -> int:
    """The bucketed FFT box of a member: 4R rounded up to a multiple of 16."""
    return int(16 * math.ceil(4.0 * radius / 16.0))


def lattice(N: int, spacing: float, clip: float, ncells: int, rng) -> np.ndarray:
    """The `ncells` points of a hexagonal lattice of the given spacing nearest
    the grid centre within `clip`, jittered by U(-3, 3) (fewer if the circle
    holds fewer)."""
    c = N / 2.0
    kmax = int(clip / spacing) + 2
    pts = []
    for a in range(-kmax, kmax + 1):
        for b in range(-kmax, kmax + 1):
            x = spacing * (a + 0.5 * b)
            y = spacing * (math.sqrt(3.0) / 2.0) * b
            if x * x + y * y <= clip * clip:
                pts.append((x, y))
    pts.sort(key=lambda q: (q[0] ** 2 + q[1] ** 2, q[0], q[1]))
    pts = np.array(pts[:max(1, ncells)], dtype=np.float64) + c
    return pts + rng.uniform(-3.0, 3.0, size=pts.shape)


def sweep_members(n: int = 256, seed: int = 1) -> list[Member]:
    """The seeded uneven sweep (numpy default_rng(seed); draws per member in a
    fixed order: grid, log cell count, radius, contractility, turnover)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        N = int(GRIDS[int(rng.integers(len(GRIDS)))])
        want = int(round(math.exp(rng.uniform(math.log(8.0), math.log(128.0)))))
        R = float(rng.uniform(16.0, 32.0))
        contract = float(rng.uniform(0.5, 2.0))
        turnover = float(rng.uniform(0.5, 2.0))
        M = box_for_radius(R)
        z = M // 2 + 1
        clip = N / 2.0 - z - 6.0          # every zone stays on the grid while cells move a few sites
        centres = lattice(N, 2.0 * R, clip, want, rng)
        out.append(Member(k, N, R, z, centres, contract, turnover, seed * 100003 + k))
    return out


def default_cache_path() -> str:
    root = os.environ.get("PFAG_CACHE_DIR") or os.path.join(os.path.expanduser("~"), ".cache", "pfag")
    return os.path.join(root, "launch_shapes.json")


class BatchedSweep:
    """All members on one GPU (fused path), stepped as one graph per step."""

    def __init__(self, members: list[Member], precision: int = 32, relax_cap: int | None = None,
                 host_init: bool = False):
        """host_init: upload the host generator's fields (OrganoidConfig.initial_state)
        instead of generating them on the device (small members, parity tests)."""
        # members of a bucket next to one another (the autotuner's groups)
        self.members = sorted(members, key=lambda m: (m.bucket(), m.index))
        self.precision = precision
        self.sims = []
        dtype = np.float64 if precision == 64 else np.float32
        try:
            for m in self.members:
                cfg = m.config()
                s = capi.Simulation(cfg.params(), precision, capi.PATH_FUSED)
                self.sims.append(s)
                if relax_cap:
                    s.set_relax_cap(relax_cap)
                if host_init:
                    s.upload(*cfg.initial_state(dtype))
                else:
                    s.seed_organoid(m.centres, m.radius, m.env_radius(), m.seed)
            self.batch = capi.Batch(self.sims)
        except Exception:
            self.close()
            raise

    @property
    def sites(self) -> int:
        return sum(m.sites for m in self.members)

    def buckets(self) -> dict[str, list[int]]:
        out: dict[str, list[int]] = {}
        for i, m in enumerate(self.members):
            out.setdefault(m.bucket(), []).append(i)
        return out

    def set_shapes(self, shapes: dict[str, dict]):
        for key, idx in self.buckets().items():
            sh = shapes.get(key)
            if sh:
                for i in idx:
                    self.sims[i].set_launch_shape(int(sh["coop_blocks"]), int(sh["update_warps"]))
                    if sh.get("lumen_tma"):
                        self.sims[i].set_lumen_tiles(True)

    def step(self, it0: int, nsteps: int = 1):
        self.batch.step(it0, nsteps)

    def step_async(self, it0: int, nsteps: int = 1):
        self.batch.step_async(it0, nsteps)

    def sync(self):
        self.batch.sync()

    def member_sim(self, index: int) -> capi.Simulation:
        """The simulation of the member with the given sweep index."""
        for m, s in zip(self.members, self.sims):
            if m.index == index:
                return s
        raise KeyError(index)

    def close(self):
        b = getattr(self, "batch", None)
        if b is not None:
            b.close()
            self.batch = None
        for s in self.sims:
            s.close()
        self.sims = []

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


# candidate launch shapes: (persistent-kernel block cap, phi-update warp budget); 0 = the default
SHAPES = ((0, 0), (296, 0), (148, 0), (74, 2368), (37, 1184))


def _time_batch(sims, steps: int) -> float:
    """Seconds per step of the given members stepped as one batch (after the
    warm-up steps that capture their graphs)."""
    b = capi.Batch(sims)
    try:
        b.step(0, 3)
        t0 = time.perf_counter()
        b.step(3, steps)
        return (time.perf_counter() - t0) / steps
    finally:
        b.close()


def autotune(members: list[Member], precision: int = 32, cache_path: str | None = None, sample: int = 8,
             steps: int = 4, shapes=SHAPES) -> dict[str, dict]:
    """Per bucket of `members`, the launch shape with the shortest step of
    fresh copies of up to `sample` of its members (generated on the device,
    stepped together, then freed: the sweep's own state is not touched); cached
    in JSON under the bucket key (box size, grid, cell-count class, precision),
    so a later sweep with the same buckets reuses the choice without timing."""
    path = cache_path or default_cache_path()
    try:
        with open(path) as f:
            cache = json.load(f)
    except (OSError, ValueError):
        cache = {}
    groups: dict[str, list[Member]] = {}
    for m in sorted(members, key=lambda m: (m.bucket(), m.index)):
        groups.setdefault(m.bucket(), []).append(m)
    chosen = {}
    for key, ms in groups.items():
        ckey = f"{key}_fp{precision}"
        if ckey not in cache:
            trial = BatchedSweep(ms[:sample], precision)
            try:
                best = None
                for coop, upd in shapes:
                    for sim in trial.sims:
                        sim.set_launch_shape(coop, upd)
                    t = _time_batch(trial.sims, steps)
                    if best is None or t < best[0]:
                        best = (t, coop, upd)
                # the lumen / ECM relaxation on TMA-staged tiles, at the best shape
                tma = 0
                try:
                    for sim in trial.sims:
                        sim.set_launch_shape(best[1], best[2])
                        sim.set_lumen_tiles(True)
                except capi.PfagError:
                    pass                       # not available for this bucket (FP64, small grid)
                else:
                    t = _time_batch(trial.sims, steps)
                    if t < best[0]:
                        best, tma = (t, best[1], best[2]), 1
            finally:
                trial.close()
            cache[ckey] = {"coop_blocks": best[1], "update_warps": best[2], "lumen_tma": tma,
                           "ms_per_step": round(best[0] * 1e3, 4), "members_timed": min(sample, len(ms))}
        chosen[key] = cache[ckey]
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    with open(path, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    return chosen
