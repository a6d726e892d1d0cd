"""Generate the long-horizon fixtures tests/golden/long_{cfg0,cfg1}.npz.

The reference's own FP64 step (oracle/_ref/libref_fp64.so, the reference's
sources built by oracle/build_ref.py) runs the seeded 7-cell organoid (cfg0:
256^2, zone_size 65) and the 64-cell organoid (cfg1: 1024^2, zone_size 129)
for 1000 steps on the host.  At the checkpoints 1, 10, 100 and 1000 it stores
per cell: the area s_n, the centroid (xc, yc), the perimeter and the rho mass
(tests/shape.py defines both).  Beside it the C restatement of the step
(oracle/pfag_oracle.c, bit-exact against the reference build) records every
step's reshaping iteration count per cell and the last two rdev values of each
loop.  The two runs of a configuration go in separate processes.  cfg1 takes
about 70 minutes of one host core per run.

    python tests/golden/make_long_golden.py [--only cfg0|cfg1] [--steps 1000]
"""
from __future__ import annotations

import argparse
import math
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

CHECKPOINTS = (1, 10, 100, 1000)


def _ref_worker(name, nsteps, q):
    sys.path.insert(0, ROOT)
    from multicellular_phase_field_active_gel_organoids_b200.params import CONFIGS
    from oracle.refrun import RefLib
    from tests.shape import perimeter, rho_mass
    cfg = CONFIGS[name]()
    p = cfg.params()
    r = RefLib("fp64", p)
    r.load(*cfg.initial_state(np.float64))
    out = {}
    t0 = time.time()
    for k in range(nsteps):
        r.step(k)
        if k + 1 in CHECKPOINTS or k + 1 == nsteps:
            st = r.state()
            c = k + 1
            out[f"s_{c}"] = st["s"]
            out[f"xc_{c}"] = st["xc"]
            out[f"yc_{c}"] = st["yc"]
            out[f"perimeter_{c}"] = perimeter(st["phi"], float(p["dx"]))
            out[f"rho_mass_{c}"] = rho_mass(st["rho"], float(p["dx"]))
            print(f"{name} reference step {c}: {time.time() - t0:.0f} s", flush=True)
    out["reference_seconds"] = np.array(time.time() - t0)
    q.put(("ref", out))


def _port_worker(name, nsteps, q):
    sys.path.insert(0, ROOT)
    from multicellular_phase_field_active_gel_organoids_b200.params import CONFIGS
    from oracle.port import Port
    cfg = CONFIGS[name]()
    p = cfg.params()
    port = Port(p, 64)
    port.load(*cfg.initial_state(np.float64))
    iters = np.zeros((nsteps, port.ncells), np.int32)
    trace = np.zeros((nsteps, port.ncells, 2))
    for k in range(nsteps):
        port.step(k)
        iters[k] = port.cell_iters()
        trace[k] = port.rdev_trace()
    port.close()
    q.put(("port", {"cell_iters": iters, "rdev_trace": trace}))


def make(name: str, nsteps: int):
    from multicellular_phase_field_active_gel_organoids_b200.params import CONFIGS
    p = CONFIGS[name]().params()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=w, args=(name, nsteps, q)) for w in (_ref_worker, _port_worker)]
    for pr in procs:
        pr.start()
    got = {}
    for _ in procs:
        kind, val = q.get()
        got[kind] = val
    for pr in procs:
        pr.join()
    thr = float(p["rtol"]) * 2.0 * math.pi * float(p["R"]) * float(p["wi"]) * float(p["rdt"])
    out = dict(got["ref"])
    out.update(got["port"])
    out["steps"] = np.array(nsteps)
    out["reshaping_threshold"] = np.array(thr)
    path = os.path.join(HERE, f"long_{name}.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=("cfg0", "cfg1"))
    ap.add_argument("--steps", type=int, default=1000)
    a = ap.parse_args()
    names = [a.only] if a.only else ["cfg0", "cfg1"]
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=make, args=(n, a.steps)) for n in names]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join()


if __name__ == "__main__":
    main()
