"""Long-horizon parity report (run on a GPU box; writes one JSON file).

Part 1, the 7-cell organoid (256^2, zone_size 65): the reference's own FP64
step (oracle/_ref/libref_fp64.so, on the host) against the plain FP64 GPU
path, the fused FP64 path and the fused FP32 path, after 1, 10, 100 and
--cfg0-steps steps.  Reported per field: relative L-inf over the whole grid
and over the sites where the reference's |phi_n| > 1e-6 (phi underflows to a
staircase of multiples of 2^-54 far from a cell, where the reference's own
branches |grad phi| > 0 decide; there the GPU and host builds may round
differently), per-cell areas (relative), centroids (exact match) and the
velocity of the last step.  Beside it, the C restatement of the step
(oracle/pfag_oracle.c, bit-exact against the reference build) runs the same
steps on the host and records every step's reshaping iteration count per
cell and the last two rdev values of each loop; the report gives the first
step at which a GPU path takes a different number of reshaping iterations
than the host, and how far from the loop's threshold the host's rdev was
there (a decision taken within rounding of the threshold).

The plain FP64 path runs twice: with its parallel reductions and with the
serial-order sums (pfag_set_serial_sums: the areas, sum_ecm and the reshaping
checks' rdev sums taken one thread per sum in the reference's host order), to
show how far the first reshaping-count difference moves when the summation
order is the reference's and only the state's rounding differs.

Part 2, the 64-cell organoid (1024^2, zone_size 129): the fused FP32 path
after each of --cfg1-checkpoints steps against the plain FP64 path and, at
the checkpoints tests/golden/long_cfg1.npz holds (the reference's own FP64
run, 1000 steps), against the reference: per-cell area, centroid, perimeter
(sum |grad phi| dx, central differences) and rho mass (sum rho dx^2), as the
largest relative (or absolute, for centroids) difference over cells.  The
plain FP64 path is compared with the reference at those checkpoints too.

    python tests/long_parity.py --out long_parity.json
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from multicellular_phase_field_active_gel_organoids_b200 import capi  # noqa: E402
from multicellular_phase_field_active_gel_organoids_b200.params import CONFIGS  # noqa: E402
from oracle import refrun  # noqa: E402
from tests.shape import perimeter, rho_mass  # noqa: E402


def rel(a, b, mask=None):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if mask is not None:
        a, b = a[mask], b[mask]
    if not b.size:
        return 0.0
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


def field_report(got, ref):
    mask = np.abs(ref["phi"]) > 1e-6
    return {
        "phi": rel(got["phi"], ref["phi"]), "phi_masked": rel(got["phi"], ref["phi"], mask),
        "rho": rel(got["rho"], ref["rho"]), "rho_masked": rel(got["rho"], ref["rho"], mask),
        "lum": rel(got["lum"], ref["lum"]), "ECM": rel(got["ECM"], ref["ECM"]),
        "areas": rel(got["s"], ref["s"]),
        "centres_equal": bool(np.array_equal(got["xc"], ref["xc"]) and np.array_equal(got["yc"], ref["yc"])),
    }


def gpu_state(sim):
    phi, rho, lum, ecm = sim.download()
    xc, yc = sim.centres()
    return {"phi": phi, "rho": rho, "lum": lum, "ECM": ecm, "s": sim.areas()[0], "xc": xc, "yc": yc}


def _port_worker(params, init, nsteps, q):
    try:
        from oracle.port import Port
        port = Port(params, 64)
        port.load(*init)
        iters = np.zeros((nsteps, port.ncells), np.int32)
        trace = np.zeros((nsteps, port.ncells, 2))
        for k in range(nsteps):
            port.step(k)
            iters[k] = port.cell_iters()
            trace[k] = port.rdev_trace()
        port.close()
        q.put(("ok", (iters, trace)))
    except Exception as e:  # pragma: no cover - reported to the parent
        q.put(("err", repr(e)))


def part1(nsteps: int) -> dict:
    cfg = CONFIGS["cfg0"]()
    p = cfg.params()
    init = cfg.initial_state(np.float64)
    checkpoints = sorted({c for c in (1, 10, 100, nsteps) if c <= nsteps})
    # the host restatement (per-step iteration counts) runs beside the reference
    ctx = mp.get_context("spawn")
    pq = ctx.Queue()
    pw = ctx.Process(target=_port_worker, args=(p, init, nsteps, pq))
    pw.start()
    t0 = time.time()
    ref = refrun.run_reference(p, init, nsteps, snapshots=checkpoints[:-1], velocity=True, timeout=7200)
    t_ref = time.time() - t0
    status, val = pq.get(timeout=7200)
    pw.join()
    if status != "ok":
        raise RuntimeError("host restatement failed: " + val)
    host_iters, host_trace = val
    thr = float(p["rtol"]) * 2.0 * math.pi * float(p["R"]) * float(p["wi"]) * float(p["rdt"])
    refs = dict(ref["snapshots"])
    refs[nsteps] = ref
    report = {"config": "cfg0: 256x256, 7 cells R=20, zone_size 65 (box 128)", "steps": nsteps,
              "reference_host_seconds": round(t_ref, 1), "reshaping_threshold": thr, "paths": {}}
    for name, prec, path, serial in (("plain_f64", 64, capi.PATH_PLAIN, False),
                                     ("plain_f64_serial_sums", 64, capi.PATH_PLAIN, True),
                                     ("fused_f64", 64, capi.PATH_FUSED, False),
                                     ("fused_f32", 32, capi.PATH_FUSED, False)):
        dtype = np.float64 if prec == 64 else np.float32
        rows = {}
        iters = np.zeros_like(host_iters)
        t0 = time.time()
        with capi.Simulation(p, prec, path) as sim:
            sim.set_relax_cap(100000)
            if serial:
                sim.set_serial_sums(True)
            sim.upload(*cfg.initial_state(dtype))
            for k in range(nsteps):
                if k == nsteps - 1:
                    sim.set_debug(1)
                sim.step(k, 1)
                iters[k] = sim.cell_iters()
                if k + 1 in checkpoints:
                    rows[str(k + 1)] = field_report(gpu_state(sim), refs[k + 1])
            vx, vy = sim.velocity()
            rvx, rvy = ref["velocity"]
            rows[str(nsteps)]["velocity"] = max(rel(vx, rvx), rel(vy, rvy))
        entry = {"checkpoints": rows, "gpu_seconds": round(time.time() - t0, 2),
                 "reshaping_iterations_host": int(host_iters.sum()), "reshaping_iterations_gpu": int(iters.sum())}
        diff = np.argwhere(iters != host_iters)
        if diff.size:
            k, n = (int(v) for v in diff[0])
            prev, last = host_trace[k, n]
            entry["first_iteration_difference"] = {
                "step": k + 1, "cell": n, "host_iterations": int(host_iters[k, n]), "gpu_iterations": int(iters[k, n]),
                "host_rdev_before_exit_rel_to_threshold": (prev - thr) / thr,
                "host_rdev_at_exit_rel_to_threshold": (last - thr) / thr,
                "steps_with_differences": int(np.unique(diff[:, 0]).size)}
        else:
            entry["first_iteration_difference"] = None
        report["paths"][name] = entry
    return report


def shape_measures(state, dx: float):
    return perimeter(state["phi"], dx), rho_mass(state["rho"], dx)


def compare(a, b, dx):
    """Per-cell differences of state `a` against `b` (the reference side)."""
    pa, ma = shape_measures(a, dx)
    pb, mb = shape_measures(b, dx)
    return {
        "area_rel_max": float(np.max(np.abs(a["s"] - b["s"]) / np.abs(b["s"]))),
        "centroid_max_abs": int(max(np.max(np.abs(a["xc"] - b["xc"])), np.max(np.abs(a["yc"] - b["yc"])))),
        "perimeter_rel_max": float(np.max(np.abs(pa - pb) / np.abs(pb))),
        "rho_mass_rel_max": float(np.max(np.abs(ma - mb) / np.maximum(np.abs(mb), 1e-300))),
    }


def compare_golden(a, gold, c, dx):
    pa, ma = shape_measures(a, dx)
    return {
        "area_rel_max": float(np.max(np.abs(a["s"] - gold[f"s_{c}"]) / np.abs(gold[f"s_{c}"]))),
        "centroid_max_abs": int(max(np.max(np.abs(a["xc"] - gold[f"xc_{c}"])),
                                    np.max(np.abs(a["yc"] - gold[f"yc_{c}"])))),
        "perimeter_rel_max": float(np.max(np.abs(pa - gold[f"perimeter_{c}"]) / np.abs(gold[f"perimeter_{c}"]))),
        "rho_mass_rel_max": float(np.max(np.abs(ma - gold[f"rho_mass_{c}"]) / np.abs(gold[f"rho_mass_{c}"]))),
    }


def part2(checkpoints) -> dict:
    cfg = CONFIGS["cfg1"]()
    p = cfg.params()
    dx = float(p["dx"])
    gpath = os.path.join(ROOT, "tests", "golden", "long_cfg1.npz")
    gold = np.load(gpath) if os.path.exists(gpath) else None
    gsteps = {int(k.split("_")[1]) for k in gold.files if k.startswith("s_")} if gold is not None else set()
    report = {"config": "cfg1: 1024x1024, 64 cells R=24, zone_size 129 (box 256)",
              "reference_checkpoints": sorted(gsteps), "checkpoints": {}}
    sims = {}
    done = 0
    try:
        for name, prec, path in (("plain_f64", 64, capi.PATH_PLAIN), ("fused_f32", 32, capi.PATH_FUSED)):
            s = capi.Simulation(p, prec, path)
            s.set_relax_cap(100000)
            s.upload(*cfg.initial_state(np.float64 if prec == 64 else np.float32))
            sims[name] = s
        for c in checkpoints:
            row = {}
            for name, s in sims.items():
                t0 = time.time()
                s.step(done, c - done)
                row[f"seconds_{name}"] = round(time.time() - t0, 2)
            done = c
            a = gpu_state(sims["plain_f64"])
            b = gpu_state(sims["fused_f32"])
            row["fused_f32_vs_plain_f64"] = compare(b, a, dx)
            row["fused_f32_vs_plain_f64"]["phi_linf"] = float(np.max(np.abs(np.asarray(b["phi"], np.float64)
                                                                             - a["phi"])))
            if c in gsteps:
                row["fused_f32_vs_reference"] = compare_golden(b, gold, c, dx)
                row["plain_f64_vs_reference"] = compare_golden(a, gold, c, dx)
            report["checkpoints"][str(c)] = row
            print(c, row, flush=True)
    except capi.PfagError as e:
        report["stopped"] = f"after {done} steps: {e}"
    finally:
        for s in sims.values():
            s.close()
    return report


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default="long_parity.json")
    ap.add_argument("--cfg0-steps", type=int, default=1000)
    ap.add_argument("--cfg1-checkpoints", default="1000,10000,50000")
    ap.add_argument("--skip-cfg0", action="store_true")
    ap.add_argument("--skip-cfg1", action="store_true")
    a = ap.parse_args()
    out = {}
    if not a.skip_cfg0:
        out["cfg0_vs_reference"] = part1(a.cfg0_steps)
        with open(a.out, "w") as f:
            json.dump(out, f, indent=1)
    if not a.skip_cfg1:
        out["cfg1_f32"] = part2([int(x) for x in a.cfg1_checkpoints.split(",")])
    with open(a.out, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out, indent=1))
    return 0


if __name__ == "__main__":
    sys.exit(main())
