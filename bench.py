#!/usr/bin/env python3
"""Benchmark of the organoid time step on B200 (one process per GPU).

Workload: the 1024x1024, 64-cell organoid (zone_size 129, FFT box 256), the
reference's step (main_code/run_with_active_gels.cpp:101-185) advanced by the
fused path.  Metric: site-updates/s = Ntot * N_s^2 cell-grid sites per step,
whole job.  Each GPU advances its own organoid replica (the step shards by
cell only with a psi all-reduce; replicas are what runs here), so scaling is
weak.  Between timed steps L2 is flushed by writing a 256 MiB buffer; each
step is timed with CUDA events on the context's stream.

  python bench.py --gpus N --steps K --warmup W            # this framework
  python bench.py --impl reference --steps K --warmup W    # reference on the host cores
  python bench.py --gpus N --shard                         # one organoid's cells split over the N GPUs
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "site-updates/s/B200 (cells x grid x steps), fast vs plain FP64 at stated error"
UNIT = "site-updates/s"
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", type=int, default=32, choices=[32, 64])
    ap.add_argument("--config", default="cfg1")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-compare", action="store_true")
    ap.add_argument("--members", type=int, default=256, help="cfg3: organoids in the batched sweep")
    ap.add_argument("--no-tune", action="store_true", help="cfg3: default launch shapes (no autotuning)")
    ap.add_argument("--pairs", type=int, default=32, help="cfg4: coarse/fine training pairs")
    ap.add_argument("--lumen-tma", action="store_true",
                    help="run the first lumen/ECM relaxation iterations on TMA-staged tiles (pfag_set_lumen_tiles)")
    ap.add_argument("--shard", action="store_true",
                    help="split one organoid's cells over the ranks (psi all-reduce, neighbour halo): strong scaling")
    return ap.parse_args()


def dist_info():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return ws, rank, local


class Dist:
    """Barrier and max-over-ranks of scalars (torch.distributed only when N > 1)."""

    def __init__(self, ws, rank, local, backend):
        self.ws, self.rank = ws, rank
        self.td = None
        if ws > 1:
            import datetime
            import torch
            import torch.distributed as td
            if backend == "nccl":
                torch.cuda.set_device(local)
            td.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=300))
            self.td, self.torch, self.backend = td, torch, backend

    def barrier(self):
        if self.td:
            self.td.barrier()

    def max(self, x: float) -> float:
        if not self.td:
            return x
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = self.torch.tensor([x], dtype=self.torch.float64, device=dev)
        self.td.all_reduce(t, op=self.td.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.td:
            return x
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = self.torch.tensor([x], dtype=self.torch.float64, device=dev)
        self.td.all_reduce(t, op=self.td.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.td:
            self.td.barrier()
            self.td.destroy_process_group()


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms in the background."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self) -> dict:
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for k, nm in enumerate(names[1:], start=5):
                    if r[k].lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# DRAM bytes (read + write) of one launch of the dominant kernel, from the
# committed ncu captures (dram__bytes_read.sum + dram__bytes_write.sum, one cold
# launch) of the fused FP32 step: (config, kernel) -> (bytes, profile file).
NCU_TRAFFIC = {
    ("cfg1", "kr_boxA"): (97.0e6, "profiles/fused_cfg1_f32_top_kernels.md"),
    ("cfg1", "kr_boxB"): (58.0e6, "profiles/fused_cfg1_f32_top_kernels.md"),
    ("cfg1", "kf_update_rows"): (77.8e6, "profiles/fused_cfg1_f32_top_kernels.md"),
    ("cfg1", "kr_boxC2"): (55.9e6, "profiles/fused_cfg1_f32_top_kernels.md"),
    ("cfg1", "kr_boxD2"): (70.1e6, "profiles/fused_cfg1_f32_top_kernels.md"),
    ("cfg1", "kf_resh_first"): (59.2e6, "profiles/fused_cfg1_f32_top_kernels.md"),
    ("cfg1", "kf_hpsi"): (28.2e6, "profiles/fused_cfg1_f32_top_kernels.md"),
    ("cfg1", "kf_relax_loops"): (19.2e6, "profiles/fused_cfg1_f32_top_kernels.md"),
}


def footprints(cfg, xc, yc):
    """Sites of the union over cells of the FFT boxes and of the zone + ring
    regions (the parts of a shared [N][N] array the box and update passes touch)."""
    N, z, M = cfg.N, cfg.zone_size, cfg.box
    ub = np.zeros((N, N), bool)
    ur = np.zeros((N, N), bool)
    for i, j in zip(np.asarray(xc), np.asarray(yc)):
        ub[max(i - z + 1, 0):i - z + 1 + M, max(j - z + 1, 0):j - z + 1 + M] = True
        ur[max(i - z - 1, 0):i + z + 1, max(j - z - 1, 0):j + z + 1] = True
    return int(ub.sum()), int(ur.sum())


def kernel_bytes(cfg, precision: int, iters: dict, ubox: int, uring: int) -> dict:
    """Algorithmic bytes per launch of the fused kernels: every array element
    the launch must read or write, each counted once per launch.  A per-cell
    array counts over the cells' boxes (box = Ntot M^2 sites), zones
    (zone = Ntot (2z)^2) or zone + ring regions (ring = Ntot (2z+2)^2); a
    neighbour cell's phi read on a cell's box is the same array and is not
    counted again; a shared [N][N] array counts once over the union of the
    regions the launch touches (ubox, uring sites) or over the grid."""
    w = precision // 8
    n, N, z = cfg.ncells, cfg.N, cfg.zone_size
    M, Wz = cfg.box, 2 * z + 2
    box = n * M * M
    zone = n * (2 * z) * (2 * z)
    ring = n * Wz * Wz
    lum_it = max(iters.get("lum_iters", 1), 1)
    ecm_it = max(iters.get("ecm_iters", 1), 1)
    cell_it = max(iters.get("cell_iters_sum", n), n)
    out = {
        # reads phi, rho (per cell), lum, ECM (shared); writes pi_xx + i pi_yy, pi_xy (complex),
        # R and the class byte
        "kr_boxA": box * (2 * w + 2 * w + 2 * w + w + 1) + ubox * 2 * w,
        # reads the two row spectra (pi_xy's primary columns only: half of it) and the class map;
        # writes the packed velocity spectrum
        "kr_boxB": box * (2 * w + w + 1 + 2 * w),
        # reads the velocity spectrum and rho; writes Fx and the row term
        "kr_boxC2": box * (2 * w + w + 2 * w),
        # reads Fx, the row term, rho, R; writes rho in place
        "kr_boxD2": box * 5 * w,
        # reads phi, rho, hfunc (per cell), psi and the coupling term G (shared); writes phin, J_x, J_y
        "kf_update_rows": ring * 6 * w + uring * 2 * w,
        # reads phi, rho, hfunc (per cell), psi, h(lum), h(ECM) (shared); writes phin, J_x, J_y
        "kf_update_tiled": ring * 6 * w + uring * 3 * w,
        # FP32: reads h(lum), h(ECM), writes G
        "kf_gel_coupling": N * N * 3 * w,
        # reshaping iteration 1: read P and J (x, y), write Q and phi (P), over every zone
        "kf_resh_first": zone * 5 * w,
        # per launch: further reshaping iterations (read P, J_x, J_y, write Q, phi), the next
        # step's centroid sums (read phi over B_n, about a zone) and lumen / ECM iterations
        # beyond the second (read P, J_x, J_y, write Q)
        "kf_relax_loops": ((2 * z) * (2 * z) * 5 * w * (cell_it - n) + zone * w +
                           N * N * 4 * w * (max(lum_it - 2, 0) + max(ecm_it - 2, 0))),
        # reads phi on the zones (hfunc elsewhere in B_n), lum, ECM; writes hfunc (zones), psi, h(lum), h(ECM)
        "kf_hpsi": N * N * (2 * w + 3 * w) + zone * 2 * w,
        # read lum, ECM, psi, h(lum), h(ECM); write lumn, ECMn
        "kfl_update": N * N * 7 * w,
        # read lum, lumn, ECM, ECMn; write 4 normal components
        "kfl_normals": N * N * 8 * w,
        # per launch (two launches per step): read P, Jx, Jy, write Q per active field
        "kl_relax": N * N * 4 * w * (min(lum_it, 2) + min(ecm_it, 2)) // 2,
        "kl_relax_tma": N * N * 4 * w * (min(lum_it, 2) + min(ecm_it, 2)) // 2,
        # power-of-two boxes of 16, 512 or 1024 (shared-memory radix-4 passes): A as kr_boxA; B reads both
        # row spectra and the class map, writes the velocity spectrum; C reads it and rho, writes the
        # fluxes' spectrum; D transforms it back along the columns; E reads it, rho and R, writes rho
        "kf_boxA": box * (2 * w + 2 * w + 2 * w + w + 1) + ubox * 2 * w,
        "kf_boxB": box * (2 * w + 2 * w + 1 + 2 * w),
        "kf_boxC": box * (2 * w + w + 2 * w),
        "kf_boxD": box * 4 * w,
        "kf_boxE": box * (2 * w + w + w + w),
        # boxes that are not a power of two (Bluestein passes)
        # stresses: reads phi, rho (per cell), lum, ECM (shared); writes Y1 (complex), pi_xy (real), R, class
        "kg_stress": box * (2 * w + 2 * w + w + w + 1) + ubox * 2 * w,
        # rows: reads Y1 (complex) and pi_xy (real); writes Y1 and pi_xy's half spectra
        "kbl_rowsA": box * (2 * w + w + 2 * w + w),
        # columns: Y1 read and written, pi_xy's half spectra read and written
        "kbl_colsB": box * (4 * w + 2 * w),
        # reads both spectra (pi_xy's half) and the class map, writes the velocity spectrum
        "kg_velocity": box * (2 * w + w + 1 + 2 * w),
        # inverse columns: Y1 read and written
        "kbl_colsC": box * 4 * w,
        # inverse rows: reads Y1 and rho; writes Fx and Fy
        "kbl_rowsD1": box * (2 * w + w + 2 * w),
        # row derivative: reads Fy and R; writes dt R + the row term over Fy
        "kbl_rowsD2": box * 3 * w,
        # column derivative: reads Fx, writes it differentiated
        "kbl_colsE": box * 2 * w,
        # the new rho: reads both terms and rho, writes rho
        "kbl_rho": box * 4 * w,
    }
    return out


def step_bytes(cfg, precision: int) -> int:
    """Compulsory state traffic of one step: per cell, phi and rho read and
    written over the zone; the shared psi, lumen and ECM read and written
    (B_step = Ntot Z 4w + N^2 6w, Z = (2 zone_size)^2)."""
    w = precision // 8
    Z = (2 * cfg.zone_size) ** 2
    return cfg.ncells * Z * 4 * w + cfg.N * cfg.N * 6 * w


def run_ours(args, ws, rank, local, dist: Dist):
    from multicellular_phase_field_active_gel_organoids_b200 import capi
    from multicellular_phase_field_active_gel_organoids_b200.params import CONFIGS

    capi.lib()   # loads libpfag.so and, with it, the CUDA runtime the library uses
    rt = ctypes.CDLL("libcudart.so.12")
    if rt.cudaSetDevice(local) != 0:
        raise RuntimeError(f"cudaSetDevice({local}) failed")
    cfg = CONFIGS[args.config]()
    p = cfg.params()
    prec = args.precision
    dtype = np.float64 if prec == 64 else np.float32
    sites = cfg.ncells * cfg.N * cfg.N
    init = cfg.initial_state(dtype)

    # L2 flush buffer and events through the CUDA runtime (no torch on the step path)
    flush = ctypes.c_void_p()
    assert rt.cudaMalloc(ctypes.byref(flush), ctypes.c_size_t(L2_FLUSH_BYTES)) == 0
    rt.cudaEventCreate.argtypes = [ctypes.POINTER(ctypes.c_void_p)]
    rt.cudaEventRecord.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    rt.cudaEventSynchronize.argtypes = [ctypes.c_void_p]
    rt.cudaEventElapsedTime.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.c_void_p, ctypes.c_void_p]
    rt.cudaMemsetAsync.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t, ctypes.c_void_p]
    rt.cudaStreamSynchronize.argtypes = [ctypes.c_void_p]

    sim = capi.Simulation(p, prec, capi.PATH_FUSED)
    if args.lumen_tma:
        sim.set_lumen_tiles(True)
    sim.upload(*init)
    stream = ctypes.c_void_p(sim.stream())
    nev = args.steps
    ev0 = [ctypes.c_void_p() for _ in range(nev)]
    ev1 = [ctypes.c_void_p() for _ in range(nev)]
    for e in ev0 + ev1:
        rt.cudaEventCreate(ctypes.byref(e))
    # warm-up (W >= 3 untimed steps)
    it = 0
    for _ in range(max(args.warmup, 3)):
        sim.step(it, 1)
        it += 1
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    dist.barrier()
    rt.cudaStreamSynchronize(stream)
    launches = 0
    t_wall0 = time.perf_counter()
    for k in range(nev):
        rt.cudaMemsetAsync(flush, k & 0xff, L2_FLUSH_BYTES, stream)
        rt.cudaEventRecord(ev0[k], stream)
        sim.step_async(it, 1)
        launches += sim.launch_count()
        rt.cudaEventRecord(ev1[k], stream)
        it += 1
    rt.cudaStreamSynchronize(stream)
    t_wall1 = time.perf_counter()
    dist.barrier()
    clocks = sampler.stop()
    sim.sync()
    ms = []
    for k in range(nev):
        f = ctypes.c_float()
        rt.cudaEventElapsedTime(ctypes.byref(f), ev0[k], ev1[k])
        ms.append(f.value)
    # per-kernel device time: CUDA events on the launching stream around every
    # launch, over a second pass of the same steps right after the timed region
    # (the timed steps replay one CUDA graph per step, which has no room for
    # per-launch events; kernel durations are the same, the launch gaps are not)
    nprof = min(nev, 50)
    capi.check(capi.lib().pfag_set_profile(sim.h, 1))
    capi.lib().pfag_profile_read(sim.h, None, None, None, 0)   # clear
    for k in range(nprof):
        rt.cudaMemsetAsync(flush, k & 0xff, L2_FLUSH_BYTES, stream)
        sim.step_async(it, 1)
        it += 1
    rt.cudaStreamSynchronize(stream)
    names = ctypes.create_string_buffer(64 * 64)
    kms = (ctypes.c_double * 64)()
    kl = (ctypes.c_long * 64)()
    capi.lib().pfag_profile_read.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_int]
    nk = capi.lib().pfag_profile_read(sim.h, names, kms, kl, 64)
    ktimes = {}
    for k in range(nk):
        nm = names.raw[64 * k:64 * (k + 1)].split(b"\0")[0].decode()
        ktimes[nm] = (kms[k], kl[k])
    capi.lib().pfag_set_profile(sim.h, 0)
    stats = sim.stats()
    step_ms_local = float(np.mean(ms))
    total_ms_local = float(np.sum(ms))
    total_ms = dist.max(total_ms_local)
    value = sites * nev * ws / (total_ms * 1e-3)

    # roofline of the dominant kernel
    iters_per_step = {"cell_iters_sum": stats["cell_iters_sum"], "lum_iters": stats["lum_iters"],
                      "ecm_iters": stats["ecm_iters"]}
    xc, yc = sim.centres()
    ubox, uring = footprints(cfg, xc, yc)
    kb = kernel_bytes(cfg, prec, iters_per_step, ubox, uring)
    top = max(ktimes.items(), key=lambda kv: kv[1][0]) if ktimes else ("none", (0.0, 1))
    top_name, (top_ms, top_launches) = top
    peak, peak_kind = measured_peak_hbm()
    per_launch_ms = top_ms / max(top_launches, 1)
    achieved = kb.get(top_name, 0) / (per_launch_ms * 1e-3) / 1e9 if per_launch_ms > 0 else 0.0
    total_k_ms = sum(v[0] for v in ktimes.values()) or 1.0
    traffic = NCU_TRAFFIC.get((args.config, top_name)) if prec == 32 else None
    b_step = step_bytes(cfg, prec)
    step_ms = float(np.mean(ms))
    step_gbs = b_step / (step_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": top_name, "achieved": round(achieved, 1), "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "algorithmic_bytes_per_launch": int(kb.get(top_name, 0)),
                "launch_ms": round(per_launch_ms, 5),
                "traffic": traffic[0] if traffic else None,
                "traffic_source": traffic[1] if traffic else None,
                "share": round(top_ms / total_k_ms, 3),
                "step_bytes": int(b_step), "step_achieved": round(step_gbs, 1),
                "step_frac": round(step_gbs / peak, 4),
                "timing": f"per-launch CUDA events over {nprof} eager profiled steps after the timed region",
                "per_kernel_ms_per_step": {k: round(v[0] / nprof, 4) for k, v in sorted(ktimes.items())},
                "per_kernel_gbs": {k: round(kb[k] / (v[0] / max(v[1], 1) * 1e-3) / 1e9, 1)
                                   for k, v in ktimes.items() if k in kb and v[0] > 0},
                "per_kernel_frac": {k: round(kb[k] / (v[0] / max(v[1], 1) * 1e-3) / 1e9 / peak, 3)
                                    for k, v in ktimes.items() if k in kb and v[0] > 0}}
    sim.close()

    # end to end through the public C ABI: pinned host buffers in, K steps, state out
    e2e = run_e2e(args, cfg, p, prec, init, rt, capi, sites, dist)

    result = {"value": value, "ms_per_step": dist.max(step_ms_local), "roofline": roofline, "e2e": e2e,
              "gpu_launches": int(dist.sum(launches)), "clocks": clocks, "stats": stats,
              "wall_ms": (t_wall1 - t_wall0) * 1e3}
    if rank == 0 and ws == 1 and not args.no_compare:
        result["compare"] = compare_paths(cfg, p, capi)
    rt.cudaFree(flush)
    return result


def run_e2e(args, cfg, p, prec, init, rt, capi, sites, dist):
    nsteps = args.steps
    dtype = np.float64 if prec == 64 else np.float32
    host = [np.ascontiguousarray(x, dtype=dtype) for x in init]
    outs = [np.empty_like(x) for x in host]
    rt.cudaHostRegister.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint]
    rt.cudaHostUnregister.argtypes = [ctypes.c_void_p]
    for a in host + outs:
        rt.cudaHostRegister(a.ctypes.data, a.nbytes, 0)
    # every step's areas, f0 and centres land in pinned host rows
    obs = [np.empty((nsteps, cfg.ncells), np.float64), np.empty((nsteps, cfg.ncells), np.float64),
           np.empty((nsteps, cfg.ncells), np.int32), np.empty((nsteps, cfg.ncells), np.int32)]
    for a in obs:
        rt.cudaHostRegister(a.ctypes.data, a.nbytes, 0)
    sim = capi.Simulation(p, prec, capi.PATH_FUSED)
    if args.lumen_tma:
        sim.set_lumen_tiles(True)
    L = capi.lib()
    dist.barrier()
    t0 = time.perf_counter()
    sim.upload(*host)                       # H2D of the initial state
    for k in range(nsteps):
        sim.step_async(k, 1)                # the step through the C ABI, no host wait
        capi.check(L.pfag_observables_async(sim.h, *[ctypes.c_void_p(a[k].ctypes.data) for a in obs]))
    capi.check(L.pfag_download(sim.h, *[ctypes.c_void_p(a.ctypes.data) for a in outs]))
    sim.sync()                              # device errors of the run
    t1 = time.perf_counter()
    dist.barrier()
    sim.close()
    for a in host + outs + obs:
        rt.cudaHostUnregister(a.ctypes.data)
    el = dist.max(t1 - t0)
    h2d = sum(a.nbytes for a in host)
    d2h = sum(a.nbytes for a in outs) + nsteps * cfg.ncells * (8 + 8 + 4 + 4)
    return {"value": sites * nsteps * dist.ws / el, "unit": UNIT,
            "h2d_bytes_per_step": int(h2d / nsteps), "d2h_bytes_per_step": int(d2h / nsteps),
            "steps": nsteps, "note": "pfag_upload from pinned host buffers, pfag_step_async per step with its areas, "
                                     "f0 and centres copied to pinned host rows (pfag_observables_async), "
                                     "pfag_download of the final state"}


def compare_paths(cfg, p, capi, nsteps=20):
    """fast (FP32 fused) and fused FP64 against the plain FP64 path after nsteps."""
    res = {}
    for key, prec, path in (("plain_f64", 64, capi.PATH_PLAIN), ("fused_f64", 64, capi.PATH_FUSED),
                            ("fused_f32", 32, capi.PATH_FUSED)):
        dtype = np.float64 if prec == 64 else np.float32
        with capi.Simulation(p, prec, path) as sim:
            sim.upload(*cfg.initial_state(dtype))
            sim.step(0, 3)
            t0 = time.perf_counter()
            sim.step(3, nsteps - 3)
            el = time.perf_counter() - t0
            phi, rho, _, _ = sim.download()
            res[key] = dict(phi=phi.astype(np.float64), rho=rho.astype(np.float64), s=sim.areas()[0],
                            rate=cfg.ncells * cfg.N * cfg.N * (nsteps - 3) / el)
    base = res["plain_f64"]
    out = {"steps": nsteps, "plain_f64_rate": base["rate"]}
    for key in ("fused_f64", "fused_f32"):
        r = res[key]
        mask = np.abs(base["phi"]) > 1e-6
        out[key] = {"rate": r["rate"],
                    "area_rel_max": float(np.max(np.abs(r["s"] - base["s"]) / np.abs(base["s"]))),
                    "phi_abs_max": float(np.max(np.abs(r["phi"] - base["phi"]))),
                    "phi_abs_max_where_phi_gt_1e-6": float(np.max(np.abs(r["phi"] - base["phi"])[mask])),
                    "rho_rel_linf": float(np.max(np.abs(r["rho"] - base["rho"])) / np.max(np.abs(base["rho"])))}
    return out


def run_batched(args, ws, rank, local, dist: Dist):
    """Config 3: the seeded uneven sweep (members generated on the device),
    one graph launch per step over every member; each GPU its own replica."""
    from multicellular_phase_field_active_gel_organoids_b200 import batched as B
    from multicellular_phase_field_active_gel_organoids_b200 import capi

    capi.lib()
    rt = ctypes.CDLL("libcudart.so.12")
    if rt.cudaSetDevice(local) != 0:
        raise RuntimeError(f"cudaSetDevice({local}) failed")
    rt.cudaEventCreate.argtypes = [ctypes.POINTER(ctypes.c_void_p)]
    rt.cudaEventRecord.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    rt.cudaEventElapsedTime.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.c_void_p, ctypes.c_void_p]
    rt.cudaMemsetAsync.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t, ctypes.c_void_p]
    rt.cudaStreamSynchronize.argtypes = [ctypes.c_void_p]
    prec = args.precision
    members = B.sweep_members(args.members, seed=1)
    t0 = time.perf_counter()
    shapes = {} if args.no_tune else B.autotune(members, prec)
    t_tune = time.perf_counter() - t0
    sw = B.BatchedSweep(members, prec)
    sw.set_shapes(shapes)
    sites = sw.sites
    flush = ctypes.c_void_p()
    assert rt.cudaMalloc(ctypes.byref(flush), ctypes.c_size_t(L2_FLUSH_BYTES)) == 0
    stream = ctypes.c_void_p(sw.batch.stream())
    it = 0
    for _ in range(max(args.warmup, 3)):
        sw.step(it, 1)
        it += 1
    nev = args.steps
    ev0 = [ctypes.c_void_p() for _ in range(nev)]
    ev1 = [ctypes.c_void_p() for _ in range(nev)]
    for e in ev0 + ev1:
        rt.cudaEventCreate(ctypes.byref(e))
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    dist.barrier()
    rt.cudaStreamSynchronize(stream)
    launches = 0
    for k in range(nev):
        rt.cudaMemsetAsync(flush, k & 0xff, L2_FLUSH_BYTES, stream)
        rt.cudaEventRecord(ev0[k], stream)
        sw.step_async(it, 1)
        launches += sw.batch.launch_count()
        rt.cudaEventRecord(ev1[k], stream)
        it += 1
    rt.cudaStreamSynchronize(stream)
    dist.barrier()
    clocks = sampler.stop()
    sw.sync()
    ms = []
    for k in range(nev):
        f = ctypes.c_float()
        rt.cudaEventElapsedTime(ctypes.byref(f), ev0[k], ev1[k])
        ms.append(f.value)
    total_ms = dist.max(float(np.sum(ms)))
    value = sites * nev * ws / (total_ms * 1e-3)
    # step-level roofline: the members' compulsory state bytes per step
    peak, peak_kind = measured_peak_hbm()
    b_step = sum(step_bytes(m.config(), prec) for m in sw.members)
    step_ms = float(np.mean(ms))
    step_gbs = b_step / (step_ms * 1e-3) / 1e9
    # end to end through the public batch API: every step's areas, f0 and
    # centres of every member copied to pinned host rows
    obs = [(np.empty(m.ncells), np.empty(m.ncells), np.empty(m.ncells, np.int32), np.empty(m.ncells, np.int32))
           for m in sw.members]
    rt.cudaHostRegister.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint]
    rt.cudaHostUnregister.argtypes = [ctypes.c_void_p]
    for row in obs:
        for a in row:
            rt.cudaHostRegister(a.ctypes.data, a.nbytes, 0)
    L = capi.lib()
    dist.barrier()
    te0 = time.perf_counter()
    for k in range(nev):
        sw.step_async(it, 1)
        it += 1
        for s, row in zip(sw.sims, obs):
            capi.check(L.pfag_observables_async(s.h, *[ctypes.c_void_p(a.ctypes.data) for a in row]))
    sw.sync()
    te = dist.max(time.perf_counter() - te0)
    for row in obs:
        for a in row:
            rt.cudaHostUnregister(a.ctypes.data)
    d2h = sum(a.nbytes for row in obs for a in row)
    e2e = {"value": sites * nev * ws / te, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": int(d2h),
           "steps": nev, "note": "pfag_batch_step_async per step (one graph launch over every member) with every "
                                 "member's areas, f0 and centres copied to pinned host rows; member states are "
                                 "generated on the device (pfag_seed_organoid), so no state crosses PCIe"}
    buckets = {k: len(v) for k, v in sw.buckets().items()}
    sw.close()
    rt.cudaFree(flush)
    return {"value": value, "ms_per_step": dist.max(step_ms), "e2e": e2e, "clocks": clocks,
            "gpu_launches": int(dist.sum(launches)), "sites": sites, "members": len(members),
            "roofline": {"bound": "hbm", "kernel": None, "achieved": round(step_gbs, 1), "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": round(step_gbs / peak, 4), "traffic": None,
                         "step_bytes": int(b_step), "step_achieved": round(step_gbs, 1),
                         "step_frac": round(step_gbs / peak, 4),
                         "note": "step level: the members' compulsory state bytes per step over the batch step time"},
            "tuning": {"seconds": round(t_tune, 1), "shapes": shapes, "buckets": buckets}}


def cpu_reference_rate(cfg_name: str, steps: int, warmup: int, precision: str = "fp32"):
    """The reference's own step (oracle/_ref, g++ build, serial) on the host."""
    from multicellular_phase_field_active_gel_organoids_b200.params import CONFIGS
    from oracle import refrun
    if not refrun.available(precision):
        return None
    code = f"""
import sys, time, json, numpy as np
sys.path.insert(0, {ROOT!r})
from multicellular_phase_field_active_gel_organoids_b200.params import CONFIGS
from oracle.refrun import RefLib
cfg = CONFIGS[{cfg_name!r}]()
r = RefLib({precision!r}, cfg.params())
r.load(*cfg.initial_state(np.float64 if {precision!r} == 'fp64' else np.float32))
for k in range({warmup}): r.step(k)
t = time.perf_counter()
for k in range({steps}): r.step({warmup} + k)
el = time.perf_counter() - t
print('RESULT', json.dumps({{'el': el}}))
"""
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=1800)
    line = [l for l in out.stdout.splitlines() if l.startswith("RESULT")]
    if not line:
        raise RuntimeError("reference run failed: " + out.stderr[-2000:])
    el = json.loads(line[0].split(" ", 1)[1])["el"]
    cfg = CONFIGS[cfg_name]()
    return cfg.ncells * cfg.N * cfg.N * steps / el, el


def main():
    args = parse()
    ws, rank, local = dist_info()
    from multicellular_phase_field_active_gel_organoids_b200.params import CONFIGS
    if args.config == "cfg3":
        return main_batched(args, ws, rank, local)
    if args.config == "cfg4":
        return main_corrector(args, ws, rank, local)
    if args.shard and args.impl == "ours":
        return main_sharded(args, ws, rank, local)
    cfg = CONFIGS[args.config]()
    config = {"workload": f"{args.config}: {cfg.N}x{cfg.N} periodic grid, {cfg.ncells} cells R={cfg.radius:g} "
                          f"on a jittered hexagonal lattice, zone_size {cfg.zone_size} (FFT box {cfg.box}), "
                          f"dx=1 dt=1e-3", "grid": cfg.N, "cells": cfg.ncells, "zone_size": cfg.zone_size,
              "box": cfg.box, "l2": "flushed between timed steps (256 MiB write)",
              "replicas": ws}
    if args.impl == "reference":
        if rank != 0:
            return 0
        k = max(1, min(args.steps, 8))
        w = 1 if args.warmup > 0 else 0
        rate, el = cpu_reference_rate(args.config, k, w, "fp32")
        sample = (f"{k} reference steps of the full {args.config} workload after {w} warm-up step, "
                  f"shipped FP32 build (g++ -O3, OpenACC pragmas inert), one process")
        line = {"metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": k, "warmup": w,
                "ms_per_step": el / k * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic (seeded organoid, same generator as our arm)", "config": config,
                "impl": "reference",
                "cpu_baseline": {"value": rate, "unit": UNIT, "cores": 1, "kind": "reference",
                                 "host_cores": os.cpu_count(), "sample": sample},
                "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    dist = Dist(ws, rank, local, "nccl")
    res = run_ours(args, ws, rank, local, dist)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            r = cpu_reference_rate(args.config, 2, 1, "fp32")
            if r:
                cpu = {"value": r[0], "unit": UNIT, "cores": 1, "kind": "reference", "host_cores": os.cpu_count(),
                       "sample": "2 steps (after 1 warm-up) of the full workload, reference FP32 build, 1 core "
                                 "(the reference's host code is serial without OpenACC)"}
        except Exception as e:  # pragma: no cover - reported, not fatal
            cpu = {"error": str(e)[:200]}
    dist.close()
    if rank != 0:
        return 0
    line = {"metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": res["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == 32 else "f64",
            "data": "synthetic (seeded organoid inputs generated in-process; no dataset)",
            "config": dict(config, path="fused", precision=("f32 with f64 areas/loop sums" if args.precision == 32
                                                            else "f64"),
                           parallelism=f"replicas x{ws}",
                           lumen_tiles="TMA-staged" if args.lumen_tma else "per-thread copies"),
            "roofline": res["roofline"], "cpu_baseline": cpu, "e2e": res["e2e"],
            "gpu_launches": res["gpu_launches"], "clocks": res["clocks"],
            "active_site_updates_per_s": res["value"] * (2 * cfg.zone_size) ** 2 / cfg.N ** 2,
            "relax_iters_last_step": res["stats"]}
    if "compare" in res:
        line["compare_vs_plain_f64"] = res["compare"]
    print(json.dumps(line))
    return 0


def main_sharded(args, ws, rank, local):
    """One organoid (cfg) with its cells split over the ranks by contiguous
    ranges (sharded.DistShard over NCCL): per step a halo of two phi planes
    with the neighbouring ranks and an all-reduce of psi.  Total work is fixed
    as N grows (strong scaling); value = the organoid's site-updates / the
    slowest rank's time.  Each step is timed with CUDA events on the context's
    stream, the L2 flush between steps outside them."""
    import datetime
    import torch
    import torch.distributed as td
    from multicellular_phase_field_active_gel_organoids_b200 import capi, sharded
    from multicellular_phase_field_active_gel_organoids_b200.params import CONFIGS
    torch.cuda.set_device(local)
    if ws == 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        if "MASTER_PORT" not in os.environ:
            import socket
            so = socket.socket()
            so.bind(("127.0.0.1", 0))
            os.environ["MASTER_PORT"] = str(so.getsockname()[1])
            so.close()
        os.environ.setdefault("RANK", "0")
        os.environ.setdefault("WORLD_SIZE", "1")
    td.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    cfg = CONFIGS[args.config]()
    prec = args.precision
    dtype = np.float64 if prec == 64 else np.float32
    sites = cfg.ncells * cfg.N * cfg.N
    sh = sharded.DistShard(cfg.params(), cfg.initial_state(dtype), precision=prec)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    it = 0
    for _ in range(max(args.warmup, 3)):
        sh.step(it, 1)
        it += 1
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    td.barrier()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches = 0
    with torch.cuda.stream(sh.stream):
        for k in range(args.steps):
            flush.fill_(k & 0xff)
            ev[k][0].record(sh.stream)
            sharded.run_steps(sh.ex, sh, it, 1)
            launches += sh.sim.launch_count()
            ev[k][1].record(sh.stream)
            it += 1
    torch.cuda.synchronize()
    td.barrier()
    clocks = sampler.stop()
    sh.sim.sync()
    total = torch.tensor([sum(a.elapsed_time(b) for a, b in ev)], dtype=torch.float64, device="cuda")
    td.all_reduce(total, op=td.ReduceOp.MAX)
    nl = torch.tensor([launches], dtype=torch.float64, device="cuda")
    td.all_reduce(nl, op=td.ReduceOp.SUM)
    stats = sh.sim.stats()
    sh.close()
    td.destroy_process_group()
    if rank != 0:
        return 0
    total_ms = float(total.item())
    value = sites * args.steps / (total_ms * 1e-3)
    plane = cfg.N * cfg.N * (8 if prec == 64 else 4)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32" if prec == 32 else "f64",
            "data": "synthetic (seeded organoid inputs generated in-process; no dataset)",
            "config": {"workload": f"{args.config}: {cfg.N}x{cfg.N} grid, {cfg.ncells} cells, zone_size "
                                   f"{cfg.zone_size} (FFT box {cfg.box}), cells split over {ws} rank(s)",
                       "grid": cfg.N, "cells": cfg.ncells, "zone_size": cfg.zone_size, "box": cfg.box,
                       "l2": "flushed between timed steps (256 MiB write)", "path": "fused",
                       "parallelism": f"cell shards x{ws}", "cells_per_rank": [b - a for a, b in sh.bounds]},
            "exchange_bytes_per_step_per_rank": {"psi_allreduce": plane, "halo": 2 * plane} if ws > 1 else {},
            "roofline": None, "cpu_baseline": None, "e2e": None,
            "gpu_launches": int(nl.item()), "clocks": clocks, "relax_iters_last_step": stats}
    print(json.dumps(line))
    return 0


def main_corrector(args, ws, rank, local):
    """Config 4: the 64-cell organoid at half resolution (512^2, dx = 2,
    dt = 4e-3) with the learned corrector every 10 coarse steps, against the
    fine method (1024^2, dx = 1, dt = 1e-3) over the same physical time.  The
    network is trained first on coarse/fine pairs of seeded organoids (16-96
    cells) generated by the fine method; the metric is the fine-equivalent
    rate (64 x 1024^2 sites x the fine steps covered, per second)."""
    import torch
    from multicellular_phase_field_active_gel_organoids_b200 import capi
    from multicellular_phase_field_active_gel_organoids_b200 import corrector as C
    from multicellular_phase_field_active_gel_organoids_b200.params import CONFIGS

    config = {"workload": "cfg4: the cfg1 organoid (1024^2, 64 cells, R = 24) at half resolution (512^2, dx = 2, "
                          "dt = 4e-3, zone_size 65) with a 5-layer 3x3 BF16 conv net (32 channels, GELU, FP32 "
                          "accumulation on tcgen05) correcting phi and rho every 10 coarse steps",
              "pairs": args.pairs, "intervals": args.steps, "l2": "not flushed (steps of one run)",
              "parallelism": f"replicas x{ws}"}
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no learned coarse-grid "
                                                                  "method; its fine step is the cfg1 reference arm"}))
        return 0
    capi.lib()
    torch.cuda.set_device(local)
    t0 = time.perf_counter()
    nseed = max(1, args.pairs // 4)
    feats, targs = C.make_pairs(range(1000, 1000 + nseed), ncells_range=(16, 96), checkpoints=4)
    sc = C.fit_scales(feats, targs)
    X, T = C.scaled(feats, targs, sc)
    del feats, targs
    t_data = time.perf_counter() - t0
    net = C.ConvNet(seed=0)
    t0 = time.perf_counter()
    hist = C.train(net, X, T, iters=600, batch=16, lr=2e-3)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    n_boxes = int(X.shape[0])
    del X, T
    fcfg = CONFIGS["cfg1"]()
    intervals = max(args.steps, 3)
    fine_steps = 40 * intervals
    with capi.Simulation(fcfg.params(), 32, capi.PATH_FUSED) as fs:
        fs.set_relax_cap(100000)
        fs.upload(*fcfg.initial_state(np.float32))
        fs.step(0, 20)
        F0 = C.state_tensors(fs)
        torch.cuda.synchronize()
        tf0 = time.perf_counter()
        fs.step(20, fine_steps)
        tf = time.perf_counter() - tf0
        ref = C.restrict(C.state_tensors(fs)[0])
    sites = fcfg.ncells * fcfg.N * fcfg.N
    res = {}
    for name, corrected in (("uncorrected", False), ("corrected", True)):
        run = C.CorrectedRun(net, sc, fcfg)
        try:
            run.start_from_fine(F0)
            run.run(1, corrected=corrected)          # warm-up interval (graph capture)
            run.start_from_fine(F0)
            torch.cuda.synchronize()
            tc0 = time.perf_counter()
            run.run(intervals, corrected=corrected)
            run.cs.sync()
            tc = time.perf_counter() - tc0
            area, per = C.shape_errors(run.state_on_coarse()[0], ref)
            res[name] = {"seconds": tc, "fine_equivalent_rate": sites * fine_steps / tc, "area_rel_err": area,
                         "perimeter_rel_err": per}
        finally:
            run.close()
    fine_rate = sites * fine_steps / tf
    cor = res["corrected"]
    line = {"metric": METRIC, "value": cor["fine_equivalent_rate"], "unit": UNIT, "n_gpus": ws,
            "steps": intervals * 10, "warmup": 10, "ms_per_step": cor["seconds"] / (intervals * 10) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 step, bf16 network",
            "data": "synthetic (seeded organoids; training pairs generated in-process by the fine method)",
            "config": config, "cpu_baseline": None,
            "e2e": {"value": cor["fine_equivalent_rate"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0, "note": "device-resident run through the public API; the state "
                                                     "starts from the fine run on the device"},
            "gpu_launches": None,
            "corrector": {"fine_rate": fine_rate, "speedup_vs_fine": cor["fine_equivalent_rate"] / fine_rate,
                          "uncorrected": res["uncorrected"], "corrected": cor, "training_boxes": n_boxes,
                          "loss_first_last": [hist[0], hist[-1]], "data_seconds": round(t_data, 1),
                          "train_seconds": round(t_train, 1), "scales": sc.as_dict()}}
    if rank == 0:
        print(json.dumps(line))
    return 0


def main_batched(args, ws, rank, local):
    config = {"workload": f"cfg3: batched uneven sweep of {args.members} seeded organoids (seed 1): grids 256^2, "
                          "512^2 or 1024^2, cell counts log-uniform in [8, 128] capped by the grid, radii U(16, 32), "
                          "FFT boxes 4R rounded up to a multiple of 16 (64..128), contractility and turnover x "
                          "U(0.5, 2); one graph launch per step over every member",
              "members": args.members, "l2": "flushed between timed steps (256 MiB write)", "replicas": ws,
              "path": "fused", "precision": "f32 with f64 areas/loop sums" if args.precision == 32 else "f64",
              "parallelism": f"replicas x{ws}"}
    if args.impl == "reference":
        if rank != 0:
            return 0
        # the reference's own step on the host for a bounded sample: the first
        # 256^2 members of the same sweep, one step each
        from multicellular_phase_field_active_gel_organoids_b200 import batched as B
        from oracle import refrun
        ms = [m for m in B.sweep_members(args.members, seed=1) if m.N == 256][:4]
        el = 0.0
        sites = 0
        for m in ms:
            code = f"""
import sys, time, json, numpy as np
sys.path.insert(0, {ROOT!r})
from multicellular_phase_field_active_gel_organoids_b200 import batched as B
from oracle.refrun import RefLib
m = [x for x in B.sweep_members({args.members}, seed=1) if x.index == {m.index}][0]
cfg = m.config()
r = RefLib('fp32', cfg.params())
r.load(*cfg.initial_state(np.float32))
r.step(0)
t = time.perf_counter()
r.step(1)
print('RESULT', json.dumps({{'el': time.perf_counter() - t}}))
"""
            out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=1800)
            line = [l for l in out.stdout.splitlines() if l.startswith("RESULT")]
            if not line:
                raise RuntimeError("reference run failed: " + out.stderr[-2000:])
            el += json.loads(line[0].split(" ", 1)[1])["el"]
            sites += m.sites
        rate = sites / el
        line = {"metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": 1, "warmup": 1,
                "ms_per_step": el * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic (seeded sweep members, same generator as our arm)",
                "config": config, "impl": "reference",
                "cpu_baseline": {"value": rate, "unit": UNIT, "cores": 1, "kind": "reference",
                                 "host_cores": os.cpu_count(),
                                 "sample": f"one step (after one warm-up step) of each of the first {len(ms)} "
                                           "256^2 members, shipped FP32 build, one process"},
                "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0
    dist = Dist(ws, rank, local, "nccl")
    res = run_batched(args, ws, rank, local, dist)
    dist.close()
    if rank != 0:
        return 0
    line = {"metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": res["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.precision == 32 else "f64",
            "data": "synthetic (seeded organoids generated on the device; no dataset)",
            "config": dict(config, sites_per_step=res["sites"]), "roofline": res["roofline"], "cpu_baseline": None,
            "e2e": res["e2e"], "gpu_launches": res["gpu_launches"], "clocks": res["clocks"], "tuning": res["tuning"]}
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
