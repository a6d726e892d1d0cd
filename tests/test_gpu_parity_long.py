"""Parity on the benchmark organoid and over long horizons.

1. cfg1, the benchmark organoid (1024^2, 64 cells, zone_size 129, box 256):
   the plain FP64 and the fused FP64 paths against the reference's own FP64
   run (oracle/_ref/libref_fp64.so on the host) after 2 steps: phi, rho,
   lumen, ECM and the second step's per-cell velocity to relative L-inf 1e-9,
   areas to 1e-10, centres exact.
2. cfg0 (256^2, 7 cells, zone_size 65) over 100 steps against the
   reference's FP64 run: centres exact at every checkpoint, areas 1e-10,
   rho and lumen/ECM 1e-8, phi 1e-9 on the sites where the reference's
   |phi| > 1e-6 and 1e-7 on the full field, velocity of step 100 1e-8, and
   every step's per-cell reshaping iteration count equal to the count of the
   C restatement of the reference step (tests/golden/long_cfg0.npz).
3. cfg0 over 1000 steps against tests/golden/long_cfg0.npz (the reference's
   FP64 run, tests/golden/make_long_golden.py): centres exact, areas 1e-7,
   perimeters and rho masses 1e-6, the total reshaping iteration count equal,
   and the steps whose count differs from the reference's (a loop exit taken
   within rounding of its threshold) few and none in the first 100.
4. cfg1 in FP32 (the benchmark path) over 1000 steps against the reference's
   FP64 run (tests/golden/long_cfg1.npz): per-cell area 1e-4, centroids within
   one grid site, perimeter and rho mass 1e-3.

Why the full-field phi bound is wider than 1e-9 and why iteration counts can
differ after ~150 steps: a reshaping loop stops the first time its summed
change falls below a threshold (cell_phase_functions.cpp:473-576); the sums
are taken in another order than the host build's, over states that differ at
the rounding level, so an exit decision within ~1e-7 of the threshold can go
the other way; one extra iteration moves phi by ~1e-6.
"""
import os

import numpy as np
import pytest

from multicellular_phase_field_active_gel_organoids_b200 import capi
from multicellular_phase_field_active_gel_organoids_b200.params import CONFIGS
from oracle import refrun
from tests.shape import perimeter, rel, rel_each, rho_mass

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

PATHS = {"plain_f64": (64, capi.PATH_PLAIN), "fused_f64": (64, capi.PATH_FUSED)}


def _golden(name):
    path = os.path.join(GOLDEN, f"long_{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"{path} not generated (tests/golden/make_long_golden.py)")
    return np.load(path)


def _state(sim):
    phi, rho, lum, ecm = sim.download()
    xc, yc = sim.centres()
    return {"phi": phi, "rho": rho, "lum": lum, "ECM": ecm, "s": sim.areas()[0], "xc": xc, "yc": yc}


@pytest.fixture(scope="module")
def cfg1_ref():
    cfg = CONFIGS["cfg1"]()
    return cfg, refrun.run_reference(cfg.params(), cfg.initial_state(), 2, velocity=True)


@pytest.mark.parametrize("name", list(PATHS))
def test_cfg1_two_steps_match_reference(cfg1_ref, name):
    cfg, ref = cfg1_ref
    prec, path = PATHS[name]
    with capi.Simulation(cfg.params(), prec, path) as sim:
        sim.set_relax_cap(100000)
        sim.upload(*cfg.initial_state())
        sim.step(0, 1)
        sim.set_debug(1)
        sim.step(1, 1)
        got = _state(sim)
        vx, vy = sim.velocity()
    assert np.array_equal(got["xc"], ref["xc"]) and np.array_equal(got["yc"], ref["yc"])
    errs = {k: rel(got[k], ref[k]) for k in ("phi", "rho", "lum", "ECM", "s")}
    rvx, rvy = ref["velocity"]
    errs["velocity"] = max(rel(vx, rvx), rel(vy, rvy))
    print(name, errs)
    assert all(errs[k] <= 1e-9 for k in ("phi", "rho", "lum", "ECM", "velocity")), errs
    assert errs["s"] <= 1e-10, errs


@pytest.fixture(scope="module")
def cfg0_ref100():
    cfg = CONFIGS["cfg0"]()
    return cfg, refrun.run_reference(cfg.params(), cfg.initial_state(), 100, snapshots=[1, 10], velocity=True,
                                     timeout=1800)


@pytest.mark.parametrize("name", list(PATHS))
def test_cfg0_hundred_steps_match_reference(cfg0_ref100, name):
    cfg, ref = cfg0_ref100
    gold = _golden("cfg0")
    host_iters = gold["cell_iters"]
    prec, path = PATHS[name]
    refs = dict(ref["snapshots"])
    refs[100] = ref
    iters = np.zeros((100, cfg.ncells), np.int32)
    report = {}
    with capi.Simulation(cfg.params(), prec, path) as sim:
        sim.set_relax_cap(100000)
        sim.upload(*cfg.initial_state())
        for k in range(100):
            if k == 99:
                sim.set_debug(1)
            sim.step(k, 1)
            iters[k] = sim.cell_iters()
            if k + 1 in refs:
                got, r = _state(sim), refs[k + 1]
                mask = np.abs(r["phi"]) > 1e-6
                e = {"phi": rel(got["phi"], r["phi"]), "phi_masked": rel(got["phi"], r["phi"], mask),
                     "rho": rel(got["rho"], r["rho"]), "lum": rel(got["lum"], r["lum"]),
                     "ECM": rel(got["ECM"], r["ECM"]), "s": rel(got["s"], r["s"])}
                report[k + 1] = e
                assert np.array_equal(got["xc"], r["xc"]) and np.array_equal(got["yc"], r["yc"]), k + 1
                assert e["phi_masked"] <= 1e-9 and e["phi"] <= 1e-7, (k + 1, e)
                assert e["rho"] <= 1e-8 and e["lum"] <= 1e-8 and e["ECM"] <= 1e-8, (k + 1, e)
                assert e["s"] <= 1e-10, (k + 1, e)
        vx, vy = sim.velocity()
    rvx, rvy = ref["velocity"]
    vel = max(rel(vx, rvx), rel(vy, rvy))
    print(name, report, "velocity", vel)
    assert vel <= 1e-8
    diff = np.argwhere(iters != host_iters[:100])
    assert diff.size == 0, f"first reshaping count difference at step {diff[0][0] + 1}, cell {diff[0][1]}"


@pytest.mark.parametrize("name", list(PATHS))
def test_cfg0_thousand_steps_against_reference_fixture(name):
    gold = _golden("cfg0")
    cfg = CONFIGS["cfg0"]()
    p = cfg.params()
    dx = float(p["dx"])
    nsteps = int(gold["steps"])
    host_iters = gold["cell_iters"]
    prec, path = PATHS[name]
    iters = np.zeros_like(host_iters)
    with capi.Simulation(p, prec, path) as sim:
        sim.set_relax_cap(100000)
        sim.upload(*cfg.initial_state())
        for k in range(nsteps):
            sim.step(k, 1)
            iters[k] = sim.cell_iters()
        got = _state(sim)
    c = nsteps
    assert np.array_equal(got["xc"], gold[f"xc_{c}"]) and np.array_equal(got["yc"], gold[f"yc_{c}"])
    e = {"s": rel_each(got["s"], gold[f"s_{c}"]),
         "perimeter": rel_each(perimeter(got["phi"], dx), gold[f"perimeter_{c}"]),
         "rho_mass": rel_each(rho_mass(got["rho"], dx), gold[f"rho_mass_{c}"])}
    steps_differing = np.unique(np.argwhere(iters != host_iters)[:, 0])
    print(name, e, "iterations", int(iters.sum()), int(host_iters.sum()), "steps differing", steps_differing.size,
          "first", (int(steps_differing[0]) + 1) if steps_differing.size else None)
    assert e["s"] <= 1e-7 and e["perimeter"] <= 1e-6 and e["rho_mass"] <= 1e-6, e
    assert int(iters.sum()) == int(host_iters.sum())
    assert steps_differing.size <= 50
    assert not steps_differing.size or steps_differing[0] >= 100


def test_cfg1_fp32_thousand_steps_against_reference_fixture():
    gold = _golden("cfg1")
    cfg = CONFIGS["cfg1"]()
    p = cfg.params()
    dx = float(p["dx"])
    c = int(gold["steps"])
    with capi.Simulation(p, 32, capi.PATH_FUSED) as sim:
        sim.set_relax_cap(100000)
        sim.upload(*cfg.initial_state(np.float32))
        sim.step(0, c)
        got = _state(sim)
    e = {"s": rel_each(got["s"], gold[f"s_{c}"]),
         "perimeter": rel_each(perimeter(got["phi"], dx), gold[f"perimeter_{c}"]),
         "rho_mass": rel_each(rho_mass(got["rho"], dx), gold[f"rho_mass_{c}"]),
         "centroid": int(max(np.max(np.abs(got["xc"] - gold[f"xc_{c}"])), np.max(np.abs(got["yc"] - gold[f"yc_{c}"]))))}
    print("fused_f32 cfg1", c, "steps", e)
    assert e["s"] <= 1e-4 and e["centroid"] <= 1, e
    assert e["perimeter"] <= 1e-3 and e["rho_mass"] <= 1e-3, e
