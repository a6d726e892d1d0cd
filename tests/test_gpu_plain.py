"""Plain path (one kernel per reference function, cuFFT) against the reference's
own FP64 run on the same inputs.  Tolerances: FP64 relative L-inf 1e-9 on phi,
rho, lumen, ECM and velocity; areas relative 1e-10; centres exact.  FP32:
per-cell area relative 1e-4 against the FP64 reference."""
import numpy as np
import pytest

from multicellular_phase_field_active_gel_organoids_b200 import capi
from multicellular_phase_field_active_gel_organoids_b200.params import CONFIGS
from oracle import refrun

pytestmark = pytest.mark.gpu


def rel_linf(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def run_gpu(cfg, nsteps, precision=64, path=capi.PATH_PLAIN, velocity=False):
    p = cfg.params()
    dtype = np.float64 if precision == 64 else np.float32
    with capi.Simulation(p, precision, path) as sim:
        sim.upload(*cfg.initial_state(dtype))
        if velocity:
            sim.set_debug(1)
        sim.step(0, nsteps)
        phi, rho, lum, ecm = sim.download()
        s, _ = sim.areas()
        xc, yc = sim.centres()
        vel = sim.velocity() if velocity else None
        st = sim.stats()
    return dict(phi=phi, rho=rho, lum=lum, ECM=ecm, s=s, xc=xc, yc=yc, velocity=vel, stats=st)


@pytest.fixture(scope="module")
def tiny_ref():
    cfg = CONFIGS["tiny"]()
    return cfg, refrun.run_reference(cfg.params(), cfg.initial_state(), 5, velocity=True)


@pytest.mark.parametrize("path", [capi.PATH_PLAIN])
def test_fp64_tiny_matches_reference(tiny_ref, path):
    cfg, ref = tiny_ref
    got = run_gpu(cfg, 5, 64, path, velocity=True)
    assert np.array_equal(got["xc"], ref["xc"]) and np.array_equal(got["yc"], ref["yc"])
    for k in ("phi", "rho", "lum", "ECM"):
        assert rel_linf(got[k], ref[k]) <= 1e-9, k
    assert rel_linf(got["s"], ref["s"]) <= 1e-10
    vx, vy = got["velocity"]
    rvx, rvy = ref["velocity"]
    assert rel_linf(vx, rvx) <= 1e-9 and rel_linf(vy, rvy) <= 1e-9


def test_fp32_tiny_area_within_1e4(tiny_ref):
    cfg, ref = tiny_ref
    got = run_gpu(cfg, 5, 32, capi.PATH_PLAIN)
    assert np.array_equal(got["xc"], ref["xc"])
    assert rel_linf(got["s"], ref["s"]) <= 1e-4
    assert rel_linf(got["phi"], ref["phi"]) <= 1e-3


def test_fp64_cfg0_three_steps():
    cfg = CONFIGS["cfg0"]()
    ref = refrun.run_reference(cfg.params(), cfg.initial_state(), 3)
    got = run_gpu(cfg, 3, 64)
    assert np.array_equal(got["xc"], ref["xc"]) and np.array_equal(got["yc"], ref["yc"])
    for k in ("phi", "rho", "lum", "ECM"):
        assert rel_linf(got[k], ref[k]) <= 1e-9, k
    assert rel_linf(got["s"], ref["s"]) <= 1e-10
