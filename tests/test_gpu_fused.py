"""Fused path (zone-restricted kernels, hand-written FFT, persistent relaxation
loops) against the reference's own FP64 run and against the plain path.
FP64 tolerances: relative L-inf 1e-9 on phi, rho, lumen, ECM and velocity,
areas 1e-10, centres exact.  FP32 (FP64 islands for areas and loop sums):
per-cell area 1e-4 against the FP64 reference."""
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


def run_gpu(cfg, nsteps, precision, path, velocity=False):
    dtype = np.float64 if precision == 64 else np.float32
    with capi.Simulation(cfg.params(), precision, path) as sim:
        sim.set_relax_cap(100000)
        sim.upload(*cfg.initial_state(dtype))
        if velocity:
            sim.set_debug(1)
        sim.step(0, nsteps)
        phi, rho, lum, ecm = sim.download()
        out = dict(phi=phi, rho=rho, lum=lum, ECM=ecm, s=sim.areas()[0], xc=sim.centres()[0],
                   yc=sim.centres()[1], iters=sim.cell_iters(), stats=sim.stats())
        if velocity:
            out["velocity"] = sim.velocity()
    return out


@pytest.fixture(scope="module")
def tiny_ref():
    cfg = CONFIGS["tiny"]()
    return cfg, refrun.run_reference(cfg.params(), cfg.initial_state(), 5, velocity=True)


def test_fused_fp64_tiny_matches_reference(tiny_ref):
    cfg, ref = tiny_ref
    got = run_gpu(cfg, 5, 64, capi.PATH_FUSED, velocity=True)
    assert np.array_equal(got["xc"], ref["xc"]) and np.array_equal(got["yc"], ref["yc"])
    errs = {k: rel_linf(got[k], ref[k]) for k in ("phi", "rho", "lum", "ECM", "s")}
    assert all(errs[k] <= 1e-9 for k in ("phi", "rho", "lum", "ECM")), errs
    assert errs["s"] <= 1e-10, errs
    vx, vy = got["velocity"]
    rvx, rvy = ref["velocity"]
    assert rel_linf(vx, rvx) <= 1e-9 and rel_linf(vy, rvy) <= 1e-9


def test_fused_fp32_tiny_area(tiny_ref):
    cfg, ref = tiny_ref
    got = run_gpu(cfg, 5, 32, capi.PATH_FUSED)
    assert np.array_equal(got["xc"], ref["xc"])
    assert rel_linf(got["s"], ref["s"]) <= 1e-4


def test_fp32_lumen_relaxation_on_tma_tiles():
    """cfg0 (256^2) with the FP32 lumen / ECM relaxation on TMA-staged tiles
    (pfag_set_lumen_tiles, kl_relax_tma) over 5 steps (the first eager, the
    rest graph replays): the same iteration counts as with the per-thread
    copies and the same fields to FP32 rounding (the same formula per site,
    compiled in another kernel), and within FP32 of the plain FP64 path; the
    knob is refused on a grid too small for the tiles."""
    cfg = CONFIGS["cfg0"]()
    init = cfg.initial_state(np.float32)
    out = {}
    for tma in (False, True):
        with capi.Simulation(cfg.params(), 32, capi.PATH_FUSED) as sim:
            sim.set_relax_cap(100000)
            sim.set_lumen_tiles(tma)
            sim.upload(*init)
            sim.step(0, 5)
            out[tma] = (sim.download(), sim.stats())
    (fa, sa), (fb, sb) = out[False], out[True]
    assert (sa["lum_iters"], sa["ecm_iters"]) == (sb["lum_iters"], sb["ecm_iters"])
    for k, x, y in zip(("phi", "rho", "lum", "ECM"), fa, fb):
        d = float(np.abs(x.astype(np.float64) - y).max())
        print("tma vs copies", k, d)
        assert d <= 1e-5, (k, d)
    b = run_gpu(cfg, 5, 64, capi.PATH_PLAIN)
    assert (sb["lum_iters"], sb["ecm_iters"]) == (b["stats"]["lum_iters"], b["stats"]["ecm_iters"])
    for k, x in zip(("lum", "ECM"), fb[2:]):
        assert np.abs(x - b[k]).max() <= 1e-5, (k, np.abs(x - b[k]).max())
    tiny = CONFIGS["tiny"]()
    with capi.Simulation(tiny.params(), 32, capi.PATH_FUSED) as sim:
        with pytest.raises(capi.PfagError):
            sim.set_lumen_tiles(True)


def test_tma_wait_limit_reports_and_recovers():
    """The bounded waits of the TMA-staged lumen tiles: with the copies not
    issued (pfag_set_debug bit 2, a host-side switch: nothing is in flight)
    no stage completes, every wait gives up after its limit, the step
    reports PFAG_E_CUDA once, and the context steps normally again (no fault,
    no hang: the kernel returns)."""
    cfg = CONFIGS["cfg0"]()
    init = cfg.initial_state(np.float32)
    with capi.Simulation(cfg.params(), 32, capi.PATH_FUSED) as sim:
        sim.set_lumen_tiles(True)
        sim.upload(*init)
        sim.set_debug(2)
        with pytest.raises(capi.PfagError) as e:
            sim.step(0, 1)
        assert e.value.code == -2 and "gave up" in str(e.value)
        sim.set_debug(0)
        sim.set_relax_cap(100000)
        sim.upload(*init)
        sim.step(0, 3)
        phi, rho, lum, ecm = sim.download()
    ref = run_gpu(cfg, 3, 32, capi.PATH_FUSED)
    assert np.abs(lum - ref["lum"]).max() <= 1e-5 and np.abs(phi - ref["phi"]).max() <= 1e-5


def test_fused_vs_plain_cfg0_fp64():
    cfg = CONFIGS["cfg0"]()
    a = run_gpu(cfg, 4, 64, capi.PATH_FUSED)
    b = run_gpu(cfg, 4, 64, capi.PATH_PLAIN)
    assert np.array_equal(a["iters"], b["iters"])
    for k in ("phi", "rho", "lum", "ECM"):
        assert rel_linf(a[k], b[k]) <= 1e-9, (k, rel_linf(a[k], b[k]))
    assert rel_linf(a["s"], b["s"]) <= 1e-10


def test_fused_cfg1_fp64_and_fp32_vs_plain():
    """The benchmark workload (1024^2, 64 cells, box 256): fused FP64 against
    the plain FP64 path over 3 steps (support rectangles wider than a block's
    columns, graph replay from the second step), and the FP32 fused areas
    against them."""
    cfg = CONFIGS["cfg1"]()
    a = run_gpu(cfg, 3, 64, capi.PATH_FUSED)
    b = run_gpu(cfg, 3, 64, capi.PATH_PLAIN)
    assert np.array_equal(a["xc"], b["xc"]) and np.array_equal(a["yc"], b["yc"])
    assert np.array_equal(a["iters"], b["iters"])
    for k in ("phi", "rho", "lum", "ECM"):
        assert rel_linf(a[k], b[k]) <= 1e-9, (k, rel_linf(a[k], b[k]))
    assert rel_linf(a["s"], b["s"]) <= 1e-10
    f = run_gpu(cfg, 3, 32, capi.PATH_FUSED)
    assert np.array_equal(f["xc"], b["xc"])
    assert rel_linf(f["s"], b["s"]) <= 1e-4


def test_fused_small_box_shared_memory_path():
    """Box size 16 (zone_size 9) goes through the shared-memory radix-4 box
    passes instead of the register FFTs: fused FP64 against plain FP64."""
    from multicellular_phase_field_active_gel_organoids_b200.params import small_organoid
    cfg = small_organoid(zone_size=9)
    a = run_gpu(cfg, 2, 64, capi.PATH_FUSED)
    b = run_gpu(cfg, 2, 64, capi.PATH_PLAIN)
    assert np.array_equal(a["iters"], b["iters"])
    for k in ("phi", "rho", "lum", "ECM"):
        assert rel_linf(a[k], b[k]) <= 1e-9, (k, rel_linf(a[k], b[k]))


def test_observables_streamed_per_step():
    """pfag_observables_async after each pfag_step_async: every step's areas and
    centres arrive in host rows without a wait per step, equal to what the
    synchronous per-step calls report."""
    import ctypes
    cfg = CONFIGS["tiny"]()
    n, K = cfg.ncells, 4
    rows = [np.zeros((K, n), np.float64), np.zeros((K, n), np.float64), np.zeros((K, n), np.int32),
            np.zeros((K, n), np.int32)]
    with capi.Simulation(cfg.params(), 64, capi.PATH_FUSED) as sim:
        sim.upload(*cfg.initial_state())
        for k in range(K):
            sim.step_async(k, 1)
            capi.check(capi.lib().pfag_observables_async(sim.h, *[ctypes.c_void_p(a[k].ctypes.data) for a in rows]))
        sim.sync()
        s_last, f0_last = sim.areas()
    with capi.Simulation(cfg.params(), 64, capi.PATH_FUSED) as ref:
        ref.upload(*cfg.initial_state())
        for k in range(K):
            ref.step(k, 1)
            s, f0 = ref.areas()
            xc, yc = ref.centres()
            assert np.array_equal(rows[0][k], s) and np.array_equal(rows[1][k], f0)
            assert np.array_equal(rows[2][k], xc) and np.array_equal(rows[3][k], yc)
    assert np.array_equal(rows[0][-1], s_last) and np.array_equal(rows[1][-1], f0_last)


def test_rho_ring_after_upload_and_reupload():
    """The rho ghost ring is made to match its sources in the first step after
    every upload (its sources never change afterwards): an input whose ring
    does not match (noise on the ring) must give the plain path's rho, also
    after a second upload once the step has been captured as a graph."""
    cfg = CONFIGS["tiny"]()
    phi, rho, lum, ecm = cfg.initial_state()
    rng = np.random.default_rng(5)
    rho = rho.copy()
    for k in range(rho.shape[0]):
        rho[k, 0, :] = rng.random(rho.shape[2])
        rho[k, -1, :] = rng.random(rho.shape[2])
        rho[k, :, 0] = rng.random(rho.shape[1])
        rho[k, :, -1] = rng.random(rho.shape[1])
    out = {}
    for name, path in (("fused", capi.PATH_FUSED), ("plain", capi.PATH_PLAIN)):
        with capi.Simulation(cfg.params(), 64, path) as sim:
            sim.upload(phi, rho, lum, ecm)
            sim.step(0, 3)
            first = sim.download()
            sim.upload(phi, rho, lum, ecm)      # again, after the graph exists
            sim.step(0, 2)
            out[name] = (first, sim.download())
    for a, b in zip(out["fused"], out["plain"]):
        for x, y in zip(a, b):
            assert rel_linf(x, y) <= 1e-9


def test_zone_at_the_ghost_ring():
    """A cell whose zone starts at row and column 1, so that its zone's ring
    covers the grid's ghost row and column 0: the normals there follow the
    periodic ghost map (useful_functions.cpp:391-420) through the fused
    kernels' global-memory branch.  Fused FP64 against plain FP64, and the
    FP32 areas against them, over 3 steps."""
    from multicellular_phase_field_active_gel_organoids_b200.params import OrganoidConfig
    cfg = OrganoidConfig("edge", 64, np.array([(18.4, 18.4), (42.0, 44.0)]), 8.0, 17, 0, 3)
    a = run_gpu(cfg, 3, 64, capi.PATH_FUSED)
    b = run_gpu(cfg, 3, 64, capi.PATH_PLAIN)
    assert int(b["xc"][0]) - 17 == 1 and int(b["yc"][0]) - 17 == 1, (b["xc"], b["yc"])
    assert np.array_equal(a["xc"], b["xc"]) and np.array_equal(a["yc"], b["yc"])
    assert np.array_equal(a["iters"], b["iters"])
    for k in ("phi", "rho", "lum", "ECM"):
        assert rel_linf(a[k], b[k]) <= 1e-9, (k, rel_linf(a[k], b[k]))
    assert rel_linf(a["s"], b["s"]) <= 1e-10
    f = run_gpu(cfg, 3, 32, capi.PATH_FUSED)
    assert np.array_equal(f["xc"], b["xc"])
    assert rel_linf(f["s"], b["s"]) <= 1e-4
    assert rel_linf(f["phi"], b["phi"]) <= 1e-3


def test_box_not_a_power_of_two():
    """zone_size 13 gives an FFT box of 24: the fused path's Bluestein
    spectral passes (inner length 64).  Fused FP64 against plain FP64 (fields, areas, velocity)
    over 3 steps, and the FP32 areas against them."""
    from multicellular_phase_field_active_gel_organoids_b200.params import small_organoid
    cfg = small_organoid(zone_size=13)
    a = run_gpu(cfg, 3, 64, capi.PATH_FUSED, velocity=True)
    b = run_gpu(cfg, 3, 64, capi.PATH_PLAIN, velocity=True)
    assert np.array_equal(a["xc"], b["xc"]) and np.array_equal(a["iters"], b["iters"])
    for k in ("phi", "rho", "lum", "ECM"):
        assert rel_linf(a[k], b[k]) <= 1e-9, (k, rel_linf(a[k], b[k]))
    assert rel_linf(a["s"], b["s"]) <= 1e-10
    for va, vb in zip(a["velocity"], b["velocity"]):
        assert rel_linf(va, vb) <= 1e-9
    f = run_gpu(cfg, 3, 32, capi.PATH_FUSED)
    assert np.array_equal(f["xc"], b["xc"])
    assert rel_linf(f["s"], b["s"]) <= 1e-4


def test_default_zone_size_200():
    """The reference's default zone_size 200: zones 400 columns wide (a
    reshaping thread takes several columns) and an FFT box of 398 (Bluestein
    spectral passes, inner length 1024), on a 512^2 grid with three cells.  Fused FP64 against
    plain FP64 over 2 steps, and the FP32 areas against them."""
    from multicellular_phase_field_active_gel_organoids_b200.params import OrganoidConfig
    pts = np.array([(256.0, 256.0), (294.0, 256.0), (237.0, 289.0)])
    cfg = OrganoidConfig("wide", 512, pts, 20.0, 200, 0, 2)
    a = run_gpu(cfg, 2, 64, capi.PATH_FUSED)
    b = run_gpu(cfg, 2, 64, capi.PATH_PLAIN)
    assert np.array_equal(a["xc"], b["xc"]) and np.array_equal(a["iters"], b["iters"])
    for k in ("phi", "rho", "lum", "ECM"):
        assert rel_linf(a[k], b[k]) <= 1e-9, (k, rel_linf(a[k], b[k]))
    assert rel_linf(a["s"], b["s"]) <= 1e-10
    f = run_gpu(cfg, 2, 32, capi.PATH_FUSED)
    assert np.array_equal(f["xc"], b["xc"])
    assert rel_linf(f["s"], b["s"]) <= 1e-4
