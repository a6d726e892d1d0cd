"""The batched sweep engine on the GPU: members stepped as one graph per step
against the reference's own FP64 run of each member (oracle/_ref), against
their solo runs, the device-side organoid generator against the host
formula, and the autotuner's cache."""
import json

import numpy as np
import pytest

from multicellular_phase_field_active_gel_organoids_b200 import batched as B
from multicellular_phase_field_active_gel_organoids_b200 import capi
from oracle import refrun
from tests.shape import rel

pytestmark = pytest.mark.gpu


def small_members(k=3):
    """The first k members of the seeded sweep on a 256^2 grid with distinct boxes."""
    out, seen = [], set()
    for m in B.sweep_members(256, seed=1):
        if m.N == 256 and m.box not in seen and m.ncells >= 2:
            out.append(m)
            seen.add(m.box)
        if len(out) == k:
            break
    return out


def test_batched_members_match_reference():
    """FP64 members (host generator inputs) advanced 4 steps as one batch
    against the reference's FP64 run of each: relative L-inf 1e-9 on phi, rho,
    lumen and ECM, areas 1e-10, centres exact."""
    ms = small_members(3)
    assert len(ms) >= 2
    refs = {m.index: refrun.run_reference(m.config().params(), m.config().initial_state(), 4) for m in ms}
    with B.BatchedSweep(ms, precision=64, relax_cap=100000, host_init=True) as sw:
        sw.step(0, 4)
        for m in ms:
            s = sw.member_sim(m.index)
            phi, rho, lum, ecm = s.download()
            xc, yc = s.centres()
            r = refs[m.index]
            assert np.array_equal(xc, r["xc"]) and np.array_equal(yc, r["yc"]), m.index
            errs = {"phi": rel(phi, r["phi"]), "rho": rel(rho, r["rho"]), "lum": rel(lum, r["lum"]),
                    "ECM": rel(ecm, r["ECM"]), "s": rel(s.areas()[0], r["s"])}
            print(m.index, m.box, m.ncells, errs)
            assert max(errs[k] for k in ("phi", "rho", "lum", "ECM")) <= 1e-9, errs
            assert errs["s"] <= 1e-10, errs


def test_batch_equals_solo_runs_fp32():
    """The graph replay of the batch runs exactly the members' own kernels:
    FP32 members after 6 steps equal their solo runs bit for bit."""
    ms = small_members(3)
    with B.BatchedSweep(ms, precision=32) as sw:
        sw.step(0, 6)
        got = {m.index: sw.member_sim(m.index).download() for m in ms}
        launches = sw.batch.launch_count()
    assert launches > 0
    for m in ms:
        cfg = m.config()
        with capi.Simulation(cfg.params(), 32, capi.PATH_FUSED) as s:
            s.seed_organoid(m.centres, m.radius, m.env_radius(), m.seed)
            s.step(0, 6)
            solo = s.download()
        for a, b in zip(got[m.index], solo):
            assert np.array_equal(a, b), m.index


def test_device_generator_matches_host_formula():
    m = small_members(1)[0]
    cfg = m.config()
    phi_h, rho_h, lum_h, ecm_h = cfg.initial_state(np.float64)
    with capi.Simulation(cfg.params(), 64, capi.PATH_FUSED) as s:
        s.seed_organoid(m.centres, m.radius, m.env_radius(), m.seed)
        phi, rho, lum, ecm = s.download()
    assert rel(phi, phi_h) <= 1e-14
    assert np.array_equal(lum, lum_h)
    cc = m.centres.mean(axis=0)
    r_env = np.sqrt(((m.centres - cc) ** 2).sum(axis=1)).max() + m.radius + 2.0
    assert np.isclose(m.env_radius(), r_env)
    assert rel(ecm, ecm_h) <= 1e-14
    band = (phi > 0.05) & (phi < 0.95)
    assert np.array_equal(rho != 0, band)
    assert np.all(np.abs(rho[band] - 1.0) <= 0.01 + 1e-15)


def test_autotune_writes_cache(tmp_path):
    ms = small_members(2)
    path = str(tmp_path / "shapes.json")
    shapes = B.autotune(ms, precision=32, cache_path=path, sample=2, steps=2)
    with open(path) as f:
        cache = json.load(f)
    assert set(shapes) == {m.bucket() for m in ms}
    for key, sh in shapes.items():
        assert cache[f"{key}_fp32"] == sh
        assert (sh["coop_blocks"], sh["update_warps"]) in B.SHAPES
        assert sh["lumen_tma"] in (0, 1)             # the 256^2 members can take TMA lumen tiles
    with B.BatchedSweep(ms, precision=32) as sw:
        sw.set_shapes(shapes)
        sw.step(0, 3)
