"""Cell sharding on the GPU: the organoid's cells split over 2 and 3
fused-path contexts on one device (sharded.LocalShards: psi summed over the
shards and the neighbour planes copied between the parts of each step)
against the reference's own FP64 run (oracle/_ref) and against the
unsharded fused step; the torch.distributed form (sharded.DistShard) on one
rank; the split step's error behaviour."""
import numpy as np
import pytest

from multicellular_phase_field_active_gel_organoids_b200 import capi, sharded
from multicellular_phase_field_active_gel_organoids_b200.params import hex_ring_organoid, small_organoid
from oracle import refrun
from tests.shape import rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cfg0_ref4():
    cfg = hex_ring_organoid()
    return cfg, refrun.run_reference(cfg.params(), cfg.initial_state(), 4)


def _check_against(ref, sh, tol_fields=1e-9, tol_areas=1e-10):
    phi, rho, lum, ecm = sh.download()
    xc, yc = sh.centres()
    assert np.array_equal(xc, ref["xc"]) and np.array_equal(yc, ref["yc"])
    errs = {"phi": rel(phi, ref["phi"]), "rho": rel(rho, ref["rho"]), "lum": rel(lum, ref["lum"]),
            "ECM": rel(ecm, ref["ECM"]), "s": rel(sh.areas(), ref["s"])}
    print(errs)
    assert max(errs[k] for k in ("phi", "rho", "lum", "ECM")) <= tol_fields, errs
    assert errs["s"] <= tol_areas, errs
    # every shard updates lum and ECM from the same psi: identical copies
    for k in range(1, len(sh.sims)):
        _, _, l2, e2 = sh.fields(k)
        assert np.array_equal(l2, lum) and np.array_equal(e2, ecm)


@pytest.mark.parametrize("nshards", [2, 3])
def test_shards_match_reference_fp64(cfg0_ref4, nshards):
    cfg, ref = cfg0_ref4
    with sharded.LocalShards(cfg.params(), cfg.initial_state(np.float64), nshards, precision=64,
                             relax_cap=100000) as sh:
        sh.step(0, 4)
        _check_against(ref, sh)


def test_one_cell_per_shard_matches_reference():
    """Three cells, three shards: both neighbour planes of every shard come from other shards."""
    cfg = small_organoid()
    p = cfg.params()
    assert int(p["Ntot"]) == 3
    ref = refrun.run_reference(p, cfg.initial_state(), 4)
    with sharded.LocalShards(p, cfg.initial_state(np.float64), 3, precision=64, relax_cap=100000) as sh:
        sh.step(0, 4)
        _check_against(ref, sh)


def test_shards_on_bluestein_boxes():
    """The reference's default zone_size 200 (FFT box 398: the Bluestein
    passes, whose stress kernel reads the neighbour planes) on a 512^2 grid
    with three cells, one per shard: FP64 against the unsharded fused step
    after 2 steps (psi summed in another grouping: rounding only)."""
    from multicellular_phase_field_active_gel_organoids_b200.params import OrganoidConfig
    pts = np.array([(256.0, 256.0), (294.0, 256.0), (237.0, 289.0)])
    cfg = OrganoidConfig("wide", 512, pts, 20.0, 200, 0, 2)
    init = cfg.initial_state(np.float64)
    with capi.Simulation(cfg.params(), 64, capi.PATH_FUSED) as s:
        s.set_relax_cap(100000)
        s.upload(*init)
        s.step(0, 2)
        one = s.download()
        a1 = s.areas()[0]
        c1 = s.centres()
    with sharded.LocalShards(cfg.params(), init, 3, precision=64, relax_cap=100000) as sh:
        sh.step(0, 2)
        got = sh.download()
        assert rel(sh.areas(), a1) <= 1e-12
        xc, yc = sh.centres()
    assert np.array_equal(xc, c1[0]) and np.array_equal(yc, c1[1])
    for a, b in zip(got, one):
        assert rel(a, b) <= 1e-12


def test_shards_fp32_close_to_unsharded():
    """FP32: psi summed per shard then over shards rounds differently from one running sum."""
    cfg = hex_ring_organoid()
    init = cfg.initial_state(np.float32)
    with capi.Simulation(cfg.params(), 32, capi.PATH_FUSED) as s:
        s.upload(*init)
        s.step(0, 6)
        one = s.download()
        a1 = s.areas()[0]
    with sharded.LocalShards(cfg.params(), init, 3, precision=32) as sh:
        sh.step(0, 3)
        sh.step(3, 3)               # the parts replay their graphs from the second step on
        assert all(s.launch_count() > 0 for s in sh.sims)
        got = sh.download()
        a3 = sh.areas()
    assert rel(a3, a1) <= 1e-5
    assert np.abs(got[0] - one[0]).max() <= 1e-4
    assert np.abs(got[1] - one[1]).max() <= 1e-4 * max(1.0, float(np.abs(one[1]).max()))


def test_dist_shard_one_rank_equals_unsharded(tmp_path):
    """DistShard on a one-rank NCCL group: the halo is the shard's own planes
    and psi needs no sum, so the split step equals the whole step bit for bit."""
    import torch
    import torch.distributed as dist
    cfg = small_organoid()
    init = cfg.initial_state(np.float32)
    with capi.Simulation(cfg.params(), 32, capi.PATH_FUSED) as s:
        s.upload(*init)
        s.step(0, 5)
        whole = s.download()
    dist.init_process_group("nccl", init_method=f"file://{tmp_path}/rdv", rank=0, world_size=1,
                            device_id=torch.device("cuda", 0))
    try:
        with sharded.DistShard(cfg.params(), init, precision=32) as sh:
            sh.step(0, 2)
            sh.step(2, 3)
            got = sh.sim.download()
    finally:
        dist.destroy_process_group()
    for a, b in zip(got, whole):
        assert np.array_equal(a, b)


def test_split_step_errors():
    cfg = small_organoid()
    with capi.Simulation(cfg.params(), 64, capi.PATH_FUSED) as s:
        s.upload(*cfg.initial_state(np.float64))
        with pytest.raises(capi.PfagError) as e:
            s.step_tail(0)                      # no head
        assert e.value.code == -1               # PFAG_E_ARG
        s.step_head(0)
        with pytest.raises(capi.PfagError):
            s.step_head(0)                      # head twice
        with pytest.raises(capi.PfagError):
            s.step(0, 1)                        # whole step between the parts
        s.step_tail(0)
        s.sync()
        s.step(1, 1)
    with capi.Simulation(cfg.params(), 64, capi.PATH_PLAIN) as s:
        with pytest.raises(capi.PfagError) as e:
            s.shard_enable()
        assert e.value.code == -5               # PFAG_E_UNSUPPORTED
