"""A sweep on one GPU (sweep.Sweep, one graph launch per step over every
member): three members of the `tiny` organoid with different friction, eta
and cell count advanced together match the reference's own FP64 run of each
member (relative L-inf 1e-9, areas 1e-10, centres exact), end in exactly the
state each reaches alone, and Sweep.run writes each member's files and
parameter file into the reference's folder layout."""
import os

import numpy as np
import pytest

from multicellular_phase_field_active_gel_organoids_b200 import capi, fileio, sweep
from multicellular_phase_field_active_gel_organoids_b200.params import small_organoid

from oracle import refrun
from tests.shape import rel

pytestmark = pytest.mark.gpu

MEMBERS = [{"ncells": 3, "friction": 1.0, "eta": 0.03}, {"ncells": 3, "friction": 2.0, "eta": 0.05},
           {"ncells": 2, "friction": 1.0, "eta": 0.03}]


def test_sweep_members_equal_solo_runs(tmp_path):
    cfg = small_organoid()
    base = cfg.params()
    init = cfg.initial_state(np.float32)
    with sweep.Sweep(MEMBERS, base, init, precision=32) as sw:
        sw.step(0, 4)
        together = sw.states()
    for m, got in zip(MEMBERS, together):
        p = sweep.member_params(m, base)
        n = m["ncells"]
        with capi.Simulation(p, 32, capi.PATH_FUSED) as sim:
            sim.upload(init[0][:n], init[1][:n], init[2], init[3])
            sim.step(0, 4)
            solo = sim.download()
        for a, b in zip(got, solo):
            np.testing.assert_array_equal(a, b)
    with sweep.Sweep(MEMBERS, base, init, precision=32) as sw:
        dirs = sw.run(str(tmp_path), nsteps=3, nsaving=2)
    for d, m in zip(dirs, MEMBERS):
        assert os.path.exists(os.path.join(d, "constants.txt"))
        phi, rho, lum, ecm = fileio.read_state_files(d, m["ncells"], 64, 32)
        assert phi.shape == (m["ncells"], 64, 64) and np.isfinite(phi).all()


def test_sweep_members_match_reference():
    cfg = small_organoid()
    base = cfg.params()
    init = cfg.initial_state(np.float64)
    refs = [refrun.run_reference(sweep.member_params(m, base),
                                 (init[0][:m["ncells"]], init[1][:m["ncells"]], init[2], init[3]), 4)
            for m in MEMBERS]
    with sweep.Sweep(MEMBERS, base, init, precision=64, relax_cap=100000) as sw:
        assert sw.batch is not None
        sw.step(0, 4)
        got = [(s.download(), s.areas()[0], s.centres()) for s in sw.sims]
    for m, ref, (state, s_area, (xc, yc)) in zip(MEMBERS, refs, got):
        assert np.array_equal(xc, ref["xc"]) and np.array_equal(yc, ref["yc"]), m
        for a, k in zip(state, ("phi", "rho", "lum", "ECM")):
            assert rel(a, ref[k]) <= 1e-9, (m, k, rel(a, ref[k]))
        assert rel(s_area, ref["s"]) <= 1e-10, m
