"""Snapshots written while the run goes on (snapshots.py over
pfag_snapshot_async / pfag_write_text_snapshot): the reference's main loop on
the `tiny` organoid for 6 iterations with nsaving 5 (snapshots before steps 0
and 5), fused FP64 path.  The final ini_*.bin files must hold the reference's
5-step state (tests/golden/tiny_ref_fp64.npz, relative L-inf 1e-9), and the
data_int text files must match, value for value, the ones the reference's own
main writes for the same run (oracle/_ref/ref_main_fp64, host build)."""
import os
import tempfile

import numpy as np
import pytest

from multicellular_phase_field_active_gel_organoids_b200 import capi, fileio, snapshots
from multicellular_phase_field_active_gel_organoids_b200.params import small_organoid
from oracle import refrun

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def _rel(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / max(np.abs(b).max(), 1e-300))


def test_async_snapshots_match_reference_files():
    cfg = small_organoid(steps=5)
    p = cfg.params()
    g = np.load(os.path.join(HERE, "golden", "tiny_ref_fp64.npz"))
    with tempfile.TemporaryDirectory() as ours, tempfile.TemporaryDirectory() as ref:
        with capi.Simulation(p, 64, capi.PATH_FUSED) as sim:
            sim.upload(*cfg.initial_state(np.float64))
            snapshots.run(sim, 6, 5, ours, text=True)
        phi, rho, lum, ecm = fileio.read_state_files(ours, 3, 64, 64)
        for name, a in (("phi", phi), ("rho", rho), ("lum", lum), ("ECM", ecm)):
            assert _rel(a, g[name]) <= 1e-9, name
        binary = refrun.main_binary("ref_main", "fp64")
        if not os.path.exists(binary):
            pytest.skip("reference main not built")
        refrun.run_main_binary(binary, p, cfg.initial_state(np.float64), ref)
        for step in (0, 5):
            names = [f"phi_cell_{k}_step_{step}.dat" for k in (1, 2, 3)] + \
                    [f"rho_cell_{k}_step_{step}.dat" for k in (1, 2, 3)] + [f"lumen_step_{step}.dat", f"ECM_step_{step}.dat"]
            for nm in names:
                a = fileio.read_text_snapshot(os.path.join(ours, "data_int", nm), 64)
                b = fileio.read_text_snapshot(os.path.join(ref, "data_int", nm), 64)
                assert np.abs(a - b).max() <= 1e-9 * max(np.abs(b).max(), 1e-300) + 1e-15, nm
