"""The reference's own main, linked against the drop-in libraries, on the GPU.

oracle/_ref/dropin_main_fp{64,32} is main_code/run_with_active_gels.cpp with
its host files, built from the reference sources, whose step functions are
dropin/libpfag_dropin_fp{64,32}.so over the B200 library.  It reads
ini_*.bin files written by fileio.py, runs the `tiny` organoid (64x64, 3
cells, zone_size 17) for 5 steps and writes its snapshot files; they must
match the reference's own 5-step state (tests/golden/tiny_ref_fp64.npz):
relative L-inf 1e-9 in FP64, through both drop-in paths (per-function
kernels, and the fused step run by find_centres_cells).  The FP32 drop-in
(fused) is held to 1e-4 absolute on phi and rho against the reference's
FP32 run (tests/golden/tiny_ref_fp32.npz).
"""
import os
import tempfile

import numpy as np
import pytest

from multicellular_phase_field_active_gel_organoids_b200.params import small_organoid
from oracle import refrun

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _run(prec, path):
    binary = refrun.main_binary("dropin_main", prec)
    if not os.path.exists(binary):
        pytest.skip("drop-in main not built (build() with the reference checkout present)")
    cfg = small_organoid(steps=5)
    dt = np.float64 if prec == "fp64" else np.float32
    with tempfile.TemporaryDirectory() as d:
        (phi, rho, lum, ecm), err = refrun.run_main_binary(binary, cfg.params(), cfg.initial_state(dt), d,
                                                           env={"PFAG_DROPIN_PATH": path})
    assert "pfag drop-in" not in err
    return phi, rho, lum, ecm


@pytest.mark.parametrize("path", ["plain", "fused"])
def test_dropin_main_fp64_matches_reference(path):
    g = np.load(os.path.join(HERE, "golden", "tiny_ref_fp64.npz"))
    phi, rho, lum, ecm = _run("fp64", path)
    for name, a in (("phi", phi), ("rho", rho), ("lum", lum), ("ECM", ecm)):
        assert _rel(a, g[name]) <= 1e-9, (path, name, _rel(a, g[name]))


def test_dropin_main_fp32_fused_close_to_reference_fp32():
    g = np.load(os.path.join(HERE, "golden", "tiny_ref_fp32.npz"))
    phi, rho, lum, ecm = _run("fp32", "fused")
    assert np.abs(phi - g["phi"]).max() <= 1e-4
    assert np.abs(rho - g["rho"]).max() <= 1e-4
