"""The drop-in boundary and the reference's state files, on the CPU.

* The drop-in libraries (dropin/libpfag_dropin_fp{32,64}.so) export the
  reference's step functions with their exact C++ signatures
  (functions/useful_functions.h:10-48, rho_functions.h:10-26,
  cell_phase_functions.h:18-39) in float and in double.
* The state-file format (multicellular_phase_field_active_gel_organoids_b200/
  fileio.py) round-trips, keeps the FP32 8-byte record layout, and the
  reference's own main (oracle/_ref/ref_main_fp64, built from the reference
  sources) run on files written by it reproduces the golden 5-step state of
  the `tiny` organoid bit for bit.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from multicellular_phase_field_active_gel_organoids_b200 import build as B
from multicellular_phase_field_active_gel_organoids_b200 import fileio
from multicellular_phase_field_active_gel_organoids_b200.params import small_organoid
from oracle import refrun

HERE = os.path.dirname(os.path.abspath(__file__))

# Demangled signatures, float build; the double build has `double` for `float`
# except in the cufftComplex (float2) scratch pointers.
SIGNATURES = [
    "saving_out_functions(int, float*, float*, float*, float*, float*, float*, float*, float*)",
    "find_centres_cells(float*, int*, int*)",
    "create_turnover_rates_tensions(float*, float*, float*, float*, float*, float*, float*, float*, float*, int*, int*)",
    "compute_hfunc_3d_tables_kernels_loop_n(float*, float*, int*, int*)",
    "compute_all_hfunc_2d_tables_kernels(float*, float*, float*, float*)",
    "compute_normal_grad_phi(float*, float*)",
    "boundary_conditions_cells(float*)",
    "compute_prod_norm_delta(float*, float*, float*, int*, int*)",
    "compute_psi_kernels(float*, float*)",
    "sum_s_kernels(float*, float*, float*)",
    "update_all_cortices(float*, float*, float*, int*, int*, float*, float*, float*, float*, float*, float*, "
    "float*, float*, int, int, float2*, float2*, float2*, float2*, float2*, float2*, float2*, float2*, float2*, "
    "float2*, float2*)",
    "update_lumen_and_ECM(float*, float*, float*, float*, float*, float*, float*)",
    "boundary_conditions_lumen_and_ECM(float*, float*)",
    "reshaping_lumen_or_ECM(int, float*, float*, float)",
    "compute_normal_to_phi(float*, float*, float*, float*)",
    "update_all_cells(int, float*, float*, float*, float*, float*, float*, float*, int*, int*, float*, float*)",
    "reshaping_cells(int, float*, float*, float*, float*, float*, int*, int*)",
    "copy_cell_tables_1_by_1(int, float*, float*)",
    "copy_tables_ECM_or_lumen(float*, float*)",
]


def _exports(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", "-C", lib], capture_output=True, text=True, check=True)
    return {line.split(" ", 2)[2] for line in out.stdout.splitlines() if " T " in line}


@pytest.mark.parametrize("prec", [32, 64])
def test_dropin_exports_reference_signatures(prec):
    lib = B.dropin_lib(prec)
    if not os.path.exists(lib):
        pytest.skip("drop-in library not built")
    got = _exports(lib)
    for sig in SIGNATURES:
        want = sig if prec == 32 else sig.replace("float*", "double*").replace(
            "float)", "double)").replace("float2", "float2")
        assert want in got, f"missing {want}"


@pytest.mark.parametrize("prec", [32, 64])
def test_state_files_round_trip(prec, tmp_path):
    dt = np.float32 if prec == 32 else np.float64
    rng = np.random.default_rng(3)
    phi = rng.random((3, 8, 8)).astype(dt)
    rho = rng.random((3, 8, 8)).astype(dt)
    lum, ecm = rng.random((8, 8)).astype(dt), rng.random((8, 8)).astype(dt)
    fileio.write_state_files(str(tmp_path), phi, rho, lum, ecm, prec)
    for k in range(3):
        assert os.path.getsize(tmp_path / f"ini_cell_{k + 1}.bin") == 8 * 64
    back = fileio.read_state_files(str(tmp_path), 3, 8, prec)
    for a, b in zip((phi, rho, lum, ecm), back):
        np.testing.assert_array_equal(a, b)
    if prec == 32:
        # record k = (x[k], x[k+1]); a cell's last record carries the next cell's first value
        raw = np.fromfile(tmp_path / "ini_cell_1.bin", dtype=np.float32)
        np.testing.assert_array_equal(raw[1:-1:2], phi[0].ravel()[1:])
        assert raw[-1] == phi[1, 0, 0]


def test_text_snapshot_round_trip(tmp_path):
    t = np.random.default_rng(1).random((5, 5))
    p = str(tmp_path / "phi_cell_1_step_0.dat")
    fileio.write_text_snapshot(p, t)
    np.testing.assert_allclose(fileio.read_text_snapshot(p, 5), t, rtol=0, atol=5e-16)


def test_reference_main_reads_and_writes_our_files():
    binary = refrun.main_binary("ref_main", "fp64")
    if not os.path.exists(binary):
        pytest.skip("reference main not built (needs the reference checkout)")
    cfg = small_organoid(steps=5)
    g = np.load(os.path.join(HERE, "golden", "tiny_ref_fp64.npz"))
    with tempfile.TemporaryDirectory() as d:
        (phi, rho, lum, ecm), _ = refrun.run_main_binary(binary, cfg.params(), cfg.initial_state(np.float64), d)
    for name, a in (("phi", phi), ("rho", rho), ("lum", lum), ("ECM", ecm)):
        np.testing.assert_array_equal(a, g[name], err_msg=name)
