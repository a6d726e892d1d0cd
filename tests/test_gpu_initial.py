"""The initial-condition generator on the GPU (pfag_generate_initial,
initial.py) against the reference's own initial-condition program
(initialisation_code/prepare_initial_files.cpp built on the host,
oracle/_ref/ref_prepare_fp{64,32}) on the same parameter set: six cells of
radius 8 on the program's ring in a 96^2 grid.  The files the reference
writes (ini_*.bin) are compared with what the generator writes through
initial.prepare_initial_files."""
import os
import tempfile

import numpy as np
import pytest

from multicellular_phase_field_active_gel_organoids_b200 import fileio, initial
from multicellular_phase_field_active_gel_organoids_b200.params import ring_params
from oracle import refrun

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _reference(prec):
    binary = refrun.main_binary("ref_prepare", prec)
    if not os.path.exists(binary):
        pytest.skip("reference initial-condition program not built")
    with tempfile.TemporaryDirectory() as d:
        return refrun.run_prepare_binary(binary, ring_params(), d)


def _ours(precision):
    with tempfile.TemporaryDirectory() as d:
        initial.prepare_initial_files(d, ring_params(), precision, text=True)
        assert os.path.exists(os.path.join(d, "data_ini_to_plot", "ini_cell_1.dat"))
        return fileio.read_state_files(d, 6, 96, precision)


def test_generator_fp64_matches_reference():
    ref = _reference("fp64")
    got = _ours(64)
    for name, a, b in zip(("phi", "rho", "lum", "ECM"), got, ref):
        assert _rel(a, b) <= 1e-9, (name, _rel(a, b))


def test_generator_fp32_close_to_reference_fp32():
    ref = _reference("fp32")
    got = _ours(32)
    for name, a, b in zip(("phi", "rho", "lum", "ECM"), got, ref):
        assert np.abs(np.asarray(a, np.float64) - b).max() <= 1e-4 * max(np.abs(b).max(), 1e-3), name
