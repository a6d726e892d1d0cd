"""pfag_areas_noalloc: the allocation-free area reduction.

It exists for callers that may not allocate device memory (device memory owned
by another allocator or an OpenACC data region, or a latency-critical loop that
cannot afford cudaMalloc's device synchronisation).  This file is named so that
pytest collects it last.  The test builds the cell h-functions with the
per-function entry points, then checks that two calls in a row of the
allocation-free entry point give the areas and area forces of the existing
entry point (pfag_fn_sum_s_kernels) to relative 1e-12, and that a cell count
beyond its static scratch is refused.
"""
import ctypes

import numpy as np
import pytest

from multicellular_phase_field_active_gel_organoids_b200 import capi
from multicellular_phase_field_active_gel_organoids_b200.params import CONFIGS

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _cudart():
    capi.lib()
    rt = ctypes.CDLL("libcudart.so.12")
    rt.cudaMalloc.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t]
    rt.cudaFree.argtypes = [ctypes.c_void_p]
    rt.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    rt.cudaMemset.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t]
    rt.cudaStreamSynchronize.argtypes = [ctypes.c_void_p]
    return rt


def _noalloc():
    f = capi.lib().pfag_areas_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                  ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


@pytest.mark.parametrize("precision", [64, 32])
def test_noalloc_areas_match_existing_entry_point(precision):
    cfg = CONFIGS["tiny"]()
    p = cfg.params()
    dtype = np.float64 if precision == 64 else np.float32
    rt = _cudart()
    f = _noalloc()
    with capi.Simulation(p, precision, capi.PATH_PLAIN) as sim:
        sim.upload(*cfg.initial_state(dtype))
        sim.fn("find_centres_cells")
        sim.fn("compute_hfunc_3d_tables_kernels_loop_n")
        s_ref = np.empty(sim.ncells, np.float64)
        f0_ref = np.empty(sim.ncells, np.float64)
        sim.fn("sum_s_kernels", ctypes.c_void_p(s_ref.ctypes.data), ctypes.c_void_p(f0_ref.ctypes.data))
        hptr, count = sim.device_field("hfunc_cell")
        assert count == sim.ncells * sim.N * sim.N
        # the test, not the entry point, owns the output buffers
        d_s, d_f0 = ctypes.c_void_p(), ctypes.c_void_p()
        nbytes = 8 * sim.ncells
        assert rt.cudaMalloc(ctypes.byref(d_s), nbytes) == 0
        assert rt.cudaMalloc(ctypes.byref(d_f0), nbytes) == 0
        try:
            for call in range(2):
                rt.cudaMemset(d_s, 0xff, nbytes)
                rt.cudaMemset(d_f0, 0xff, nbytes)
                rc = f(ctypes.c_void_p(hptr), precision, sim.ncells, sim.N, p["dx"], p["alpha"], p["s0"],
                       d_s, d_f0, ctypes.c_void_p(sim.stream()))
                assert rc == 0, capi.lib().pfag_last_error().decode()
                assert rt.cudaStreamSynchronize(ctypes.c_void_p(sim.stream())) == 0
                s = np.empty(sim.ncells, np.float64)
                f0 = np.empty(sim.ncells, np.float64)
                assert rt.cudaMemcpy(ctypes.c_void_p(s.ctypes.data), d_s, nbytes, 2) == 0
                assert rt.cudaMemcpy(ctypes.c_void_p(f0.ctypes.data), d_f0, nbytes, 2) == 0
                np.testing.assert_allclose(s, s_ref, rtol=TOL, atol=0, err_msg=f"call {call}")
                np.testing.assert_allclose(f0, f0_ref, rtol=TOL, atol=TOL * np.abs(f0_ref).max(),
                                           err_msg=f"call {call}")
        finally:
            rt.cudaFree(d_s)
            rt.cudaFree(d_f0)


def test_noalloc_rejects_more_cells_than_its_scratch():
    f = _noalloc()
    dummy = ctypes.c_void_p(16)   # never dereferenced: the size check comes first
    rc = f(dummy, 64, 1025, 64, 1.0, 1.0, 1.0, dummy, dummy, None)
    assert rc == -1   # PFAG_E_ARG
    assert b"1024" in capi.lib().pfag_last_error()
