"""The C ABI library: it loads, exports every entry point include/pfag.h
declares, and reports errors (no GPU needed for these)."""
import ctypes
import os
import re

import numpy as np
import pytest

from multicellular_phase_field_active_gel_organoids_b200 import build, capi
from multicellular_phase_field_active_gel_organoids_b200.params import CONFIGS

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module", autouse=True)
def _lib():
    build.build()
    return capi.lib()


def declared_functions():
    text = open(os.path.join(ROOT, "include", "pfag.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pfag_\w+)\s*\(", text)))


def test_header_declares_the_reference_functions():
    names = declared_functions()
    for fn in ("find_centres_cells", "create_turnover_rates_tensions", "compute_hfunc_3d_tables_kernels_loop_n",
               "compute_all_hfunc_2d_tables_kernels", "compute_normal_grad_phi", "compute_prod_norm_delta",
               "compute_psi_kernels", "sum_s_kernels", "update_all_cortices", "update_lumen_and_ECM",
               "reshaping_lumen_or_ECM", "compute_normal_to_phi", "update_all_cells", "reshaping_cells",
               "saving_out_functions"):
        assert f"pfag_fn_{fn}" in names


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_covers_exports():
    declared = set(declared_functions())
    assert set(capi.EXPORTS) <= declared


def test_invalid_parameters_are_rejected_before_any_device_work():
    p = CONFIGS["tiny"]().params()
    bad = dict(p, zone_size=40)          # 2*40+2 > 64: the zone cannot fit the grid
    with pytest.raises(capi.PfagError) as e:
        capi.Simulation(bad, 64, capi.PATH_PLAIN)
    assert e.value.code == -3
    with pytest.raises(capi.PfagError):
        capi.Simulation(dict(p, friction=0.0), 64, capi.PATH_PLAIN)
    with pytest.raises(capi.PfagError):
        capi.Simulation(p, 16, capi.PATH_PLAIN)


def test_params_struct_roundtrip():
    p = CONFIGS["cfg1"]().params()
    s = capi.make_params(p)
    assert s.N_s == 1024 and s.Ntot == 64 and s.zone_size == 129
    assert abs(s.wi - np.sqrt(2.0)) < 1e-15 and s.a_tan_basal == p["a_ort_basal"] * p["epsilon_bas"]
