"""Sweep expansion and member parameter sets (sweep.py), on the CPU.

The member lists must equal, in order, what the reference's own expansion
(main_code/setup_simulation.py:17-47) produces for the same dictionaries
(tests/golden/sweep_expand.json, made by tests/golden/make_sweep_golden.py),
and a member's parameter set must carry its placeholder values under the
constants_template.cpp names, with the template's derived values recomputed."""
import json
import os

import numpy as np

from multicellular_phase_field_active_gel_organoids_b200 import sweep
from multicellular_phase_field_active_gel_organoids_b200.params import small_organoid

HERE = os.path.dirname(os.path.abspath(__file__))


def test_expand_matches_reference_order():
    cases = json.load(open(os.path.join(HERE, "golden", "sweep_expand.json")))
    for case in cases:
        d = {k: (np.array(v) if isinstance(v, list) else v) for k, v in case["input"].items()}
        got = [{k: float(v) for k, v in m.items()} for m in sweep.expand(d)]
        assert got == case["members"]


def test_member_params_mapping():
    base = small_organoid().params()
    p = sweep.member_params({"ncells": 2.0, "gen_ap": 3.0, "a_ort_lat": 50.0, "epsilon_lat": 2.0, "xi_lumen": 0.3},
                            base)
    assert p["N_ini"] == 2 and p["Ntot"] == 2 and p["N_current"] == 2
    assert p["matgenrate_apical"] == 3.0 and p["matgenrate_basal"] == 3.0      # basal = apical (:74)
    assert p["a_ort_lateral"] == 50.0 and p["a_tan_lateral"] == 100.0          # a_tan = a_ort * epsilon (:61)
    assert p["xi_lum"] == 0.3
    assert p["N_s"] == base["N_s"] and p["zone_size"] == base["zone_size"]


def test_member_dirs_reference_names(tmp_path):
    import datetime
    d = sweep.member_dirs(3, str(tmp_path), datetime.date(2022, 6, 6))
    assert [os.path.basename(x) for x in d] == ["2022_06_06_0", "2022_06_06_1", "2022_06_06_2"]
