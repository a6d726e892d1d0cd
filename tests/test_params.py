"""Parameter derivation (constants_template.cpp rules) and the seeded configurations."""
import math

import numpy as np

from multicellular_phase_field_active_gel_organoids_b200.params import CONFIGS, derive, TEMPLATE_DEFAULTS


def test_template_derivations():
    p = derive({"Nsteps": 101, "nsaving": 10, "N_ini": 6, "R0": 2.0})
    assert p["Ntotsave"] == 11 and p["random_ontime"] == 102 and p["rdev_ini"] == 2 * p["rdev_threshold"]
    assert p["Ntot"] == 6 and p["N_current"] == 6 and p["R"] == 2.0
    assert abs(p["s0"] - (3.14159265359 * 4.0 + 0.01)) < 1e-12
    assert p["gamma_cell"] == TEMPLATE_DEFAULTS["eta"] * 1.5
    assert p["matgenrate_basal"] == p["matgenrate_apical"] and p["degrate_basal"] == p["degrate_apical"]


def test_cfg1_geometry():
    cfg = CONFIGS["cfg1"]()
    assert cfg.ncells == 64 and cfg.N == 1024 and cfg.box == 256
    r = np.sqrt(((cfg.centres - 512.0) ** 2).sum(axis=1))
    assert r.max() <= 220.0 + 3.0 * math.sqrt(2) + 1e-9
    # every zone fits the grid interior
    assert (cfg.centres.min() - cfg.zone_size - 2 >= 1) and (cfg.centres.max() + cfg.zone_size + 2 <= 1023)


def test_initial_state_is_seeded_and_in_range():
    cfg = CONFIGS["tiny"]()
    a = cfg.initial_state()
    b = cfg.initial_state()
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    phi, rho, lum, ecm = a
    assert phi.min() >= 0 and phi.max() <= 1 and np.all(lum == 0)
    assert 0.98 <= rho[rho > 0].min() and rho.max() <= 1.01
    assert ecm.min() >= 0 and ecm.max() <= 1
