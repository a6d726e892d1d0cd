"""Parameter set of the time step and the seeded organoid configurations.

The parameter names, defaults and derivation rules mirror the reference's
functions/constants_template.cpp:4-129 (the drop-in parameter set), with the
jinja2 placeholders filled by the values main_code/setup_simulation.py:15 uses
(ncells=6, epsilon_*=1, a_ort_*=100, b_*=1, gen_ap=1, deg_ap=100,
viscosity_*=1, friction=1, eta=0.03, xi_lumen=0.15, eta_lum_cells=0,
alpha_ECM=0.002, eta_ecm_cells=0.001).

Organoid configurations are in grid units (dx = 1), so the interface width wi,
the reference radius R0 = R and the target area s0 are rescaled per
configuration: wi = sqrt(2), R0 = R = cell radius, s0 = pi R^2.  The
reshaping relaxation's 1-D equilibrium is a logistic of width wi/sqrt(2), so
with wi = sqrt(2) the initial profile 0.5 (1 - tanh((r - R)/2)) =
1 / (1 + exp(r - R)) is that equilibrium (the reference's own logistic
profile, initialisation_functions.cpp:135).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# constants_template.cpp defaults, placeholders from setup_simulation.py:15
TEMPLATE_DEFAULTS: dict[str, float] = {
    "threshold_reshaping_steps": 100000, "riprint": 100000, "rdev_threshold": 5,
    "Nsteps": 11, "ncontinue": 0, "ndisplay": 5, "nsaving": 10,
    "dx": 0.01, "dt": 0.002, "N_s": 1200, "L": 120,
    "R0": 1.0, "sigma": 0.2, "N_ini": 6, "zone_size": 200, "Rint": 1.0,
    "coupling_PF_AG": 1.0, "seuil_gel": 0.1, "gen_ontime": 0, "active_gel_ontime": 0,
    "contract_ontime": 0,
    "epsilon_ap": 1.0, "epsilon_bas": 1.0, "epsilon_lat": 1.0,
    "a_ort_lateral": 100.0, "a_ort_apical": 100.0, "a_ort_basal": 100.0,
    "b_ap": 1.0, "b_bas": 1.0, "b_lat": 1.0,
    "matgenrate_apical": 1.0, "degrate_apical": 100.0,
    "matgenrate_lateral": 1.0, "degrate_lateral": 100.0,
    "friction": 1.0, "viscosity_ap": 1.0, "viscosity_bas": 1.0, "viscosity_lat": 1.0,
    "tau": 1.0, "alpha": 1.0, "beta": 1.0, "eta": 0.03,
    "tau_lum": 1.0, "beta_lum_cells": 1.0, "eta_lum_cells": 0.0, "xi_lum": 0.15,
    "alpha_ECM": 0.002, "tau_ECM": 1.0, "beta_ECM_cells": 1.0, "eta_ECM_cells": 0.001,
    "xi_ECM": 0.0, "beta_lum_ECM": 1.0,
    "wi": 0.07, "rho0": 0.001, "tol": 0.01, "rimax": 1000000, "rtol": 0.001, "rdt": 0.001,
}

INT_KEYS = {"threshold_reshaping_steps", "riprint", "rdev_threshold", "rdev_ini", "Nsteps",
            "ncontinue", "ndisplay", "nsaving", "Ntotsave", "N_s", "L", "N_ini", "Ntot",
            "N_current", "zone_size", "random_ontime", "gen_ontime", "active_gel_ontime",
            "contract_ontime", "rimax"}


def derive(base: dict[str, float]) -> dict[str, float]:
    """Fill the derived values exactly as constants_template.cpp computes them."""
    p = dict(TEMPLATE_DEFAULTS)
    p.update(base)
    p.setdefault("R", p["R0"])                                         # :26
    p.setdefault("s0", 3.14159265359 * p["R0"] * p["R0"] + 0.01)      # :27
    p["Ntot"] = p["N_ini"]                                             # :35
    p["N_current"] = p.get("N_current", p["N_ini"])                    # :36
    p["Ntotsave"] = 1 + (int(p["Nsteps"]) - 1) // int(p["nsaving"])   # :14
    p["random_ontime"] = int(p["Nsteps"]) + 1                          # :45
    p["rdev_ini"] = 2 * int(p["rdev_threshold"])                       # :7
    p["Rout"] = math.sqrt(p["Rint"] ** 2 + p["N_ini"] * p["s0"] / 3.14159265359)  # :29
    p["a_tan_lateral"] = p["a_ort_lateral"] * p["epsilon_lat"]        # :61
    p["a_tan_apical"] = p["a_ort_apical"] * p["epsilon_ap"]           # :62
    p["a_tan_basal"] = p["a_ort_basal"] * p["epsilon_bas"]            # :63
    p.setdefault("matgenrate_basal", p["matgenrate_apical"])          # :74
    p.setdefault("degrate_basal", p["degrate_apical"])                # :75
    p["gamma_cell"] = p["eta"] * 1.5                                  # :88
    p["gamma_lum_cells"] = p["eta_lum_cells"] * 1.1                   # :94
    p["gamma_ECM_cells"] = p["eta_ECM_cells"] * 1.1                   # :102
    for k in INT_KEYS:
        if k in p:
            p[k] = int(p[k])
    return p


def write_param_file(p: dict[str, float], path: str) -> None:
    """Key/value file read by the oracle builds of the reference (PFAG_REF_PARAMS)."""
    with open(path, "w") as f:
        for k in sorted(p):
            v = p[k]
            f.write(f"{k} {int(v)}\n" if k in INT_KEYS else f"{k} {float(v)!r}\n")


@dataclass
class OrganoidConfig:
    """A seeded organoid: grid, cells, zone, parameters and initial fields."""
    name: str
    N: int
    centres: np.ndarray            # (Ntot, 2) float, grid coordinates (i, j)
    radius: float
    zone_size: int
    seed: int = 0
    steps: int = 1000
    overrides: dict = field(default_factory=dict)

    @property
    def ncells(self) -> int:
        return int(self.centres.shape[0])

    @property
    def box(self) -> int:
        return 2 * self.zone_size - 2

    def params(self) -> dict[str, float]:
        base = {
            "N_s": self.N, "N_ini": self.ncells, "zone_size": self.zone_size,
            "dx": 1.0, "dt": 1e-3, "R0": self.radius, "wi": math.sqrt(2.0),
            "s0": math.pi * self.radius ** 2, "alpha_ECM": 0.002 * 1e-4, "rdev_threshold": 50000,
            "Nsteps": self.steps + 1, "nsaving": max(self.steps, 1),
            "ndisplay": 1 << 30,      # silences the reference's per-step stderr reports
        }
        base.update(self.overrides)
        return derive(base)

    def initial_state(self, dtype=np.float64):
        """phi, rho (Ntot, N, N), lum, ECM (N, N), built in float64 then cast."""
        N, n = self.N, self.ncells
        ii, jj = np.meshgrid(np.arange(N, dtype=np.float64), np.arange(N, dtype=np.float64),
                             indexing="ij")
        phi = np.empty((n, N, N), dtype=np.float64)
        for c, (ci, cj) in enumerate(self.centres):
            r = np.sqrt((ii - ci) ** 2 + (jj - cj) ** 2)
            phi[c] = 0.5 * (1.0 - np.tanh((r - self.radius) / 2.0))
        rng = np.random.default_rng(self.seed)
        noise = rng.uniform(-1.0, 1.0, size=(n, N, N))
        rho = np.where((phi > 0.05) & (phi < 0.95), 1.0, 0.0) * (1.0 + 0.01 * noise)
        lum = np.zeros((N, N), dtype=np.float64)
        cc = self.centres.mean(axis=0)
        r_env = np.sqrt(((self.centres - cc) ** 2).sum(axis=1)).max() + self.radius + 2.0
        r = np.sqrt((ii - cc[0]) ** 2 + (jj - cc[1]) ** 2)
        ecm = 0.5 * (1.0 + np.tanh((r - r_env) / 2.0))
        return (phi.astype(dtype), rho.astype(dtype), lum.astype(dtype), ecm.astype(dtype))


def hex_ring_organoid(name="cfg0", N=256, radius=20.0, spacing=38.0, zone_size=65, steps=1000,
                      seed=0) -> OrganoidConfig:
    """One central disc plus a hexagonal ring of six (the 7-cell organoid)."""
    c = N / 2.0
    pts = [(c, c)] + [(c + spacing * math.cos(k * math.pi / 3), c + spacing * math.sin(k * math.pi / 3))
                      for k in range(6)]
    return OrganoidConfig(name, N, np.array(pts), radius, zone_size, seed, steps)


def jittered_hex_organoid(name="cfg1", N=1024, ncells=64, radius=24.0, spacing=48.0, clip=220.0,
                          jitter=3.0, zone_size=129, steps=10000, seed=0) -> OrganoidConfig:
    """Discs on a jittered hexagonal lattice clipped to a circle: the `ncells`
    lattice points nearest the grid centre (all within `clip`), each moved by
    U(-jitter, jitter) in both coordinates (numpy default_rng(seed))."""
    c = N / 2.0
    pts = []
    kmax = int(clip / spacing) + 2
    for a in range(-kmax, kmax + 1):
        for b in range(-kmax, kmax + 1):
            x = spacing * (a + 0.5 * b)
            y = spacing * (math.sqrt(3.0) / 2.0) * b
            if x * x + y * y <= clip * clip:
                pts.append((x, y))
    pts.sort(key=lambda q: (q[0] ** 2 + q[1] ** 2, q[0], q[1]))
    if len(pts) < ncells:
        raise ValueError("lattice too sparse for the requested cell count")
    pts = np.array(pts[:ncells]) + c
    rng = np.random.default_rng(seed + 1000)
    pts = pts + rng.uniform(-jitter, jitter, size=pts.shape)
    return OrganoidConfig(name, N, pts, radius, zone_size, seed, steps)


def small_organoid(name="tiny", N=64, radius=8.0, zone_size=17, steps=10, seed=0) -> OrganoidConfig:
    """Three touching discs on a 64x64 grid: the golden-fixture case."""
    c = N / 2.0
    d = 2.0 * radius - 1.0
    pts = [(c + d * math.cos(2 * math.pi * k / 3) * 0.6, c + d * math.sin(2 * math.pi * k / 3) * 0.6)
           for k in range(3)]
    return OrganoidConfig(name, N, np.array(pts), radius, zone_size, seed, steps)


def ring_params(N: int = 96, ncells: int = 6, radius: float = 8.0, zone_size: int = 17) -> dict:
    """Parameter set of the reference's initial-condition program
    (initialisation_code/prepare_initial_files.cpp): `ncells` cells of radius
    `radius` (R0 = R) that it places on a ring of radius ncells*0.9*R/dx/pi,
    in grid units with the same rescaling as the configurations above; two
    snapshot slots (before and after the shaping)."""
    return derive({"N_s": N, "N_ini": ncells, "zone_size": zone_size, "dx": 1.0, "dt": 1e-3, "R0": radius,
                   "wi": math.sqrt(2.0), "s0": math.pi * radius ** 2, "alpha_ECM": 0.002 * 1e-4,
                   "rdev_threshold": 50000, "Nsteps": 2, "nsaving": 1, "ndisplay": 1 << 30})


CONFIGS = {
    "cfg0": lambda: hex_ring_organoid(),
    "cfg1": lambda: jittered_hex_organoid(),
    # the same organoid with the reference's default zone_size (200: FFT box 398)
    "cfg1z200": lambda: jittered_hex_organoid(name="cfg1z200", zone_size=200),
    "tiny": lambda: small_organoid(),
}
