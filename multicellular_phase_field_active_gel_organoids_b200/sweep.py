"""Parameter sweeps in one process on one GPU.

The reference sweeps by expanding a dictionary of parameter arrays into one
member per combination (main_code/setup_simulation.py:29-47), rendering one
constants.cpp per member into its own folder (:66-78, :94-115) and submitting
one batch job per folder (:119-127).  Here the same expansion gives the same
members in the same order, each member's parameter set is the one its
constants.cpp would hold (written as a key/value file into the member's
folder), and all members advance together on one GPU: one context (device
state and CUDA graph) per member and, on the fused path, one graph launch per
step over every member (capi.Batch, the batched engine of batched.py), so small
organoids that do not fill the GPU alone run side by side.  Every member starts from the
same initial state files, as the reference copies the same ini_*.bin files
into every folder (:101-103); a member with N_ini cells reads the first N_ini.
"""
from __future__ import annotations

import datetime
import os

import numpy as np

from . import capi, fileio, params as P
from .snapshots import SnapshotWriter

# constants_template.cpp placeholders and the constants they set (:34-101)
PLACEHOLDERS = {
    "ncells": "N_ini", "epsilon_ap": "epsilon_ap", "epsilon_bas": "epsilon_bas", "epsilon_lat": "epsilon_lat",
    "a_ort_lat": "a_ort_lateral", "a_ort_ap": "a_ort_apical", "a_ort_bas": "a_ort_basal",
    "b_ap": "b_ap", "b_bas": "b_bas", "b_lat": "b_lat", "gen_ap": "matgenrate_apical", "deg_ap": "degrate_apical",
    "friction": "friction", "viscosity_ap": "viscosity_ap", "viscosity_bas": "viscosity_bas",
    "viscosity_lat": "viscosity_lat", "eta": "eta", "eta_lum_cells": "eta_lum_cells", "xi_lumen": "xi_lum",
    "alpha_ECM": "alpha_ECM", "eta_ecm_cells": "eta_ECM_cells",
}


def _lengths(d: dict):
    return [len(v) if isinstance(v, np.ndarray) else 0 for v in d.values()]


def expand(constants: dict) -> list[dict]:
    """The members of a sweep, in the reference's order (setup_simulation.py:29-47):
    the key whose value array is longest (as numpy's argsort ranks the lengths)
    is expanded first, value by value, and the rest recursively; keys holding a
    scalar are fixed.  Values are numpy arrays, as in the reference's dictionary."""
    out = []
    d = dict(constants)
    keys = list(d.keys())
    lens = _lengths(constants)
    first = np.argsort(lens)[::-1]
    if lens[first[0]] > 0:
        key = keys[first[0]]
        for v in constants[key]:
            d[key] = v
            if sum(_lengths(d)) == 0:
                out.append(dict(d))
            else:
                out += expand(d)
    return out


def member_params(member: dict, base: dict | None = None) -> dict:
    """The parameter set a member's constants.cpp holds: the template's fixed
    values (and `base`, e.g. the grid and zone of a configuration) with the
    member's placeholder values, derived as the template derives them."""
    p = dict(base or {})
    for k, v in member.items():
        if k not in PLACEHOLDERS:
            raise KeyError(f"{k} is not a constants_template.cpp placeholder")
        p[PLACEHOLDERS[k]] = float(v) if k != "ncells" else int(v)
    for k in ("Ntot", "N_current", "Ntotsave", "random_ontime", "rdev_ini", "Rout", "a_tan_lateral", "a_tan_apical",
              "a_tan_basal", "gamma_cell", "gamma_lum_cells", "gamma_ECM_cells", "matgenrate_basal",
              "degrate_basal"):
        p.pop(k, None)          # recomputed from the member's values
    return P.derive(p)


def member_dirs(n: int, root: str, day: datetime.date | None = None) -> list[str]:
    """Folder names of the reference: <YYYY_MM_DD>_<i> (setup_simulation.py:90-97)."""
    day = day or datetime.date.today()
    tag = "_".join(str(day).split("-"))
    return [os.path.join(root, f"{tag}_{i}") for i in range(n)]


class Sweep:
    """All members of a sweep advanced together on one GPU."""

    def __init__(self, members: list[dict], base: dict, initial, precision: int = 32,
                 path: int = capi.PATH_FUSED, relax_cap: int | None = None):
        """`initial` = (phi, rho, lum, ECM) with at least max(N_ini) cells."""
        self.params = [member_params(m, base) for m in members]
        self.sims = []
        self.batch = None
        phi, rho, lum, ecm = initial
        dtype = np.float64 if precision == 64 else np.float32
        try:
            for p in self.params:
                s = capi.Simulation(p, precision, path)
                if relax_cap:
                    s.set_relax_cap(relax_cap)
                n = int(p["N_ini"])
                s.upload(*(np.ascontiguousarray(a, dtype=dtype) for a in (phi[:n], rho[:n], lum, ecm)))
                self.sims.append(s)
            if path == capi.PATH_FUSED:
                self.batch = capi.Batch(self.sims)
        except Exception:
            self.close()
            raise

    def _step_async(self, it: int) -> None:
        if self.batch is not None:
            self.batch.step_async(it, 1)      # one graph launch over every member
        else:
            for s in self.sims:
                s.step_async(it, 1)

    def step(self, it0: int, nsteps: int = 1) -> None:
        """nsteps steps of every member."""
        for k in range(nsteps):
            self._step_async(it0 + k)
        if self.batch is not None:
            self.batch.sync()
        for s in self.sims:
            s.sync()

    def run(self, root: str, nsteps: int, nsaving: int, text: bool = False, day=None) -> list[str]:
        """The reference's main loop for every member (a snapshot at every it
        with it % nsaving == 0, then the step), each member writing its files
        into its own folder with its parameter file; returns the folders."""
        dirs = member_dirs(len(self.sims), root, day)
        writers = []
        try:
            for d, p, s in zip(dirs, self.params, self.sims):
                os.makedirs(d, exist_ok=True)
                P.write_param_file(p, os.path.join(d, "constants.txt"))
                writers.append(SnapshotWriter(s, d, text=text, slots=2))
            for it in range(nsteps):
                if it % nsaving == 0:
                    for w in writers:
                        w.save(it)
                self._step_async(it)
            if self.batch is not None:
                self.batch.sync()
            for s in self.sims:
                s.sync()
        finally:
            for w in writers:
                w.close()
        return dirs

    def states(self):
        return [s.download() for s in self.sims]

    def close(self):
        if self.batch is not None:
            self.batch.close()
            self.batch = None
        for s in self.sims:
            s.close()
        self.sims = []

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def read_initial_files(directory: str, ncells: int, N: int, precision: int):
    """The shared initial state of a sweep from a folder of ini_*.bin files."""
    return fileio.read_state_files(directory, ncells, N, precision)
