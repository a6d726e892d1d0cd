"""Initial conditions: the reference's prepare_initial_files program on the GPU.

initialisation_code/prepare_initial_files.cpp builds the organoid a run
starts from: N_ini cells on a ring (logistic profiles), lumen inside the ring
and ECM outside in the space the cells leave, a cortex density from each
cell's phase, then one pass of the step's shaping (the cells' reshaping
loops, rho refitted to the reshaped cells, the lumen/ECM update and reshaping)
and writes ini_cell_k.bin, ini_rho_k.bin, ini_lumen.bin, ini_ECM.bin (plus
text copies under data_ini_to_plot/).  `generate()` runs the same sequence
through pfag_generate_initial on the device and returns the state;
`prepare_initial_files()` also writes the files, byte-compatible with the
reference's (the run program reads them back).
"""
from __future__ import annotations

import os

import numpy as np

from . import capi, fileio


def generate(params: dict, precision: int = 64, rho0: float | None = None, tol: float | None = None):
    """(phi, rho, lum, ECM) of the reference's snapshot slot 1 after the shaping.
    rho0 and tol default to the parameter set's values (constants_template.cpp)."""
    rho0 = float(params.get("rho0", 0.001) if rho0 is None else rho0)
    tol = float(params.get("tol", 0.01) if tol is None else tol)
    with capi.Simulation(params, precision, capi.PATH_PLAIN) as sim:
        sim.generate_initial(rho0, tol, make_fields=True)
        return sim.download()


def prepare_initial_files(directory: str, params: dict, precision: int = 64, rho0: float | None = None,
                          tol: float | None = None, text: bool = False):
    """generate() and write its state as the reference's ini_*.bin files in
    `directory` (and, with `text`, data_ini_to_plot/ini_cell_k.dat etc. in the
    reference's "%lg" layout).  Returns the state."""
    phi, rho, lum, ecm = generate(params, precision, rho0, tol)
    fileio.write_state_files(directory, phi, rho, lum, ecm, precision)
    if text:
        d = os.path.join(directory, "data_ini_to_plot")
        os.makedirs(d, exist_ok=True)
        for k in range(phi.shape[0]):
            _write_lg(os.path.join(d, f"ini_cell_{k + 1}.dat"), phi[k])
            _write_lg(os.path.join(d, f"ini_rho_{k + 1}.dat"), rho[k])
        _write_lg(os.path.join(d, "ini_lumen.dat"), lum)
        _write_lg(os.path.join(d, "ini_ECM.dat"), ecm)
    return phi, rho, lum, ecm


def _write_lg(path: str, table) -> None:
    # "%lg": six significant digits, as prepare_initial_files.cpp:127-201 prints them
    t = np.asarray(table, dtype=np.float64)
    with open(path, "w") as f:
        for row in t:
            f.write("".join(f"{v:g}\n" for v in row))
            f.write("\n")
