"""ctypes wrapper of the C restatement (oracle/lib/liboracle_fp{32,64}.so).

TEST INFRASTRUCTURE ONLY: the checker for tests/, smoke() and bench.py's CPU
baseline leg.  `Port(params, precision)` holds one organoid state on the host
and advances it with the restated reference step.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

_FIELDS = [(n, ctypes.c_int) for n in ("N_s", "Ntot", "zone_size", "N_current", "rdev_threshold", "rimax")] + [
    (n, ctypes.c_double) for n in (
        "dx", "dt", "R", "s0", "sigma", "coupling_PF_AG", "tau", "alpha", "beta", "eta",
        "tau_lum", "beta_lum_cells", "eta_lum_cells", "xi_lum",
        "alpha_ECM", "tau_ECM", "beta_ECM_cells", "eta_ECM_cells", "xi_ECM", "beta_lum_ECM",
        "wi", "rtol", "rdt", "friction",
        "a_tan_apical", "a_tan_basal", "a_tan_lateral", "a_ort_apical", "a_ort_basal", "a_ort_lateral",
        "b_ap", "b_bas", "b_lat", "matgenrate_apical", "matgenrate_basal", "matgenrate_lateral",
        "degrate_apical", "degrate_basal", "degrate_lateral", "viscosity_ap", "viscosity_bas", "viscosity_lat")]


class PfoParams(ctypes.Structure):
    _fields_ = _FIELDS


def lib_path(precision: int) -> str:
    return os.path.join(HERE, "lib", f"liboracle_fp{precision}.so")


class Port:
    def __init__(self, params: dict, precision: int = 64):
        path = lib_path(precision)
        if not os.path.exists(path):
            from oracle import build_ref
            build_ref.build_port()
        self.lib = ctypes.CDLL(path)
        L = self.lib
        vp = ctypes.c_void_p
        L.pfo_create.restype = vp
        L.pfo_create.argtypes = [ctypes.POINTER(PfoParams)]
        L.pfo_destroy.argtypes = [vp]
        L.pfo_load.argtypes = [vp, vp, vp, vp, vp]
        L.pfo_step.argtypes = [vp, ctypes.c_int]
        L.pfo_field.restype = vp
        L.pfo_field.argtypes = [vp, ctypes.c_char_p]
        L.pfo_centres.restype = vp
        L.pfo_centres.argtypes = [vp, ctypes.c_int]
        L.pfo_cell_iters.restype = vp
        L.pfo_cell_iters.argtypes = [vp]
        L.pfo_iters.argtypes = [vp, ctypes.c_int]
        L.pfo_rdev_trace.restype = vp
        L.pfo_rdev_trace.argtypes = [vp]
        p = PfoParams()
        for name, t in _FIELDS:
            setattr(p, name, t(params[name]).value)
        self._p = p
        self.h = L.pfo_create(ctypes.byref(p))
        self.N = int(params["N_s"])
        self.ncells = int(params["Ntot"])
        self.dtype = np.float64 if precision == 64 else np.float32

    def close(self):
        if self.h:
            self.lib.pfo_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load(self, phi, rho, lum, ecm):
        a = [np.ascontiguousarray(x, dtype=self.dtype) for x in (phi, rho, lum, ecm)]
        self.lib.pfo_load(self.h, *[ctypes.c_void_p(x.ctypes.data) for x in a])

    def step(self, it: int):
        rc = self.lib.pfo_step(self.h, int(it))
        if rc != 0:
            raise RuntimeError(f"oracle step failed ({rc})")

    def _arr(self, name, count, dtype=None):
        p = self.lib.pfo_field(self.h, name.encode())
        dt = dtype or self.dtype
        ct = ctypes.c_double if dt == np.float64 else ctypes.c_float
        return np.frombuffer((ct * count).from_address(p), dtype=dt).copy()

    def state(self):
        n, N = self.ncells, self.N
        xc = np.frombuffer((ctypes.c_int * n).from_address(self.lib.pfo_centres(self.h, 0)), np.int32).copy()
        yc = np.frombuffer((ctypes.c_int * n).from_address(self.lib.pfo_centres(self.h, 1)), np.int32).copy()
        it = np.frombuffer((ctypes.c_int * n).from_address(self.lib.pfo_cell_iters(self.h)), np.int32).copy()
        return {"phi": self._arr("phi", n * N * N).reshape(n, N, N), "rho": self._arr("rho", n * N * N).reshape(n, N, N),
                "lum": self._arr("lum", N * N).reshape(N, N), "ECM": self._arr("ECM", N * N).reshape(N, N),
                "s": self._arr("s", n), "xc": xc, "yc": yc, "cell_iters": it,
                "lum_iters": self.lib.pfo_iters(self.h, 0), "ecm_iters": self.lib.pfo_iters(self.h, 1)}


    def cell_iters(self) -> np.ndarray:
        """Reshaping iteration count of every cell in the last step."""
        n = self.ncells
        return np.frombuffer((ctypes.c_int * n).from_address(self.lib.pfo_cell_iters(self.h)), np.int32).copy()

    def rdev_trace(self) -> np.ndarray:
        """(Ntot, 2): the last two rdev values of every cell's reshaping loop in
        the last step (the one before the exit test and the one that passed it)."""
        n = self.ncells
        p = self.lib.pfo_rdev_trace(self.h)
        return np.frombuffer((ctypes.c_double * (2 * n)).from_address(p), np.float64).reshape(n, 2).copy()


def run_port(params: dict, init, nsteps: int, precision: int = 64):
    p = Port(params, precision)
    p.load(*init)
    for k in range(nsteps):
        p.step(k)
    st = p.state()
    p.close()
    return st
