"""Run the reference's own step (oracle/_ref/libref_fp{32,64}.so) on an
in-memory state.  TEST INFRASTRUCTURE ONLY: imported by tests/, the golden
fixture script and bench.py's CPU baseline leg, never by the product.

The library holds the reference's globals, so one process serves one
configuration; `run_reference()` therefore runs in a fresh subprocess by
default.
"""
from __future__ import annotations

import ctypes
import multiprocessing as mp
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def lib_path(precision: str = "fp64") -> str:
    return os.path.join(HERE, "_ref", f"libref_{precision}.so")


def available(precision: str = "fp64") -> bool:
    return os.path.exists(lib_path(precision))


class RefLib:
    def __init__(self, precision: str, params: dict):
        self.precision = precision
        self.dtype = np.float64 if precision == "fp64" else np.float32
        self.lib = ctypes.CDLL(lib_path(precision), mode=ctypes.RTLD_LOCAL)
        L = self.lib
        L.pfag_ref_param_set.argtypes = [ctypes.c_char_p, ctypes.c_double]
        L.pfag_ref_param_set.restype = ctypes.c_int
        L.pfag_ref_array.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_long)]
        L.pfag_ref_array.restype = ctypes.c_void_p
        L.pfag_ref_step.argtypes = [ctypes.c_int, ctypes.c_int]
        for k, v in params.items():
            if L.pfag_ref_param_set(k.encode(), float(v)) != 0:
                raise KeyError(k)
        if L.pfag_ref_init() != 0:
            raise RuntimeError("reference init failed")
        self.N = int(params["N_s"])
        self.ncells = int(params["N_ini"])

    def load(self, phi, rho, lum, ecm):
        d = self.dtype
        a = [np.ascontiguousarray(x, dtype=d) for x in (phi, rho, lum, ecm)]
        self.lib.pfag_ref_load(*[x.ctypes.data_as(ctypes.c_void_p) for x in a])
        self.lib.pfag_ref_prepare()

    def step(self, it: int, save: bool = False):
        self.lib.pfag_ref_step(int(it), 1 if save else 0)

    def step_with_velocity(self, it: int):
        """One step; returns the per-cell velocity Re(IFFT(v))/M^2 on the FFT box
        (vx, vy of shape (Ntot, M, M)), read from the shim's capture of the
        inverse transforms (per cell: vx, vy, rho in rho_functions.cpp:449-464)."""
        M = 2 * int(self.lib_param("zone_size")) - 2
        n = self.ncells
        buf = np.zeros(3 * n * M * M, dtype=np.float64)
        self.lib.pfag_shim_capture.argtypes = [ctypes.c_void_p, ctypes.c_long]
        self.lib.pfag_shim_capture_len.restype = ctypes.c_long
        self.lib.pfag_shim_capture(buf.ctypes.data_as(ctypes.c_void_p), buf.size)
        self.step(it)
        got = self.lib.pfag_shim_capture_len()
        self.lib.pfag_shim_capture(None, 0)
        if got != buf.size:
            raise RuntimeError(f"captured {got} values, expected {buf.size}")
        v = buf.reshape(n, 3, M, M) / float(M * M)
        return v[:, 0].copy(), v[:, 1].copy()

    def lib_param(self, name: str) -> float:
        self.lib.pfag_ref_param_get.restype = ctypes.c_double
        self.lib.pfag_ref_param_get.argtypes = [ctypes.c_char_p]
        return self.lib.pfag_ref_param_get(name.encode())

    def array(self, name: str) -> np.ndarray:
        cnt = ctypes.c_long(0)
        p = self.lib.pfag_ref_array(name.encode(), ctypes.byref(cnt))
        if not p:
            raise KeyError(name)
        if name in ("xcenters", "ycenters"):
            t = ctypes.c_int
            dt = np.int32
        else:
            t = ctypes.c_double if self.dtype == np.float64 else ctypes.c_float
            dt = self.dtype
        buf = (t * cnt.value).from_address(p)
        return np.frombuffer(buf, dtype=dt).copy()

    def state(self):
        N, n = self.N, self.ncells
        return {
            "phi": self.array("phi").reshape(n, N, N), "rho": self.array("rho").reshape(n, N, N),
            "lum": self.array("lum").reshape(N, N), "ECM": self.array("ECM").reshape(N, N),
            "s": self.array("s"), "xc": self.array("xcenters"), "yc": self.array("ycenters"),
        }


def _worker(precision, params, init, nsteps, start_it, extra, velocity, q):
    try:
        r = RefLib(precision, params)
        r.load(*init)
        out_steps = {}
        vel = None
        for k in range(nsteps):
            if velocity and k == nsteps - 1:
                vel = r.step_with_velocity(start_it + k)
            else:
                r.step(start_it + k)
            if extra and (k + 1) in extra:
                out_steps[k + 1] = r.state()
        st = r.state()
        st["snapshots"] = out_steps
        st["velocity"] = vel
        q.put(("ok", st))
    except Exception as e:  # pragma: no cover - reported to the parent
        q.put(("err", repr(e)))


def run_reference(params: dict, init, nsteps: int, precision: str = "fp64", start_it: int = 0,
                  snapshots=None, velocity: bool = False, timeout: float = 3600.0):
    """Run `nsteps` reference steps from `init` = (phi, rho, lum, ECM) in a
    spawned subprocess and return the final state dict (plus snapshots, and the
    last step's per-cell velocity when `velocity` is set)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_worker, args=(precision, params, init, nsteps, start_it,
                                          set(snapshots or []), velocity, q))
    p.start()
    import queue
    import time
    t_end = time.time() + timeout
    while True:
        try:
            status, val = q.get(timeout=1.0)
            break
        except queue.Empty:
            if not p.is_alive():
                raise RuntimeError(f"reference subprocess exited with code {p.exitcode} without a result")
            if time.time() > t_end:
                p.kill()
                raise RuntimeError("reference run timed out")
    p.join()
    if status != "ok":
        raise RuntimeError("reference run failed: " + val)
    return val


def main_binary(kind: str, precision: str = "fp64") -> str:
    """oracle/_ref/{ref_main,dropin_main}_fp{32,64}: the reference's own main
    linked with its step files (ref_main) or with the package's drop-in
    libraries (dropin_main)."""
    return os.path.join(HERE, "_ref", f"{kind}_{precision}")


def run_main_binary(binary: str, params: dict, init, workdir: str, env: dict | None = None,
                    timeout: float = 600.0):
    """Run a build of the reference's main in `workdir`: write the parameter
    file and the ini_*.bin state files of `init` = (phi, rho, lum, ECM), run
    Nsteps steps as main does, and return the state of the last snapshot slot
    read back from the ini_*.bin files main writes (phi, rho, lum, ECM), with
    the process's stderr."""
    import subprocess
    import sys
    sys.path.insert(0, os.path.dirname(HERE))
    from multicellular_phase_field_active_gel_organoids_b200 import fileio, params as P
    prec = 64 if binary.endswith("fp64") else 32
    os.makedirs(os.path.join(workdir, "data_int"), exist_ok=True)
    pfile = os.path.join(workdir, "params.txt")
    P.write_param_file(params, pfile)
    fileio.write_state_files(workdir, *init, precision=prec)
    e = dict(os.environ)
    e["PFAG_REF_PARAMS"] = pfile
    e.update(env or {})
    r = subprocess.run([binary], cwd=workdir, env=e, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"{os.path.basename(binary)} exited with {r.returncode}:\n{r.stderr[-3000:]}")
    n, N = int(params["N_ini"]), int(params["N_s"])
    return fileio.read_state_files(workdir, n, N, prec), r.stderr


def run_prepare_binary(binary: str, params: dict, workdir: str, timeout: float = 600.0):
    """Run a build of the reference's initial-condition program
    (oracle/_ref/ref_prepare_fp{32,64}) in `workdir` with the parameter set
    `params`; return the state it writes (ini_*.bin: phi, rho, lum, ECM)."""
    import subprocess
    import sys
    sys.path.insert(0, os.path.dirname(HERE))
    from multicellular_phase_field_active_gel_organoids_b200 import fileio, params as P
    prec = 64 if binary.endswith("fp64") else 32
    os.makedirs(os.path.join(workdir, "data_ini_to_plot"), exist_ok=True)
    pfile = os.path.join(workdir, "params.txt")
    P.write_param_file(params, pfile)
    e = dict(os.environ)
    e["PFAG_REF_PARAMS"] = pfile
    r = subprocess.run([binary], cwd=workdir, env=e, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"{os.path.basename(binary)} exited with {r.returncode}:\n{r.stderr[-3000:]}")
    n, N = int(params["N_ini"]), int(params["N_s"])
    return fileio.read_state_files(workdir, n, N, prec)
