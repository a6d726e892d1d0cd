"""ctypes binding of libpfag (include/pfag.h) and a small host-side driver.

This is the Python mirror of the reference's step interface: a `Simulation`
holds the device state of one organoid and advances it with the same step the
reference's main loop runs (main_code/run_with_active_gels.cpp:101-185).
There is no CPU fallback: if libpfag.so cannot be loaded the import fails.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpfag.so")

PFAG_OK = 0
PATH_PLAIN = 0
PATH_FUSED = 1

ERRORS = {-1: "PFAG_E_ARG", -2: "PFAG_E_CUDA", -3: "PFAG_E_ZONE", -4: "PFAG_E_EMPTY_CELL",
          -5: "PFAG_E_UNSUPPORTED", -6: "PFAG_E_RELAX"}


class PfagParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("N_s", "Ntot", "zone_size", "N_current", "rdev_threshold", "rimax")] + [
        (n, ctypes.c_double) for n in (
            "dx", "dt", "R", "s0", "sigma", "coupling_PF_AG",
            "tau", "alpha", "beta", "eta",
            "tau_lum", "beta_lum_cells", "eta_lum_cells", "xi_lum",
            "alpha_ECM", "tau_ECM", "beta_ECM_cells", "eta_ECM_cells", "xi_ECM", "beta_lum_ECM",
            "wi", "rtol", "rdt", "friction",
            "a_tan_apical", "a_tan_basal", "a_tan_lateral",
            "a_ort_apical", "a_ort_basal", "a_ort_lateral",
            "b_ap", "b_bas", "b_lat",
            "matgenrate_apical", "matgenrate_basal", "matgenrate_lateral",
            "degrate_apical", "degrate_basal", "degrate_lateral",
            "viscosity_ap", "viscosity_bas", "viscosity_lat")]


class PfagStats(ctypes.Structure):
    _fields_ = [("cell_iters_max", ctypes.c_int), ("cell_iters_sum", ctypes.c_int), ("lum_iters", ctypes.c_int),
                ("ecm_iters", ctypes.c_int), ("relax_failures", ctypes.c_int), ("sum_ecm", ctypes.c_double)]


class PfagError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None

EXPORTS = [
    "pfag_last_error", "pfag_version", "pfag_create", "pfag_destroy", "pfag_upload", "pfag_download",
    "pfag_step", "pfag_step_async", "pfag_sync", "pfag_get_areas", "pfag_get_centres", "pfag_get_stats",
    "pfag_get_cell_iters", "pfag_set_relax_cap", "pfag_set_serial_sums", "pfag_set_debug", "pfag_get_velocity", "pfag_device_state", "pfag_stream", "pfag_launch_count",
    "pfag_fn_find_centres_cells", "pfag_fn_create_turnover_rates_tensions",
    "pfag_fn_compute_hfunc_3d_tables_kernels_loop_n", "pfag_fn_compute_all_hfunc_2d_tables_kernels",
    "pfag_fn_compute_normal_grad_phi", "pfag_fn_compute_prod_norm_delta", "pfag_fn_compute_psi_kernels",
    "pfag_fn_sum_s_kernels", "pfag_fn_update_all_cortices", "pfag_fn_update_lumen_and_ECM",
    "pfag_fn_reshaping_lumen_or_ECM", "pfag_fn_compute_normal_to_phi", "pfag_fn_update_all_cells",
    "pfag_fn_reshaping_cells", "pfag_fn_copy_back", "pfag_fn_saving_out_functions",
    "pfag_generate_initial", "pfag_observables_async", "pfag_snapshot_async", "pfag_snapshot_wait", "pfag_write_text_snapshot",
    "pfag_seed_organoid", "pfag_set_launch_shape", "pfag_batch_create", "pfag_batch_step", "pfag_batch_step_async", "pfag_batch_sync",
    "pfag_batch_stream", "pfag_batch_launch_count", "pfag_batch_destroy",
    "pfag_upload_device", "pfag_conv3x3", "pfag_conv3x3_wgrad", "pfag_conv_act_bwd", "pfag_conv_flip", "pfag_adam",
    "pfag_conv_mse", "pfag_corrector_gather", "pfag_corrector_apply",
    "pfag_shard_enable", "pfag_step_head", "pfag_step_tail", "pfag_sum_planes", "pfag_device_field",
    "pfag_set_lumen_tiles",
]


def lib() -> ctypes.CDLL:
    """Load libpfag.so (raises OSError when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"libpfag.so not built at {LIB_PATH}; run the package build first")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.pfag_last_error.restype = ctypes.c_char_p
        L.pfag_create.argtypes = [ctypes.POINTER(PfagParams), ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
        L.pfag_destroy.argtypes = [vp]
        L.pfag_upload.argtypes = [vp, vp, vp, vp, vp]
        L.pfag_download.argtypes = [vp, vp, vp, vp, vp]
        L.pfag_step.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.pfag_step_async.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.pfag_sync.argtypes = [vp]
        L.pfag_get_areas.argtypes = [vp, vp, vp]
        L.pfag_get_centres.argtypes = [vp, vp, vp]
        L.pfag_get_stats.argtypes = [vp, ctypes.POINTER(PfagStats)]
        L.pfag_set_debug.argtypes = [vp, ctypes.c_int]
        L.pfag_get_cell_iters.argtypes = [vp, vp]
        L.pfag_set_relax_cap.argtypes = [vp, ctypes.c_int]
        L.pfag_set_serial_sums.argtypes = [vp, ctypes.c_int]
        L.pfag_get_velocity.argtypes = [vp, vp, vp]
        L.pfag_device_state.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp),
                                        ctypes.POINTER(vp)]
        L.pfag_device_field.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_long)]
        L.pfag_set_profile.argtypes = [vp, ctypes.c_int]
        L.pfag_profile_read.argtypes = [vp, vp, vp, vp, ctypes.c_int]
        L.pfag_stream.argtypes = [vp]
        L.pfag_stream.restype = vp
        L.pfag_launch_count.argtypes = [vp]
        L.pfag_launch_count.restype = ctypes.c_long
        L.pfag_set_launch_shape.argtypes = [vp, ctypes.c_int, ctypes.c_long]
        L.pfag_set_lumen_tiles.argtypes = [vp, ctypes.c_int]
        L.pfag_seed_organoid.argtypes = [vp, vp, ctypes.c_double, ctypes.c_double, ctypes.c_ulonglong]
        L.pfag_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(vp)]
        L.pfag_batch_step.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.pfag_batch_step_async.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.pfag_batch_sync.argtypes = [vp]
        L.pfag_batch_stream.argtypes = [vp]
        L.pfag_batch_stream.restype = vp
        L.pfag_batch_launch_count.argtypes = [vp]
        L.pfag_batch_launch_count.restype = ctypes.c_long
        L.pfag_batch_destroy.argtypes = [vp]
        L.pfag_shard_enable.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp)]
        L.pfag_step_head.argtypes = [vp, ctypes.c_int]
        L.pfag_step_tail.argtypes = [vp, ctypes.c_int]
        L.pfag_sum_planes.argtypes = [vp, ctypes.POINTER(vp), ctypes.c_int, ctypes.c_long, ctypes.c_int, vp]
        i, f = ctypes.c_int, ctypes.c_float
        L.pfag_upload_device.argtypes = [vp, vp, vp, vp, vp]
        L.pfag_conv3x3.argtypes = [vp, vp, vp, vp, vp, i, i, i, i, i, i, vp, vp]
        L.pfag_conv3x3_wgrad.argtypes = [vp, vp, vp, vp, i, i, i, i, i, vp, vp]
        L.pfag_conv_act_bwd.argtypes = [vp, vp, vp, i, i, i, i, i, vp]
        L.pfag_conv_flip.argtypes = [vp, vp, i, i, vp]
        L.pfag_adam.argtypes = [vp, vp, vp, vp, vp, vp, i, f, f, f, f, i, vp]
        L.pfag_conv_mse.argtypes = [vp, vp, vp, vp, i, i, i, i, i, f, vp]
        L.pfag_corrector_gather.argtypes = [vp, vp, f, f, f]
        L.pfag_corrector_apply.argtypes = [vp, vp, f, f]
        L.pfag_generate_initial.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_int]
        L.pfag_observables_async.argtypes = [vp, vp, vp, vp, vp]
        L.pfag_snapshot_async.argtypes = [vp, vp, vp, vp, vp]
        L.pfag_snapshot_async.restype = ctypes.c_long
        L.pfag_snapshot_wait.argtypes = [vp, ctypes.c_long]
        L.pfag_write_text_snapshot.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_char_p]
        for name in EXPORTS:
            if name.startswith("pfag_fn_"):
                f = getattr(L, name)
                if name == "pfag_fn_reshaping_lumen_or_ECM":
                    f.argtypes = [vp, ctypes.c_int]
                elif name == "pfag_fn_sum_s_kernels":
                    f.argtypes = [vp, vp, vp]
                elif name == "pfag_fn_saving_out_functions":
                    f.argtypes = [vp, vp, vp, vp, vp]
                else:
                    f.argtypes = [vp]
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != PFAG_OK:
        raise PfagError(rc, lib().pfag_last_error().decode())


def make_params(p: dict) -> PfagParams:
    s = PfagParams()
    s.N_s = int(p["N_s"]); s.Ntot = int(p["Ntot"]); s.zone_size = int(p["zone_size"])
    s.N_current = int(p["N_current"]); s.rdev_threshold = int(p["rdev_threshold"]); s.rimax = int(p["rimax"])
    for name, _ in PfagParams._fields_[6:]:
        setattr(s, name, float(p[name]))
    return s


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


class Simulation:
    """Device state of one organoid plus the step (plain or fused path)."""

    def __init__(self, params: dict, precision: int = 64, path: int = PATH_PLAIN):
        self.params = dict(params)
        self.precision = precision
        self.path = path
        self.dtype = np.float64 if precision == 64 else np.float32
        self.N = int(params["N_s"])
        self.ncells = int(params["Ntot"])
        self.M = 2 * int(params["zone_size"]) - 2
        self._p = make_params(params)
        h = ctypes.c_void_p()
        check(lib().pfag_create(ctypes.byref(self._p), precision, path, ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().pfag_destroy(self.h)
            self.h = None

    def __del__(self):  # pragma: no cover - interpreter shutdown ordering
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def upload(self, phi, rho, lum, ecm):
        arrs = [np.ascontiguousarray(x, dtype=self.dtype) for x in (phi, rho, lum, ecm)]
        n, N = self.ncells, self.N
        assert arrs[0].size == n * N * N and arrs[1].size == n * N * N
        assert arrs[2].size == N * N and arrs[3].size == N * N
        check(lib().pfag_upload(self.h, *[_ptr(a) for a in arrs]))

    def download(self):
        n, N = self.ncells, self.N
        phi = np.empty((n, N, N), self.dtype)
        rho = np.empty((n, N, N), self.dtype)
        lum = np.empty((N, N), self.dtype)
        ecm = np.empty((N, N), self.dtype)
        check(lib().pfag_download(self.h, _ptr(phi), _ptr(rho), _ptr(lum), _ptr(ecm)))
        return phi, rho, lum, ecm

    def step(self, it0: int, nsteps: int = 1):
        check(lib().pfag_step(self.h, int(it0), int(nsteps)))

    def step_async(self, it0: int, nsteps: int = 1):
        check(lib().pfag_step_async(self.h, int(it0), int(nsteps)))

    def sync(self):
        check(lib().pfag_sync(self.h))

    def areas(self):
        s = np.empty(self.ncells, np.float64)
        f0 = np.empty(self.ncells, np.float64)
        check(lib().pfag_get_areas(self.h, _ptr(s), _ptr(f0)))
        return s, f0

    def centres(self):
        xc = np.empty(self.ncells, np.int32)
        yc = np.empty(self.ncells, np.int32)
        check(lib().pfag_get_centres(self.h, _ptr(xc), _ptr(yc)))
        return xc, yc

    def stats(self) -> dict:
        st = PfagStats()
        check(lib().pfag_get_stats(self.h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in PfagStats._fields_}

    def cell_iters(self):
        it = np.empty(self.ncells, np.int32)
        check(lib().pfag_get_cell_iters(self.h, _ptr(it)))
        return it

    def set_relax_cap(self, cap: int):
        check(lib().pfag_set_relax_cap(self.h, int(cap)))

    def set_serial_sums(self, on: bool = True):
        """Plain path: take the areas, sum_ecm and the relaxation checks' sums
        in the reference's serial host order (one thread per cell)."""
        check(lib().pfag_set_serial_sums(self.h, 1 if on else 0))

    def upload_device(self, phi: int, rho: int, lum: int, ecm: int):
        """State from device buffers (pointers) of the context's element type."""
        check(lib().pfag_upload_device(self.h, *[ctypes.c_void_p(int(x)) for x in (phi, rho, lum, ecm)]))

    def seed_organoid(self, centres, radius: float, env_radius: float, seed: int):
        """Generate the seeded organoid on the device (pfag_seed_organoid)."""
        c = np.ascontiguousarray(centres, dtype=np.float64).reshape(-1, 2)
        if c.shape[0] != self.ncells:
            raise ValueError(f"{c.shape[0]} centres for {self.ncells} cells")
        check(lib().pfag_seed_organoid(self.h, _ptr(c), float(radius), float(env_radius), int(seed)))

    def set_launch_shape(self, coop_blocks: int = 0, update_warps: int = 0):
        check(lib().pfag_set_launch_shape(self.h, int(coop_blocks), int(update_warps)))

    def set_lumen_tiles(self, tma: bool):
        """TMA-staged lumen / ECM relaxation tiles on (True) or off (pfag_set_lumen_tiles)."""
        check(lib().pfag_set_lumen_tiles(self.h, 1 if tma else 0))

    def set_debug(self, flags: int = 1):
        check(lib().pfag_set_debug(self.h, int(flags)))

    def velocity(self):
        shape = (self.ncells, self.M, self.M)
        vx = np.empty(shape, self.dtype)
        vy = np.empty(shape, self.dtype)
        check(lib().pfag_get_velocity(self.h, _ptr(vx), _ptr(vy)))
        return vx, vy

    def device_field(self, name: str):
        """(device pointer, element count) of a named state array."""
        p = ctypes.c_void_p()
        n = ctypes.c_long()
        check(lib().pfag_device_field(self.h, name.encode(), ctypes.byref(p), ctypes.byref(n)))
        return int(p.value or 0), int(n.value)

    def launch_count(self) -> int:
        return int(lib().pfag_launch_count(self.h))

    def stream(self) -> int:
        return int(lib().pfag_stream(self.h) or 0)

    def shard_enable(self):
        """(lo, hi) device pointers of the neighbour planes of a shard
        (pfag_shard_enable): phi of the cells before local cell 0 and after
        local cell ncells-1."""
        lo, hi = ctypes.c_void_p(), ctypes.c_void_p()
        check(lib().pfag_shard_enable(self.h, ctypes.byref(lo), ctypes.byref(hi)))
        return int(lo.value), int(hi.value)

    def step_head(self, it: int):
        check(lib().pfag_step_head(self.h, int(it)))

    def step_tail(self, it: int):
        check(lib().pfag_step_tail(self.h, int(it)))

    def generate_initial(self, rho0: float, tol: float, make_fields: bool = True):
        """prepare_initial_files.cpp:53-117 on the device (plain-path context):
        the initial fields (make_fields) and their one-shot shaping."""
        check(lib().pfag_generate_initial(self.h, float(rho0), float(tol), 1 if make_fields else 0))

    def fn(self, name: str, *args):
        """Call one per-function entry point, e.g. fn("find_centres_cells")."""
        f = getattr(lib(), "pfag_fn_" + name)
        check(f(self.h, *args))


def sum_planes(out: int, parts, count: int, precision: int, stream: int = 0) -> None:
    """out[i] = parts[0][i] + parts[1][i] + ... in order, on the device
    (pfag_sum_planes; device pointers as ints)."""
    arr = (ctypes.c_void_p * len(parts))(*[int(p) for p in parts])
    check(lib().pfag_sum_planes(ctypes.c_void_p(int(out)), arr, len(parts), int(count), int(precision),
                                ctypes.c_void_p(int(stream))))


class Batch:
    """Fused-path simulations advanced together: one graph launch per step over
    every member (pfag_batch_*).  The members stay owned by the caller."""

    def __init__(self, sims):
        self.sims = list(sims)
        arr = (ctypes.c_void_p * len(self.sims))(*[s.h for s in self.sims])
        h = ctypes.c_void_p()
        check(lib().pfag_batch_create(arr, len(self.sims), ctypes.byref(h)))
        self.h = h

    def step(self, it0: int, nsteps: int = 1):
        check(lib().pfag_batch_step(self.h, int(it0), int(nsteps)))

    def step_async(self, it0: int, nsteps: int = 1):
        check(lib().pfag_batch_step_async(self.h, int(it0), int(nsteps)))

    def sync(self):
        check(lib().pfag_batch_sync(self.h))

    def stream(self) -> int:
        return lib().pfag_batch_stream(self.h) or 0

    def launch_count(self) -> int:
        return int(lib().pfag_batch_launch_count(self.h))

    def close(self):
        if self.h:
            lib().pfag_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
