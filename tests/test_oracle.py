"""The oracle, pinned: the CPU cuFFT shim against numpy.fft, and the C
restatement (oracle/pfag_oracle.c) against the golden fixtures the reference
itself produced (tests/golden/make_golden.py) and against the reference build
run live (bit-exact: same transforms, same operation order)."""
import ctypes
import os

import numpy as np
import pytest

from multicellular_phase_field_active_gel_organoids_b200.params import CONFIGS
from oracle import build_ref, port, refrun

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module", autouse=True)
def _built():
    build_ref.build_port()


def _shim():
    path = port.lib_path(64)
    L = ctypes.CDLL(path)
    L.pfag_shim_fft2d_f64.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
    return L


@pytest.mark.parametrize("shape", [(8, 8), (32, 32), (126, 126), (128, 128), (398, 398), (7, 12), (199, 10), (1, 5)])
def test_fft_shim_matches_numpy(shape):
    L = _shim()
    rng = np.random.default_rng(1)
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    for sign, ref in ((-1, np.fft.fft2(a)), (1, np.fft.ifft2(a) * a.size)):
        b = np.ascontiguousarray(a.astype(np.complex128))
        L.pfag_shim_fft2d_f64(shape[0], shape[1], b.ctypes.data, sign)
        assert np.max(np.abs(b - ref)) / np.max(np.abs(ref)) < 1e-14


@pytest.mark.parametrize("prec", [64, 32])
def test_port_reproduces_golden(prec):
    g = np.load(os.path.join(GOLDEN, f"tiny_ref_fp{prec}.npz"))
    cfg = CONFIGS["tiny"]()
    dtype = np.float64 if prec == 64 else np.float32
    p = port.Port(cfg.params(), prec)
    p.load(*cfg.initial_state(dtype))
    p.step(0)
    st1 = p.state()
    assert np.array_equal(st1["phi"], g["phi_1"]) and np.array_equal(st1["rho"], g["rho_1"])
    for k in range(1, int(g["steps"])):
        p.step(k)
    st = p.state()
    for key in ("phi", "rho", "lum", "ECM", "s", "xc", "yc"):
        assert np.array_equal(st[key], g[key]), key


@pytest.mark.skipif(not refrun.available("fp64"), reason="reference oracle build absent")
def test_reference_build_reproduces_golden():
    g = np.load(os.path.join(GOLDEN, "tiny_ref_fp64.npz"))
    cfg = CONFIGS["tiny"]()
    r = refrun.run_reference(cfg.params(), cfg.initial_state(), int(g["steps"]), velocity=True)
    for key in ("phi", "rho", "lum", "ECM", "s", "xc"):
        assert np.array_equal(r[key], g[key]), key
    assert np.array_equal(r["velocity"][0], g["vx"])


@pytest.mark.skipif(not refrun.available("fp64"), reason="reference oracle build absent")
def test_port_matches_reference_cfg0_first_step():
    # the first cfg0 step runs ~513 reshaping iterations per cell: a long, stiff pin
    cfg = CONFIGS["cfg0"]()
    init = cfg.initial_state()
    a = port.run_port(cfg.params(), init, 1, 64)
    b = refrun.run_reference(cfg.params(), init, 1)
    for key in ("phi", "rho", "lum", "ECM", "s", "xc", "yc"):
        assert np.array_equal(a[key], b[key]), key
    assert a["cell_iters"].tolist() == [514, 513, 513, 513, 513, 513, 513]


def test_port_reports_empty_cell():
    cfg = CONFIGS["tiny"]()
    phi, rho, lum, ecm = cfg.initial_state()
    phi[1] = np.minimum(phi[1], 0.4)          # no site above 0.5: the reference divides by zero
    p = port.Port(cfg.params(), 64)
    p.load(phi, rho, lum, ecm)
    with pytest.raises(RuntimeError, match="-4"):
        p.step(0)


def test_port_reports_zone_outside_grid():
    cfg = CONFIGS["tiny"]()
    phi, rho, lum, ecm = cfg.initial_state()
    phi[0] = 0.0
    phi[0, 2:6, 2:6] = 1.0                     # centroid near the corner: zone leaves the grid
    p = port.Port(cfg.params(), 64)
    p.load(phi, rho, lum, ecm)
    with pytest.raises(RuntimeError, match="-3"):
        p.step(0)
