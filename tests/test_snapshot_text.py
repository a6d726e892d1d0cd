"""The reference's text snapshot layout ("%.15f" per line, a blank line after
each row, main_code/run_with_active_gels.cpp:215-229) written by the
library's host formatter (pfag_write_text_snapshot) must be byte-identical to
C printf's "%.15f" (Python's "%.15f" formatting is the same correctly rounded
conversion), including exact decimal ties, tiny values, negative zero and
values beyond the formatter's integer range."""
import ctypes

import numpy as np
import pytest

from multicellular_phase_field_active_gel_organoids_b200 import capi


def _reference_text(t):
    return "".join("".join("%.15f\n" % v for v in row) + "\n" for row in np.asarray(t, np.float64))


@pytest.mark.parametrize("prec", [32, 64])
def test_text_snapshot_bytes(prec, tmp_path):
    dt = np.float64 if prec == 64 else np.float32
    rng = np.random.default_rng(7)
    N = 64
    t = rng.random((N, N)).astype(dt)
    edge = [0.0, -0.0, 1.0, 0.5, 2.5e-16, 5e-16, 1.5e-15, 7.5e-16, 1e-300, -1e-300, 5e-324, 0.9999999999999995,
            0.1, 0.2, 0.3, 1 / 3, 1e-5, -0.123456789012345678, 12345.678, 8999.9999999999995, -3.7e5, 1e20,
            float(np.float32(0.1)), 0.000000000000001, 0.0000000000000005, 0.0000000000000015]
    t.ravel()[:len(edge)] = np.array(edge, dtype=np.float64).astype(dt)
    t.ravel()[len(edge):len(edge) + 200] = (rng.integers(0, 10 ** 6, 200) * 0.5e-15).astype(dt)  # decimal ties
    t = np.ascontiguousarray(t)
    p = tmp_path / "snap.dat"
    capi.check(capi.lib().pfag_write_text_snapshot(ctypes.c_void_p(t.ctypes.data), prec, N, str(p).encode()))
    assert p.read_text() == _reference_text(t)
