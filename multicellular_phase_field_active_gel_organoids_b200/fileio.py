"""The reference's state files, read and written byte for byte.

Binary state files (main_code/run_with_active_gels.cpp:193-251 writes them,
functions/initialisation_functions.cpp:10-58 reads them):
  ini_cell_<k>.bin, ini_rho_<k>.bin   k = 1 .. N_ini, one cell each
  ini_lumen.bin, ini_ECM.bin          the shared fields
Each file holds N_s*N_s records in row-major order, and every record is
8 bytes: the reference reads and writes `sizeof(&x)` bytes (the size of a
pointer) from the address of element x.  In the FP64 build a record is exactly
one double.  In the FP32 build it is the float x followed by the float stored
after it in memory (the next element; after a slice's last element, the next
slice's first one, or whatever follows the buffer).  Readers use the first
4 bytes of each record; the reference's own reader also stores the second
4 bytes into the element after x, which the next record then overwrites.
There is no header: the precision is that of the build.

Text snapshots (run_with_active_gels.cpp:215-229, :253-267):
  data_int/phi_cell_<k>_step_<T>.dat, data_int/rho_cell_<k>_step_<T>.dat,
  data_int/lumen_step_<T>.dat, data_int/ECM_step_<T>.dat
one "%.15f" value per line, a blank line after every grid row.
"""
from __future__ import annotations

import os

import numpy as np

_DT = {32: np.float32, 64: np.float64}


def _records(flat: np.ndarray, after, precision: int) -> bytes:
    """8-byte records of the 1-D array `flat`; `after` is the value stored past
    its end in memory (FP32 only)."""
    if precision == 64:
        return np.ascontiguousarray(flat, dtype=np.float64).tobytes()
    a = np.ascontiguousarray(flat, dtype=np.float32)
    nxt = np.empty_like(a)
    nxt[:-1] = a[1:]
    nxt[-1] = np.float32(0.0 if after is None else after)
    return np.stack([a, nxt], axis=1).tobytes()


def _read_records(path: str, count: int, precision: int) -> np.ndarray:
    raw = np.fromfile(path, dtype=np.uint8)
    if raw.size != 8 * count:
        raise ValueError(f"{path}: {raw.size} bytes, expected {8 * count} ({count} records of 8 bytes)")
    if precision == 64:
        return raw.view(np.float64).copy()
    return raw.view(np.float32)[0::2].copy()


def write_state_files(directory: str, phi, rho, lum, ecm, precision: int) -> None:
    """Write ini_cell_k.bin, ini_rho_k.bin, ini_lumen.bin and ini_ECM.bin as
    the reference writes them from one snapshot slot: phi/rho (ncells, N, N)
    laid out as consecutive cells, so a cell's last record carries the next
    cell's first value (0 after the last cell and after the shared fields)."""
    if precision not in _DT:
        raise ValueError("precision must be 32 or 64")
    dt = _DT[precision]
    phi = np.asarray(phi, dtype=dt)
    rho = np.asarray(rho, dtype=dt)
    n, N, _ = phi.shape
    os.makedirs(directory, exist_ok=True)
    for name, tab in (("cell", phi), ("rho", rho)):
        for k in range(n):
            after = tab[k + 1, 0, 0] if k + 1 < n else None
            with open(os.path.join(directory, f"ini_{name}_{k + 1}.bin"), "wb") as f:
                f.write(_records(tab[k].ravel(), after, precision))
    for name, tab in (("lumen", lum), ("ECM", ecm)):
        with open(os.path.join(directory, f"ini_{name}.bin"), "wb") as f:
            f.write(_records(np.asarray(tab, dtype=dt).ravel(), None, precision))


def read_state_files(directory: str, ncells: int, N: int, precision: int):
    """Read the four kinds of state files back: phi, rho (ncells, N, N), lum,
    ECM (N, N), in the build's precision."""
    if precision not in _DT:
        raise ValueError("precision must be 32 or 64")
    NN = N * N
    phi = np.stack([_read_records(os.path.join(directory, f"ini_cell_{k + 1}.bin"), NN, precision)
                    for k in range(ncells)]).reshape(ncells, N, N)
    rho = np.stack([_read_records(os.path.join(directory, f"ini_rho_{k + 1}.bin"), NN, precision)
                    for k in range(ncells)]).reshape(ncells, N, N)
    lum = _read_records(os.path.join(directory, "ini_lumen.bin"), NN, precision).reshape(N, N)
    ecm = _read_records(os.path.join(directory, "ini_ECM.bin"), NN, precision).reshape(N, N)
    return phi, rho, lum, ecm


def read_text_snapshot(path: str, N: int) -> np.ndarray:
    """One data_int/*.dat snapshot as an (N, N) float64 array."""
    with open(path) as f:
        rows = f.read().split("\n\n")
    vals = [float(v) for r in rows for v in r.split()]
    if len(vals) != N * N:
        raise ValueError(f"{path}: {len(vals)} values, expected {N * N}")
    return np.array(vals, dtype=np.float64).reshape(N, N)


def write_text_snapshot(path: str, table) -> None:
    """Write an (N, N) table in the reference's text layout."""
    t = np.asarray(table, dtype=np.float64)
    with open(path, "w") as f:
        for row in t:
            f.write("".join(f"{v:.15f}\n" for v in row))
            f.write("\n")
