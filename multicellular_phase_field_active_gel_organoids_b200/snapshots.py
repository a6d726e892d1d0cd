"""Snapshot output that overlaps the steps.

The reference saves the state into a snapshot slot every nsaving steps
(saving_out_functions, useful_functions.cpp:66-99) and writes the slots after
the run (run_with_active_gels.cpp:193-269): ini_cell_k.bin, ini_rho_k.bin,
ini_lumen.bin, ini_ECM.bin (8-byte records) and, per slot, the text files
data_int/{phi,rho}_cell_k_step_T.dat and data_int/{lumen,ECM}_step_T.dat.

`SnapshotWriter` keeps that output layout but writes while the run goes on:
`save(it)` queues a device copy of the state (pfag_snapshot_async: a
device-to-device copy on the step's stream, then a copy to pinned host memory
on a second stream) and returns; a writer thread waits for the host copy and
writes the files (binary with numpy, text with the library's multi-threaded
"%.15f" formatter).  `slots` pinned buffers bound how many snapshots can be in
flight; `save` blocks only when all of them are.
"""
from __future__ import annotations

import ctypes
import os
import queue
import threading

import numpy as np

from . import capi, fileio


class _Pinned:
    """Page-locked host buffers for one snapshot (phi, rho, lum, ECM)."""

    def __init__(self, rt, ncells, N, dtype):
        self.rt = rt
        self.ptrs = []
        self.arrays = []
        for shape in ((ncells, N, N), (ncells, N, N), (N, N), (N, N)):
            nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
            p = ctypes.c_void_p()
            if rt.cudaHostAlloc(ctypes.byref(p), ctypes.c_size_t(nbytes), 0) != 0:
                raise MemoryError(f"cudaHostAlloc of {nbytes} bytes failed")
            self.ptrs.append(p)
            buf = (ctypes.c_char * nbytes).from_address(p.value)
            self.arrays.append(np.frombuffer(buf, dtype=dtype).reshape(shape))

    def free(self):
        for p in self.ptrs:
            self.rt.cudaFreeHost(p)
        self.ptrs, self.arrays = [], []


class SnapshotWriter:
    """Asynchronous saver of a capi.Simulation's state in the reference's files."""

    def __init__(self, sim: "capi.Simulation", directory: str, text: bool = True, slots: int = 2):
        capi.lib()
        self.rt = ctypes.CDLL("libcudart.so.12")
        self.rt.cudaHostAlloc.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t, ctypes.c_uint]
        self.rt.cudaFreeHost.argtypes = [ctypes.c_void_p]
        self.sim = sim
        self.dir = directory
        self.text = text
        self.prec = 64 if sim.dtype == np.float64 else 32
        os.makedirs(directory, exist_ok=True)
        if text:
            os.makedirs(os.path.join(directory, "data_int"), exist_ok=True)
        self.bufs = [_Pinned(self.rt, sim.ncells, sim.N, sim.dtype) for _ in range(slots)]
        self.free = queue.Queue()
        for k in range(slots):
            self.free.put(k)
        self.work = queue.Queue()
        self.error = None
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()

    def save(self, it: int) -> None:
        """Queue the current state as the snapshot of step `it` (the state the
        next step starts from, as saving_out_functions sees it)."""
        if self.error:
            raise self.error
        k = self.free.get()
        b = self.bufs[k]
        t = capi.lib().pfag_snapshot_async(self.sim.h, *b.ptrs)
        if t < 0:
            self.free.put(k)
            capi.check(int(t))
        self.work.put((t, k, int(it)))

    def _run(self):
        while True:
            item = self.work.get()
            if item is None:
                return
            t, k, it = item
            try:
                capi.check(capi.lib().pfag_snapshot_wait(self.sim.h, t))
                self._write(self.bufs[k].arrays, it)
            except Exception as e:  # reported by the next save() / close()
                self.error = e
            finally:
                self.free.put(k)

    def _write(self, arrays, it):
        phi, rho, lum, ecm = arrays
        fileio.write_state_files(self.dir, phi, rho, lum, ecm, self.prec)
        if not self.text:
            return
        L = capi.lib()
        d = os.path.join(self.dir, "data_int")

        def txt(table, name):
            a = np.ascontiguousarray(table)
            capi.check(L.pfag_write_text_snapshot(ctypes.c_void_p(a.ctypes.data), self.prec, self.sim.N,
                                                  os.path.join(d, name).encode()))

        for n in range(phi.shape[0]):
            txt(phi[n], f"phi_cell_{n + 1}_step_{it}.dat")
            txt(rho[n], f"rho_cell_{n + 1}_step_{it}.dat")
        txt(lum, f"lumen_step_{it}.dat")
        txt(ecm, f"ECM_step_{it}.dat")

    def close(self) -> None:
        """Wait for every queued snapshot to be written, then free the buffers."""
        self.work.put(None)
        self.thread.join()
        for b in self.bufs:
            b.free()
        self.bufs = []
        if self.error:
            raise self.error

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def run(sim: "capi.Simulation", nsteps: int, nsaving: int, directory: str, text: bool = True, start_it: int = 0):
    """The reference's main loop (run_with_active_gels.cpp:101-185): a snapshot
    of the state at every step it with it % nsaving == 0, then the step, for
    it = start_it .. start_it + nsteps - 1; snapshots written in the reference's
    layout while the run goes on."""
    with SnapshotWriter(sim, directory, text=text) as w:
        for it in range(start_it, start_it + nsteps):
            if it % nsaving == 0:
                w.save(it)
            sim.step_async(it, 1)
        sim.sync()
