"""CPU oracle for the SPH step — TEST INFRASTRUCTURE ONLY.

ctypes front-end of sph_oracle.c, the serial FP64 restatement of the
reference's step (cwang2015/sources; see the C file's header for the
reference lines it follows).  PARITY UNPINNED: the reference ships no golden
vectors for this path and cannot be compiled here; known-answer tests in
tests/ pin the restatement instead, and a separate numpy restatement of the
same Fortran agrees with it bit for bit (tests/test_oracle_numpy.py).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package, as the checker; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from sources_b200.abi import PhaseArrays, PhaseHost, Params

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libsph_oracle.so")
_lib = None


def build() -> str:
    subprocess.run(["sh", os.path.join(_HERE, "build_oracle.sh")], check=True)
    return _SO


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(_HERE, "sph_oracle.c")
        if not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(src):
            build()
        L = C.CDLL(_SO)
        L.or_create.restype = C.c_void_p
        L.or_create.argtypes = [C.POINTER(Params), C.c_int]
        L.or_upload_phase.argtypes = [C.c_void_p, C.c_int, C.POINTER(PhaseHost)]
        L.or_download_phase.argtypes = [C.c_void_p, C.c_int, C.POINTER(PhaseHost)]
        L.or_single_step.argtypes = [C.c_void_p, C.c_int]
        L.or_time_integration.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.or_export_pairs.restype = C.c_int64
        L.or_export_pairs.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_int64]
        L.or_set_search_mode.argtypes = [C.c_void_p, C.c_int]
        L.or_nfail.argtypes = [C.c_void_p, C.c_int]
        L.or_destroy.argtypes = [C.c_void_p]
        L.or_kernel.argtypes = [C.c_int, C.c_double, C.POINTER(C.c_double), C.c_double,
                                C.POINTER(C.c_double), C.POINTER(C.c_double)]
        _lib = L
    return _lib


def kernel(skf: int, r: float, dx, h: float):
    """W and grad W of m_particles.f90:1469-1602 for one pair."""
    d = (C.c_double * 2)(*dx)
    w = C.c_double()
    g = (C.c_double * 2)()
    lib().or_kernel(skf, r, d, h, C.byref(w), g)
    return w.value, (g[0], g[1])


class Oracle:
    """Serial FP64 reference step on a Scene (see sources_b200.scenes).

    search='direct' visits pairs exactly as direct_find does (O(N^2));
    search='cells' uses a cell list that visits the same candidates in the
    same order, so results are bit-identical and large scenes stay cheap."""

    def __init__(self, scene, search: str = "cells"):
        self.L = lib()
        self.params = scene.params
        self.h = self.L.or_create(C.byref(scene.params), len(scene.phases))
        if not self.h:
            raise RuntimeError("or_create failed")
        self.L.or_set_search_mode(self.h, 1 if search == "cells" else 0)
        self.phases = [p.copy() for p in scene.phases]
        for k, P in enumerate(self.phases):
            rc = self.L.or_upload_phase(self.h, k + 1, C.byref(P.host_struct()))
            if rc:
                raise RuntimeError(f"or_upload_phase -> {rc}")
        self.itimestep = 0
        self.time = 0.0

    def single_step(self, itimestep: int) -> int:
        return self.L.or_single_step(self.h, itimestep)

    def time_integration(self, maxtimestep: int) -> int:
        it = C.c_int(self.itimestep)
        t = C.c_double(self.time)
        rc = self.L.or_time_integration(self.h, maxtimestep, C.byref(it), C.byref(t))
        self.itimestep, self.time = it.value, t.value
        return rc

    def download(self, phase: int) -> PhaseArrays:
        P = self.phases[phase - 1]
        out = PhaseArrays(P.n, P.ntotal, P.material, P.dspp)
        h = out.host_struct()
        rc = self.L.or_download_phase(self.h, phase, C.byref(h))
        if rc:
            raise RuntimeError(f"or_download_phase -> {rc}")
        out.nfail = h.nfail
        return out

    def pairs(self, which: int):
        n = self.L.or_export_pairs(self.h, which, None, None, 0)
        pi = np.zeros(max(n, 1), dtype=np.int32)
        pj = np.zeros(max(n, 1), dtype=np.int32)
        self.L.or_export_pairs(self.h, which, pi.ctypes.data_as(C.POINTER(C.c_int32)),
                               pj.ctypes.data_as(C.POINTER(C.c_int32)), n)
        return pi[:n], pj[:n]

    def close(self):
        if self.h:
            self.L.or_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
