"""sources_b200 — B200 (sm_100a) two-phase SPH step of cwang2015/sources.

The product is libsphg.so (C ABI, include/sphg.h).  This package is the
Python host mirror of the reference's interface for the step: `Solver` owns
one libsphg context and exposes the reference's entry points by name:

    Solver.single_step(itimestep)         single_step / single_step_for_water /
                                          single_step_for_soil (declarations_sph.f90:1131,1439,1530)
    Solver.time_integration(maxtimestep)  time_integration / _for_water / _for_soil (:525,794,978)

There is no CPU fallback: constructing a Solver without the built library or
without a CUDA device raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi
from .abi import (PhaseArrays, PhaseHost, Params, Stats, SPHG_FP32, SPHG_FP64, SPHG_PAIRS_CROSS,
                  SPHG_PAIRS_FIRST, SPHG_PAIRS_SECOND, SPHG_SOIL, SPHG_WATER, default_params)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsphg.so")

# every entry point of include/sphg.h
EXPORTS = ("sphg_default_params", "sphg_create", "sphg_upload_phase", "sphg_single_step",
           "sphg_time_integration", "sphg_download_phase", "sphg_export_pairs", "sphg_stats",
           "sphg_set_stream", "sphg_kernel_profile", "sphg_kernel_report", "sphg_destroy",
           "sphg_strerror", "sphg_sum_density_noalloc", "sphg_set_scenes", "sphg_upload_scene_ids",
           "sphg_set_tuning", "sphg_read_case", "sphg_write_tecplot_phase", "sphg_write_tecplot",
           "sphg_gemm_bf16_tn", "sphg_gemm_wait_probe", "sphg_export_xv_device", "sphg_import_xv_device", "sphg_group_create",
           "sphg_group_time_integration", "sphg_group_destroy", "sphg_scene_default", "sphg_scene_size",
           "sphg_make_scene", *sorted(_GNN_SIGNATURES := {
               # message-passing network kernels (include/sphg_learn.h); P pointer,
               # I int, L 64-bit count, F float, D double, S size_t pointer
               "sphg_gemm_bf16_ws": "PPIIIPPP",
               "sphg_gnn_edge_layer": "PPPPPPLIPPPPPP",
               "sphg_gnn_edge_layer_nodes": "PPPPIPPLIPPPPPPP",
               "sphg_gnn_edge_encoder": "PPIPPPPPP",
               "sphg_gnn_node_mlp": "PIPPPPPPPP",
               "sphg_gnn_scan_bytes": "IP",
               "sphg_gnn_graph_count": "PPIPPPPPPLP",
               "sphg_gnn_graph_fill": "PPIPPPPPP",
               "sphg_gnn_node_features": "PPPIPIIFFPP",
               "sphg_gnn_edge_features": "PPPPPLLDPP",
               "sphg_gnn_f32_to_bf16": "PPLP",
               "sphg_gnn_relu_bwd": "PPPPLP",
               "sphg_gnn_colsum": "PLIPP",
               "sphg_gnn_transpose": "PIPLIP",
               "sphg_gnn_segsum": "PPPIIFP",
               "sphg_gnn_segsum_bf16": "PPPIIFP",
               "sphg_gnn_segsum_cat": "PPPPILIFP",
               "sphg_gnn_segsum_bwd": "PPPLIFP",
               "sphg_gnn_gather_bwd": "PPPPILIP",
               "sphg_gnn_node_concat": "PPPLIP",
               "sphg_gnn_node_concat_bwd": "PPPLIP",
               "sphg_gnn_mse": "PIPIPLFFPPP",
               "sphg_gnn_adam": "PPPPPPIIFFFFIIP",
               "sphg_gnn_stride_update": "PIPPPPIIIDP",
               "sphg_gnn_number_density": "PPPIDPP",
               "sphg_gnn_gate_sums": "PPPPPIDPP",
           }))

_lib = None


class SPHError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        msg = load().sphg_strerror(code).decode() if _lib is not None else str(code)
        super().__init__(f"{where}: {msg} (status {code})")


def load(path: str = LIB_PATH):
    """Load libsphg.so (built in-tree by sources_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"libsphg.so not built ({path}); run python -m sources_b200.build")
    L = C.CDLL(path)
    P = C.c_void_p
    L.sphg_default_params.argtypes = [C.POINTER(Params)]
    L.sphg_default_params.restype = None
    L.sphg_create.argtypes = [C.POINTER(Params), C.c_int, C.POINTER(P)]
    L.sphg_upload_phase.argtypes = [P, C.c_int, C.POINTER(PhaseHost)]
    L.sphg_single_step.argtypes = [P, C.c_int]
    L.sphg_time_integration.argtypes = [P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    L.sphg_download_phase.argtypes = [P, C.c_int, C.POINTER(PhaseHost)]
    L.sphg_export_pairs.argtypes = [P, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_int64,
                                    C.POINTER(C.c_int64)]
    L.sphg_stats.argtypes = [P, C.POINTER(Stats)]
    L.sphg_set_stream.argtypes = [P, P]
    L.sphg_kernel_profile.argtypes = [P, C.c_int]
    L.sphg_kernel_report.argtypes = [P, C.c_char_p, C.c_int64]
    L.sphg_destroy.argtypes = [P]
    L.sphg_destroy.restype = None
    L.sphg_strerror.argtypes = [C.c_int]
    L.sphg_strerror.restype = C.c_char_p
    L.sphg_set_scenes.argtypes = [P, C.c_int, C.POINTER(abi.SceneRow)]
    L.sphg_upload_scene_ids.argtypes = [P, C.c_int, C.POINTER(C.c_int32)]
    L.sphg_set_tuning.argtypes = [P, C.POINTER(abi.Tuning)]
    L.sphg_gemm_bf16_tn.argtypes = [P, P, P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P, P]
    L.sphg_gemm_wait_probe.argtypes = [P, P, C.c_int, C.c_int, C.c_int, C.c_longlong, P, P]
    L.sphg_read_case.argtypes = [C.c_char_p, C.POINTER(Params), C.POINTER(abi.Case)]
    L.sphg_write_tecplot_phase.argtypes = [C.c_char_p, C.c_int, C.POINTER(PhaseHost), C.POINTER(C.c_int32)]
    L.sphg_write_tecplot.argtypes = [P, C.c_char_p, C.c_char_p, C.c_int, C.POINTER(C.c_int32),
                                     C.POINTER(C.c_int32)]
    L.sphg_sum_density_noalloc.argtypes = [C.POINTER(Params), C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p]
    L.sphg_group_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.POINTER(P)]
    L.sphg_group_time_integration.argtypes = [P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    L.sphg_group_destroy.argtypes = [P]
    L.sphg_group_destroy.restype = None
    L.sphg_scene_default.argtypes = [C.c_int, C.POINTER(abi.SceneSpec)]
    L.sphg_scene_default.restype = None
    L.sphg_scene_size.argtypes = [C.POINTER(abi.SceneSpec), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                  C.POINTER(C.c_int32)]
    L.sphg_make_scene.argtypes = [C.POINTER(abi.SceneSpec), C.POINTER(Params), C.POINTER(PhaseHost),
                                  C.POINTER(PhaseHost)]
    L.sphg_export_xv_device.argtypes = [P, C.c_int, P, P]
    L.sphg_import_xv_device.argtypes = [P, C.c_int, P, P]
    codes = {"P": C.c_void_p, "I": C.c_int, "L": C.c_longlong, "F": C.c_float, "D": C.c_double}
    for name, sig in _GNN_SIGNATURES.items():
        getattr(L, name).argtypes = [codes[c] for c in sig]
    _lib = L
    return L


def read_case(path: str, params: Params | None = None):
    """Read a reference case file (read_cas, declarations_sph.f90:61).
    Returns (params, case) with the file's values applied to `params`
    (reference defaults if None)."""
    L = load()
    p = params if params is not None else default_params()
    c = abi.Case()
    rc = L.sphg_read_case(path.encode(), C.byref(p), C.byref(c))
    if rc:
        raise SPHError(rc, f"sphg_read_case({path}): {c.bad_values} bad value(s)")
    return p, c


def scene_spec(kind: int, **sizes) -> "abi.SceneSpec":
    """sphg_scene_default of a scene kind (abi.SPHG_SCENE_*), with any field
    of sphg_scene_spec overridden by keyword."""
    L = load()
    s = abi.SceneSpec()
    L.sphg_scene_default(kind, C.byref(s))
    for k, v in sizes.items():
        setattr(s, k, v)
    return s


def make_scene(spec: "abi.SceneSpec"):
    """A scene built by the library's own generators (sphg_make_scene):
    (params, [PhaseArrays per phase])."""
    L = load()
    nph = C.c_int32()
    nt, nv = (C.c_int32 * 2)(), (C.c_int32 * 2)()
    _check(L.sphg_scene_size(C.byref(spec), C.byref(nph), nt, nv), "sphg_scene_size")
    mats = [SPHG_WATER, SPHG_SOIL] if nph.value == 2 else \
        [SPHG_WATER if spec.kind == abi.SPHG_SCENE_DAM_BREAK else SPHG_SOIL]
    phases = [PhaseArrays(nt[k] + nv[k], nt[k], mats[k], spec.dx) for k in range(nph.value)]
    hosts = [P.host_struct() for P in phases]
    p = Params()
    _check(L.sphg_make_scene(C.byref(spec), C.byref(p), C.byref(hosts[0]),
                             C.byref(hosts[1]) if len(hosts) > 1 else None), "sphg_make_scene")
    return p, phases


def write_tecplot_phase(path: str, P: PhaseArrays, zone=None, append: bool = False):
    """Tecplot ASCII zone of one phase from host arrays."""
    L = load()
    z = None if zone is None else np.ascontiguousarray(zone, dtype=np.int32)
    _check(L.sphg_write_tecplot_phase(path.encode(), 1 if append else 0, C.byref(P.host_struct()),
                                      None if z is None else z.ctypes.data_as(C.POINTER(C.c_int32))),
           "sphg_write_tecplot_phase")


def _check(rc: int, where: str):
    if rc != 0:
        raise SPHError(rc, where)


class Solver:
    """One libsphg context holding a Scene's phases on the GPU."""

    def __init__(self, scene, params: Params | None = None):
        self.L = load()
        self.params = params if params is not None else scene.params
        self.nphase = len(scene.phases)
        self.meta = [(p.n, p.ntotal, p.material, p.dspp) for p in scene.phases]
        h = C.c_void_p()
        _check(self.L.sphg_create(C.byref(self.params), self.nphase, C.byref(h)), "sphg_create")
        self.h = h
        for k, P in enumerate(scene.phases):
            self.upload(k + 1, P)
        self.itimestep = 0
        self.time = 0.0

    def upload(self, phase: int, P: PhaseArrays):
        _check(self.L.sphg_upload_phase(self.h, phase, C.byref(P.host_struct())), "sphg_upload_phase")

    def single_step(self, itimestep: int):
        _check(self.L.sphg_single_step(self.h, itimestep), "sphg_single_step")

    def time_integration(self, maxtimestep: int):
        it = C.c_int(self.itimestep)
        t = C.c_double(self.time)
        rc = self.L.sphg_time_integration(self.h, maxtimestep, C.byref(it), C.byref(t))
        self.itimestep, self.time = it.value, t.value
        _check(rc, "sphg_time_integration")

    def download(self, phase: int, into: PhaseArrays | None = None, fields=None) -> PhaseArrays:
        n, nt, mat, dspp = self.meta[phase - 1]
        out = into if into is not None else PhaseArrays(n, nt, mat, dspp)
        h = out.host_struct(fields)
        _check(self.L.sphg_download_phase(self.h, phase, C.byref(h)), "sphg_download_phase")
        out.nfail = h.nfail
        return out

    def export_xv(self, phase: int, x_dev: int | None, v_dev: int | None):
        """Positions / velocities (original order) into device arrays given
        by address, on the context's stream."""
        _check(self.L.sphg_export_xv_device(self.h, phase, C.c_void_p(x_dev or 0), C.c_void_p(v_dev or 0)),
               "sphg_export_xv_device")

    def import_xv(self, phase: int, x_dev: int | None, v_dev: int | None):
        _check(self.L.sphg_import_xv_device(self.h, phase, C.c_void_p(x_dev or 0), C.c_void_p(v_dev or 0)),
               "sphg_import_xv_device")

    def pairs(self, which: int):
        n = C.c_int64()
        _check(self.L.sphg_export_pairs(self.h, which, None, None, 0, C.byref(n)), "sphg_export_pairs")
        pi = np.zeros(max(n.value, 1), dtype=np.int32)
        pj = np.zeros(max(n.value, 1), dtype=np.int32)
        _check(self.L.sphg_export_pairs(self.h, which, pi.ctypes.data_as(C.POINTER(C.c_int32)),
                                        pj.ctypes.data_as(C.POINTER(C.c_int32)), n.value, C.byref(n)),
               "sphg_export_pairs")
        return pi[:n.value], pj[:n.value]

    def stats(self) -> Stats:
        s = Stats()
        _check(self.L.sphg_stats(self.h, C.byref(s)), "sphg_stats")
        return s

    def set_scenes(self, rows):
        """rows: [(dt, water_b, water_c, soil_phi), ...] per scene."""
        arr = (abi.SceneRow * len(rows))(*[abi.SceneRow(*r) for r in rows])
        _check(self.L.sphg_set_scenes(self.h, len(rows), arr), "sphg_set_scenes")

    def upload_scene_ids(self, phase: int, ids):
        a = np.ascontiguousarray(ids, dtype=np.int32)
        _check(self.L.sphg_upload_scene_ids(self.h, phase, a.ctypes.data_as(C.POINTER(C.c_int32))),
               "sphg_upload_scene_ids")

    def set_tuning(self, cell_factor: float = 1.0, reorder_interval: int = 10, x_split: int = 0,
                   state_order: int = 0):
        t = abi.Tuning(cell_factor, reorder_interval, x_split, state_order)
        _check(self.L.sphg_set_tuning(self.h, C.byref(t)), "sphg_set_tuning")

    def write_tecplot(self, path_first: str, path_second: str | None = None, append: bool = False,
                      zone_first=None, zone_second=None):
        """Tecplot ASCII output of every phase (output, declarations_sph.f90:1703)."""
        z = [None if a is None else np.ascontiguousarray(a, dtype=np.int32) for a in (zone_first, zone_second)]
        zp = [None if a is None else a.ctypes.data_as(C.POINTER(C.c_int32)) for a in z]
        _check(self.L.sphg_write_tecplot(self.h, path_first.encode(), None if path_second is None else
                                         path_second.encode(), 1 if append else 0, zp[0], zp[1]),
               "sphg_write_tecplot")

    def set_stream(self, stream_handle: int | None):
        _check(self.L.sphg_set_stream(self.h, C.c_void_p(stream_handle or 0)), "sphg_set_stream")

    def profile(self, enable: bool):
        _check(self.L.sphg_kernel_profile(self.h, 1 if enable else 0), "sphg_kernel_profile")

    def kernel_report(self) -> dict:
        import json
        buf = C.create_string_buffer(1 << 16)
        _check(self.L.sphg_kernel_report(self.h, buf, len(buf)), "sphg_kernel_report")
        return json.loads(buf.value.decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.sphg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class SolverGroup:
    """Several Solvers stepped together (sphg_group_*): after the first step,
    one CUDA graph per step holds every context's step as a parallel branch.
    Results equal stepping each Solver in turn.  All members must be at the
    same itimestep; the group must not be stepped once a member is closed."""

    def __init__(self, solvers):
        self.L = load()
        self.solvers = list(solvers)
        arr = (C.c_void_p * len(self.solvers))(*[sv.h.value for sv in self.solvers])
        h = C.c_void_p()
        _check(self.L.sphg_group_create(arr, len(self.solvers), C.byref(h)), "sphg_group_create")
        self.h = h

    def time_integration(self, maxtimestep: int):
        n = len(self.solvers)
        its = (C.c_int * n)(*[sv.itimestep for sv in self.solvers])
        ts = (C.c_double * n)(*[sv.time for sv in self.solvers])
        rc = self.L.sphg_group_time_integration(self.h, maxtimestep, its, ts)
        for k, sv in enumerate(self.solvers):
            sv.itimestep, sv.time = its[k], ts[k]
        _check(rc, "sphg_group_time_integration")

    def close(self):
        if getattr(self, "h", None):
            self.L.sphg_group_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
