"""ctypes mirrors of include/sphg.h and the Fortran-layout host arrays.

The structs here are byte-for-byte the C structs of the header; the field
comments there cite the reference lines each field replaces.  `PhaseArrays`
owns numpy arrays laid out like the reference's `particles` components
(m_particles.f90:223-300): vectors as x(2,n) (numpy shape (n, 2), C order,
which is Fortran (2, n)), scalars as (n).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

SPHG_ABI_VERSION = 2

SPHG_OK = 0
SPHG_ERR_PAIR_OVERFLOW = 1
SPHG_ERR_OUT_OF_DOMAIN = 2
SPHG_ERR_BAD_KERNEL = 3
SPHG_ERR_BAD_ARG = 4
SPHG_ERR_CUDA = 5
SPHG_ERR_TIMEOUT = 6
SPHG_ERR_NONFINITE = 7
SPHG_ERR_UNSUPPORTED = 8
SPHG_ERR_STATE = 9
SPHG_ERR_NO_DEVICE = 10

SPHG_WATER = 1
SPHG_SOIL = 2
SPHG_FP64 = 0
SPHG_FP32 = 1
SPHG_PAIRS_FIRST = 0
SPHG_PAIRS_SECOND = 1
SPHG_PAIRS_CROSS = 2


def f32(v: float) -> float:
    """Value of a Fortran default-real (single precision) literal."""
    return float(np.float32(v))


class Material(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "rho0", "b", "gamma", "c", "viscosity",
        "k", "porosity", "permeability", "G", "E", "niu", "cohesion", "phi")]


class Params(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "abi_version", "dim", "skf", "single_phase", "first_material",
        "summation_density", "average_velocity", "visc_artificial",
        "artificial_density", "soil_artificial_stress", "volume_fraction",
        "water_artificial_volume", "volume_fraction_renorm",
        "stress_integration", "yield_criterion", "plasticity",
        "integrate_scheme", "precision", "reorder_interval", "renorm_interval")] + [
        (n, C.c_double) for n in (
            "gravity", "numeric_gravity", "alpha", "beta", "etq", "dd", "p1", "p2",
            "delta", "epsilon", "dt", "x_min", "x_max", "y_min", "y_max")] + [
        ("max_interaction", C.c_int64),
        ("water", Material),
        ("soil", Material),
        ("forchheimer_b", C.c_double),
    ]


_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int32)

VEC_FIELDS = ("x", "vx", "dvx", "av", "v_min")
SCALAR_FIELDS = ("rho", "rho_min", "drho", "p", "c", "mass", "hsml",
                 "vof", "vof_min", "dvof", "vof2",
                 "sxx", "sxy", "syy", "dsxx", "dsxy", "dsyy", "dp",
                 "sxx_min", "sxy_min", "syy_min", "p_min",
                 "epsilon_p", "vcc", "txx", "tyy", "txy")
INT_FIELDS = ("itype", "fail")


class PhaseHost(C.Structure):
    _fields_ = ([("ntotal", C.c_int32), ("nvirt", C.c_int32), ("material", C.c_int32),
                 ("nfail", C.c_int32), ("dspp", C.c_double)]
                + [(n, _DP) for n in VEC_FIELDS]
                + [(n, _DP) for n in SCALAR_FIELDS]
                + [(n, _IP) for n in INT_FIELDS])


class SceneRow(C.Structure):
    _fields_ = [("dt", C.c_double), ("water_b", C.c_double), ("water_c", C.c_double), ("soil_phi", C.c_double)]


class Tuning(C.Structure):
    _fields_ = [("cell_factor", C.c_double), ("reorder_interval", C.c_int32), ("x_split", C.c_int32),
                ("state_order", C.c_int32)]


class Case(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("print_step", "save_step", "nnps", "single_phase", "dry_soil",
                                         "with_nozzle", "first_material", "second_material",
                                         "unknown_keywords", "bad_values")] + [
        ("inlet_velocity", C.c_double), ("dt", C.c_double), ("results", (C.c_char * 256) * 3),
        ("particle_size", C.c_char * 32), ("operating_mode", C.c_char * 32)]


SPHG_SCENE_DAM_BREAK, SPHG_SCENE_GRANULAR_COLUMN, SPHG_SCENE_TWO_PHASE = 1, 2, 3


class SceneSpec(C.Structure):
    _fields_ = [("kind", C.c_int32), ("skf", C.c_int32), ("precision", C.c_int32), ("_pad", C.c_int32)] + [
        (n, C.c_double) for n in ("dx", "box_w", "box_h", "col_w", "col_h", "water_h", "phi_deg", "porosity",
                                  "permeability", "forchheimer_b")]


class Stats(C.Structure):
    _fields_ = [("niac", C.c_int64 * 3), ("maxiac", C.c_int32 * 2), ("miniac", C.c_int32 * 2),
                ("noiac", C.c_int32 * 2), ("nfail", C.c_int32), ("n_out_of_domain", C.c_int32),
                ("itimestep", C.c_int32), ("_pad", C.c_int32), ("time", C.c_double),
                ("last_step_ms", C.c_double)]


def default_params() -> Params:
    """Reference defaults: param.f90:10-133 and type(numerical)
    m_particles.f90:31-55 (single-precision literals kept as the Fortran
    compiler stores them, e.g. gravity = -9.8 is -9.800000190734863)."""
    p = Params()
    p.abi_version = SPHG_ABI_VERSION
    p.dim = 2
    p.skf = 4                      # m_particles.f90:141
    p.single_phase = 0
    p.first_material = SPHG_WATER
    p.summation_density = 0        # param.f90:79
    p.average_velocity = 1         # :80
    p.visc_artificial = 1          # :86
    p.artificial_density = 1       # :95
    p.soil_artificial_stress = 1   # :96
    p.volume_fraction = 1          # :98
    p.water_artificial_volume = 1  # :99
    p.volume_fraction_renorm = 1   # :100
    p.stress_integration = 1       # :92
    p.yield_criterion = 2          # :93
    p.plasticity = 3               # :94
    p.integrate_scheme = 1         # :78
    p.precision = SPHG_FP64
    p.reorder_interval = 10
    p.renorm_interval = 40         # declarations_sph.f90:1415
    p.gravity = f32(-9.8)          # declarations_sph.f90:13
    p.numeric_gravity = f32(-9.8)  # m_particles.f90:40
    p.alpha, p.beta, p.etq = 0.1, 0.0, 0.1   # m_particles.f90:44 (d0 literals)
    p.dd, p.p1, p.p2 = 0.1, 12.0, 4.0        # :47
    p.delta = 0.1                            # :50
    p.epsilon = f32(0.001)                   # :53
    p.dt = 0.0
    p.x_min, p.x_max, p.y_min, p.y_max = -10.0, 10.0, -10.0, 10.0  # param.f90:23-25
    p.max_interaction = 10 * 2000            # param.f90:14
    return p


class PhaseArrays:
    """Host arrays of one phase, in the reference's particle order."""

    def __init__(self, n: int, ntotal: int, material: int, dspp: float = 0.0, alloc=None):
        """alloc(shape, dtype) -> zeroed array; e.g. pinned host memory."""
        self.n = int(n)
        self.ntotal = int(ntotal)
        self.nvirt = int(n - ntotal)
        self.material = int(material)
        self.dspp = float(dspp)
        self.nfail = 0
        mk = alloc or (lambda shape, dtype: np.zeros(shape, dtype=dtype))
        for f in VEC_FIELDS:
            setattr(self, f, mk((self.n, 2), np.float64))
        for f in SCALAR_FIELDS:
            setattr(self, f, mk((self.n,), np.float64))
        for f in INT_FIELDS:
            setattr(self, f, mk((self.n,), np.int32))

    def nbytes(self, fields=None) -> int:
        tot = 0
        for f in VEC_FIELDS + SCALAR_FIELDS + INT_FIELDS:
            if fields is None or f in fields:
                tot += getattr(self, f).nbytes
        return tot

    def copy(self, alloc=None) -> "PhaseArrays":
        o = PhaseArrays(self.n, self.ntotal, self.material, self.dspp, alloc=alloc)
        for f in VEC_FIELDS + SCALAR_FIELDS + INT_FIELDS:
            getattr(o, f)[...] = getattr(self, f)
        o.nfail = self.nfail
        return o

    def host_struct(self, fields=None) -> PhaseHost:
        """PhaseHost pointing at these arrays (all fields, or only `fields`)."""
        h = PhaseHost()
        h.ntotal, h.nvirt, h.material, h.dspp = self.ntotal, self.nvirt, self.material, self.dspp
        for f in VEC_FIELDS + SCALAR_FIELDS:
            if fields is None or f in fields:
                a = getattr(self, f)
                assert a.flags["C_CONTIGUOUS"] and a.dtype == np.float64
                setattr(h, f, a.ctypes.data_as(_DP))
        for f in INT_FIELDS:
            if fields is None or f in fields:
                a = getattr(self, f)
                assert a.flags["C_CONTIGUOUS"] and a.dtype == np.int32
                setattr(h, f, a.ctypes.data_as(_IP))
        return h
