"""The library's scene generators (sphg_make_scene, host code, no GPU)
against sources_b200/scenes.py: the three workloads at their full sizes and
at other sizes, kernels and precisions, bit for bit in every array and in
every field of the parameters, except the inverse-Tait water density and the
mass made from it: numpy's vectorised pow and the C library's pow round some
of those powers differently (by one ulp), so rho and mass agree to 1e-15
relative."""
import ctypes as C

import numpy as np
import pytest

from sources_b200 import abi, make_scene, scene_spec, scenes
from sources_b200.abi import SPHG_FP32, SPHG_FP64, Params

FIELDS = ("x", "vx", "p", "c", "hsml", "vof", "sxx", "sxy", "syy", "drho", "dvx", "itype")
POW_FIELDS = ("rho", "mass")


def params_equal(a: Params, b: Params):
    return C.string_at(C.addressof(a), C.sizeof(Params)) == C.string_at(C.addressof(b), C.sizeof(Params))


def check(py, p, phases):
    assert params_equal(py.params, p)
    assert len(py.phases) == len(phases)
    for A, B in zip(py.phases, phases):
        assert (A.n, A.ntotal, A.material, A.dspp) == (B.n, B.ntotal, B.material, B.dspp)
        for f in FIELDS:
            assert np.array_equal(getattr(A, f), getattr(B, f)), f
        for f in POW_FIELDS:
            a, b = getattr(A, f), getattr(B, f)
            assert np.all(np.abs(a - b) <= 1e-15 * np.abs(a)), f


def test_workloads_at_full_size(lib):
    check(scenes.dam_break(), *make_scene(scene_spec(abi.SPHG_SCENE_DAM_BREAK)))
    check(scenes.granular_column(), *make_scene(scene_spec(abi.SPHG_SCENE_GRANULAR_COLUMN)))
    check(scenes.two_phase(), *make_scene(scene_spec(abi.SPHG_SCENE_TWO_PHASE)))


@pytest.mark.parametrize("skf,prec", [(1, SPHG_FP64), (2, SPHG_FP32), (3, SPHG_FP64), (4, SPHG_FP32)])
def test_other_sizes_kernels_and_precisions(lib, skf, prec):
    check(scenes.dam_break(width=0.05, height=0.1, tank_w=0.2, tank_h=0.15, dx=0.005, skf=skf, precision=prec),
          *make_scene(scene_spec(abi.SPHG_SCENE_DAM_BREAK, col_w=0.05, col_h=0.1, box_w=0.2, box_h=0.15, skf=skf,
                                 precision=prec)))
    check(scenes.granular_column(width=0.04, height=0.02, box_w=0.12, box_h=0.05, dx=0.002, skf=skf, phi_deg=31.0,
                                 precision=prec),
          *make_scene(scene_spec(abi.SPHG_SCENE_GRANULAR_COLUMN, col_w=0.04, col_h=0.02, box_w=0.12, box_h=0.05,
                                 skf=skf, phi_deg=31.0, precision=prec)))
    check(scenes.two_phase(width=0.2, height=0.1, block_w=0.05, block_h=0.03, water_h=0.06, dx=0.002, skf=skf,
                           porosity=0.35, permeability=2e-3, phi_deg=25.0, precision=prec, forchheimer_b=3.0),
          *make_scene(scene_spec(abi.SPHG_SCENE_TWO_PHASE, box_w=0.2, box_h=0.1, col_w=0.05, col_h=0.03,
                                 water_h=0.06, skf=skf, porosity=0.35, permeability=2e-3, phi_deg=25.0,
                                 precision=prec, forchheimer_b=3.0)))


def test_bad_specs_are_rejected(lib):
    from sources_b200.abi import SPHG_ERR_BAD_ARG
    for kw in ({"dx": 0.0}, {"kind": 7}, {"skf": 5}, {"col_w": -1.0}, {"precision": 3}):
        s = scene_spec(abi.SPHG_SCENE_TWO_PHASE)
        for k, v in kw.items():
            setattr(s, k, v)
        n, nt, nv = C.c_int32(), (C.c_int32 * 2)(), (C.c_int32 * 2)()
        assert lib.sphg_scene_size(C.byref(s), C.byref(n), nt, nv) == SPHG_ERR_BAD_ARG
    # views whose sizes differ from sphg_scene_size's
    s = scene_spec(abi.SPHG_SCENE_DAM_BREAK, col_w=0.05, col_h=0.1, box_w=0.2, box_h=0.15)
    P = abi.PhaseArrays(10, 5, abi.SPHG_WATER, 0.005)
    p = Params()
    assert lib.sphg_make_scene(C.byref(s), C.byref(p), C.byref(P.host_struct()), None) == SPHG_ERR_BAD_ARG
