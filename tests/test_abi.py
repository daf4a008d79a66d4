"""The C-ABI boundary on the CPU: libsphg.so loads, exports every entry point
include/sphg.h declares, its structs have the layout ctypes mirrors, its
defaults are the reference's, and argument validation answers without a GPU.
No compute call runs here."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from sources_b200 import EXPORTS, abi, load
from sources_b200.abi import Params, PhaseHost, Stats, default_params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sphg.h")


def header_functions():
    inc = os.path.dirname(HEADER)
    txt = "".join(open(os.path.join(inc, f)).read() for f in sorted(os.listdir(inc)) if f.endswith(".h"))
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(sphg_[a-z0-9_]+)\s*\(", txt)))


def test_header_and_python_agree_on_exports():
    assert sorted(EXPORTS) == header_functions()


def test_library_exports_every_header_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", lib._name], capture_output=True, text=True).stdout
    syms = {l.split()[-1] for l in out.splitlines() if l.strip()}
    for f in header_functions():
        assert f in syms, f
        assert hasattr(lib, f)


def _c_layout():
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "sphg.h"
#include "sphg_learn.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu\n", sizeof(sphg_params), sizeof(sphg_phase_host), sizeof(sphg_stats_t),
         sizeof(sphg_material), offsetof(sphg_params, soil));
  printf("%zu %zu %zu %zu\n", offsetof(sphg_phase_host, x), offsetof(sphg_phase_host, txy),
         offsetof(sphg_phase_host, fail), offsetof(sphg_params, max_interaction));
  printf("%zu %zu\n", offsetof(sphg_stats_t, time), offsetof(sphg_stats_t, last_step_ms));
  printf("%zu %zu %zu %zu %zu\n", sizeof(sphg_case), offsetof(sphg_case, results), offsetof(sphg_case, operating_mode),
         sizeof(sphg_scene), sizeof(sphg_tuning));
  printf("%zu %zu %zu %zu\n", sizeof(SphgGemmEpi), offsetof(SphgGemmEpi, nedge), sizeof(sphg_gnn_node),
         sizeof(sphg_gnn_grid));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", exe, c], check=True)
        return [int(v) for v in subprocess.run([exe], capture_output=True, text=True).stdout.split()]


def test_struct_layout_matches_ctypes():
    v = _c_layout()
    assert v[0] == C.sizeof(Params)
    assert v[1] == C.sizeof(PhaseHost)
    assert v[2] == C.sizeof(Stats)
    assert v[3] == C.sizeof(abi.Material)
    assert v[4] == Params.soil.offset
    assert v[5] == PhaseHost.x.offset and v[6] == PhaseHost.txy.offset and v[7] == PhaseHost.fail.offset
    assert v[8] == Params.max_interaction.offset
    assert v[9] == Stats.time.offset and v[10] == Stats.last_step_ms.offset
    assert v[11] == C.sizeof(abi.Case) and v[12] == abi.Case.results.offset
    assert v[13] == abi.Case.operating_mode.offset
    assert v[14] == C.sizeof(abi.SceneRow) and v[15] == C.sizeof(abi.Tuning)
    from sources_b200 import learn
    assert v[16] == C.sizeof(learn.GemmEpi) and v[17] == learn.GemmEpi.nedge.offset
    assert v[18] == learn.NODE_DTYPE.itemsize and v[19] == C.sizeof(learn.Grid)


def test_default_params_match_reference_defaults(lib):
    p = Params()
    lib.sphg_default_params(C.byref(p))
    q = default_params()
    for name, _ in Params._fields_:
        if name in ("water", "soil"):
            continue
        assert getattr(p, name) == getattr(q, name), name
    assert p.gravity == -9.800000190734863     # -9.8 default-real literal
    assert p.epsilon == 0.0010000000474974513  # 0.001 default-real literal
    assert p.skf == 4 and p.plasticity == 3 and p.yield_criterion == 2


def test_strerror_covers_every_status(lib):
    for code in range(0, 11):
        s = lib.sphg_strerror(code).decode()
        assert s and s != "unknown status"
    assert lib.sphg_strerror(99).decode() == "unknown status"


def test_create_validates_before_touching_the_device(lib):
    p = default_params()
    p.dt = 1e-5
    h = C.c_void_p()
    p.skf = 5
    assert lib.sphg_create(C.byref(p), 2, C.byref(h)) == abi.SPHG_ERR_BAD_KERNEL
    p.skf = 1
    p.integrate_scheme = 2   # Verlet: outside the implemented scope
    assert lib.sphg_create(C.byref(p), 2, C.byref(h)) == abi.SPHG_ERR_UNSUPPORTED
    p.integrate_scheme = 1
    p.yield_criterion = 1    # Mohr-Coulomb
    assert lib.sphg_create(C.byref(p), 2, C.byref(h)) == abi.SPHG_ERR_UNSUPPORTED
    p.yield_criterion = 2
    assert lib.sphg_create(C.byref(p), 3, C.byref(h)) == abi.SPHG_ERR_BAD_ARG
    p.dt = 0.0
    assert lib.sphg_create(C.byref(p), 2, C.byref(h)) == abi.SPHG_ERR_BAD_ARG
    p.dt = 1e-5
    for b in (-1.0, float("nan"), float("inf")):   # Forchheimer coefficient
        p.forchheimer_b = b
        assert lib.sphg_create(C.byref(p), 2, C.byref(h)) == abi.SPHG_ERR_BAD_ARG
    p.forchheimer_b = 0.0
    p.abi_version = abi.SPHG_ABI_VERSION - 1   # a caller built against an older header
    assert lib.sphg_create(C.byref(p), 2, C.byref(h)) == abi.SPHG_ERR_BAD_ARG
    p.abi_version = abi.SPHG_ABI_VERSION
    assert lib.sphg_create(None, 2, C.byref(h)) == abi.SPHG_ERR_BAD_ARG
    assert lib.sphg_single_step(None, 1) == abi.SPHG_ERR_BAD_ARG
    # groups: no contexts, too many, a null member
    g = C.c_void_p()
    none = (C.c_void_p * 2)(None, None)
    assert lib.sphg_group_create(none, 0, C.byref(g)) == abi.SPHG_ERR_BAD_ARG
    assert lib.sphg_group_create(none, 33, C.byref(g)) == abi.SPHG_ERR_BAD_ARG
    assert lib.sphg_group_create(none, 2, C.byref(g)) == abi.SPHG_ERR_BAD_ARG
    assert lib.sphg_group_time_integration(None, 1, None, None) == abi.SPHG_ERR_BAD_ARG
    lib.sphg_group_destroy(None)
    assert lib.sphg_stats(None, None) == abi.SPHG_ERR_BAD_ARG


def test_create_without_device_reports_no_device(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    p = default_params()
    p.dt = 1e-5
    h = C.c_void_p()
    assert lib.sphg_create(C.byref(p), 2, C.byref(h)) == abi.SPHG_ERR_NO_DEVICE
    assert not h.value


def test_solver_fails_loudly_without_library(tmp_path):
    import sources_b200 as sb
    saved = sb._lib
    try:
        sb._lib = None
        with pytest.raises(RuntimeError, match="not built"):
            sb.load(str(tmp_path / "missing.so"))
    finally:
        sb._lib = saved


def test_fortran_bindings_name_exported_symbols(lib):
    """Every bind(C, name=...) of the Fortran interface module names a symbol
    the library exports (the module itself needs a Fortran compiler, which
    this image does not have)."""
    src = open(os.path.join(ROOT, "sources_b200", "fortran", "sphg_iface.f90")).read()
    names = set(re.findall(r'bind\(C,\s*name="(sphg_[a-z0-9_]+)"\)', src))
    out = subprocess.run(["nm", "-D", "--defined-only", lib._name], capture_output=True, text=True).stdout
    syms = {l.split()[-1] for l in out.splitlines() if l.strip()}
    assert len(names) >= 15
    assert names <= syms, sorted(names - syms)
