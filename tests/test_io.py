"""Case-file reader (read_cas, declarations_sph.f90:61-335) and Tecplot
writer (output, declarations_sph.f90:1703-1810) of libsphg: host code, no
GPU needed except for the context-level writer."""
import math

import numpy as np
import pytest

from sources_b200 import SPHError, read_case, scenes, write_tecplot_phase
from sources_b200.abi import SPHG_FP64, SPHG_SOIL, SPHG_WATER

CASE = """# two-phase run
PRINT STEP = 100
SAVE STEP = 500
particle pairs find method = 1
RESULTS FILE = 'f_xv.dat', 'f_state.dat',
               'f_other.dat'
SINGLE PHASE = .false.
FIRST PHASE = water
SECOND PHASE = soil

WATER PROPERTY = 1000., 1.6e5, 7., 20., 1.0d-3
SOIL PROPERTY = 1850., 7.0e5, 0.84e6, 0.3, 24.7
DARCY PARAMETER = 0.4, 1.0e-3
SOIL FAILURE CRITERIA = 0., 0.3456
TIME STEP SIZE = 1.0e-5
NOT A KEYWORD = 3
INTEGRATION SCHEME = 1
&
TIME STEP SIZE = 99.0
"""


def test_read_case(tmp_path, lib):
    f = tmp_path / "run.cas"
    f.write_text(CASE)
    p, c = read_case(str(f))
    assert c.print_step == 100 and c.save_step == 500 and c.nnps == 1
    assert [c.results[i].value.decode() for i in range(3)] == ["f_xv.dat", "f_state.dat", "f_other.dat"]
    assert c.single_phase == 0 and p.single_phase == 0
    assert c.first_material == SPHG_WATER and c.second_material == SPHG_SOIL
    assert (p.water.rho0, p.water.b, p.water.gamma, p.water.c, p.water.viscosity) == (1000.0, 1.6e5, 7.0, 20.0, 1e-3)
    assert (p.soil.rho0, p.soil.k, p.soil.E, p.soil.niu, p.soil.c) == (1850.0, 7.0e5, 0.84e6, 0.3, 24.7)
    assert (p.soil.porosity, p.soil.permeability) == (0.4, 1.0e-3)
    assert (p.soil.cohesion, p.soil.phi) == (0.0, 0.3456)
    assert p.dt == 1.0e-5                     # the '&' line ends the file
    assert c.unknown_keywords == 1 and c.bad_values == 0


def test_read_case_errors(tmp_path, lib):
    with pytest.raises(SPHError):
        read_case(str(tmp_path / "missing.cas"))
    f = tmp_path / "bad.cas"
    f.write_text("TIME STEP SIZE = fast\n")
    with pytest.raises(SPHError):
        read_case(str(f))


def _read_tecplot(path):
    lines = open(path).read().splitlines()
    zone = [i for i, l in enumerate(lines) if "ZONE" in l][0]
    header = " ".join(lines[:zone])
    names = [t.strip().strip('"') for t in header.split("=", 1)[1].replace(",", " ").split()]
    n = int(lines[zone].split("I=")[1].split()[0])
    vals = np.array([float(t) for l in lines[zone + 1:] for t in l.split()])
    return names, n, vals.reshape(len(names), n)


@pytest.mark.parametrize("name", ["dam_break", "granular_column"])
def test_tecplot_writer(tmp_path, lib, name):
    s = scenes.small(name, precision=SPHG_FP64)
    P = s.phases[0]
    P.vof2[:] = 0.25
    zone = np.arange(P.n, dtype=np.int32) % 7
    out = tmp_path / "out.dat"
    write_tecplot_phase(str(out), P, zone)
    names, n, blocks = _read_tecplot(str(out))
    assert n == P.n
    col = dict(zip(names, blocks))
    assert np.allclose(col["X"], P.x[:, 0], rtol=1e-14) and np.allclose(col["Y"], P.x[:, 1], rtol=1e-14)
    assert np.allclose(col["rho"], P.rho, rtol=1e-14) and np.array_equal(col["zone"], zone)
    if P.material == SPHG_WATER:
        assert names == ["X", "Y", "Pressure", "VoF", "vx", "vy", "rho", "zone", "VoF2", "mass"]
        assert np.allclose(col["VoF2"], 0.25)
    else:
        assert names == ["X", "Y", "Pressure", "VoF", "ep", "sxy", "sxx", "syy", "vx", "vy", "rho", "mass",
                         "sigma_yy", "zone"]
        assert np.allclose(col["sigma_yy"], -P.p + P.syy, rtol=1e-14, atol=1e-9)
    write_tecplot_phase(str(out), P, zone, append=True)
    assert open(out).read().count("ZONE") == 2


@pytest.mark.gpu
def test_context_tecplot_matches_download(tmp_path, cuda_ok):
    from sources_b200 import Solver
    s = scenes.small("two_phase", precision=SPHG_FP64)
    with Solver(s) as g:
        g.time_integration(3)
        a, b = tmp_path / "w.dat", tmp_path / "s.dat"
        g.write_tecplot(str(a), str(b))
        for k, path in ((1, a), (2, b)):
            d = g.download(k)
            names, n, blocks = _read_tecplot(str(path))
            col = dict(zip(names, blocks))
            assert n == d.n
            assert np.allclose(col["X"], d.x[:, 0], rtol=1e-14) and np.allclose(col["rho"], d.rho, rtol=1e-14)
            assert np.allclose(col["vy"], d.vx[:, 1], rtol=1e-14, atol=1e-300)
