"""Full-state transfers of a phase larger than the staging area (C ABI).

Uploads and downloads move every field of a phase through one device staging
area of at most 2^26 doubles; a phase above 1.81M particles (37 doubles each)
goes through it in groups of fields, with one permutation launch per group.
The 912,016-particle workload fits in one group, so this test makes a wider
two-phase scene (9.5 x 1.0 m at dx 2 mm: 1.9M water particles) and checks,
after steps that reordered the state:

* download -> upload (the in-place refill of the same particles) -> download
  returns every array bit for bit, in both precisions' storage;
* the refilled context then steps exactly as one that was never refilled.
"""
import numpy as np
import pytest

from sources_b200 import Solver, scenes
from sources_b200.abi import INT_FIELDS, SCALAR_FIELDS, SPHG_FP32, VEC_FIELDS

pytestmark = pytest.mark.gpu

STAGING_DOUBLES = 1 << 26
DOUBLES_PER_PARTICLE = 37


def test_grouped_transfers_round_trip_and_keep_the_trajectory(cuda_ok):
    s = scenes.two_phase(width=9.5, precision=SPHG_FP32)
    water = s.phases[0]
    assert water.n * DOUBLES_PER_PARTICLE > STAGING_DOUBLES      # the grouped path
    with Solver(s) as trip, Solver(s) as full:
        trip.time_integration(12)                                 # past the first reorder
        full.time_integration(12)
        first = [trip.download(k + 1) for k in range(2)]
        for k, P in enumerate(first):
            trip.upload(k + 1, P)
        again = [trip.download(k + 1) for k in range(2)]
        for A, B in zip(first, again):
            for f in VEC_FIELDS + SCALAR_FIELDS + INT_FIELDS:
                assert np.array_equal(getattr(A, f), getattr(B, f)), f
        trip.time_integration(2)
        full.time_integration(2)
        for k in range(2):
            a, b = full.download(k + 1), trip.download(k + 1)
            for f in ("x", "vx", "rho", "p", "vof", "drho", "dvx"):
                assert np.array_equal(getattr(a, f), getattr(b, f)), (k, f)


def test_registered_host_arrays_round_trip(cuda_ok):
    """Arrays page-locked by sphg_register_phases (as a Fortran host would do
    after ALLOCATE: plain host memory, small arrays of both phases side by
    side) move bit for bit; registering twice and unregistering twice are
    both accepted, and the arrays stay ordinary memory after."""
    import ctypes as C
    from sources_b200 import load
    from sources_b200.abi import PhaseHost
    L = load()
    s = scenes.small("two_phase", precision=SPHG_FP32)
    with Solver(s) as g:
        g.time_integration(12)
        host = [g.download(k + 1) for k in range(2)]          # plain numpy (pageable) arrays
        views = (PhaseHost * 2)(*[P.host_struct() for P in host])
        assert L.sphg_register_phases(views, 2) == 0
        assert L.sphg_register_phases(views, 2) == 0
        for k, P in enumerate(host):
            g.download(k + 1, into=P)
            g.upload(k + 1, P)
        again = [g.download(k + 1) for k in range(2)]
        assert L.sphg_unregister_phases(views, 2) == 0
        assert L.sphg_unregister_phases(views, 2) == 0
        for A, B in zip(host, again):
            for f in VEC_FIELDS + SCALAR_FIELDS + INT_FIELDS:
                assert np.array_equal(getattr(A, f), getattr(B, f)), f
        host[0].x[0, 0] += 1.0                                  # still ordinary memory
