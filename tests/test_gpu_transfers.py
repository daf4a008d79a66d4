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
