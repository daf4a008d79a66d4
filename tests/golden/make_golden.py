"""Writes tests/golden/oracle_small.npz: outputs of the CPU oracle on the three
reduced scenes, kept as regression fixtures (they pin the oracle against its
own past, not against the reference, which ships no outputs).

    python tests/golden/make_golden.py

For each scene (dam_break, granular_column, two_phase; FP64, jittered, with
seeded velocities): the right-hand side of single_step(1), and the state after
five leapfrog steps.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import Oracle                      # noqa: E402
from sources_b200 import scenes                # noqa: E402
from sources_b200.abi import SPHG_FP64         # noqa: E402

RHS = ("drho", "dvx", "av", "p")
STATE = ("x", "vx", "rho", "p")
SOIL = ("sxx", "sxy", "syy", "dsxx", "dp")
WATER2 = ("dvof", "vof2")


def scene(name):
    s = scenes.jitter(scenes.small(name, precision=SPHG_FP64), 0.0002, seed=2024)
    rng = np.random.default_rng(2024)
    for P in s.phases:
        P.vx[:P.ntotal] = rng.normal(0, 0.02, size=(P.ntotal, 2))
    return s


def outputs():
    out = {}
    for name in ("dam_break", "granular_column", "two_phase"):
        s = scene(name)
        o = Oracle(s)
        assert o.single_step(1) == 0
        for k, P in enumerate(s.phases, start=1):
            d = o.download(k)
            fields = RHS + (SOIL if P.material == 2 else ()) + (WATER2 if P.material == 1 and len(s.phases) == 2 else ())
            for f in fields:
                out[f"{name}/rhs/{k}/{f}"] = np.asarray(getattr(d, f)).copy()
        o = Oracle(s)
        assert o.time_integration(5) == 0
        for k, P in enumerate(s.phases, start=1):
            d = o.download(k)
            for f in STATE + (("sxx", "syy") if P.material == 2 else ()):
                out[f"{name}/step5/{k}/{f}"] = np.asarray(getattr(d, f)).copy()
    return out


if __name__ == "__main__":
    np.savez_compressed(os.path.join(HERE, "oracle_small.npz"), **outputs())
    print("wrote", os.path.join(HERE, "oracle_small.npz"))
