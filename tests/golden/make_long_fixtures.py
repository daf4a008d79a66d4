"""Writes tests/golden/oracle_two_phase_912k_500.npz: the CPU oracle's state of
the 912,016-particle two-phase collapse (4.0 x 1.0 m, dx 2 mm, soil block
1.0 x 0.4 m under 0.8 m of water) after 500 leapfrog steps, FP64.

    python tests/golden/make_long_fixtures.py [--full PATH]

The serial oracle needs about ten minutes for these 500 steps, too long for a
test, so the test compares against this file.  The full state is ~100 MB, so
the file keeps every STRIDE-th particle of each phase (in the reference's
particle order, virtual particles included) and the whole-phase summaries
(field maxima and sums) needed to scale errors.  --full PATH also writes the
complete state there (npz, not committed) for a whole-field comparison.
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import Oracle                      # noqa: E402
from sources_b200 import scenes                # noqa: E402
from sources_b200.abi import SPHG_FP64         # noqa: E402

STEPS = 500
STRIDE = 128
FIELDS = ("x", "vx", "rho", "p", "vof", "sxx", "sxy", "syy", "drho", "dvx", "epsilon_p")
OUT = os.path.join(HERE, "oracle_two_phase_912k_500.npz")


def run(full_path=None):
    s = scenes.two_phase(precision=SPHG_FP64)
    o = Oracle(s)
    t = time.time()
    assert o.time_integration(STEPS) == 0
    print(f"oracle: {STEPS} steps of {s.n_particles} particles in {time.time() - t:.0f} s")
    out = {"steps": np.int64(STEPS), "stride": np.int64(STRIDE), "time": np.float64(o.time),
           "n_particles": np.int64(s.n_particles)}
    full = {}
    for k in (1, 2):
        d = o.download(k)
        out[f"{k}/n"] = np.int64(d.n)
        out[f"{k}/nfail"] = np.int64(d.nfail)
        for f in FIELDS + ("fail",):
            a = np.asarray(getattr(d, f))
            out[f"{k}/{f}"] = a[::STRIDE].copy()
            out[f"{k}/{f}/absmax"] = np.float64(np.abs(a).max()) if a.size else np.float64(0)
            full[f"{k}/{f}"] = a.copy()
    np.savez_compressed(OUT, **out)
    print("wrote", OUT)
    if full_path:
        np.savez(full_path, **full)
        print("wrote", full_path)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--full", default=None)
    a = ap.parse_args()
    run(a.full)
