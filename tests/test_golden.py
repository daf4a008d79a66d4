"""The CPU oracle against the committed fixtures of tests/golden/ (written by
tests/golden/make_golden.py): the right-hand side and five leapfrog steps of
the three reduced scenes must come out bit for bit as recorded.  This guards
the oracle against unintended change; the reference itself ships no outputs
to record."""
import importlib.util
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def test_oracle_reproduces_the_golden_fixtures():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    ref = np.load(os.path.join(HERE, "golden", "oracle_small.npz"))
    out = mg.outputs()
    assert sorted(out) == sorted(ref.files)
    for k in ref.files:
        assert np.array_equal(out[k], ref[k]), k
