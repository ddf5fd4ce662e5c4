"""The oracle against its committed golden fixtures (tests/golden/, made by
tests/golden/make_golden.py): every value recomputed bit for bit, so a change
of the restatement cannot pass unnoticed."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))


def test_oracle_reproduces_golden_fixtures():
    import make_golden
    ref = np.load(os.path.join(HERE, "golden", "oracle_small.npz"))
    got = make_golden.compute()
    assert sorted(ref.files) == sorted(got)
    for k in ref.files:
        assert np.array_equal(np.asarray(got[k]), ref[k]), k
