"""The oracle against its committed golden fixtures (tests/golden/, made by
tests/golden/make_golden.py): integer outputs (counts, event-sequence hashes)
recomputed exactly, floating-point outputs to a few ulp (their last bits depend
on the host libm and compiler), so a change of the restatement cannot pass
unnoticed."""
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
        g = np.asarray(got[k])
        if np.issubdtype(ref[k].dtype, np.floating):
            np.testing.assert_allclose(g, ref[k], rtol=1e-14, atol=0, err_msg=k)
        else:
            assert np.array_equal(g, ref[k]), k
