"""The oracle reproduces the committed golden fixtures (regression pin of
the CPU restatement; fixtures written by tests/golden/make_golden.py)."""
import os
import sys

import numpy as np
import pytest

from conftest import rel_l2

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402


@pytest.mark.parametrize("name", sorted(make_golden.CASES))
def test_oracle_matches_golden(built, name):
    g = np.load(os.path.join(HERE, "golden", name + ".npz"))
    _, freqs, t, r, y, llog = make_golden.compute(name)
    assert list(freqs) == list(g["freqs"])
    assert list(llog) == list(g["llog"])
    for k, v in (("tsgt", t), ("rsgt", r), ("synn", y)):
        assert v.shape == g[k].shape
        assert rel_l2(v, g[k]) <= 1e-12, k
