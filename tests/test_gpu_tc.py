"""Tensor-core split contraction (tcgen05) against an FP64 sum of the same
piece products: ragged row/column tails, several frequencies per launch,
fp16 and bf16 pieces, both stage depths."""
import pytest

import dsmsgt


@pytest.mark.gpu
@pytest.mark.parametrize("fmt", [0, 1])
@pytest.mark.parametrize("bk", [32, 64])
def test_tc_contraction_matches_fp64(built, fmt, bk):
    r = dsmsgt.tc_selftest(M=300, N=600, K=192, nfreq=3, fmt=fmt, bk=bk)
    assert r["ref_max"] > 0
    # FP32 accumulation of 3*192 products of magnitude <= 4
    assert r["max_err"] <= 1e-5 * r["ref_max"], r


@pytest.mark.gpu
def test_tc_contraction_one_tile(built):
    r = dsmsgt.tc_selftest(M=5, N=7, K=32, nfreq=1, fmt=0, bk=32)
    assert r["max_err"] <= 1e-6 * r["ref_max"], r
