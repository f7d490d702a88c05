"""Tensor-core split contraction (tcgen05) against an FP64 sum of the same
piece products: ragged row/column tails, several frequencies per launch,
fp16 and bf16 pieces, both stage depths, every accumulation option."""
import pytest

import dsmsgt


@pytest.mark.gpu
@pytest.mark.parametrize("fmt", [0, 1])
@pytest.mark.parametrize("bk", [32, 64])
@pytest.mark.parametrize("flags", [0, 1, 2, 3])
def test_tc_contraction_matches_fp64(built, fmt, bk, flags):
    r = dsmsgt.tc_selftest(M=300, N=600, K=192, nfreq=3, fmt=fmt, bk=bk, flags=flags)
    assert r["ref_max"] > 0
    # tensor-core FP32 accumulation of 3*192 products of magnitude <= 8
    assert r["max_err"] <= 2e-5 * r["ref_max"], r


@pytest.mark.gpu
@pytest.mark.parametrize("flags", [0, 3])
def test_tc_contraction_one_tile(built, flags):
    r = dsmsgt.tc_selftest(M=5, N=7, K=32, nfreq=1, fmt=0, bk=32, flags=flags)
    assert r["max_err"] <= 1e-6 * r["ref_max"], r
