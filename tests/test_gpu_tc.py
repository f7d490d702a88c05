"""Tensor-core split contraction (tcgen05) against an FP64 sum of the same
piece products: ragged row/column tails, several frequencies per launch,
fp16 and bf16 pieces, both stage depths, order directions and hi*hi chunk
lengths (0: one chunk per tile)."""
import pytest

import dsmsgt


@pytest.mark.gpu
@pytest.mark.parametrize("fmt", [0, 1])
@pytest.mark.parametrize("bk", [32, 64])
@pytest.mark.parametrize("flags,chunk", [(0, 0), (1, 1), (1, 2), (0, 5)])
def test_tc_contraction_matches_fp64(built, fmt, bk, flags, chunk):
    r = dsmsgt.tc_selftest(M=300, N=600, K=192, nfreq=3, fmt=fmt, bk=bk, flags=flags, chunk=chunk)
    assert r["ref_max"] > 0
    # tensor-core FP32 accumulation of 3*192 products of magnitude <= 8
    assert r["max_err"] <= 2e-5 * r["ref_max"], r


@pytest.mark.gpu
@pytest.mark.parametrize("flags,chunk", [(0, 0), (1, 2)])
def test_tc_contraction_one_tile(built, flags, chunk):
    r = dsmsgt.tc_selftest(M=5, N=7, K=32, nfreq=1, fmt=0, bk=32, flags=flags, chunk=chunk)
    assert r["max_err"] <= 1e-6 * r["ref_max"], r


@pytest.mark.gpu
def test_tc_chunked_accumulation_is_length_independent(built):
    """With the hi*hi products summed in short chunks and the chunks added
    in FP64, the error no longer grows with the number of orders."""
    e = {}
    for K in (256, 4096):
        r = dsmsgt.tc_selftest(M=512, N=256, K=K, nfreq=1, fmt=0, bk=32, flags=1, chunk=2)
        e[K] = r["max_err"] / r["ref_max"]
    assert e[4096] < 4e-7, e
    assert e[4096] < 3.0 * e[256] + 1e-7, e
