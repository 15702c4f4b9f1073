"""Exact float re-rank (float_rescore_topk, src/search/float_rescore.cpp:80-164):
the oracle against the reference's own code on CPU, and the GPU kernel through
the C ABI against the oracle. Scores and orders are compared bit for bit."""
import numpy as np
import pytest

from oracle.oracle import oracle_float_rescore, reference_float_rescore
from vectorcache_b200.synthetic import power_law


def _case(dim, n, nq, k, seed):
    rng = np.random.default_rng(seed)
    corpus = power_law(n, dim, seed=seed)
    q = power_law(nq, dim, seed=seed + 1)
    ids = rng.integers(0, n, size=(nq, k)).astype(np.uint64)
    if k >= 3:
        ids[:, -1] = n + 5  # out of range -> -inf, sorted last
        corpus[3] = corpus[7]  # equal scores: order by id
        ids[0, :2] = [7, 3]
    return q, corpus, ids


@pytest.mark.parametrize("dim", [8, 24, 128, 200, 1536])
def test_oracle_matches_reference(oracle, reference, dim):
    q, corpus, ids = _case(dim, 300, 6, 17, seed=dim)
    s1, i1 = oracle_float_rescore(oracle, q, corpus, ids)
    s2, i2 = reference_float_rescore(reference, q, corpus, ids)
    assert np.array_equal(i1, i2)
    assert np.array_equal(s1.view(np.uint32), s2.view(np.uint32))
    assert np.isneginf(s1[:, -1]).all()
    row = i1[0].tolist()
    assert row.index(3) + 1 == row.index(7)  # equal scores: lower id first, adjacent


@pytest.mark.gpu
@pytest.mark.parametrize("dim,k", [(8, 1), (24, 10), (128, 64), (200, 100), (1536, 256), (768, 1000)])
def test_gpu_matches_oracle(oracle, dim, k):
    import vectorcache_b200 as vcb

    q, corpus, ids = _case(dim, 2000, 9, k, seed=dim + k)
    want_s, want_i = oracle_float_rescore(oracle, q, corpus, ids)
    got = vcb.rescore(q, corpus, vcb.SearchResults(np.zeros(ids.shape, np.float32), ids))
    assert np.array_equal(got.ids, want_i)
    assert np.array_equal(got.scores.view(np.uint32), want_s.view(np.uint32))
