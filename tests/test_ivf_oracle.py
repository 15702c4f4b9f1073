"""The bucketed (IVF) search restatement in the C oracle against the
reference's own score_prepared_into (src/search/search.cpp:1156-1264), which
scores a bucket's residual codes into per-query heaps with a score offset
<q_hat, encode_c> and an id map. Same residual rows, probes and offsets on
both sides; scores and ids must agree bit for bit."""
import numpy as np
import pytest

from vectorcache_b200.synthetic import ivf_case


def _oracle_ivf(oracle, case, bits, k, tq):
    shift = scale = None
    if tq:
        shift, scale = oracle.fit_calibration(case["residuals"][case["calib_slots"]], bits)
    packed, alpha = oracle.encode(case["residuals"], bits, shift, scale)
    flat = oracle.codes_flat(packed, bits, case["residuals"].shape[1])
    prep = oracle.prepare_queries(case["q"], bits, shift, scale)
    s, i = oracle.ivf_search(prep, flat, alpha, case["ids"], case["start"], case["size"], case["probes"],
                             case["n_probe"], case["offsets"], k)
    return s, i, shift, scale


@pytest.mark.parametrize("dim,bits,k,tq", [(104, 4, 10, True), (128, 2, 1, False), (256, 3, 64, True),
                                           (64, 4, 130, False)])
def test_oracle_matches_reference_ivf(oracle, reference, dim, bits, k, tq):
    case = ivf_case(n=3000, dim=dim, n_buckets=23, nq=12, max_probe=7, seed=dim + bits)
    s_o, i_o, shift, scale = _oracle_ivf(oracle, case, bits, k, tq)
    s_r, i_r = reference.ivf_search(case["q"], bits, case["residuals"], case["ids"], case["start"], case["size"],
                                    case["probes"], case["n_probe"], case["offsets"], k, shift, scale)
    assert np.array_equal(i_o, i_r)
    assert np.array_equal(s_o.view(np.uint32), s_r.view(np.uint32))


def test_ivf_equals_flat_when_offsets_are_zero_and_all_buckets_probed(oracle):
    # With every bucket probed and zero offsets the IVF composition is a flat
    # search over the slots (ids mapped), so it must equal the flat top-k.
    case = ivf_case(n=1500, dim=128, n_buckets=9, nq=6, max_probe=9, seed=3, all_probed=True)
    case["offsets"][:] = 0.0
    bits, k = 4, 10
    packed, alpha = oracle.encode(case["residuals"], bits)
    flat = oracle.codes_flat(packed, bits, 128)
    prep = oracle.prepare_queries(case["q"], bits)
    s, i = oracle.ivf_search(prep, flat, alpha, case["ids"], case["start"], case["size"], case["probes"],
                             case["n_probe"], case["offsets"], k)
    valid = np.concatenate([np.arange(int(st), int(st + sz)) for st, sz in zip(case["start"], case["size"])])
    scores = oracle.float_scores(prep, flat[valid], alpha[valid])
    ids = case["ids"][valid]
    for r in range(6):
        order = sorted(range(len(valid)), key=lambda j: (-scores[r, j], ids[j]))[:k]
        assert np.array_equal(i[r], ids[order])
        assert np.array_equal(s[r], scores[r, order])
