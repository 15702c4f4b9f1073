"""GPU search at the benchmark configurations' own sizes against the CPU oracle.

The small parity cases give every scan CTA a single 2048-vector block. Here
the scan plan carries each CTA's top-k state across many blocks (the tiling
the 1M-vector benchmark runs), and the first benchmark configuration runs at
its full size: 100,000 x 128 Gaussian-mixture rows, 1,000 queries, k = 10,
4-bit, no TQ+ — codes, alpha, integer and float scores of every (query,
vector) and the top-10 are compared bit for bit. The 1536-d power-law cases
cover 2-bit, 3-bit and 4-bit codes with k = 10 and k = 64 at 200,000 rows with
TQ+ calibrated on 10,000 of them.

Tolerance: none. Codes, alpha, LUT sums and float scores are bit-exact and
top-k ids and scores identical (score desc, ties by lower id), as in
oracle/tq_oracle.c's restatement of the reference's avx2_perm0 path.
"""
import numpy as np
import pytest

import vectorcache_b200 as vcb
from vectorcache_b200.synthetic import gaussian_mixture, power_law

pytestmark = pytest.mark.gpu

BLOCK = 2048  # vectors per scan block


def bits_equal(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def mismatch_rows(a, b):
    return int(np.count_nonzero(np.any(np.asarray(a) != np.asarray(b), axis=1)))


def build(db, bits, calib):
    idx = vcb.TurboQuantIndex(db.shape[1], bits)
    if calib is not None:
        idx.calibrate(calib)
    idx.add(db)
    idx.prepare()
    return idx


def check_codes(oracle, idx, db, bits, calib):
    shift = scale = None
    if calib is not None:
        shift, scale = oracle.fit_calibration(calib, bits)
        sh, sc = idx.calibration()
        assert bits_equal(sh, shift) and bits_equal(sc, scale)
    packed, alpha = oracle.encode(db, bits, shift, scale)
    got = idx.packed()
    assert bits_equal(got, packed), f"{mismatch_rows(got, packed)} rows of codes differ"
    assert bits_equal(idx.alpha(), alpha)
    return packed, alpha, shift, scale


def test_config1_full_size(oracle):
    """100k x 128 mixture, 1k queries, k=10, 4-bit, no TQ+."""
    db, q = gaussian_mixture(100_000, 1_000, 128, seed=2024)
    idx = build(db, 4, None)
    packed, alpha, _, _ = check_codes(oracle, idx, db, 4, None)
    flat = oracle.codes_flat(packed, 4, 128)
    assert bits_equal(idx.codes_flat(), flat)
    plan = idx.scan_plan(q.shape[0], 10)
    assert plan["range_vectors"] >= 2 * BLOCK, plan
    prep = oracle.prepare_queries(q, 4)
    got = idx.prepare_queries(q)
    for key in ("q_rot", "bias_corr", "luts", "lut_scale", "lut_bias"):
        assert bits_equal(got[key], prep[key]), key
    # every (query, vector) score, in chunks of 250 queries
    want_top_s, want_top_i = [], []
    for s in range(0, q.shape[0], 250):
        sub = {key: v[s:s + 250] for key, v in prep.items()}
        ints, scores = idx.dense_scores(q[s:s + 250])
        assert np.array_equal(ints, oracle.int_scores(sub["luts"], flat))
        want = oracle.float_scores(sub, flat, alpha)
        assert bits_equal(scores, want)
        ts, ti = oracle.topk(want, 10)
        want_top_s.append(ts)
        want_top_i.append(ti)
    want_s, want_i = np.concatenate(want_top_s), np.concatenate(want_top_i)
    res = idx.search(q, 10)
    assert np.array_equal(res.ids, want_i)
    assert bits_equal(res.scores, want_s)
    # the oracle's own search_flat composition gives the same top-10
    os_, oi = oracle.search_flat(q, 4, packed, alpha, 10)
    assert np.array_equal(oi, want_i) and bits_equal(os_, want_s)
    idx.close()


# (gen, dim, n, bits, TQ+, [(queries, k), ...]); every search here plans at
# least two scan blocks per CTA (asserted).
CASES = [
    ("mix", 128, 300_000, 4, True, [(1024, 10), (512, 64), (64, 10)]),
    ("mix", 128, 500_000, 4, False, [(2048, 10)]),
    ("pl", 1536, 200_000, 2, True, [(256, 10), (256, 64)]),
    ("pl", 1536, 200_000, 4, True, [(256, 64), (256, 10)]),
    ("pl", 1536, 200_000, 3, True, [(256, 10)]),
]

_DATA = {}


def data(gen, dim, n):
    key = (gen, dim, n)
    if key not in _DATA:
        if gen == "mix":
            db, q = gaussian_mixture(n, 2048, dim, seed=n + dim)
        else:
            db, q = power_law(n, dim, seed=n + dim), power_law(256, dim, seed=n + dim + 1)
        _DATA.clear()  # keep one data set in memory
        _DATA[key] = (db, q)
    return _DATA[key]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}{c[1]}_n{c[2]}_b{c[3]}{'_tq' if c[4] else ''}")
def test_multi_block_ranges(oracle, case):
    gen, dim, n, bits, tq, searches = case
    db, q_all = data(gen, dim, n)
    calib = db[:10_000] if tq else None
    idx = build(db, bits, calib)
    packed, alpha, shift, scale = check_codes(oracle, idx, db, bits, calib)
    for nq, k in searches:
        q = q_all[:nq]
        plan = idx.scan_plan(nq, k)
        assert plan["range_vectors"] >= 2 * BLOCK and plan["split_batches"] == 1, plan
        res = idx.search(q, k)
        ws, wi = oracle.search_flat(q, bits, packed, alpha, k, shift, scale)
        assert np.array_equal(res.ids, wi), (nq, k)
        assert bits_equal(res.scores, ws), (nq, k)
    idx.close()


# One and two queries per CTA: split by 256-group batch over few blocks
# (1536-d 4-bit: 3 batches; 768-d 3-bit: 2; register prefetch ring), or whole
# rows with the codes streamed through shared-memory slots (128-d).
ONE_TWO = [
    ("pl", 1536, 200_000, 4, True),
    ("pl", 768, 200_000, 3, True),
    ("mix", 128, 300_000, 4, True),
]


@pytest.mark.parametrize("case", ONE_TWO, ids=lambda c: f"{c[0]}{c[1]}_n{c[2]}_b{c[3]}")
def test_one_and_two_queries(oracle, case):
    gen, dim, n, bits, tq = case
    db, q_all = data(gen, dim, n)
    calib = db[:10_000] if tq else None
    idx = build(db, bits, calib)
    packed, alpha, shift, scale = check_codes(oracle, idx, db, bits, calib)
    for nq in (1, 2):
        for k in (10, 32):
            plan = idx.scan_plan(nq, k)
            split = plan["split_batches"] > 1
            # whole rows: shared-memory slots, except one query over 2- or
            # 4-bit codes (a register ring on four CTAs per SM)
            staged = not split and (nq == 2 or bits == 3)
            assert plan["q_per_cta"] == nq and split == (dim > 256) and (plan["stages"] > 0) == staged, plan
            q = q_all[:nq]
            res = idx.search(q, k)
            ws, wi = oracle.search_flat(q, bits, packed, alpha, k, shift, scale)
            assert np.array_equal(res.ids, wi), (nq, k)
            assert bits_equal(res.scores, ws), (nq, k)
    idx.close()


# Whole-row scans too large for the oracle: top-10 against every vector's
# score from the dense-scores kernel (itself checked against the oracle above
# and in test_gpu_parity), ties by lower id. Two queries (and one query over
# 3-bit codes) stream through shared-memory slots, one query over 4-bit codes
# keeps a register ring on four CTAs per SM.
#   1.3M x 1024 4-bit: the LUT is streamed in 256-group chunks beside the slots;
#   1.3M x 768 3-bit: resident LUT, 3-bit lookups;
#   10M x 128 4-bit: several blocks per CTA (the slots carry over blocks).
STAGED_LARGE = [(1_300_000, 1024, 4), (1_300_000, 768, 3), (10_000_000, 128, 4)]


@pytest.mark.parametrize("case", STAGED_LARGE, ids=lambda c: f"n{c[0]}_d{c[1]}_b{c[2]}")
def test_whole_rows_match_dense_scores(case):
    torch = pytest.importorskip("torch")
    from vectorcache_b200.synthetic import power_law_torch

    n, dim, bits = case
    dev = torch.device("cuda", 0)
    idx = vcb.TurboQuantIndex(dim, bits)
    part = 1_300_000 if n <= 1_300_000 else 2_000_000
    for s in range(0, n, part):
        x = power_law_torch(min(part, n - s), dim, seed=40 + s // part, device=dev)
        if s == 0:
            idx.calibrate_device(x[:10_000])
        idx.add_device(x)
        del x
    idx.prepare()
    torch.cuda.empty_cache()
    q = power_law(2, dim, seed=41)
    ids = np.arange(n)
    for nq in (1, 2):
        plan = idx.scan_plan(nq, 10)
        staged = nq == 2 or bits == 3
        assert (plan["stages"] > 0) == staged and plan["split_batches"] == 1 and plan["q_per_cta"] == nq, plan
        if n > 5_000_000:
            assert plan["range_vectors"] >= 2 * BLOCK, plan
        res = idx.search(q[:nq], 10)
        _, scores = idx.dense_scores(q[:nq])
        for i in range(nq):
            top = np.lexsort((ids, -scores[i]))[:10]
            assert np.array_equal(res.ids[i], top), (nq, i)
            assert bits_equal(res.scores[i], scores[i][top]), (nq, i)
    idx.close()


# One query over 1M rows splits by 256-group batch on four CTAs per SM (8 code
# groups in flight per thread); smaller split scans keep two CTAs per SM. The
# top-10 of one and of two queries against every vector's score from the
# dense-scores kernel, ties by lower id.
ONE_QUERY_SPLIT = [(1_000_000, 1536, 4), (1_000_000, 768, 3)]


@pytest.mark.parametrize("case", ONE_QUERY_SPLIT, ids=lambda c: f"n{c[0]}_d{c[1]}_b{c[2]}")
def test_one_query_split_matches_dense_scores(case):
    torch = pytest.importorskip("torch")
    from vectorcache_b200.synthetic import power_law_torch

    n, dim, bits = case
    dev = torch.device("cuda", 0)
    idx = vcb.TurboQuantIndex(dim, bits)
    x = power_law_torch(n, dim, seed=52, device=dev)
    idx.calibrate_device(x[:10_000])
    idx.add_device(x)
    idx.prepare()
    del x
    torch.cuda.empty_cache()
    q = power_law(2, dim, seed=53)
    ids = np.arange(n)
    for nq in (1, 2):
        plan = idx.scan_plan(nq, 10)
        assert plan["split_batches"] > 1 and plan["q_per_cta"] == nq, plan
        res = idx.search(q[:nq], 10)
        _, scores = idx.dense_scores(q[:nq])
        for i in range(nq):
            top = np.lexsort((ids, -scores[i]))[:10]
            assert np.array_equal(res.ids[i], top), (nq, i)
            assert bits_equal(res.scores[i], scores[i][top]), (nq, i)
    idx.close()
