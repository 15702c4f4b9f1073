"""GPU path through the C ABI against the golden vectors and the CPU oracle.

Codes, packed bit planes, codes_flat, alpha, query LUT state, integer LUT sums
and float scores are compared bit for bit; top-k ids and scores must be
identical (ties broken by lower id)."""
import numpy as np
import pytest

import vectorcache_b200 as vcb
from conftest import golden_cases, load_golden
from vectorcache_b200.synthetic import gaussian_mixture, power_law

pytestmark = pytest.mark.gpu


def bits_equal(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def build_index(db, bits, calib=None):
    idx = vcb.TurboQuantIndex(db.shape[1], bits)
    if calib is not None:
        idx.calibrate(calib)
    idx.add(db)
    idx.prepare()
    return idx


@pytest.mark.parametrize("name", golden_cases())
def test_golden(name):
    g = load_golden(name)
    idx = build_index(g["db"], g["bits"], g["calib"] if g["tq"] else None)
    if g["tq"]:
        sh, sc = idx.calibration()
        assert bits_equal(sh, g["shift"]) and bits_equal(sc, g["scale"])
    assert bits_equal(idx.packed(), g["packed"])
    assert bits_equal(idx.codes_flat(), g["codes_flat"])
    assert bits_equal(idx.alpha(), g["alpha"])
    prep = idx.prepare_queries(g["q"])
    for key in ("q_rot", "bias_corr", "luts", "lut_scale", "lut_bias"):
        assert bits_equal(prep[key], g[key]), key
    res = idx.search(g["q"], g["k"])
    assert np.array_equal(res.ids, g["top_ids"])
    assert bits_equal(res.scores, g["top_scores"])


CASES = [
    # gen, dim, n, nq, bits, tq
    ("mix", 128, 3000, 33, 4, False),
    ("mix", 128, 2500, 17, 2, True),
    ("pl", 1536, 1100, 9, 4, True),
    ("pl", 1536, 700, 5, 2, True),
    ("pl", 768, 2049, 13, 3, True),
    ("pl", 384, 1500, 8, 4, False),
    ("pl", 256, 4097, 6, 3, False),
    ("mix", 104, 777, 11, 4, True),
    ("mix", 200, 513, 7, 2, False),
    ("pl", 2048, 300, 5, 4, True),
    ("mix", 8, 100, 4, 4, False),
    ("mix", 96, 64, 3, 3, True),
    # the remaining register layouts of the pipelined encode (512, 1024, 520)
    # and a dim that takes the per-warp row kernel (1000)
    ("pl", 512, 1000, 5, 4, True),
    ("mix", 1024, 700, 4, 2, False),
    ("mix", 520, 900, 5, 4, True),
    ("pl", 1000, 600, 3, 3, True),
    # wider than 2048: the shared-memory row kernels
    ("mix", 3072, 300, 4, 3, True),
    ("mix", 4096, 257, 3, 4, False),
    ("mix", 16384, 70, 2, 2, True),
]


def make_data(gen, dim, n, nq, seed):
    if gen == "mix":
        return gaussian_mixture(n, nq, dim, seed=seed)
    return power_law(n, dim, seed=seed), power_law(nq, dim, seed=seed + 7)


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}{c[1]}_n{c[2]}_b{c[4]}{'_tq' if c[5] else ''}")
def test_against_oracle(oracle, case):
    gen, dim, n, nq, bits, tq = case
    db, q = make_data(gen, dim, n, nq, seed=dim + n)
    calib = db[: min(n, 1000)] if tq else None
    shift = scale = None
    if tq:
        shift, scale = oracle.fit_calibration(calib, bits)
    idx = build_index(db, bits, calib)
    if tq:
        sh, sc = idx.calibration()
        assert bits_equal(sh, shift) and bits_equal(sc, scale)
    packed, alpha = oracle.encode(db, bits, shift, scale)
    assert bits_equal(idx.packed(), packed)
    flat = oracle.codes_flat(packed, bits, dim)
    assert bits_equal(idx.codes_flat(), flat)
    assert bits_equal(idx.alpha(), alpha)
    prep = oracle.prepare_queries(q, bits, shift, scale)
    got = idx.prepare_queries(q)
    for key in ("q_rot", "bias_corr", "luts", "lut_scale", "lut_bias"):
        assert bits_equal(got[key], prep[key]), key
    ints, scores = idx.dense_scores(q)
    assert np.array_equal(ints, oracle.int_scores(prep["luts"], flat))
    want_scores = oracle.float_scores(prep, flat, alpha)
    assert bits_equal(scores, want_scores)
    for k in (1, 10, 64, 256):
        res = idx.search(q, k)
        ws, wi = oracle.topk(want_scores, k)
        assert np.array_equal(res.ids, wi), k
        assert bits_equal(res.scores, ws), k
    # One and two queries: with several 256-group batches (dim > 512 at 3/4
    # bits, > 1024 at 2 bits) the scan splits the work by batch.
    for m in (1, 2):
        for k in (1, 10):
            res = idx.search(q[:m], k)
            ws, wi = oracle.topk(want_scores[:m], k)
            assert np.array_equal(res.ids, wi), (m, k)
            assert bits_equal(res.scores, ws), (m, k)


def test_profile_by_launch():
    """Profiling mode times every launch: per class and per launch name."""
    db = power_law(3000, 256, seed=5)
    idx = build_index(db, 4)
    q = power_law(8, 256, seed=6)
    idx.set_profiling(True)
    idx.read_profile()
    idx.search(q, 10)
    prof = idx.read_profile()
    idx.set_profiling(False)
    by = prof["by_launch"]
    assert by["scan kernel"][1] >= 1 and by["query prep kernel"][1] >= 1
    assert sum(ms for ms, _ in by.values()) == pytest.approx(prof["prep_ms"] + prof["scan_ms"] + prof["merge_ms"])
    assert idx.read_profile()["by_launch"] == {}
