"""The CPU oracle against golden vectors produced by the reference's own code
(tests/golden/make_golden.py). Everything is compared bit for bit."""
import numpy as np
import pytest

from conftest import golden_cases, load_golden


def bits_equal(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def test_codebook_tables(oracle, tables):
    for key in tables:
        if not key.endswith("_centroids"):
            continue
        bits = int(key.split("_")[0][1:])
        dim = int(key.split("_")[1][1:])
        b, c = oracle.codebook(bits, dim)
        assert bits_equal(c, tables[key]), key
        assert bits_equal(b, tables[key.replace("centroids", "boundaries")]), key


def test_codebook_midpoint_rule(oracle):
    # test_codebook.cpp:7-24: boundaries are the f32 midpoints of f32 centroids.
    for bits in (2, 3, 4):
        for dim in (8, 128, 200, 768):
            b, c = oracle.codebook(bits, dim)
            mid = ((c[:-1] + c[1:]) * np.float32(0.5)).astype(np.float32)
            assert bits_equal(b, mid)
            assert np.all(np.diff(c) > 0)


def test_rotation_tables(oracle, tables):
    for dim in (8, 104, 128, 1536):
        s, p = oracle.rotation(dim)
        assert bits_equal(s, tables[f"d{dim}_signs"])
        assert np.array_equal(p, tables[f"d{dim}_perm"])
        assert sorted(p.tolist()) == list(range(dim))


def test_beta_cdf(oracle, tables):
    for a, t, want in tables["beta_cdf"]:
        assert oracle.beta_cdf_aa(a, t) == want


@pytest.mark.parametrize("name", golden_cases())
def test_encode_and_search(oracle, name):
    g = load_golden(name)
    bits, dim = g["bits"], g["dim"]
    shift = scale = None
    if g["tq"]:
        shift, scale = oracle.fit_calibration(g["calib"], bits)
        assert bits_equal(shift, g["shift"]) and bits_equal(scale, g["scale"])
    packed, alpha = oracle.encode(g["db"], bits, shift, scale)
    assert bits_equal(packed, g["packed"])
    assert bits_equal(alpha, g["alpha"])
    flat = oracle.codes_flat(packed, bits, dim)
    assert bits_equal(flat, g["codes_flat"])
    prep = oracle.prepare_queries(g["q"], bits, shift, scale)
    for key in ("q_rot", "bias_corr", "luts", "lut_scale", "lut_bias"):
        assert bits_equal(prep[key], g[key]), key
    s, i = oracle.search_flat(g["q"], bits, packed, alpha, g["k"], shift, scale)
    assert np.array_equal(i, g["top_ids"])
    assert bits_equal(s, g["top_scores"])


def test_topk_order_ties(oracle):
    # topk_heap.hpp:19-22 / test_topk_heap.cpp: equal scores go to the lower id.
    scores = np.array([[1.0, 3.0, 3.0, 2.0, 3.0, -1.0]], np.float32)
    s, i = oracle.topk(scores, 4)
    assert i.tolist() == [[1, 2, 4, 3]]
    assert s.tolist() == [[3.0, 3.0, 3.0, 2.0]]
    s, i = oracle.topk(scores, 10)  # k_eff = min(k, n)
    assert i.shape == (1, 6)
