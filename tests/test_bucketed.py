"""Bucketed (IVF) index on the GPU through the C ABI.

* the partition is well formed and deterministic (every row in exactly one
  bucket, no bucket above max_bucket_size, slot layout aligned, encode
  centroids = member means, routing centroids = their normalized means);
* routing scores and probe offsets are fp32 dot products checked against fp64
  to 1e-5;
* the residual codes equal the oracle's encoding of x_hat - encode_c;
* search results equal the C oracle's restatement of the reference's
  score_prepared_into composition (tests/test_ivf_oracle.py pins that oracle to
  the reference) on the same probes and offsets: ids and scores bit for bit;
* recall against exact brute force grows with n_probe.
"""
import numpy as np
import pytest

import vectorcache_b200 as vcb
from vectorcache_b200.synthetic import vmf_mixture

TOL = 1e-5  # fp32 routing / offset dot products against fp64


def bits_equal(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def test_params_are_validated_before_any_device_work():
    with pytest.raises(vcb.InvalidArgument):
        vcb.BucketedTurboQuantIndex(100, 4, vcb.BucketParams(n_probe=0))
    with pytest.raises(vcb.InvalidArgument):
        vcb.BucketedTurboQuantIndex(100, 4, vcb.BucketParams(max_bucket_size=1))


def _data(n, nq, dim, seed):
    db = vmf_mixture(n, dim, seed=seed, clusters=60)
    q = vmf_mixture(nq, dim, seed=seed + 1, clusters=60)
    return db, q


def _build(db, bits, params, calib=None):
    idx = vcb.BucketedTurboQuantIndex(db.shape[1], bits, params)
    if calib is not None:
        idx.calibrate(calib)
    idx.add(db)
    idx.prepare()
    return idx


@pytest.fixture(scope="module")
def small():
    db, q = _data(12000, 24, 100, seed=11)
    params = vcb.BucketParams(n_probe=8, max_bucket_size=300, energy_soft=150, kmeans_iters=3, seed=7)
    return db, q, params


@pytest.mark.gpu
def test_partition_invariants_and_determinism(small):
    db, q, params = small
    idx = _build(db, 4, params)
    inf = idx.info()
    assert inf["dim_padded"] == 104 and inf["size"] == db.shape[0]
    lay = idx.layout()
    nb = inf["n_buckets"]
    sizes = lay["bucket_size"].astype(np.int64)
    assert sizes.sum() == db.shape[0] and sizes.min() >= 1 and sizes.max() <= params.max_bucket_size
    starts = lay["slot_start"].astype(np.int64)
    assert np.all(starts % 256 == 0) and starts[-1] == inf["n_slots"]
    assert np.all(np.diff(starts) == (sizes + 255) // 256 * 256)
    labels = lay["labels"]
    seen = np.zeros(db.shape[0], np.int64)
    x_hat = idx.rows()
    route, enc = idx.centroids()
    for b in range(nb):
        ids = lay["slot_ids"][starts[b]:starts[b] + sizes[b]]
        assert np.all(np.diff(ids.astype(np.int64)) > 0)  # members sorted by id
        assert np.all(labels[ids] == b)
        assert np.all(lay["slot_ids"][starts[b] + sizes[b]:starts[b + 1]] == 0xFFFFFFFF)
        seen[ids] += 1
        mean = x_hat[ids].astype(np.float64).mean(axis=0)
        assert np.max(np.abs(enc[b] - mean)) < 1e-6
        assert np.max(np.abs(route[b] - mean / np.linalg.norm(mean))) < 1e-6
    assert np.all(seen == 1)
    # x_hat: unit rows padded with zeros
    assert np.allclose(np.linalg.norm(x_hat, axis=1), 1.0, atol=1e-6)
    assert np.all(x_hat[:, 100:] == 0)
    again = _build(db, 4, params)
    lay2 = again.layout()
    assert all(np.array_equal(lay[key], lay2[key]) for key in lay)
    assert all(bits_equal(a, b) for a, b in zip(idx.centroids(), again.centroids()))
    idx.close()
    again.close()


@pytest.mark.gpu
@pytest.mark.parametrize("bits,k,tq", [(4, 10, False), (4, 64, True), (2, 10, True), (3, 1, False)])
def test_search_matches_oracle(oracle, small, bits, k, tq):
    db, q, params = small
    idx = _build(db, bits, params, calib=db[:2000] if tq else None)
    eng = idx.engine()
    shift = scale = None
    if tq:
        shift, scale = eng.calibration()
    lay = idx.layout()
    route, enc = idx.centroids()
    x_hat = idx.rows()
    starts = lay["slot_start"].astype(np.int64)
    sizes = lay["bucket_size"].astype(np.int64)
    # residual codes: the oracle's encoding of x_hat - encode_c in slot order
    ns = idx.info()["n_slots"]
    resid = np.zeros((ns, 104), np.float32)
    for b in range(len(sizes)):
        ids = lay["slot_ids"][starts[b]:starts[b] + sizes[b]]
        resid[starts[b]:starts[b] + sizes[b]] = x_hat[ids] - enc[b]
    packed, alpha = oracle.encode(resid, bits, shift, scale)
    flat = oracle.codes_flat(packed, bits, 104)
    got_flat = eng.codes_flat()[:ns]
    got_alpha = eng.alpha()[:ns]
    valid = lay["slot_ids"] != 0xFFFFFFFF
    assert bits_equal(got_flat[valid], flat[valid])
    assert bits_equal(got_alpha[valid], alpha[valid])

    tr = idx.search_trace(q, k)
    qh = tr["q_hat"]
    # routing scores against fp64, and the probes are the best-routed buckets
    _, rs = idx.route(q)
    r64 = qh.astype(np.float64) @ route.astype(np.float64).T
    assert np.max(np.abs(rs - r64)) < TOL
    for r in range(q.shape[0]):
        order = sorted(range(rs.shape[1]), key=lambda b: (-rs[r, b], b))[: tr["probes"].shape[1]]
        assert np.array_equal(tr["probes"][r], order)
    off64 = np.einsum("qd,qpd->qp", qh.astype(np.float64), enc[tr["probes"]].astype(np.float64))
    assert np.max(np.abs(tr["offsets"] - off64)) < TOL

    prep = oracle.prepare_queries(qh, bits, shift, scale)
    n_probe = np.full(q.shape[0], tr["probes"].shape[1], np.uint32)
    ws, wi = oracle.ivf_search(prep, got_flat, got_alpha, lay["slot_ids"].astype(np.uint64), starts, sizes,
                               tr["probes"], n_probe, tr["offsets"], k)
    assert np.array_equal(tr["ids"], wi[:, : tr["ids"].shape[1]])
    assert bits_equal(tr["scores"], ws[:, : tr["scores"].shape[1]])
    idx.close()


@pytest.mark.gpu
def test_rerank_matches_oracle(oracle, small):
    # rerank_k: the scan's top rerank_k candidates, re-scored with the exact
    # float <q_hat, x_hat> in the reference's float_rescore_topk order, top k kept.
    from oracle.oracle import oracle_float_rescore

    db, q, params = small
    p = vcb.BucketParams(**{**params.__dict__, "rerank_k": 40})
    idx = _build(db, 4, p)
    eng = idx.engine()
    lay = idx.layout()
    tr = idx.search_trace(q, 40)  # the scan's top-40 (k >= rerank_k: no re-rank)
    res = idx.search(q, 10)       # re-ranked top-10
    prep = oracle.prepare_queries(tr["q_hat"], 4)
    n_probe = np.full(q.shape[0], tr["probes"].shape[1], np.uint32)
    ns = idx.info()["n_slots"]
    ws, wi = oracle.ivf_search(prep, eng.codes_flat()[:ns], eng.alpha()[:ns], lay["slot_ids"].astype(np.uint64),
                               lay["slot_start"].astype(np.int64), lay["bucket_size"].astype(np.int64), tr["probes"],
                               n_probe, tr["offsets"], 40)
    assert np.array_equal(tr["ids"], wi)
    rs, ri = oracle_float_rescore(oracle, tr["q_hat"], idx.rows(), wi)
    assert np.array_equal(res.ids, ri[:, :10])
    assert bits_equal(res.scores, rs[:, :10])
    idx.close()


@pytest.mark.gpu
def test_per_query_probe_counts(small):
    db, q, params = small
    idx = _build(db, 4, params)
    counts = (np.arange(q.shape[0]) % 8 + 1).astype(np.uint32)
    mixed = idx.search(q, 10, n_probe=8, n_probe_per_query=counts)
    for c in np.unique(counts):
        rows = np.nonzero(counts == c)[0]
        alone = idx.search(q[rows], 10, n_probe=int(c))
        assert np.array_equal(mixed.ids[rows], alone.ids)
        assert bits_equal(mixed.scores[rows], alone.scores)
    idx.close()


@pytest.mark.gpu
def test_query_passes_match_small_batches(small):
    # 20,000 queries exceed one pass (at most 16,384 queries); with per-query
    # probe counts and re-ranking the passes must give exactly what the same
    # queries give in batches that fit one pass.
    db, _, params = small
    p = vcb.BucketParams(**{**params.__dict__, "rerank_k": 20})
    idx = _build(db, 4, p)
    q = vmf_mixture(20_000, db.shape[1], seed=19, clusters=60)
    counts = (np.arange(q.shape[0]) % 13 + 1).astype(np.uint32)
    whole = idx.search(q, 10, n_probe=13, n_probe_per_query=counts)
    for s in range(0, q.shape[0], 5000):
        part = idx.search(q[s:s + 5000], 10, n_probe=13, n_probe_per_query=counts[s:s + 5000])
        assert np.array_equal(whole.ids[s:s + 5000], part.ids)
        assert bits_equal(whole.scores[s:s + 5000], part.scores)
    idx.close()


@pytest.mark.gpu
def test_recall_grows_with_n_probe(small):
    db, q, params = small
    idx = _build(db, 4, params)
    x = db / np.linalg.norm(db, axis=1, keepdims=True)
    qn = q / np.linalg.norm(q, axis=1, keepdims=True)
    exact = np.argsort(-(qn.astype(np.float64) @ x.astype(np.float64).T), axis=1, kind="stable")[:, :10]
    nb = idx.info()["n_buckets"]
    recalls = []
    for npb in (1, 4, 16, min(nb, 256)):
        res = idx.search(q, 10, n_probe=npb)
        hits = sum(len(set(res.ids[r].tolist()) & set(exact[r].tolist())) for r in range(q.shape[0]))
        recalls.append(hits / (10 * q.shape[0]))
    assert all(b >= a - 0.02 for a, b in zip(recalls, recalls[1:]))
    assert recalls[-1] >= 0.85
    idx.close()


@pytest.mark.gpu
def test_add_after_prepare_keeps_invariants(small):
    db, q, params = small
    idx = _build(db[:8000], 4, params)
    _, enc0 = idx.centroids()
    idx.add(db[8000:])
    idx.prepare()
    lay = idx.layout()
    sizes = lay["bucket_size"].astype(np.int64)
    assert sizes.sum() == db.shape[0] and sizes.max() <= params.max_bucket_size
    _, enc1 = idx.centroids()
    # buckets that were not split keep their encode centroid (frozen at birth)
    kept = sum(any(bits_equal(e, f) for f in enc1) for e in enc0)
    assert kept >= len(enc0) // 2
    res = idx.search(q, 10)
    assert res.ids.shape == (q.shape[0], 10)
    idx.close()


@pytest.mark.gpu
def test_floor_schedules_at_many_buckets(oracle):
    # Passes of >= 4096 queries take 32 first probes from n_probe 128 on, with
    # an extra floor after 8 probes; smaller passes take 8 first probes below
    # n_probe 256 and no middle floor. Both must return the exhaustive top-k
    # of the probed buckets: the same queries in one pass and in passes below
    # 4096 agree bit for bit, and both equal the oracle's scan of every probed
    # bucket (no floor) on the routing's probes and offsets.
    db = vmf_mixture(120_000, 100, seed=41, clusters=300)
    params = vcb.BucketParams(n_probe=128, max_bucket_size=300, energy_soft=150, kmeans_iters=3, seed=5)
    idx = _build(db, 4, params)
    nb = idx.info()["n_buckets"]
    assert nb >= 512
    q = vmf_mixture(4608, 100, seed=42, clusters=300)
    eng = idx.engine()
    lay = idx.layout()
    ns = idx.info()["n_slots"]
    flat, alpha = eng.codes_flat()[:ns], eng.alpha()[:ns]
    slot_ids = lay["slot_ids"].astype(np.uint64)
    starts, sizes = lay["slot_start"].astype(np.int64), lay["bucket_size"].astype(np.int64)
    for n_probe in (128, 512):
        whole = idx.search(q, 10, n_probe=n_probe)
        for s in range(0, q.shape[0], 1536):
            part = idx.search(q[s:s + 1536], 10, n_probe=n_probe)
            assert np.array_equal(whole.ids[s:s + 1536], part.ids), (n_probe, s)
            assert bits_equal(whole.scores[s:s + 1536], part.scores), (n_probe, s)
        sub = slice(0, 512)
        tr = idx.search_trace(q[sub], 10, n_probe=n_probe)
        prep = oracle.prepare_queries(tr["q_hat"], 4)
        counts = np.full(tr["probes"].shape[0], n_probe, np.uint32)
        ws, wi = oracle.ivf_search(prep, flat, alpha, slot_ids, starts, sizes, tr["probes"], counts,
                                   tr["offsets"], 10)
        assert np.array_equal(whole.ids[sub], wi), n_probe
        assert bits_equal(whole.scores[sub], ws), n_probe
    # Per-query counts under a 512 cap (the learned probe's form): in a pass of
    # >= 4096 queries every query above 32 probes takes 32 first probes; in
    # smaller passes only those from 256 on. Same top-k both ways, equal to the
    # exhaustive scan of each query's own probes.
    npq = np.random.default_rng(43).integers(1, 513, q.shape[0]).astype(np.uint32)
    npq[:64] = np.arange(1, 65)  # every count around the 8 / 32 first-probe splits
    whole = idx.search(q, 10, n_probe=512, n_probe_per_query=npq)
    for s in range(0, q.shape[0], 1536):
        part = idx.search(q[s:s + 1536], 10, n_probe=512, n_probe_per_query=npq[s:s + 1536])
        assert np.array_equal(whole.ids[s:s + 1536], part.ids), s
        assert bits_equal(whole.scores[s:s + 1536], part.scores), s
    sub = slice(0, 512)
    tr = idx.search_trace(q[sub], 10, n_probe=512, n_probe_per_query=npq[sub])
    prep = oracle.prepare_queries(tr["q_hat"], 4)
    ws, wi = oracle.ivf_search(prep, flat, alpha, slot_ids, starts, sizes, tr["probes"], npq[sub],
                               tr["offsets"], 10)
    assert np.array_equal(whole.ids[sub], wi)
    assert bits_equal(whole.scores[sub], ws)
    idx.close()
