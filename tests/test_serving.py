"""Serving loop (continuous batching) on the GPU: every request's result is the
same as the same search run alone, whatever it was batched or overlapped with;
an open-loop Poisson replay completes with sane latencies; the learned probe
runs inside the server; the HBM budget bounds the number of slots."""
import numpy as np
import pytest

import vectorcache_b200 as vcb
from vectorcache_b200.bucketed import search_learned_device
from vectorcache_b200.probe import ProbeMLP
from vectorcache_b200.synthetic import gaussian_mixture, vmf_mixture

pytestmark = pytest.mark.gpu


def bits_equal(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.fixture(scope="module")
def indexes():
    db, _ = gaussian_mixture(40000, 10, 128, seed=3)
    flat = vcb.TurboQuantIndex(128, 4)
    flat.calibrate(db[:2000])
    flat.add(db)
    flat.prepare()
    xb = vmf_mixture(30000, 100, seed=5, clusters=300)
    bkt = vcb.BucketedTurboQuantIndex(100, 4, vcb.BucketParams(max_bucket_size=400, energy_soft=200, rerank_k=40))
    bkt.add(xb)
    bkt.prepare()
    yield flat, bkt, db, xb
    flat.close()
    bkt.close()


def _alone(flat, bkt, target, fid, q, k, npb):
    if target == fid:
        return flat.search(q, k)
    return bkt.search(q, k, n_probe=npb)


def test_results_same_alone_and_in_the_mix(indexes):
    flat, bkt, db, xb = indexes
    srv = vcb.Server(max_slots=4, max_batch=512)
    fid = srv.add_flat(flat, 64)
    bid = srv.add_bucketed(bkt, 64, 32)
    srv.start()
    assert srv.info()["slots"] >= 1
    rng = np.random.default_rng(0)
    reqs = []
    for _ in range(160):
        target = int(rng.integers(0, 2))
        nq = int(rng.integers(1, 65))
        k = int(rng.choice([10, 64]))
        npb = int(rng.choice([8, 32]))
        src = db if target == fid else xb
        q = src[rng.integers(0, src.shape[0], nq)] + rng.normal(0, 0.01, (nq, src.shape[1])).astype(np.float32)
        reqs.append((target, q, k, npb, srv.submit(target, q, k, npb if target == bid else 0)))
    got = [r.wait() for *_, r in reqs]  # all served before the indexes are used directly
    for (target, q, k, npb, _), (s, i, lat) in zip(reqs, got):
        want = _alone(flat, bkt, target, fid, q, k, npb)
        assert np.array_equal(i, want.ids) and bits_equal(s, want.scores)
        assert lat > 0
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["batches"] <= len(reqs)
    srv.close()


def test_poisson_replay(indexes):
    flat, bkt, db, xb = indexes
    srv = vcb.Server(max_slots=3, max_batch=1024)
    fid = srv.add_flat(flat, 64)
    bid = srv.add_bucketed(bkt, 64, 32)
    srv.start()
    rng = np.random.default_rng(1)
    rate, dur = 20000.0, 0.25  # queries / s, seconds
    t, trace = 0.0, []
    while t < dur * 1e6:
        nq = int(rng.integers(1, 257))
        t += rng.exponential(nq / rate * 1e6)
        target = int(rng.integers(0, 2))
        src = db if target == fid else xb
        q = src[rng.integers(0, src.shape[0], nq)]
        trace.append((t, target, q, int(rng.choice([10, 64])), 32 if target == bid else 0))
    lat, wall, results = srv.replay(trace)
    assert lat.shape == (len(trace),) and np.all(lat > 0) and wall > 0
    for (t_us, target, q, k, npb), (s, i) in list(zip(trace, results))[:20]:
        want = _alone(flat, bkt, target, fid, q, k, npb)
        assert np.array_equal(i, want.ids)
    srv.close()


def test_learned_probe_in_the_server(indexes):
    import torch

    flat, bkt, db, xb = indexes
    mlp = ProbeMLP(classes=(2, 4, 8, 16, 32), hidden=64, layers=2, seed=4)
    srv = vcb.Server(max_slots=2, max_batch=256)
    bid = srv.add_bucketed(bkt, 10, 32, mlp=mlp, coverage=0.8)
    srv.start()
    q = xb[:200] + np.random.default_rng(2).normal(0, 0.01, (200, 100)).astype(np.float32)
    r = [srv.submit(bid, q[j:j + 50], 10, 32) for j in range(0, 200, 50)]
    got = [x.wait() for x in r]
    dq = torch.from_numpy(q).cuda()
    ds = torch.empty((200, 10), dtype=torch.float32, device="cuda")
    di = torch.empty((200, 10), dtype=torch.int64, device="cuda")
    search_learned_device(bkt, dq, 10, mlp, ds, di, coverage=0.8, fallback_n_probe=32)
    torch.cuda.synchronize()
    want_i = di.cpu().numpy().view(np.uint64)
    for j, (s, i, _) in enumerate(got):
        assert np.array_equal(i, want_i[50 * j:50 * j + 50])
    srv.close()
    mlp.close()


def test_budget_bounds_the_slots(indexes):
    flat, bkt, db, xb = indexes
    probe = vcb.Server(max_slots=1, max_batch=8192)
    probe.add_flat(flat, 64)
    probe.start()
    inf = probe.info()
    probe.close()
    assert inf["slot_bytes"] > (8 << 20)  # LUTs alone: 8192 x 64 x 32 bytes
    # room for about 2.5 slots: the server stops at 1 to 3 of the 8 allowed
    srv = vcb.Server(hbm_budget_bytes=inf["resident_bytes"] + int(2.5 * inf["slot_bytes"]), max_slots=8,
                     max_batch=8192)
    srv.add_flat(flat, 64)
    srv.start()
    assert 1 <= srv.info()["slots"] <= 3
    srv.close()
    tiny = vcb.Server(hbm_budget_bytes=1 << 20, max_slots=2, max_batch=256)
    tiny.add_flat(flat, 10)
    with pytest.raises(vcb.TurboQuantError):
        tiny.start()
    tiny.close()
