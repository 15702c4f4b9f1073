"""Serving loop (continuous batching) on the GPU: every request's result is the
same as the same search run alone, whatever it was batched or overlapped with;
an open-loop Poisson replay completes with sane latencies; the learned probe
runs inside the server; a batch whose scratch does not fit the HBM budget's
arena waits until running batches free theirs."""
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


def test_requests_wait_for_memory_and_run_when_it_frees(indexes):
    # The HBM budget leaves scratch for about 1.5 full batches, with four slots
    # free: of two full batches submitted together, the second waits for the
    # first one's scratch, then runs. Both equal the same search alone.
    flat, bkt, db, xb = indexes
    roomy = vcb.Server(max_slots=4, max_batch=4096)
    fid = roomy.add_flat(flat, 64)
    roomy.start()
    resident = roomy.info()["resident_bytes"]
    need = roomy.batch_bytes(fid, 4096, 64)
    mem = roomy.memory()
    roomy.close()
    assert need > (16 << 20) and mem["max_batch_bytes"] >= need
    srv = vcb.Server(hbm_budget_bytes=resident + need + need // 2, max_slots=4, max_batch=4096)
    fid = srv.add_flat(flat, 64)
    srv.start()
    arena = srv.memory()["arena_bytes"]
    assert need <= arena < 2 * srv.batch_bytes(fid, 4096, 63)
    rng = np.random.default_rng(9)
    qa = db[rng.integers(0, db.shape[0], 4096)] + rng.normal(0, 0.01, (4096, 128)).astype(np.float32)
    qb = db[rng.integers(0, db.shape[0], 4096)] + rng.normal(0, 0.01, (4096, 128)).astype(np.float32)
    # different k: two batches, submitted back to back
    lat, wall, results = srv.replay([(0.0, fid, qa, 64, 0), (0.0, fid, qb, 63, 0)])
    mem = srv.memory()
    assert mem["memory_waits"] >= 1
    assert mem["arena_peak"] <= mem["arena_bytes"] and mem["arena_peak"] < 2 * need
    assert lat[1] > lat[0]
    for (q, k), (s, i) in zip(((qa, 64), (qb, 63)), results):
        want = flat.search(q, k)
        assert np.array_equal(i, want.ids) and bits_equal(s, want.scores)
    assert srv.stats()["completed"] == 2
    srv.close()
    tiny = vcb.Server(hbm_budget_bytes=1 << 20, max_slots=2, max_batch=256)
    tiny.add_flat(flat, 10)
    with pytest.raises(vcb.TurboQuantError):
        tiny.start()
    tiny.close()


def test_batch_sizing_matches_what_runs(indexes):
    # The arena piece of a batch is its exact scratch: batches of every size,
    # k and n_probe run inside their pieces (a piece too small fails the
    # batch), and the sizing of a full batch bounds all smaller ones tried.
    flat, bkt, db, xb = indexes
    srv = vcb.Server(max_slots=2, max_batch=512)
    fid = srv.add_flat(flat, 64)
    bid = srv.add_bucketed(bkt, 64, 32)
    srv.start()
    top = srv.memory()["max_batch_bytes"]
    rng = np.random.default_rng(4)
    for _ in range(24):
        target = int(rng.integers(0, 2))
        nq = int(rng.choice([1, 2, 3, 17, 200, 512]))
        k = int(rng.choice([1, 10, 33, 64]))
        npb = int(rng.choice([4, 32]))
        assert 0 < srv.batch_bytes(target, nq, k, npb) <= top
        src = db if target == fid else xb
        q = src[rng.integers(0, src.shape[0], nq)]
        s, i, _ = srv.submit(target, q, k, npb if target == bid else 0).wait()
        want = _alone(flat, bkt, target, fid, q, k, npb)
        assert np.array_equal(i, want.ids)
    srv.close()
