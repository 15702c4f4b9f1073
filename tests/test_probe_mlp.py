"""Learned n_probe MLP: its GPU forward pass and gradients against the float64
CPU checker (oracle/probe_oracle.py, same bf16 rounding points), training on
the GPU lowers the loss, and on a bucketed index the learned per-query n_probe
reaches the plain fixed-n_probe recall with fewer buckets scanned."""
import numpy as np
import pytest

import vectorcache_b200 as vcb
from oracle import probe_oracle as po
from vectorcache_b200.probe import DEFAULT_CLASSES, ProbeMLP, probe_labels, recall_rows
from vectorcache_b200.synthetic import vmf_mixture

pytestmark = pytest.mark.gpu

GRAD_RTOL = 2e-3  # ||g_gpu - g_cpu|| / ||g_cpu||: fp32 vs fp64 accumulation, rare bf16 activation flips


def _fake_routing(m, seed):
    rng = np.random.default_rng(seed)
    base = rng.uniform(0.3, 0.9, (m, 1))
    steps = rng.exponential(rng.uniform(1e-3, 1e-2, (m, 1)), (m, 256))
    return (base - np.cumsum(steps, axis=1)).astype(np.float32)


def test_forward_and_gradients_match_cpu_checker():
    mlp = ProbeMLP(hidden=128, layers=2, seed=3)
    top = _fake_routing(96, 1)
    raw = mlp.features(top)
    # features: scores then gaps, gap vector zero-padded
    assert np.array_equal(raw[:, :256], top)
    assert np.array_equal(raw[:, 256:511], (top[:, :-1] - top[:, 1:]).astype(np.float32))
    assert np.all(raw[:, 511] == 0)
    mean, std = raw.mean(axis=0), raw.std(axis=0) + 1e-6
    mlp.set_normalization(mean, std)
    labels = np.random.default_rng(2).integers(0, len(DEFAULT_CLASSES), 96).astype(np.uint32)
    params = mlp.params()
    x = po.inputs(raw, mlp.mean, mlp.std)
    loss_c, grad_c, logits_c = po.forward_backward(x, params, mlp.shapes(), labels)
    logits_g = mlp.forward(top)
    assert np.max(np.abs(logits_g - logits_c)) < 1e-3 * max(1.0, np.max(np.abs(logits_c)))
    loss_g, grad_g = mlp.gradients(top, labels)
    assert abs(loss_g - loss_c) < 1e-4 * max(1.0, abs(loss_c))
    rel = np.linalg.norm(grad_g - grad_c) / np.linalg.norm(grad_c)
    assert rel < GRAD_RTOL, rel
    # per layer as well
    off = 0
    for fi, fo in mlp.shapes():
        n = fi * fo + fo
        g, c = grad_g[off:off + n], grad_c[off:off + n]
        assert np.linalg.norm(g - c) <= GRAD_RTOL * np.linalg.norm(c) + 1e-9
        off += n
    mlp.close()


def test_training_on_gpu_lowers_loss():
    import torch

    mlp = ProbeMLP(hidden=128, layers=2, seed=5)
    top = _fake_routing(4096, 7)
    # a learnable rule: the label follows the first gap
    gap = top[:, 0] - top[:, 1]
    labels = np.digitize(gap, np.quantile(gap, np.linspace(0, 1, 9)[1:-1])).astype(np.uint32)
    raw = mlp.features(top)
    mlp.set_normalization(raw.mean(axis=0), raw.std(axis=0) + 1e-6)
    d_top = torch.from_numpy(top).cuda()
    d_lab = torch.from_numpy(labels.astype(np.int32)).cuda()
    first = None
    for epoch in range(30):
        for s in range(0, 4096, 512):
            loss = mlp.train_step_device(d_top[s:s + 512], d_lab[s:s + 512], 512, 256, 3e-3)
            first = loss if first is None else first
    logits = mlp.forward(top)
    acc = float(np.mean(np.argmax(logits, axis=1) == labels))
    assert loss < 0.5 * first and acc > 0.6
    mlp.close()


def test_learned_probe_gains_over_fixed_probe():
    # A scaled-down copy of the bucketed benchmark: vMF mixture (2000 clusters,
    # kappa log-uniform in [20, 200], Zipf sizes), dim 100, 4-bit, top-50
    # re-rank. The plain path's operating point is the smallest fixed n_probe
    # reaching Recall@10 >= 0.9; the network must reach (nearly) the same
    # recall while scanning clearly fewer buckets on average.
    import torch

    dim, n = 100, 200_000
    db = vmf_mixture(n, dim, seed=41)
    train_q = vmf_mixture(20_000, dim, seed=42)
    test_q = vmf_mixture(2000, dim, seed=43)
    params = vcb.BucketParams(max_bucket_size=800, energy_soft=400, expected_n=n, rerank_k=50, seed=3)
    idx = vcb.BucketedTurboQuantIndex(dim, 4, params)
    idx.add(db)
    idx.prepare()
    assert idx.info()["n_buckets"] >= 256
    x = torch.from_numpy(db).cuda()

    def exact(q):
        qq = torch.from_numpy(q).cuda()
        return torch.topk(qq @ x.T, 10, dim=1).indices.cpu().numpy()  # rows are unit vectors already

    ex_train, ex_test = exact(train_q), exact(test_q)
    fixed_rec = {}
    for p in (16, 32, 64, 128, 256):
        fixed_rec[p] = recall_rows(idx.search(test_q, 10, n_probe=p).ids, ex_test, 10).mean()
    p_op = next((p for p in fixed_rec if fixed_rec[p] >= 0.9), 256)
    classes = tuple(c for c in (1, 2, 4, 8, 16, 32, 64, 128, 256) if c <= p_op)
    labels, _ = probe_labels(lambda q, p: idx.search(q, 10, n_probe=p).ids, train_q, ex_train, classes, 10, p_op)
    mlp = ProbeMLP(classes=classes, hidden=128, layers=2, seed=9)

    def route(q):
        dq = torch.from_numpy(q).cuda()
        ts = torch.empty((q.shape[0], 256), dtype=torch.float32, device="cuda")
        ti = torch.empty((q.shape[0], 256), dtype=torch.int32, device="cuda")
        idx.route_device(dq, 256, ts, ti)
        torch.cuda.synchronize()
        return ts

    tr = route(train_q)
    raw = mlp.features(tr.cpu().numpy())
    mlp.set_normalization(raw.mean(axis=0), raw.std(axis=0) + 1e-6)
    d_lab = torch.from_numpy(labels.astype(np.int32)).cuda()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(1)
    for epoch in range(30):
        perm = torch.randperm(train_q.shape[0], device="cuda", generator=gen)
        for s in range(0, train_q.shape[0], 512):
            sel = perm[s:s + 512]
            mlp.train_step_device(tr[sel].contiguous(), d_lab[sel].contiguous(), sel.numel(), 256, 2e-3)
    te = route(test_q)
    npq = torch.empty(test_q.shape[0], dtype=torch.int32, device="cuda")
    mlp.predict_device(te, test_q.shape[0], 256, npq, coverage=0.7, min_confidence=0.0, fallback=p_op)
    torch.cuda.synchronize()
    npq = npq.cpu().numpy().astype(np.uint32)
    learned = idx.search(test_q, 10, n_probe=p_op, n_probe_per_query=npq)
    r_learned = recall_rows(learned.ids, ex_test, 10).mean()
    # What the network gains: at the same mean number of buckets scanned, its
    # per-query allocation reaches a higher recall than one fixed n_probe.
    mean_probe = int(np.ceil(npq.mean()))
    assert mean_probe < p_op, (npq.mean(), p_op, np.bincount(labels))
    r_same_cost = recall_rows(idx.search(test_q, 10, n_probe=mean_probe).ids, ex_test, 10).mean()
    assert r_learned > r_same_cost + 0.005, (r_learned, r_same_cost, mean_probe)
    # low confidence falls back to the fixed n_probe
    fb = torch.empty(test_q.shape[0], dtype=torch.int32, device="cuda")
    mlp.predict_device(te, test_q.shape[0], 256, fb, coverage=0.95, min_confidence=1.01, fallback=p_op)
    torch.cuda.synchronize()
    assert np.all(fb.cpu().numpy() == p_op)
    mlp.close()
    idx.close()
