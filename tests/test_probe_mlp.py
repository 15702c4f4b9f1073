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


def test_recall_objective_gradients_and_rules_match_cpu_checker():
    top = _fake_routing(96, 11)
    classes = DEFAULT_CLASSES
    for objective in ("classes", "recall"):
        mlp = ProbeMLP(hidden=128, layers=2, seed=4, objective=objective)
        raw = mlp.features(top)
        mlp.set_normalization(raw.mean(axis=0), raw.std(axis=0) + 1e-6)
        rng = np.random.default_rng(12)
        if objective == "recall":
            targets = rng.uniform(0, 1, (96, len(classes))).astype(np.float32)
            # the classes-objective entry points refuse a recall model
            g = np.empty(mlp.n_params, np.float32)
            lab = np.zeros(96, np.uint32)
            assert mlp._lib.tq_probe_mlp_gradients(mlp._h, top.ctypes.data, lab.ctypes.data, 96, 256, None,
                                                   g.ctypes.data) == 2
        else:
            targets = rng.integers(0, len(classes), 96).astype(np.uint32)
        x = po.inputs(raw, mlp.mean, mlp.std)
        loss_c, grad_c, _ = po.forward_backward(x, mlp.params(), mlp.shapes(), targets)
        loss_g, grad_g = mlp.gradients(top, targets)
        assert abs(loss_g - loss_c) < 1e-4 * max(1.0, abs(loss_c))
        rel = np.linalg.norm(grad_g - grad_c) / np.linalg.norm(grad_c)
        assert rel < GRAD_RTOL, (objective, rel)
        # the device prediction rule against the checker's, on the device logits
        import torch

        logits = mlp.forward(top)
        d_top = torch.from_numpy(top).cuda()
        out = torch.empty(96, dtype=torch.int32, device="cuda")
        for rule in ((0.5, 0.7, 0.95) if objective == "classes" else (0.0, 0.05, 0.2, 1.0)):
            mlp.predict_device(d_top, 96, 256, out, coverage=rule, min_confidence=0.0, fallback=512)
            torch.cuda.synchronize()
            want, margin = po.predict(logits, classes, objective, rule, 0.0, 512)
            got = out.cpu().numpy()
            sure = margin > 1e-5
            assert sure.sum() > 80
            assert np.array_equal(got[sure], want[sure]), (objective, rule)
        mlp.close()


@pytest.fixture(scope="module")
def small_bucketed():
    # A scaled-down copy of the bucketed benchmark: vMF mixture (2000 clusters,
    # kappa log-uniform in [20, 200], Zipf sizes), dim 100, 4-bit, top-50
    # re-rank. The plain path's operating point is the smallest fixed n_probe
    # reaching Recall@10 >= 0.9.
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
    labels, rec = probe_labels(lambda q, p: idx.search(q, 10, n_probe=p).ids, train_q, ex_train, classes, 10, p_op)

    def route(q):
        dq = torch.from_numpy(q).cuda()
        ts = torch.empty((q.shape[0], 256), dtype=torch.float32, device="cuda")
        ti = torch.empty((q.shape[0], 256), dtype=torch.int32, device="cuda")
        idx.route_device(dq, 256, ts, ti)
        torch.cuda.synchronize()
        return ts

    yield {"idx": idx, "test_q": test_q, "ex_test": ex_test, "p_op": p_op, "classes": classes, "labels": labels,
           "rec": rec, "tr": route(train_q), "te": route(test_q)}
    idx.close()


def _trained(setup, objective):
    import torch

    mlp = ProbeMLP(classes=setup["classes"], hidden=128, layers=2, seed=9, objective=objective)
    tr = setup["tr"]
    raw = mlp.features(tr.cpu().numpy())
    mlp.set_normalization(raw.mean(axis=0), raw.std(axis=0) + 1e-6)
    if objective == "recall":
        d_tgt = torch.from_numpy(setup["rec"].astype(np.float32)).cuda()
    else:
        d_tgt = torch.from_numpy(setup["labels"].astype(np.int32)).cuda()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(1)
    m = tr.shape[0]
    for epoch in range(30):
        perm = torch.randperm(m, device="cuda", generator=gen)
        for s in range(0, m, 512):
            sel = perm[s:s + 512]
            mlp.train_step_device(tr[sel].contiguous(), d_tgt[sel].contiguous(), sel.numel(), 256, 2e-3)
    return mlp


def _gain(setup, mlp, rule):
    """(mean n_probe, learned recall, recall of one fixed n_probe at that mean)."""
    import torch

    idx, test_q, ex_test, p_op, te = (setup[k] for k in ("idx", "test_q", "ex_test", "p_op", "te"))
    npq = torch.empty(test_q.shape[0], dtype=torch.int32, device="cuda")
    mlp.predict_device(te, test_q.shape[0], 256, npq, coverage=rule, min_confidence=0.0, fallback=p_op)
    torch.cuda.synchronize()
    npq = npq.cpu().numpy().astype(np.uint32)
    learned = idx.search(test_q, 10, n_probe=p_op, n_probe_per_query=npq)
    r_learned = recall_rows(learned.ids, ex_test, 10).mean()
    mean_probe = int(np.ceil(npq.mean()))
    r_same_cost = recall_rows(idx.search(test_q, 10, n_probe=max(mean_probe, 1)).ids, ex_test, 10).mean()
    return npq.mean(), r_learned, r_same_cost


def test_learned_probe_gains_over_fixed_probe(small_bucketed):
    # The network must reach (nearly) the plain recall while scanning clearly
    # fewer buckets on average: at the same mean number of buckets scanned, its
    # per-query allocation reaches a higher recall than one fixed n_probe.
    import torch

    setup = small_bucketed
    p_op = setup["p_op"]
    mlp = _trained(setup, "classes")
    mean_probe, r_learned, r_same_cost = _gain(setup, mlp, 0.7)
    assert np.ceil(mean_probe) < p_op, (mean_probe, p_op, np.bincount(setup["labels"]))
    assert r_learned > r_same_cost + 0.005, (r_learned, r_same_cost, mean_probe)
    # low confidence falls back to the fixed n_probe
    te, nq = setup["te"], setup["test_q"].shape[0]
    fb = torch.empty(nq, dtype=torch.int32, device="cuda")
    mlp.predict_device(te, nq, 256, fb, coverage=0.95, min_confidence=1.01, fallback=p_op)
    torch.cuda.synchronize()
    assert np.all(fb.cpu().numpy() == p_op)
    mlp.close()


def test_recall_objective_gains_over_fixed_probe(small_bucketed):
    # The recall objective: a larger trade-off never scans more buckets, and
    # some trade-off beats one fixed n_probe of the same mean cost.
    setup = small_bucketed
    mlp = _trained(setup, "recall")
    runs = [_gain(setup, mlp, lam) for lam in (0.02, 0.05, 0.1, 0.2)]
    means = [r[0] for r in runs]
    assert all(a >= b for a, b in zip(means, means[1:])), means
    assert any(np.ceil(mp) < setup["p_op"] and rl > rs + 0.005 for mp, rl, rs in runs), runs
    mlp.close()
