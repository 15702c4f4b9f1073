"""The CPU checker of the learned n_probe MLP (oracle/probe_oracle.py) on its
own: bf16 rounding matches torch's, and its backpropagation matches central
finite differences of its forward pass (float64, rounding off)."""
import numpy as np

from oracle import probe_oracle as po


def test_bf16_rounding_matches_torch():
    import torch

    x = np.random.default_rng(0).standard_normal(10000).astype(np.float32) * 10
    x[:4] = [0.0, 1.0, 1.00390625, 1.01171875]  # exact and tie cases
    want = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(po.bf16(x), want)


def test_backprop_matches_finite_differences():
    rng = np.random.default_rng(1)
    shapes = [(512, 8), (8, 8), (8, 5)]
    n = sum(a * b + b for a, b in shapes)
    params = rng.standard_normal(n) * 0.2
    x = rng.standard_normal((6, 512)) * 0.1
    labels = rng.integers(0, 5, 6)
    loss, grad, _ = po.forward_backward(x, params, shapes, labels, rounding=False)
    idx = rng.choice(n, 60, replace=False)
    eps = 1e-6
    for i in idx:
        p1, p2 = params.copy(), params.copy()
        p1[i] += eps
        p2[i] -= eps
        l1 = po.forward_backward(x, p1, shapes, labels, rounding=False)[0]
        l2 = po.forward_backward(x, p2, shapes, labels, rounding=False)[0]
        assert abs((l1 - l2) / (2 * eps) - grad[i]) < 1e-6 + 1e-4 * abs(grad[i])


def test_recall_objective_backprop_matches_finite_differences():
    rng = np.random.default_rng(2)
    shapes = [(512, 8), (8, 8), (8, 5)]
    n = sum(a * b + b for a, b in shapes)
    params = rng.standard_normal(n) * 0.2
    x = rng.standard_normal((6, 512)) * 0.1
    targets = rng.uniform(0, 1, (6, 5))
    loss, grad, logits = po.forward_backward(x, params, shapes, targets, rounding=False)
    # the loss is the mean binary cross-entropy of sigmoid(logits) against the targets
    s = 1 / (1 + np.exp(-logits))
    assert abs(loss - np.mean(-(targets * np.log(s) + (1 - targets) * np.log(1 - s)))) < 1e-12
    idx = rng.choice(n, 60, replace=False)
    eps = 1e-6
    for i in idx:
        p1, p2 = params.copy(), params.copy()
        p1[i] += eps
        p2[i] -= eps
        l1 = po.forward_backward(x, p1, shapes, targets, rounding=False)[0]
        l2 = po.forward_backward(x, p2, shapes, targets, rounding=False)[0]
        assert abs((l1 - l2) / (2 * eps) - grad[i]) < 1e-7 + 1e-4 * abs(grad[i])


def test_recall_rule_trades_recall_for_probes():
    classes = [1, 2, 4, 8]
    # predicted recall 0.5, 0.8, 0.9, 0.95 at the four classes
    r = np.array([[0.5, 0.8, 0.9, 0.95]])
    z = np.log(r / (1 - r))
    pick = lambda lam: int(po.predict(z, classes, "recall", lam, 0.0, 8)[0][0])
    assert pick(0.0) == 8                # recall only: the largest class
    assert pick(0.3) == 4                # 0.9 - 0.15 beats 0.95 - 0.3 and 0.8 - 0.075
    assert pick(2.0) == 2                # 0.8 - 0.5 beats 0.5 - 0.25
    assert pick(4.0) == 1                # probes dominate
    assert int(po.predict(z, classes, "recall", 0.3, 0.99, 8)[0][0]) == 8  # low confidence: fallback
