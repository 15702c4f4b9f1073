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
