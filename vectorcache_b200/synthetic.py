"""Seeded synthetic workloads with the shapes and distributions of the flat
TurboQuant benchmark configurations (no datasets are available offline).

* `gaussian_mixture` — 256 isotropic Gaussians, centers N(0, 1) per
  coordinate, per-cluster sigma 0.35, clipped to [0, inf) and scaled so values
  span 0..255 (a SIFT-like stand-in; 100k x 128 in the small configuration).
* `power_law` — Gaussian with per-coordinate variances lambda_i ~ i^-0.8,
  rotated by a seeded Haar-random orthogonal matrix, then L2-normalized (an
  embedding-like stand-in; 1M x 1536 in the large configuration).

The numpy versions serve parity tests; `power_law_torch` generates the same
distribution on a CUDA device for the 1M-row benchmark (different random
stream, same law).
"""
from __future__ import annotations

import numpy as np


def gaussian_mixture(n_db: int, n_q: int, dim: int, seed: int = 0, clusters: int = 256,
                     sigma: float = 0.35) -> tuple[np.ndarray, np.ndarray]:
    rng = np.random.default_rng(seed)
    centers = rng.standard_normal((clusters, dim)).astype(np.float32)

    def draw(m):
        lab = rng.integers(0, clusters, m)
        x = centers[lab] + sigma * rng.standard_normal((m, dim)).astype(np.float32)
        return np.clip(x, 0.0, None)

    db, q = draw(n_db), draw(n_q)
    scale = np.float32(255.0) / np.float32(max(float(db.max()), 1e-12))
    return (db * scale).astype(np.float32), (q * scale).astype(np.float32)


def haar_orthogonal(dim: int, seed: int) -> np.ndarray:
    """QR of a Gaussian matrix with the sign fix that makes it Haar-distributed."""
    g = np.random.default_rng(seed).standard_normal((dim, dim))
    q, r = np.linalg.qr(g)
    q *= np.sign(np.diag(r))[None, :]
    return q


def power_law_spectrum(dim: int, exponent: float = 0.8) -> np.ndarray:
    return np.arange(1, dim + 1, dtype=np.float64) ** -exponent


def power_law(n: int, dim: int, seed: int = 0, rot_seed: int = 1234) -> np.ndarray:
    rng = np.random.default_rng(seed)
    z = rng.standard_normal((n, dim)) * np.sqrt(power_law_spectrum(dim))[None, :]
    x = z @ haar_orthogonal(dim, rot_seed).T
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    return x.astype(np.float32)


def power_law_torch(n: int, dim: int, seed: int, device, rot_seed: int = 1234, chunk: int = 65536):
    """Same law as `power_law`, generated on `device` in row chunks."""
    import torch

    rot = torch.as_tensor(haar_orthogonal(dim, rot_seed).T, dtype=torch.float32, device=device)
    sd = torch.as_tensor(np.sqrt(power_law_spectrum(dim)), dtype=torch.float32, device=device)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    out = torch.empty((n, dim), dtype=torch.float32, device=device)
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        for s in range(0, n, chunk):
            e = min(n, s + chunk)
            z = torch.randn((e - s, dim), generator=gen, device=device, dtype=torch.float32) * sd
            x = z @ rot
            out[s:e] = x / torch.linalg.vector_norm(x, dim=1, keepdim=True)
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    return out
