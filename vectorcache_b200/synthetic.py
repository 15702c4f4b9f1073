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


def _vmf_directions(mu: np.ndarray, kappa: np.ndarray, rng) -> np.ndarray:
    """Samples from von Mises-Fisher distributions around unit means mu (m x d)
    with concentrations kappa (m,), by Wood's (1994) rejection sampler for the
    cosine w and a uniform tangent direction."""
    m, d = mu.shape
    b = (-2.0 * kappa + np.sqrt(4.0 * kappa ** 2 + (d - 1.0) ** 2)) / (d - 1.0)
    x0 = (1.0 - b) / (1.0 + b)
    c = kappa * x0 + (d - 1.0) * np.log(1.0 - x0 ** 2)
    w = np.empty(m)
    todo = np.arange(m)
    while todo.size:
        z = rng.beta((d - 1.0) / 2.0, (d - 1.0) / 2.0, todo.size)
        u = rng.random(todo.size)
        bb, xx, cc, kk = b[todo], x0[todo], c[todo], kappa[todo]
        ww = (1.0 - (1.0 + bb) * z) / (1.0 - (1.0 - bb) * z)
        ok = kk * ww + (d - 1.0) * np.log(1.0 - xx * ww) - cc >= np.log(u)
        w[todo[ok]] = ww[ok]
        todo = todo[~ok]
    v = rng.standard_normal((m, d))
    v -= np.sum(v * mu, axis=1, keepdims=True) * mu
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return w[:, None] * mu + np.sqrt(np.maximum(0.0, 1.0 - w ** 2))[:, None] * v


def vmf_mixture(n: int, dim: int, seed: int = 0, clusters: int = 2000, kappa_range=(20.0, 200.0),
                zipf_s: float = 1.1, centers_seed: int = 4321) -> np.ndarray:
    """Mixture of von Mises-Fisher clusters: uniform random unit centers,
    kappa log-uniform in kappa_range, cluster sizes Zipf(zipf_s) over cluster
    rank; rows are L2-normalized float32 (a GloVe-angular-like stand-in; the
    bucketed configuration uses 1.2M x 100 with 2000 clusters). The centers and
    kappas depend only on `centers_seed`, so database and query draws with
    different `seed` share the same clusters."""
    crng = np.random.default_rng(centers_seed)
    mu = crng.standard_normal((clusters, dim))
    mu /= np.linalg.norm(mu, axis=1, keepdims=True)
    kappa = np.exp(crng.uniform(np.log(kappa_range[0]), np.log(kappa_range[1]), clusters))
    p = np.arange(1, clusters + 1, dtype=np.float64) ** -zipf_s
    p /= p.sum()
    rng = np.random.default_rng(seed)
    lab = rng.choice(clusters, size=n, p=p)
    out = np.empty((n, dim), np.float32)
    chunk = 1 << 16
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        x = _vmf_directions(mu[lab[s:e]], kappa[lab[s:e]], rng)
        out[s:e] = (x / np.linalg.norm(x, axis=1, keepdims=True)).astype(np.float32)
    return out


def ivf_case(n: int, dim: int, n_buckets: int, nq: int, max_probe: int, seed: int = 0,
             all_probed: bool = False, slot_align: int = 256) -> dict:
    """A small bucketed-index layout for parity tests: unit rows assigned to
    their nearest of `n_buckets` random centers, encode centroid = fp32 mean of
    the members, residual rows in bucket order at slot-aligned starts (padding
    slots are zero rows with id 2^64-1), per-query probes (nearest centers
    first), per-query probe counts, and offsets <q, encode_c> in fp32."""
    rng = np.random.default_rng(seed)
    centers = rng.standard_normal((n_buckets, dim)).astype(np.float32)
    x = centers[rng.integers(0, n_buckets, n)] + 0.6 * rng.standard_normal((n, dim)).astype(np.float32)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    x = x.astype(np.float32)
    lab = np.argmax(x @ centers.T, axis=1)
    size = np.bincount(lab, minlength=n_buckets).astype(np.uint64)
    padded = ((size + slot_align - 1) // slot_align) * slot_align
    start = np.concatenate([[0], np.cumsum(padded)[:-1]]).astype(np.uint64)
    n_slots = int(padded.sum())
    enc_c = np.zeros((n_buckets, dim), np.float32)
    residuals = np.zeros((n_slots, dim), np.float32)
    ids = np.full(n_slots, np.iinfo(np.uint64).max, np.uint64)
    for b in range(n_buckets):
        members = np.nonzero(lab == b)[0]
        if members.size == 0:
            continue
        enc_c[b] = x[members].mean(axis=0, dtype=np.float64).astype(np.float32)
        st = int(start[b])
        residuals[st:st + members.size] = x[members] - enc_c[b]
        ids[st:st + members.size] = members
    q = rng.standard_normal((nq, dim)).astype(np.float32)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    q = q.astype(np.float32)
    route = q @ centers.T
    order = np.argsort(-route, axis=1, kind="stable")[:, :max_probe].astype(np.uint32)
    n_probe = (np.full(nq, max_probe) if all_probed else rng.integers(1, max_probe + 1, nq)).astype(np.uint32)
    offsets = np.einsum("qd,qpd->qp", q, enc_c[order]).astype(np.float32)
    valid = np.nonzero(ids != np.iinfo(np.uint64).max)[0]
    return {"x": x, "q": q, "residuals": residuals, "ids": ids, "start": start, "size": size,
            "probes": order, "n_probe": n_probe, "offsets": offsets, "encode_c": enc_c,
            "calib_slots": valid[: min(500, valid.size)]}
