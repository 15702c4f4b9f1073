"""Test infrastructure only — the CPU checker of the learned n_probe MLP.

The MLP has no counterpart in the reference, so this checker is not pinned to
reference code: it restates the network's definition (vectorcache_b200
tq_probe.cu) in float64 numpy with the same bf16 rounding points — inputs,
weights, hidden activations and the dZ operands of the backward products are
rounded to bf16 exactly where the GPU rounds them — and computes the mean loss of either training objective
(softmax cross-entropy on labels, or per-class sigmoid cross-entropy on
recall targets) and its gradients by explicit backpropagation. Also the
prediction rules. Only tests/ import it.
"""
from __future__ import annotations

import numpy as np


def bf16(x) -> np.ndarray:
    """Round float32 values to the nearest bfloat16 (ties to even), returned as
    float32 (finite inputs)."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32)


def unpack(params: np.ndarray, shapes):
    out, off = [], 0
    for fi, fo in shapes:
        w = params[off:off + fi * fo].reshape(fi, fo)
        off += fi * fo
        b = params[off:off + fo]
        off += fo
        out.append((w, b))
    return out


def inputs(raw: np.ndarray, mean: np.ndarray, std: np.ndarray) -> np.ndarray:
    """Standardized bf16 inputs: bf16(fp32(fp32(raw - mean) * fp32(1 / std)))."""
    isd = np.where(std > np.float32(1e-12), np.float32(1.0) / std.astype(np.float32), np.float32(0.0))
    v = (raw.astype(np.float32) - mean.astype(np.float32)).astype(np.float32) * isd.astype(np.float32)
    return bf16(v.astype(np.float32))


def forward_backward(x: np.ndarray, params: np.ndarray, shapes, labels: np.ndarray, rounding: bool = True):
    """x: bf16-valued inputs (m x 512). labels: m label classes (softmax
    cross-entropy) or an m x n_classes matrix of recall targets in [0, 1]
    (per-class sigmoid binary cross-entropy, mean over all entries). Returns
    (loss, grads float64, logits). rounding=False drops the bf16 rounding
    (float64 throughout) for finite-difference checks of the
    backpropagation itself."""
    rnd = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    layers = unpack(params if not rounding else params.astype(np.float32), shapes)
    m = x.shape[0]
    acts = [x.astype(np.float64)]
    zs = []
    h = acts[0]
    for li, (w, b) in enumerate(layers):
        z = h @ rnd(w).astype(np.float64) + b.astype(np.float64)
        zs.append(z)
        if li + 1 < len(layers):
            h = rnd(np.maximum(z, 0.0).astype(np.float32) if rounding else np.maximum(z, 0.0)).astype(np.float64)
            acts.append(h)
    logits = zs[-1]
    labels = np.asarray(labels)
    if labels.ndim == 2:
        # recall objective: per-class sigmoid, binary cross-entropy against
        # soft targets, mean over queries and classes
        t = labels.astype(np.float64)
        n_cls = logits.shape[1]
        loss = float(np.mean(np.maximum(logits, 0.0) - t * logits + np.log1p(np.exp(-np.abs(logits)))))
        dz = (1.0 / (1.0 + np.exp(-logits)) - t) / (m * n_cls)
    else:
        mx = logits.max(axis=1, keepdims=True)
        e = np.exp(logits - mx)
        p = e / e.sum(axis=1, keepdims=True)
        loss = float(np.mean(np.log(e.sum(axis=1)) - (logits[np.arange(m), labels] - mx[:, 0])))
        dz = p.copy()
        dz[np.arange(m), labels] -= 1.0
        dz /= m
    grads = []
    for li in range(len(layers) - 1, -1, -1):
        w, _ = layers[li]
        # the products take dZ rounded to bf16 (from fp32); the bias gradient sums dZ itself
        dzr = rnd(dz.astype(np.float32)).astype(np.float64) if rounding else dz
        gw = acts[li].T @ dzr
        gb = dz.sum(axis=0)
        grads.append((gw, gb))
        if li > 0:
            da = dzr @ rnd(w).astype(np.float64).T
            dz = da * (zs[li - 1] > 0)
    grads.reverse()
    flat = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
    return loss, flat, logits


def predict(logits: np.ndarray, classes, objective: str, coverage: float, min_confidence: float, fallback: int):
    """The prediction rules on logits (float64). Returns (n_probe per row, the
    margin of the chosen class over the runner-up: rows with a tiny margin may
    legitimately pick differently in fp32)."""
    z = np.asarray(logits, np.float64)
    cls = np.asarray(classes, np.float64)
    if objective == "recall":
        r = 1.0 / (1.0 + np.exp(-z))
        v = r - coverage * cls[None, :] / cls[-1]
        pick = np.argmax(v, axis=1)
        srt = np.sort(v, axis=1)
        margin = srt[:, -1] - srt[:, -2]
        conf = r.max(axis=1)
    else:
        e = np.exp(z - z.max(axis=1, keepdims=True))
        p = e / e.sum(axis=1, keepdims=True)
        c = np.cumsum(p, axis=1)
        reach = c >= coverage
        pick = np.where(reach.any(axis=1), reach.argmax(axis=1), z.shape[1] - 1)
        margin = np.min(np.abs(c - coverage), axis=1)
        conf = p.max(axis=1)
    out = np.where(conf < min_confidence, fallback, cls[pick].astype(np.int64))
    return out, margin
