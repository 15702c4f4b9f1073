"""Learned n_probe predictor for the bucketed index (no counterpart in the
reference).

A query's top-256 routing scores and their gaps go through a small MLP
(2 hidden layers of 128, BF16 weights, FP32 accumulation) trained and run on
the GPU by libvectorcache_b200.so (tq_probe_mlp_* in include/vectorcache_b200.h).
The classes are candidate n_probe values. Two training objectives:

* "classes": softmax cross-entropy on one label per query; a query is
  searched with the smallest n_probe whose predicted cumulative probability
  reaches `coverage`, or with the fixed fallback n_probe when the model's
  confidence is low.
* "recall": one sigmoid per class fitted to the query's measured recall at
  that class; a query is searched with the class maximizing
  predicted recall - coverage * n_probe / largest class, so `coverage` is a
  trade-off (recall given up to save the largest class's probe budget) and
  one value for all queries spends probes where the predicted gain per probe
  is largest.

Labels and recall targets come from the plain index itself (`probe_labels`):
for every training query its recall against the exact brute-force top-k at
each candidate n_probe, and the smallest candidate n_probe whose (optionally
re-ranked) top-k reaches the recall the index gets at the reference n_probe.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _check, _dev, _ptr, _stream_ptr, load_library

_SZ = C.c_size_t
_P = C.c_void_p

DEFAULT_CLASSES = (1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256)
N_INPUTS = 512
ROUTE_P = 256
OBJECTIVES = {"classes": 0, "recall": 1}  # TQ_PROBE_OBJECTIVE_CLASSES / _RECALL


def _declare_probe(lib):
    if getattr(lib, "_probe_declared", False):
        return lib
    sig = {
        "tq_probe_mlp_create": (C.c_int, [_SZ, _SZ, _P, _SZ, C.c_uint64, C.c_int, C.POINTER(_P)]),
        "tq_probe_mlp_destroy": (C.c_int, [_P]),
        "tq_probe_mlp_info": (C.c_int, [_P, C.POINTER(_SZ), C.POINTER(_SZ), C.POINTER(_SZ)]),
        "tq_probe_mlp_features": (C.c_int, [_P, _P, _SZ, _SZ, _P]),
        "tq_probe_mlp_set_normalization": (C.c_int, [_P, _P, _P]),
        "tq_probe_mlp_get_params": (C.c_int, [_P, _P]),
        "tq_probe_mlp_set_params": (C.c_int, [_P, _P]),
        "tq_probe_mlp_forward": (C.c_int, [_P, _P, _SZ, _SZ, _P]),
        "tq_probe_mlp_gradients": (C.c_int, [_P, _P, _P, _SZ, _SZ, C.POINTER(C.c_float), _P]),
        "tq_probe_mlp_train_step_device": (C.c_int, [_P, _P, _P, _SZ, _SZ, C.c_float, C.POINTER(C.c_float), _P]),
        "tq_probe_mlp_set_objective": (C.c_int, [_P, C.c_int]),
        "tq_probe_mlp_recall_gradients": (C.c_int, [_P, _P, _P, _SZ, _SZ, C.POINTER(C.c_float), _P]),
        "tq_probe_mlp_train_step_recall_device": (C.c_int, [_P, _P, _P, _SZ, _SZ, C.c_float,
                                                            C.POINTER(C.c_float), _P]),
        "tq_probe_mlp_predict_device": (C.c_int, [_P, _P, _SZ, _SZ, C.c_float, C.c_float, C.c_uint32, _P, _P, _P]),
        "tq_probe_mlp_synchronize": (C.c_int, [_P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    lib._probe_declared = True
    return lib


class ProbeMLP:
    """The MLP itself: parameters live on the device (fp32 master + bf16 copy)."""

    def __init__(self, classes=DEFAULT_CLASSES, hidden: int = 128, layers: int = 2, seed: int = 1, device: int = 0,
                 objective: str = "classes"):
        if objective not in OBJECTIVES:
            raise ValueError(f"objective must be one of {sorted(OBJECTIVES)}")
        self._lib = _declare_probe(load_library())
        self.classes = np.ascontiguousarray(classes, np.uint32)
        self.hidden, self.layers, self.device = int(hidden), int(layers), int(device)
        self.objective = objective
        h = _P()
        _check(self._lib.tq_probe_mlp_create(hidden, layers, _ptr(self.classes), len(self.classes), seed, device,
                                             C.byref(h)))
        self._h = h
        _check(self._lib.tq_probe_mlp_set_objective(h, OBJECTIVES[objective]))
        ni, npar, nc = _SZ(), _SZ(), _SZ()
        _check(self._lib.tq_probe_mlp_info(h, C.byref(ni), C.byref(npar), C.byref(nc)))
        self.n_inputs, self.n_params, self.n_classes = ni.value, npar.value, nc.value
        self.mean = np.zeros(N_INPUTS, np.float32)
        self.std = np.ones(N_INPUTS, np.float32)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.tq_probe_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # layer shapes in parameter order: (fan_in, fan_out) of each linear layer
    def shapes(self):
        dims = [N_INPUTS] + [self.hidden] * self.layers + [self.n_classes]
        return list(zip(dims[:-1], dims[1:]))

    def features(self, top_scores) -> np.ndarray:
        t = np.ascontiguousarray(top_scores, np.float32)
        out = np.empty((t.shape[0], N_INPUTS), np.float32)
        _check(self._lib.tq_probe_mlp_features(self._h, _ptr(t), t.shape[0], t.shape[1], _ptr(out)))
        return out

    def set_normalization(self, mean, std) -> None:
        self.mean = np.ascontiguousarray(mean, np.float32)
        self.std = np.ascontiguousarray(std, np.float32)
        _check(self._lib.tq_probe_mlp_set_normalization(self._h, _ptr(self.mean), _ptr(self.std)))

    def params(self) -> np.ndarray:
        out = np.empty(self.n_params, np.float32)
        _check(self._lib.tq_probe_mlp_get_params(self._h, _ptr(out)))
        return out

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.n_params
        _check(self._lib.tq_probe_mlp_set_params(self._h, _ptr(p)))

    def forward(self, top_scores) -> np.ndarray:
        t = np.ascontiguousarray(top_scores, np.float32)
        out = np.empty((t.shape[0], self.n_classes), np.float32)
        _check(self._lib.tq_probe_mlp_forward(self._h, _ptr(t), t.shape[0], t.shape[1], _ptr(out)))
        return out

    def gradients(self, top_scores, targets) -> tuple[float, np.ndarray]:
        """Mean loss and gradients for a host batch: targets are label
        classes (classes objective) or an m x n_classes recall matrix (recall
        objective)."""
        t = np.ascontiguousarray(top_scores, np.float32)
        g = np.empty(self.n_params, np.float32)
        loss = C.c_float()
        if self.objective == "recall":
            r = np.ascontiguousarray(targets, np.float32)
            if r.shape != (t.shape[0], self.n_classes):
                raise ValueError("recall targets must be m x n_classes")
            _check(self._lib.tq_probe_mlp_recall_gradients(self._h, _ptr(t), _ptr(r), t.shape[0], t.shape[1],
                                                           C.byref(loss), _ptr(g)))
        else:
            lab = np.ascontiguousarray(targets, np.uint32)
            _check(self._lib.tq_probe_mlp_gradients(self._h, _ptr(t), _ptr(lab), t.shape[0], t.shape[1],
                                                    C.byref(loss), _ptr(g)))
        return loss.value, g

    def train_step_device(self, d_top, d_targets, m: int, p: int, lr: float, stream=None) -> float:
        """One Adam step on device rows: d_targets are int32 labels (classes
        objective) or an m x n_classes float32 recall matrix (recall objective)."""
        loss = C.c_float()
        fn = (self._lib.tq_probe_mlp_train_step_recall_device if self.objective == "recall"
              else self._lib.tq_probe_mlp_train_step_device)
        _check(fn(self._h, _dev(d_top)[0], _dev(d_targets)[0], m, p, lr, C.byref(loss), _stream_ptr(stream)))
        return loss.value

    def predict_device(self, d_top, m: int, p: int, d_out, coverage: float = 0.9, min_confidence: float = 0.0,
                       fallback: int = 64, d_confidence=None, stream=None) -> None:
        """Per-query n_probe into d_out (m int32). `coverage` is the cumulative
        probability (classes objective) or the recall trade-off (recall
        objective)."""
        conf = None if d_confidence is None else _dev(d_confidence)[0]
        _check(self._lib.tq_probe_mlp_predict_device(self._h, _dev(d_top)[0], m, p, coverage, min_confidence,
                                                     fallback, _dev(d_out)[0], conf, _stream_ptr(stream)))

    def synchronize(self) -> None:
        _check(self._lib.tq_probe_mlp_synchronize(self._h))


def recall_rows(ids: np.ndarray, exact: np.ndarray, t: int) -> np.ndarray:
    """Per-query |top-t(ids) & top-t(exact)| / t."""
    a = ids[:, :t].astype(np.int64)
    e = exact[:, :t].astype(np.int64)
    hits = (a[:, :, None] == e[:, None, :]).any(axis=2).sum(axis=1)
    return hits / float(t)


def probe_labels(search_fn, queries, exact_ids, classes=DEFAULT_CLASSES, k: int = 10,
                 reference_probe: int | None = None):
    """Labels from the plain index: search_fn(queries, n_probe) -> ids (nq x >= k).

    A query's goal is the recall@k (against the exact top-k) the plain index
    reaches for it at `reference_probe` (default: the largest class); its
    label is the index of the smallest class n_probe that reaches that goal.
    Returns (labels, recall matrix nq x n_classes)."""
    classes = list(classes)
    ref = classes[-1] if reference_probe is None else reference_probe
    if ref not in classes:
        raise ValueError("reference_probe must be one of the classes")
    rec = np.stack([recall_rows(search_fn(queries, p), exact_ids, k) for p in classes], axis=1)
    goal = rec[:, classes.index(ref)] - 1e-9
    ok = rec >= goal[:, None]
    return ok.argmax(axis=1).astype(np.uint32), rec
