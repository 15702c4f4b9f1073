"""Bucketed (IVF) TurboQuant index: Python mirror of the reference README's

    vectorcache::BucketParams p;            // n_probe, max_bucket_size, energy_soft, expected_n, ...
    vectorcache::BucketedTurboQuantIndex bindex(dim, bits, p);
    bindex.calibrate(sample); bindex.add(database); bindex.prepare();
    auto bres = bindex.search(queries, k);

(README.md:56, :91-98, :113-120). All work runs in libvectorcache_b200.so
(tq_bucketed_* in include/vectorcache_b200.h); this module marshals arguments.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import (InvalidArgument, SearchResults, TurboQuantIndex, TQ_ERR_INVALID_ARGUMENT, _check, _dev, _ptr,
               _stream_ptr, load_library)

_SZ = C.c_size_t
_P = C.c_void_p


class _Params(C.Structure):
    _fields_ = [("n_probe", C.c_uint32), ("max_bucket_size", C.c_uint32), ("energy_soft", C.c_uint32),
                ("kmeans_iters", C.c_uint32), ("rerank_k", C.c_uint32), ("reserved", C.c_uint32),
                ("expected_n", C.c_uint64), ("seed", C.c_uint64)]


@dataclass
class BucketParams:
    """BucketParams of the reference README (README.md:113-120), plus
    rerank_k: when larger than k, the scan keeps rerank_k candidates that are
    re-scored with the exact float inner product before the top k is taken."""

    n_probe: int = 64
    max_bucket_size: int = 800
    energy_soft: int = 400
    expected_n: int = 0
    kmeans_iters: int = 4
    seed: int = 0x5EED5EED
    rerank_k: int = 0

    def _c(self) -> _Params:
        return _Params(self.n_probe, self.max_bucket_size, self.energy_soft, self.kmeans_iters, self.rerank_k, 0,
                       self.expected_n, self.seed)


def _declare_bucketed(lib):
    if getattr(lib, "_bucketed_declared", False):
        return lib
    u32p = C.POINTER(C.c_uint32)
    sig = {
        "tq_bucket_params_init": (None, [C.POINTER(_Params)]),
        "tq_bucketed_create": (C.c_int, [_SZ, _SZ, C.POINTER(_Params), C.c_int, C.POINTER(_P)]),
        "tq_bucketed_destroy": (C.c_int, [_P]),
        "tq_bucketed_calibrate": (C.c_int, [_P, _P, _SZ]),
        "tq_bucketed_add": (C.c_int, [_P, _P, _SZ]),
        "tq_bucketed_add_device": (C.c_int, [_P, _P, _SZ, _P]),
        "tq_bucketed_prepare": (C.c_int, [_P]),
        "tq_bucketed_search": (C.c_int, [_P, _P, _SZ, _SZ, _SZ, _P, _P, _P, C.POINTER(_SZ)]),
        "tq_bucketed_search_device": (C.c_int, [_P, _P, _SZ, _SZ, _SZ, _P, _P, _P, C.POINTER(_SZ), _P]),
        "tq_bucketed_route_device": (C.c_int, [_P, _P, _SZ, _SZ, _P, _P, _P]),
        "tq_bucketed_info": (C.c_int, [_P] + [C.POINTER(_SZ)] * 6 + [C.POINTER(C.c_int)]),
        "tq_bucketed_search_trace": (C.c_int, [_P, _P, _SZ, _SZ, _SZ, _P, _P, _P, C.POINTER(_SZ), _P, _P, _P]),
        "tq_bucketed_route": (C.c_int, [_P, _P, _SZ, _P, _P]),
        "tq_bucketed_export_layout": (C.c_int, [_P, _P, _P, _P, _P]),
        "tq_bucketed_export_centroids": (C.c_int, [_P, _P, _P]),
        "tq_bucketed_export_rows": (C.c_int, [_P, _P]),
        "tq_bucketed_engine": (C.c_int, [_P, C.POINTER(_P)]),
    }
    del u32p
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    lib._bucketed_declared = True
    return lib


class BucketedTurboQuantIndex:
    """Bucketed (IVF) TurboQuant index on one CUDA device (cosine: rows and
    queries are L2-normalized). Any dim in [1, 2048]; rows are zero-padded to a
    multiple of 8 coordinates internally."""

    def __init__(self, dim: int, bits: int, params: BucketParams | None = None, device: int = 0):
        self._lib = _declare_bucketed(load_library())
        self.params = params or BucketParams()
        h = _P()
        cp = self.params._c()
        _check(self._lib.tq_bucketed_create(dim, bits, C.byref(cp), device, C.byref(h)))
        self._h = h
        self.dim = int(dim)
        self.bits = int(bits)
        self.device = int(device)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.tq_bucketed_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _rows(self, x) -> np.ndarray:
        a = np.ascontiguousarray(x, dtype=np.float32)
        if a.ndim != 2 or a.shape[1] != self.dim:
            raise InvalidArgument(TQ_ERR_INVALID_ARGUMENT, f"expected [n, {self.dim}] float32 rows")
        return a

    # -- lifecycle ----------------------------------------------------------
    def calibrate(self, sample) -> None:
        a = self._rows(sample)
        _check(self._lib.tq_bucketed_calibrate(self._h, _ptr(a), a.shape[0]))

    def add(self, vectors) -> None:
        a = self._rows(vectors)
        _check(self._lib.tq_bucketed_add(self._h, _ptr(a), a.shape[0]))

    def add_device(self, d_vectors, n: int | None = None, stream=None) -> None:
        ptr, n = _dev(d_vectors, n)
        _check(self._lib.tq_bucketed_add_device(self._h, ptr, n, _stream_ptr(stream)))

    def prepare(self) -> None:
        _check(self._lib.tq_bucketed_prepare(self._h))

    def search(self, queries, k: int, n_probe: int = 0, n_probe_per_query=None) -> SearchResults:
        q = self._rows(queries)
        nq = q.shape[0]
        npq = None
        if n_probe_per_query is not None:
            npq = np.ascontiguousarray(n_probe_per_query, np.uint32)
        ke = _SZ(0)
        scores = np.empty(max(nq * k, 1), np.float32)
        ids = np.empty(max(nq * k, 1), np.uint64)
        _check(self._lib.tq_bucketed_search(self._h, _ptr(q), nq, k, n_probe, _ptr(npq), _ptr(scores), _ptr(ids),
                                            C.byref(ke)))
        kk = ke.value
        return SearchResults(scores[: nq * kk].reshape(nq, kk).copy(), ids[: nq * kk].reshape(nq, kk).copy())

    def search_device(self, d_queries, k: int, d_scores, d_ids, n_probe: int = 0, d_n_probe=None,
                      nq: int | None = None, stream=None) -> int:
        qp, nq = _dev(d_queries, nq)
        npp = None if d_n_probe is None else _dev(d_n_probe)[0]
        ke = _SZ(0)
        _check(self._lib.tq_bucketed_search_device(self._h, qp, nq, k, n_probe, npp, _dev(d_scores)[0],
                                                   _dev(d_ids)[0], C.byref(ke), _stream_ptr(stream)))
        return ke.value

    def route_device(self, d_queries, p: int, d_top_scores, d_top_ids, nq: int | None = None, stream=None) -> None:
        qp, nq = _dev(d_queries, nq)
        _check(self._lib.tq_bucketed_route_device(self._h, qp, nq, p, _dev(d_top_scores)[0], _dev(d_top_ids)[0],
                                                  _stream_ptr(stream)))

    # -- introspection ------------------------------------------------------
    def info(self) -> dict:
        v = [_SZ() for _ in range(6)]
        p = C.c_int()
        _check(self._lib.tq_bucketed_info(self._h, *[C.byref(x) for x in v], C.byref(p)))
        keys = ["dim", "dim_padded", "bits", "size", "n_buckets", "n_slots"]
        out = {k: x.value for k, x in zip(keys, v)}
        out["prepared"] = bool(p.value)
        return out

    def search_trace(self, queries, k: int, n_probe: int = 0, n_probe_per_query=None) -> dict:
        q = self._rows(queries)
        nq = q.shape[0]
        inf = self.info()
        npb = min(n_probe or self.params.n_probe, inf["n_buckets"])
        npq = None if n_probe_per_query is None else np.ascontiguousarray(n_probe_per_query, np.uint32)
        ke = _SZ(0)
        scores = np.empty(max(nq * k, 1), np.float32)
        ids = np.empty(max(nq * k, 1), np.uint64)
        probes = np.empty((nq, npb), np.uint32)
        offsets = np.empty((nq, npb), np.float32)
        q_hat = np.empty((nq, inf["dim_padded"]), np.float32)
        _check(self._lib.tq_bucketed_search_trace(self._h, _ptr(q), nq, k, n_probe, _ptr(npq), _ptr(scores),
                                                  _ptr(ids), C.byref(ke), _ptr(probes), _ptr(offsets),
                                                  _ptr(q_hat)))
        kk = ke.value
        return {"scores": scores[: nq * kk].reshape(nq, kk).copy(), "ids": ids[: nq * kk].reshape(nq, kk).copy(),
                "probes": probes, "offsets": offsets, "q_hat": q_hat}

    def route(self, queries) -> tuple[np.ndarray, np.ndarray]:
        q = self._rows(queries)
        inf = self.info()
        q_hat = np.empty((q.shape[0], inf["dim_padded"]), np.float32)
        scores = np.empty((q.shape[0], inf["n_buckets"]), np.float32)
        _check(self._lib.tq_bucketed_route(self._h, _ptr(q), q.shape[0], _ptr(q_hat), _ptr(scores)))
        return q_hat, scores

    def layout(self) -> dict:
        inf = self.info()
        nb, ns = inf["n_buckets"], inf["n_slots"]
        slot_start = np.empty(nb + 1, np.uint64)
        size = np.empty(nb, np.uint32)
        slot_ids = np.empty(ns, np.uint32)
        labels = np.empty(inf["size"], np.uint32)
        _check(self._lib.tq_bucketed_export_layout(self._h, _ptr(slot_start), _ptr(size), _ptr(slot_ids),
                                                   _ptr(labels)))
        return {"slot_start": slot_start, "bucket_size": size, "slot_ids": slot_ids, "labels": labels}

    def centroids(self) -> tuple[np.ndarray, np.ndarray]:
        inf = self.info()
        route = np.empty((inf["n_buckets"], inf["dim_padded"]), np.float32)
        enc = np.empty_like(route)
        _check(self._lib.tq_bucketed_export_centroids(self._h, _ptr(route), _ptr(enc)))
        return route, enc

    def rows(self) -> np.ndarray:
        inf = self.info()
        out = np.empty((inf["size"], inf["dim_padded"]), np.float32)
        _check(self._lib.tq_bucketed_export_rows(self._h, _ptr(out)))
        return out

    def engine(self) -> TurboQuantIndex:
        """The flat index over the residual slots (borrowed: do not close it)."""
        h = _P()
        _check(self._lib.tq_bucketed_engine(self._h, C.byref(h)))
        inf = self.info()
        eng = TurboQuantIndex.__new__(TurboQuantIndex)
        eng._h = h
        eng._lib = self._lib
        eng.dim = inf["dim_padded"]
        eng.bits = self.bits
        eng.device = self.device
        eng.n_byte_groups = eng.dim // (8 // self.bits)
        eng.close = lambda: None  # owned by the bucketed index
        return eng


def _declare_learned(lib):
    if getattr(lib, "_learned_declared", False):
        return lib
    fn = lib.tq_bucketed_search_learned_device
    fn.restype = C.c_int
    fn.argtypes = [_P, _P, _SZ, _SZ, _P, C.c_float, C.c_float, _SZ, _P, _P, C.POINTER(_SZ), _P]
    lib._learned_declared = True
    return lib


def search_learned_device(index: "BucketedTurboQuantIndex", d_queries, k: int, mlp, d_scores, d_ids,
                          coverage: float = 0.9, min_confidence: float = 0.0, fallback_n_probe: int = 0,
                          nq: int | None = None, stream=None) -> int:
    """One routing pass, the learned n_probe per query, then the bucket scan
    (tq_bucketed_search_learned_device)."""
    lib = _declare_learned(index._lib)
    qp, nq = _dev(d_queries, nq)
    ke = _SZ(0)
    _check(lib.tq_bucketed_search_learned_device(index._h, qp, nq, k, mlp._h, coverage, min_confidence,
                                                 fallback_n_probe, _dev(d_scores)[0], _dev(d_ids)[0], C.byref(ke),
                                                 _stream_ptr(stream)))
    return ke.value


BucketedTurboQuantIndex.search_learned_device = search_learned_device


def select_top_device(d_scores, p: int, d_top_scores, d_top_ids, ncols: int | None = None, device: int = 0,
                      stream=None) -> None:
    """Per row of a device score matrix (torch CUDA tensor, rows x ld floats),
    the top p columns, score descending, equal scores by lower column; -inf and
    NaN are never selected (tq_select_top_device, the routing's selection).
    d_top_scores (float32) and d_top_ids (int32 / uint32) are rows x p."""
    lib = load_library()
    fn = lib.tq_select_top_device
    fn.restype = C.c_int
    fn.argtypes = [_P, _SZ, _SZ, _SZ, _SZ, _P, _P, C.c_int, _P]
    rows, ld = int(d_scores.shape[0]), int(d_scores.stride(0))
    _check(fn(_dev(d_scores)[0], rows, ld, int(ncols if ncols is not None else d_scores.shape[1]), p,
              _dev(d_top_scores)[0], _dev(d_top_ids)[0], device, _stream_ptr(stream)))
