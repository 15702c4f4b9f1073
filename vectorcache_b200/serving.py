"""Serving loop: continuous batching over resident indexes (tq_server_* in
include/vectorcache_b200.h; no counterpart in the reference).

    srv = Server(device=0, hbm_budget_bytes=120 << 30, max_slots=4, max_batch=1024)
    flat_id = srv.add_flat(flat_index, max_k=64)
    bkt_id = srv.add_bucketed(bucketed_index, max_k=64, max_probe=512, mlp=probe_mlp)
    srv.start()
    req = srv.submit(flat_id, queries, k=10)
    scores, ids, latency_us = req.wait()
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _check, _ptr, load_library

_SZ = C.c_size_t
_P = C.c_void_p


class _ReplayItem(C.Structure):
    _fields_ = [("arrival_us", C.c_double), ("target", C.c_int), ("queries", _P), ("nq", _SZ), ("k", _SZ),
                ("n_probe", _SZ), ("scores", _P), ("ids", _P)]


def _declare_server(lib):
    if getattr(lib, "_server_declared", False):
        return lib
    sig = {
        "tq_server_create": (C.c_int, [C.c_int, _SZ, _SZ, _SZ, C.POINTER(_P)]),
        "tq_server_destroy": (C.c_int, [_P]),
        "tq_server_add_flat": (C.c_int, [_P, _P, _SZ, C.POINTER(C.c_int)]),
        "tq_server_add_bucketed": (C.c_int, [_P, _P, _SZ, _SZ, _P, C.c_float, C.c_float, C.POINTER(C.c_int)]),
        "tq_server_start": (C.c_int, [_P]),
        "tq_server_info": (C.c_int, [_P, C.POINTER(_SZ), C.POINTER(_SZ), C.POINTER(_SZ)]),
        "tq_server_submit": (C.c_int, [_P, C.c_int, _P, _SZ, _SZ, _SZ, _P, _P, C.POINTER(C.c_uint64)]),
        "tq_server_wait": (C.c_int, [_P, C.c_uint64, C.POINTER(_SZ), C.POINTER(C.c_double)]),
        "tq_server_stats": (C.c_int, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                      C.POINTER(_SZ)]),
        "tq_server_replay": (C.c_int, [_P, C.POINTER(_ReplayItem), _SZ, _P, C.POINTER(C.c_double)]),
        "tq_server_memory": (C.c_int, [_P, C.POINTER(_SZ), C.POINTER(_SZ), C.POINTER(_SZ), C.POINTER(C.c_uint64)]),
        "tq_server_batch_bytes": (C.c_int, [_P, C.c_int, _SZ, _SZ, _SZ, C.POINTER(_SZ)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    lib._server_declared = True
    return lib


class Request:
    """A submitted request; its host buffers stay alive until wait()."""

    def __init__(self, server, rid, queries, scores, ids):
        self._srv, self.id = server, rid
        self._keep = (queries, scores, ids)

    def wait(self):
        ke, lat = _SZ(), C.c_double()
        _check(self._srv._lib.tq_server_wait(self._srv._h, self.id, C.byref(ke), C.byref(lat)))
        _, s, i = self._keep
        nq = s.shape[0]
        kk = ke.value
        return s.ravel()[: nq * kk].reshape(nq, kk).copy(), i.ravel()[: nq * kk].reshape(nq, kk).copy(), lat.value


class Server:
    def __init__(self, device: int = 0, hbm_budget_bytes: int = 120 << 30, max_slots: int = 4,
                 max_batch: int = 1024):
        self._lib = _declare_server(load_library())
        h = _P()
        _check(self._lib.tq_server_create(device, hbm_budget_bytes, max_slots, max_batch, C.byref(h)))
        self._h = h
        self.max_batch = max_batch
        self._dims = []
        self._max_k = []

    def close(self):
        if getattr(self, "_h", None):
            self._lib.tq_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_flat(self, index, max_k: int = 64) -> int:
        t = C.c_int()
        _check(self._lib.tq_server_add_flat(self._h, index._h, max_k, C.byref(t)))
        self._dims.append(index.dim)
        self._max_k.append(max_k)
        return t.value

    def add_bucketed(self, index, max_k: int = 64, max_probe: int = 64, mlp=None, coverage: float = 0.9,
                     min_confidence: float = 0.0) -> int:
        t = C.c_int()
        _check(self._lib.tq_server_add_bucketed(self._h, index._h, max_k, max_probe, mlp._h if mlp else None,
                                                coverage, min_confidence, C.byref(t)))
        self._dims.append(index.dim)
        self._max_k.append(max_k)
        return t.value

    def start(self) -> None:
        _check(self._lib.tq_server_start(self._h))

    def info(self) -> dict:
        ns, sb, rb = _SZ(), _SZ(), _SZ()
        _check(self._lib.tq_server_info(self._h, C.byref(ns), C.byref(sb), C.byref(rb)))
        return {"slots": ns.value, "slot_bytes": sb.value, "resident_bytes": rb.value}

    def memory(self) -> dict:
        """Scratch arena: size, peak use, largest batch scratch, batches that waited for memory."""
        a, p, m = _SZ(), _SZ(), _SZ()
        w = C.c_uint64()
        _check(self._lib.tq_server_memory(self._h, C.byref(a), C.byref(p), C.byref(m), C.byref(w)))
        return {"arena_bytes": a.value, "arena_peak": p.value, "max_batch_bytes": m.value, "memory_waits": w.value}

    def batch_bytes(self, target: int, nq: int, k: int, n_probe: int = 0) -> int:
        """Arena bytes the scratch of one batch of nq queries takes."""
        b = _SZ()
        _check(self._lib.tq_server_batch_bytes(self._h, target, nq, k, n_probe, C.byref(b)))
        return b.value

    def stats(self) -> dict:
        b, q, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        p = _SZ()
        _check(self._lib.tq_server_stats(self._h, C.byref(b), C.byref(q), C.byref(c), C.byref(p)))
        return {"batches": b.value, "queries": q.value, "completed": c.value, "peak_inflight": p.value}

    def submit(self, target: int, queries, k: int, n_probe: int = 0) -> Request:
        q = np.ascontiguousarray(queries, np.float32)
        nq = q.shape[0]
        s = np.empty((nq, k), np.float32)
        i = np.empty((nq, k), np.uint64)
        rid = C.c_uint64()
        _check(self._lib.tq_server_submit(self._h, target, _ptr(q), nq, k, n_probe, _ptr(s), _ptr(i), C.byref(rid)))
        return Request(self, rid.value, q, s, i)

    def replay(self, trace):
        """trace: list of (arrival_us, target, queries [nq, dim] float32, k, n_probe).
        Returns (latencies_us, wall_s, results list of (scores, ids) with k columns)."""
        items = (_ReplayItem * len(trace))()
        keep = []
        for n, (t_us, target, q, k, n_probe) in enumerate(trace):
            q = np.ascontiguousarray(q, np.float32)
            s = np.zeros((q.shape[0], k), np.float32)
            i = np.zeros((q.shape[0], k), np.uint64)
            keep.append((q, s, i))
            items[n] = _ReplayItem(float(t_us), int(target), q.ctypes.data, q.shape[0], k, n_probe, s.ctypes.data,
                                   i.ctypes.data)
        lat = np.zeros(len(trace), np.float64)
        wall = C.c_double()
        _check(self._lib.tq_server_replay(self._h, items, len(trace), _ptr(lat), C.byref(wall)))
        return lat, wall.value, [(s, i) for _, s, i in keep]
