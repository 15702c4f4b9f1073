"""Multi-index launch: one persistent, CUDA-graph-captured scan over many flat
indexes (tq_multi_* in include/vectorcache_b200.h; no counterpart in the
reference).

    multi = MultiIndex([idx_a, idx_b, idx_c])
    multi.plan(nq=[1, 300, 4096], k=[10, 64, 10], autotune=True)
    multi.set_queries(0, qa); multi.set_queries(1, qb); multi.set_queries(2, qc)
    multi.launch(); multi.synchronize()
    scores, ids = multi.results(1)
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _check, _ptr, _stream_ptr, load_library

_SZ = C.c_size_t
_P = C.c_void_p


def _declare_multi(lib):
    if getattr(lib, "_multi_declared", False):
        return lib
    sig = {
        "tq_multi_create": (C.c_int, [_P, _SZ, C.POINTER(_P)]),
        "tq_multi_destroy": (C.c_int, [_P]),
        "tq_multi_plan": (C.c_int, [_P, _P, _P, C.c_int]),
        "tq_multi_buffers": (C.c_int, [_P, _SZ, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P), C.POINTER(_SZ)]),
        "tq_multi_launch": (C.c_int, [_P, _P]),
        "tq_multi_run_uncaptured": (C.c_int, [_P, _P]),
        "tq_multi_synchronize": (C.c_int, [_P]),
        "tq_multi_config": (C.c_int, [_P, C.POINTER(C.c_longlong), C.POINTER(C.c_int), C.POINTER(_SZ),
                                      C.POINTER(_SZ), _P, C.POINTER(_SZ)]),
        "tq_multi_direct": (C.c_int, [_P, C.POINTER(_SZ), _P]),
        "tq_copy_to_device": (C.c_int, [_P, _P, _SZ]),
        "tq_copy_to_host": (C.c_int, [_P, _P, _SZ]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    lib._multi_declared = True
    return lib


class MultiIndex:
    def __init__(self, indexes):
        self._lib = _declare_multi(load_library())
        self.indexes = list(indexes)
        arr = (_P * len(self.indexes))(*[x._h.value if hasattr(x._h, "value") else x._h for x in self.indexes])
        h = _P()
        _check(self._lib.tq_multi_create(arr, len(self.indexes), C.byref(h)))
        self._h = h
        self.nq = self.k = None

    def close(self):
        if getattr(self, "_h", None):
            self._lib.tq_multi_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def plan(self, nq, k, autotune: bool = True) -> None:
        self.nq = np.ascontiguousarray(nq, np.uint64)
        self.k = np.ascontiguousarray(k, np.uint64)
        _check(self._lib.tq_multi_plan(self._h, _ptr(self.nq), _ptr(self.k), int(bool(autotune))))

    def buffers(self, i: int):
        q, s, ids = _P(), _P(), _P()
        ke = _SZ()
        _check(self._lib.tq_multi_buffers(self._h, i, C.byref(q), C.byref(s), C.byref(ids), C.byref(ke)))
        return q.value, s.value, ids.value, ke.value

    def set_queries(self, i: int, queries) -> None:
        """Copy host rows (nq[i] x dim) into index i's query buffer."""
        q = np.ascontiguousarray(queries, np.float32)
        ptr, _, _, _ = self.buffers(i)
        _check(self._lib.tq_copy_to_device(_P(ptr), _ptr(q), q.nbytes))

    def results(self, i: int):
        _, sp, ip, ke = self.buffers(i)
        n = int(self.nq[i])
        s = np.empty((n, ke), np.float32)
        ids = np.empty((n, ke), np.uint64)
        if n and ke:
            _check(self._lib.tq_copy_to_host(_ptr(s), _P(sp), s.nbytes))
            _check(self._lib.tq_copy_to_host(_ptr(ids), _P(ip), ids.nbytes))
        return s, ids

    def launch(self, stream=None) -> None:
        _check(self._lib.tq_multi_launch(self._h, _stream_ptr(stream)))

    def run_uncaptured(self, stream=None) -> None:
        _check(self._lib.tq_multi_run_uncaptured(self._h, _stream_ptr(stream)))

    def synchronize(self) -> None:
        _check(self._lib.tq_multi_synchronize(self._h))

    def config(self) -> dict:
        rv, ctas = C.c_longlong(), C.c_int()
        ni, sm = _SZ(), _SZ()
        tuned = np.zeros(64, np.float64)
        nt = _SZ(64)
        _check(self._lib.tq_multi_config(self._h, C.byref(rv), C.byref(ctas), C.byref(ni), C.byref(sm),
                                          _ptr(tuned), C.byref(nt)))
        nd = _SZ()
        flags = np.zeros(len(self.indexes), np.uint8)
        _check(self._lib.tq_multi_direct(self._h, C.byref(nd), _ptr(flags)))
        return {"range_vectors": rv.value, "ctas": ctas.value, "items": ni.value, "smem_bytes": sm.value,
                "tuned_ms": tuned[: nt.value].tolist(), "direct_indexes": int(nd.value),
                "direct_flags": flags.tolist()}

