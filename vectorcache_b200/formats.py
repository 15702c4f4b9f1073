"""File formats of the flat index path, through the C ABI (tq_formats.cpp):

* float32 .npy matrices (the reference's NpyReader / write_npy_f32_matrix,
  include/vectorcache/datasets/npy.hpp:33-66);
* VCEX exact-top-k files (tools/query-bench.cpp:180-340), the reference's
  cache of brute-force ground truth.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import _check, _ptr, load_library

_SZ = C.c_size_t


def npy_shape(path) -> tuple[int, int]:
    r, c = _SZ(), _SZ()
    _check(load_library().tq_npy_f32_info(str(path).encode(), C.byref(r), C.byref(c)))
    return r.value, c.value


def read_npy_f32(path, row0: int = 0, nrows: int | None = None) -> np.ndarray:
    rows, cols = npy_shape(path)
    n = rows - row0 if nrows is None else nrows
    out = np.empty((n, cols), np.float32)
    _check(load_library().tq_npy_f32_read(str(path).encode(), row0, n, _ptr(out)))
    return out


def write_npy_f32(path, matrix) -> None:
    m = np.ascontiguousarray(matrix, np.float32)
    if m.ndim != 2:
        raise ValueError("matrix must be 2-D")
    _check(load_library().tq_npy_f32_write(str(path).encode(), m.shape[0], m.shape[1], _ptr(m)))


def write_vcex(path, ids, index_n: int, seed: int, source_label: str = "", split: str = "",
               query_split: str = "") -> None:
    a = np.ascontiguousarray(ids, np.uint64)
    if a.ndim != 2:
        raise ValueError("ids must be [n_queries, k]")
    _check(load_library().tq_vcex_write(str(path).encode(), _ptr(a), a.shape[0], a.shape[1], index_n, seed,
                                        source_label.encode(), split.encode(), query_split.encode()))


def read_vcex(path) -> tuple[dict, np.ndarray]:
    lib = load_library()
    nq, k = _SZ(), _SZ()
    index_n, seed = C.c_uint64(), C.c_uint64()
    p = str(Path(path)).encode()
    _check(lib.tq_vcex_read_header(p, C.byref(nq), C.byref(k), C.byref(index_n), C.byref(seed)))
    ids = np.empty((nq.value, k.value), np.uint64)
    _check(lib.tq_vcex_read_ids(p, _ptr(ids)))
    return {"n_queries": nq.value, "k": k.value, "index_n": index_n.value, "seed": seed.value}, ids
