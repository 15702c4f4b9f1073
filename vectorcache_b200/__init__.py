"""vectorcache_b200 — B200-native (sm_100a) flat TurboQuant index.

Python mirror of the reference's flat-index API (nishadtardalkar/vectorcache,
README.md:100-121 and gpu::FlatIndex in include/vectorcache/gpu/flat_index.hpp):

    index = TurboQuantIndex(dim=1536, bits=4)
    index.calibrate(sample)    # optional TQ+
    index.add(database)        # float32 [n, dim]
    index.prepare()
    res = index.search(queries, k=10)   # res.scores [nq, k_eff], res.ids [nq, k_eff]

All work runs in the CUDA library libvectorcache_b200.so through its C ABI
(include/vectorcache_b200.h); this module only marshals arguments. There is no
CPU fallback: importing works without a GPU, creating an index needs one and
raises if the compiled library is missing.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np

__all__ = [
    "TurboQuantIndex",
    "SearchResults",
    "TurboQuantError",
    "codebook",
    "rotation_tables",
    "scan_plan_shape",
    "load_library",
    "LIB_PATH",
]

LIB_PATH = Path(__file__).resolve().parent / "libvectorcache_b200.so"

TQ_OK = 0
TQ_ERR_INVALID_ARGUMENT = 1
TQ_ERR_STATE = 2
TQ_ERR_CUDA = 3
TQ_ERR_OUT_OF_MEMORY = 4
TQ_ERR_UNSUPPORTED = 5


class TurboQuantError(RuntimeError):
    """Error returned by the C ABI; `code` is the TQ_ERR_* value."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


class InvalidArgument(TurboQuantError, ValueError):
    """Mirrors std::invalid_argument in the reference."""


_lib = None
_SZ = C.c_size_t
_P = C.c_void_p


class Profile(C.Structure):
    """tq_profile: per-kernel device time between two reads."""

    _fields_ = [("prep_ms", C.c_double), ("scan_ms", C.c_double), ("merge_ms", C.c_double),
                ("encode_ms", C.c_double), ("prep_launches", C.c_uint64), ("scan_launches", C.c_uint64),
                ("merge_launches", C.c_uint64), ("encode_launches", C.c_uint64),
                ("scan_stream_bytes", C.c_uint64), ("scan_queries", C.c_uint64)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


def _declare(lib):
    sig = {
        "tq_last_error": (C.c_char_p, []),
        "tq_version": (C.c_char_p, []),
        "tq_codebook": (C.c_int, [_SZ, _SZ, _P, _P]),
        "tq_rotation_tables": (C.c_int, [_SZ, _P, _P]),
        "tq_index_create": (C.c_int, [_SZ, _SZ, C.c_uint32, C.c_int, C.POINTER(_P)]),
        "tq_index_destroy": (C.c_int, [_P]),
        "tq_index_calibrate": (C.c_int, [_P, _P, _SZ]),
        "tq_index_calibrate_device": (C.c_int, [_P, _P, _SZ, _P]),
        "tq_index_add": (C.c_int, [_P, _P, _SZ]),
        "tq_index_add_device": (C.c_int, [_P, _P, _SZ, _P]),
        "tq_index_prepare": (C.c_int, [_P]),
        "tq_index_search": (C.c_int, [_P, _P, _SZ, _SZ, _P, _P, C.POINTER(_SZ)]),
        "tq_index_search_device": (C.c_int, [_P, _P, _SZ, _SZ, _P, _P, C.POINTER(_SZ), _P]),
        "tq_index_synchronize": (C.c_int, [_P]),
        "tq_index_info": (C.c_int, [_P, C.POINTER(_SZ), C.POINTER(_SZ), C.POINTER(_SZ),
                                    C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "tq_index_export_codes_flat": (C.c_int, [_P, _P]),
        "tq_index_export_packed": (C.c_int, [_P, _P]),
        "tq_index_export_alpha": (C.c_int, [_P, _P]),
        "tq_index_export_calibration": (C.c_int, [_P, _P, _P]),
        "tq_index_prepare_queries": (C.c_int, [_P, _P, _SZ, _P, _P, _P, _P, _P]),
        "tq_index_dense_scores": (C.c_int, [_P, _P, _SZ, _P, _P]),
        "tq_index_replay_count": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
        "tq_index_scan_plan": (C.c_int, [_P, _SZ, _SZ, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                         C.POINTER(C.c_uint64), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "tq_scan_plan_shape": (C.c_int, [C.c_uint64, _SZ, _SZ, _SZ, _SZ, C.c_int, C.POINTER(C.c_int),
                                         C.POINTER(C.c_int), C.POINTER(C.c_uint64), C.POINTER(C.c_int),
                                         C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "tq_index_save": (C.c_int, [_P, C.c_char_p]),
        "tq_index_load": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(_P)]),
        "tq_index_add_npy": (C.c_int, [_P, C.c_char_p]),
        "tq_npy_f32_info": (C.c_int, [C.c_char_p, C.POINTER(_SZ), C.POINTER(_SZ)]),
        "tq_npy_f32_read": (C.c_int, [C.c_char_p, _SZ, _SZ, _P]),
        "tq_npy_f32_write": (C.c_int, [C.c_char_p, _SZ, _SZ, _P]),
        "tq_vcex_write": (C.c_int, [C.c_char_p, _P, _SZ, _SZ, C.c_uint64, C.c_uint64, C.c_char_p, C.c_char_p,
                                    C.c_char_p]),
        "tq_vcex_read_header": (C.c_int, [C.c_char_p, C.POINTER(_SZ), C.POINTER(_SZ), C.POINTER(C.c_uint64),
                                          C.POINTER(C.c_uint64)]),
        "tq_vcex_read_ids": (C.c_int, [C.c_char_p, _P]),
        "tq_rescore": (C.c_int, [_P, _SZ, _SZ, _P, _SZ, _SZ, _P, _P, C.c_int]),
        "tq_rescore_device": (C.c_int, [_P, _SZ, _SZ, _P, _SZ, _SZ, _P, _P, _P]),
        "tq_index_get_stream": (C.c_int, [_P, C.POINTER(_P)]),
        "tq_index_set_profiling": (C.c_int, [_P, C.c_int]),
        "tq_index_read_profile": (C.c_int, [_P, C.POINTER(Profile)]),
        "tq_index_profile_entries": (C.c_int, [_P, C.POINTER(_SZ)]),
        "tq_index_profile_entry": (C.c_int, [_P, _SZ, C.c_char_p, _SZ, C.POINTER(C.c_double),
                                             C.POINTER(C.c_uint64)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def load_library(path: Path | str | None = None):
    """Load (once) the compiled CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise TurboQuantError(
            TQ_ERR_UNSUPPORTED,
            f"{p} is missing: build it with `python -m vectorcache_b200.build` (no CPU fallback exists)",
        )
    lib = _declare(C.CDLL(str(p)))
    if path is None:
        _lib = lib
    return lib


def _check(rc: int) -> None:
    if rc != TQ_OK:
        msg = load_library().tq_last_error().decode()
        if rc == TQ_ERR_INVALID_ARGUMENT:
            raise InvalidArgument(rc, msg)
        raise TurboQuantError(rc, msg)


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(_P)


def _rows(x, dim: int) -> np.ndarray:
    a = np.ascontiguousarray(x, dtype=np.float32)
    if a.ndim == 1:
        if a.size % dim != 0:
            raise InvalidArgument(TQ_ERR_INVALID_ARGUMENT, "vectors size must be multiple of dim")
        a = a.reshape(-1, dim)
    if a.ndim != 2 or a.shape[1] != dim:
        raise InvalidArgument(TQ_ERR_INVALID_ARGUMENT, f"expected [n, {dim}] float32 rows")
    return a


def codebook(bits: int, dim: int) -> tuple[np.ndarray, np.ndarray]:
    """(boundaries, centroids) of the Lloyd-Max Beta codebook (codebook.cpp:203)."""
    L = 1 << bits if 2 <= bits <= 4 else 16
    b = np.zeros(max(L - 1, 1), np.float32)
    c = np.zeros(L, np.float32)
    _check(load_library().tq_codebook(bits, dim, _ptr(b), _ptr(c)))
    return b, c


def rotation_tables(dim: int) -> tuple[np.ndarray, np.ndarray]:
    """(signs, perm) of the ChaCha8 rotation (rotation.cpp:139-160)."""
    s = np.zeros(max(dim, 1), np.float32)
    p = np.zeros(max(dim, 1), np.uint32)
    _check(load_library().tq_rotation_tables(dim, _ptr(s), _ptr(p)))
    return s, p


def scan_plan_shape(n: int, nq: int, dim: int, bits: int, k: int, sms: int = 148) -> dict:
    """The scan tiling a search of nq queries with this k would use on an index
    of n vectors (dim, bits) and a device of `sms` SMs, planned on the host (no
    GPU needed): TurboQuantIndex.scan_plan's fields plus the CTAs per SM of a
    batch-split one- or two-query scan (0 when it does not split)."""
    lib = load_library()
    q, r, s, st, cps = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_int()
    rv = C.c_uint64()
    _check(lib.tq_scan_plan_shape(n, nq, dim, bits, k, sms, C.byref(q), C.byref(r), C.byref(rv), C.byref(s),
                                  C.byref(st), C.byref(cps)))
    return {"q_per_cta": q.value, "n_ranges": r.value, "range_vectors": rv.value, "split_batches": s.value,
            "stages": st.value, "split_ctas_per_sm": cps.value}


def rescore(queries, corpus, results: "SearchResults", device: int = 0) -> "SearchResults":
    """Exact float inner-product re-rank of a top-k (float_rescore_topk,
    src/search/float_rescore.cpp:80-164): each candidate is re-scored as
    <query, corpus[id]> and every row re-sorted (score desc, id asc)."""
    q = np.ascontiguousarray(queries, dtype=np.float32)
    c = np.ascontiguousarray(corpus, dtype=np.float32)
    dim = q.shape[1]
    if c.ndim != 2 or c.shape[1] != dim:
        raise InvalidArgument(TQ_ERR_INVALID_ARGUMENT, "corpus must be [n, dim] float32")
    scores = np.ascontiguousarray(results.scores, dtype=np.float32).copy()
    ids = np.ascontiguousarray(results.ids, dtype=np.uint64).copy()
    nq, k = ids.shape
    _check(load_library().tq_rescore(_ptr(q), nq, dim, _ptr(c), c.shape[0], k, _ptr(scores), _ptr(ids), device))
    return SearchResults(scores, ids)


@dataclass
class SearchResults:
    """Row-major top-k, like vectorcache::SearchResults (search.hpp:77-84)."""

    scores: np.ndarray  # float32 [nq, k]
    ids: np.ndarray     # uint64 [nq, k]

    @property
    def k(self) -> int:
        return self.scores.shape[1]

    @property
    def nq(self) -> int:
        return self.scores.shape[0]


def _stream_ptr(stream) -> int | None:
    """cudaStream_t for a *_device call. With no stream given and torch in use,
    the caller's current torch stream: device buffers handed over as torch
    tensors were produced there, so the library's work is ordered after it."""
    if stream is None:
        import sys

        torch = sys.modules.get("torch")
        if torch is not None and torch.cuda.is_available() and torch.cuda.is_initialized():
            # torch's default stream is the legacy default stream (handle 0);
            # pass cudaStreamLegacy (1) for it: a NULL stream would mean the
            # library's own non-blocking stream, which is not ordered with it.
            return int(torch.cuda.current_stream().cuda_stream) or 1
        return None
    if isinstance(stream, int):
        return stream
    return int(getattr(stream, "cuda_stream", stream))


class TurboQuantIndex:
    """Flat TurboQuant index on one CUDA device.

    Same call order and validation as the reference: dim a positive multiple of
    8 and <= 16384, bits in {2, 3, 4}; calibrate() (TQ+) before prepare();
    search() after prepare(); k_eff = min(k, size).
    """

    def __init__(self, dim: int, bits: int, device: int = 0, _handle=None):
        lib = load_library()
        h = _handle
        if h is None:
            h = _P()
            _check(lib.tq_index_create(dim, bits, 0, device, C.byref(h)))
        self._h = h
        self._lib = lib
        self.dim = int(dim)
        self.bits = int(bits)
        self.device = int(device)
        self.n_byte_groups = self.dim // (8 // self.bits)

    @classmethod
    def load(cls, path, device: int = 0) -> "TurboQuantIndex":
        """Open an index written by save(); it comes back prepared."""
        lib = load_library()
        h = _P()
        _check(lib.tq_index_load(str(path).encode(), device, C.byref(h)))
        d, b = _SZ(), _SZ()
        _check(lib.tq_index_info(h, C.byref(d), C.byref(b), None, None, None))
        return cls(d.value, b.value, device, _handle=h)

    def save(self, path) -> None:
        _check(self._lib.tq_index_save(self._h, str(path).encode()))

    def add_npy(self, path) -> None:
        """Append the rows of a float32 (rows, dim) .npy file."""
        _check(self._lib.tq_index_add_npy(self._h, str(path).encode()))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.tq_index_destroy(self._h)
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

    # -- lifecycle -----------------------------------------------------------
    def calibrate(self, sample) -> None:
        a = _rows(sample, self.dim)
        _check(self._lib.tq_index_calibrate(self._h, _ptr(a), a.shape[0]))

    def add(self, vectors) -> None:
        a = _rows(vectors, self.dim)
        _check(self._lib.tq_index_add(self._h, _ptr(a), a.shape[0]))

    def prepare(self) -> None:
        _check(self._lib.tq_index_prepare(self._h))

    def search(self, queries, k: int) -> SearchResults:
        q = _rows(queries, self.dim)
        nq = q.shape[0]
        ke = _SZ(0)
        scores = np.empty(max(nq * k, 1), np.float32)
        ids = np.empty(max(nq * k, 1), np.uint64)
        _check(self._lib.tq_index_search(self._h, _ptr(q), nq, k, _ptr(scores), _ptr(ids), C.byref(ke)))
        kk = ke.value
        return SearchResults(scores[: nq * kk].reshape(nq, kk).copy(), ids[: nq * kk].reshape(nq, kk).copy())

    # -- device-resident variants (torch tensors or raw pointers) -----------
    def add_device(self, d_vectors, n: int | None = None, stream=None) -> None:
        ptr, n = _dev(d_vectors, n)
        _check(self._lib.tq_index_add_device(self._h, ptr, n, _stream_ptr(stream)))

    def calibrate_device(self, d_sample, n: int | None = None, stream=None) -> None:
        ptr, n = _dev(d_sample, n)
        _check(self._lib.tq_index_calibrate_device(self._h, ptr, n, _stream_ptr(stream)))

    def search_device(self, d_queries, k: int, d_scores, d_ids, nq: int | None = None, stream=None) -> int:
        qp, nq = _dev(d_queries, nq)
        ke = _SZ(0)
        _check(self._lib.tq_index_search_device(self._h, qp, nq, k, _dev(d_scores)[0], _dev(d_ids)[0],
                                                C.byref(ke), _stream_ptr(stream)))
        return ke.value

    def synchronize(self) -> None:
        _check(self._lib.tq_index_synchronize(self._h))

    # -- introspection -------------------------------------------------------
    def info(self) -> dict:
        d, b, n = _SZ(), _SZ(), _SZ()
        p, c = C.c_int(), C.c_int()
        _check(self._lib.tq_index_info(self._h, C.byref(d), C.byref(b), C.byref(n), C.byref(p), C.byref(c)))
        return {"dim": d.value, "bits": b.value, "size": n.value, "prepared": bool(p.value),
                "calibrated": bool(c.value)}

    @property
    def size(self) -> int:
        return self.info()["size"]

    def codes_flat(self) -> np.ndarray:
        out = np.empty((self.size, self.n_byte_groups), np.uint8)
        _check(self._lib.tq_index_export_codes_flat(self._h, _ptr(out)))
        return out

    def packed(self) -> np.ndarray:
        out = np.empty((self.size, self.bits * self.dim // 8), np.uint8)
        _check(self._lib.tq_index_export_packed(self._h, _ptr(out)))
        return out

    def alpha(self) -> np.ndarray:
        out = np.empty(self.size, np.float32)
        _check(self._lib.tq_index_export_alpha(self._h, _ptr(out)))
        return out

    def calibration(self) -> tuple[np.ndarray, np.ndarray]:
        s = np.empty(self.dim, np.float32)
        c = np.empty(self.dim, np.float32)
        _check(self._lib.tq_index_export_calibration(self._h, _ptr(s), _ptr(c)))
        return s, c

    def prepare_queries(self, queries) -> dict:
        q = _rows(queries, self.dim)
        nq = q.shape[0]
        out = {
            "q_rot": np.empty((nq, self.dim), np.float32),
            "bias_corr": np.empty(nq, np.float32),
            "luts": np.empty((nq, self.n_byte_groups * 32), np.uint8),
            "lut_scale": np.empty(nq, np.float32),
            "lut_bias": np.empty(nq, np.float32),
        }
        _check(self._lib.tq_index_prepare_queries(
            self._h, _ptr(q), nq, _ptr(out["q_rot"]), _ptr(out["bias_corr"]), _ptr(out["luts"]),
            _ptr(out["lut_scale"]), _ptr(out["lut_bias"])))
        return out

    def dense_scores(self, queries) -> tuple[np.ndarray, np.ndarray]:
        q = _rows(queries, self.dim)
        nq, n = q.shape[0], self.size
        ints = np.empty((nq, n), np.uint32)
        scores = np.empty((nq, n), np.float32)
        _check(self._lib.tq_index_dense_scores(self._h, _ptr(q), nq, _ptr(ints), _ptr(scores)))
        return ints, scores

    def stream(self) -> int:
        """The index's own cudaStream_t (as an int)."""
        p = _P()
        _check(self._lib.tq_index_get_stream(self._h, C.byref(p)))
        return p.value or 0

    def set_profiling(self, enabled: bool) -> None:
        _check(self._lib.tq_index_set_profiling(self._h, int(bool(enabled))))

    def read_profile(self) -> dict:
        """Device time per launch class since the last read, and under
        "by_launch" per launch name: {name: (ms, launches)}."""
        prof = Profile()
        _check(self._lib.tq_index_read_profile(self._h, C.byref(prof)))
        out = prof.as_dict()
        n = _SZ()
        _check(self._lib.tq_index_profile_entries(self._h, C.byref(n)))
        by = {}
        name = C.create_string_buffer(64)
        for i in range(n.value):
            ms, cnt = C.c_double(), C.c_uint64()
            _check(self._lib.tq_index_profile_entry(self._h, i, name, 64, C.byref(ms), C.byref(cnt)))
            by[name.value.decode()] = (ms.value, cnt.value)
        out["by_launch"] = by
        return out

    def replay_count(self) -> int:
        c = C.c_uint64()
        _check(self._lib.tq_index_replay_count(self._h, C.byref(c)))
        return c.value

    def scan_plan(self, nq: int, k: int) -> dict:
        """The scan tiling a search of nq queries with this k uses."""
        q, r, s, st = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        rv = C.c_uint64()
        _check(self._lib.tq_index_scan_plan(self._h, nq, k, C.byref(q), C.byref(r), C.byref(rv), C.byref(s),
                                            C.byref(st)))
        return {"q_per_cta": q.value, "n_ranges": r.value, "range_vectors": rv.value, "split_batches": s.value,
                "stages": st.value}


def _dev(t, n: int | None = None):
    """(device pointer, rows) from a torch CUDA tensor or an int pointer."""
    if isinstance(t, int):
        return t, int(n or 0)
    ptr = t.data_ptr()
    rows = t.shape[0] if n is None else n
    return ptr, int(rows)


from .bucketed import BucketedTurboQuantIndex, BucketParams  # noqa: E402

__all__ += ["BucketedTurboQuantIndex", "BucketParams"]

from .serving import Server  # noqa: E402

__all__ += ["Server"]
