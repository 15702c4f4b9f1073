"""Test infrastructure only — ctypes loaders for the CPU checkers and the
reference's own GPU index.

* `Oracle`   — oracle/_build/libtqoracle.so, the plain-C restatement of the
               reference's flat TurboQuant arithmetic (tq_oracle.c).
* `Reference` — oracle/_ref/libtqref.so, the reference's own CPU code compiled
               in place by oracle/Makefile (only where the reference tree was
               available at build time).
* `ReferenceGpuIndex` — oracle/_ref/libtqrefgpu.so, the reference's own GPU
               flat index (make -C oracle refgpu), timed by bench.py as the GPU
               bar to beat.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
arms use this module, and only as the checker or the timed CPU baseline; the
product library never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "libtqoracle.so"
REF_SO = HERE / "_ref" / "libtqref.so"
REF_GPU_SO = HERE / "_ref" / "libtqrefgpu.so"
# The reference source tree, when the caller names one (no default location).
REF_TREE_ENV = "VCB_REFERENCE_TREE"

_SZ = C.c_size_t
_P = C.c_void_p


def _p(a):
    return None if a is None else a.ctypes.data_as(_P)


def build(reference_tree: str | os.PathLike | None = None) -> None:
    """Compile the C oracle; with `reference_tree` (or $VCB_REFERENCE_TREE) set
    and present, also compile the reference's own CPU code in place from it."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    tree = reference_tree or os.environ.get(REF_TREE_ENV)
    if tree and (Path(tree) / "src").is_dir():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", "refgpu", f"REF={tree}", f"-j{os.cpu_count() or 4}"],
                       check=True)


def nbg_of(bits: int, dim: int) -> int:
    return dim // (8 // bits)


class _Common:
    prefix = ""

    def __init__(self, path: Path):
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (python -c 'import oracle.oracle as o; o.build()')")
        self.lib = C.CDLL(str(path))

    def fn(self, name):
        return getattr(self.lib, self.prefix + name)

    def codebook(self, bits, dim):
        b = np.zeros(15, np.float32)
        c = np.zeros(16, np.float32)
        assert self.fn("codebook")(_SZ(bits), _SZ(dim), _p(b), _p(c)) == 0
        L = 1 << bits
        return b[: L - 1].copy(), c[:L].copy()

    def rotation(self, dim):
        s = np.zeros(dim, np.float32)
        p = np.zeros(dim, np.uint32)
        assert self.fn("rotation")(_SZ(dim), _p(s), _p(p)) == 0
        return s, p

    def fit_calibration(self, x, bits):
        x = np.ascontiguousarray(x, np.float32)
        n, dim = x.shape
        sh = np.zeros(dim, np.float32)
        sc = np.zeros(dim, np.float32)
        assert self.fn("fit_calibration")(_p(x), _SZ(n), _SZ(dim), _SZ(bits), _p(sh), _p(sc)) == 0
        return sh, sc

    def encode(self, x, bits, shift=None, scale=None):
        x = np.ascontiguousarray(x, np.float32)
        n, dim = x.shape
        packed = np.zeros((n, bits * dim // 8), np.uint8)
        alpha = np.zeros(n, np.float32)
        rc = self.fn("encode")(_p(x), _SZ(n), _SZ(dim), _SZ(bits), _p(shift), _p(scale), _p(packed), _p(alpha))
        assert rc == 0
        return packed, alpha

    def codes_flat(self, packed, bits, dim):
        packed = np.ascontiguousarray(packed, np.uint8)
        n = packed.shape[0]
        out = np.zeros((n, nbg_of(bits, dim)), np.uint8)
        assert self.fn("codes_flat")(_p(packed), _SZ(n), _SZ(bits), _SZ(dim), _p(out)) == 0
        return out

    def prepare_queries(self, q, bits, shift=None, scale=None):
        q = np.ascontiguousarray(q, np.float32)
        nq, dim = q.shape
        nbg = nbg_of(bits, dim)
        out = {
            "q_rot": np.zeros((nq, dim), np.float32),
            "bias_corr": np.zeros(nq, np.float32),
            "luts": np.zeros((nq, nbg * 32), np.uint8),
            "lut_scale": np.zeros(nq, np.float32),
            "lut_bias": np.zeros(nq, np.float32),
        }
        rc = self.fn("prepare_queries")(_p(q), _SZ(nq), _SZ(dim), _SZ(bits), _p(shift), _p(scale),
                                       _p(out["q_rot"]), _p(out["bias_corr"]), _p(out["luts"]),
                                       _p(out["lut_scale"]), _p(out["lut_bias"]))
        assert rc == 0
        return out


class Oracle(_Common):
    prefix = "tqo_"

    def __init__(self, path: Path = ORACLE_SO):
        super().__init__(path)
        self.lib.tqo_beta_cdf_aa.restype = C.c_double
        self.lib.tqo_beta_cdf_aa.argtypes = [C.c_double, C.c_double]
        self.lib.tqo_topk.restype = _SZ
        self.lib.tqo_search_flat.restype = _SZ

    def beta_cdf_aa(self, a, t):
        return self.lib.tqo_beta_cdf_aa(a, t)

    def int_scores(self, luts, codes_flat):
        luts = np.ascontiguousarray(luts, np.uint8)
        codes_flat = np.ascontiguousarray(codes_flat, np.uint8)
        nq, n, nbg = luts.shape[0], codes_flat.shape[0], codes_flat.shape[1]
        out = np.zeros((nq, n), np.uint32)
        self.lib.tqo_int_scores(_p(luts), _SZ(nq), _p(codes_flat), _SZ(n), _SZ(nbg), _p(out))
        return out

    def float_scores(self, prep, codes_flat, alpha):
        codes_flat = np.ascontiguousarray(codes_flat, np.uint8)
        alpha = np.ascontiguousarray(alpha, np.float32)
        nq, n, nbg = prep["luts"].shape[0], codes_flat.shape[0], codes_flat.shape[1]
        out = np.zeros((nq, n), np.float32)
        self.lib.tqo_float_scores(_p(prep["luts"]), _p(prep["lut_scale"]), _p(prep["lut_bias"]),
                                  _p(prep["bias_corr"]), _SZ(nq), _p(codes_flat), _p(alpha), _SZ(n),
                                  _SZ(nbg), _p(out))
        return out

    def topk(self, scores, k):
        scores = np.ascontiguousarray(scores, np.float32)
        nq, n = scores.shape
        s = np.zeros(max(nq * k, 1), np.float32)
        i = np.zeros(max(nq * k, 1), np.uint64)
        ke = self.lib.tqo_topk(_p(scores), _SZ(nq), _SZ(n), _SZ(k), _p(s), _p(i))
        return s[: nq * ke].reshape(nq, ke), i[: nq * ke].reshape(nq, ke)

    def search_flat(self, q, bits, packed, alpha, k, shift=None, scale=None):
        q = np.ascontiguousarray(q, np.float32)
        nq, dim = q.shape
        n = packed.shape[0]
        s = np.zeros(max(nq * k, 1), np.float32)
        i = np.zeros(max(nq * k, 1), np.uint64)
        ke = self.lib.tqo_search_flat(_p(q), _SZ(nq), _SZ(dim), _SZ(bits), _p(shift), _p(scale),
                                      _p(np.ascontiguousarray(packed)), _p(np.ascontiguousarray(alpha)),
                                      _SZ(n), _SZ(k), _p(s), _p(i))
        return s[: nq * ke].reshape(nq, ke), i[: nq * ke].reshape(nq, ke)


    def ivf_search(self, prep, codes_flat, alpha, ids, bucket_start, bucket_size, probes, n_probe, offsets, k):
        """IVF residual search over bucket-ordered slots (score_prepared_into
        composed over each query's probed buckets)."""
        codes_flat = np.ascontiguousarray(codes_flat, np.uint8)
        nq = prep["luts"].shape[0]
        nbg = codes_flat.shape[1]
        probes = np.ascontiguousarray(probes, np.uint32)
        max_probe = probes.shape[1]
        s = np.zeros((nq, k), np.float32)
        i = np.zeros((nq, k), np.uint64)
        self.lib.tqo_ivf_search(
            _p(prep["luts"]), _p(prep["lut_scale"]), _p(prep["lut_bias"]), _p(prep["bias_corr"]), _SZ(nq),
            _SZ(nbg), _p(codes_flat), _p(np.ascontiguousarray(alpha, np.float32)),
            _p(np.ascontiguousarray(ids, np.uint64)), _p(np.ascontiguousarray(bucket_start, np.uint64)),
            _p(np.ascontiguousarray(bucket_size, np.uint64)), _p(probes),
            _p(np.ascontiguousarray(n_probe, np.uint32)), _SZ(max_probe),
            _p(np.ascontiguousarray(offsets, np.float32)), _SZ(k), _p(s), _p(i))
        return s, i


class Reference(_Common):
    prefix = "tqref_"

    def ivf_search(self, q, bits, residuals, ids, bucket_start, bucket_size, probes, n_probe, offsets, k,
                   shift=None, scale=None):
        """The reference's own score_prepared_into over the same buckets: its
        encode + repack per bucket, LUTs from prepare_queries, one call per
        (query, probed bucket) in probe order, heaps sorted at the end."""
        q = np.ascontiguousarray(q, np.float32)
        nq, dim = q.shape
        probes = np.ascontiguousarray(probes, np.uint32)
        s = np.zeros((nq, k), np.float32)
        i = np.zeros((nq, k), np.uint64)
        rc = self.lib.tqref_ivf_search(
            _p(q), _SZ(nq), _SZ(dim), _SZ(bits), _p(shift), _p(scale),
            _p(np.ascontiguousarray(residuals, np.float32)), _p(np.ascontiguousarray(ids, np.uint64)),
            _p(np.ascontiguousarray(bucket_start, np.uint64)), _p(np.ascontiguousarray(bucket_size, np.uint64)),
            _SZ(len(bucket_size)), _p(probes), _p(np.ascontiguousarray(n_probe, np.uint32)), _SZ(probes.shape[1]),
            _p(np.ascontiguousarray(offsets, np.float32)), _SZ(k), _p(s), _p(i))
        if rc != 0:
            raise RuntimeError(self.lib.tqref_last_error().decode())
        return s, i

    def __init__(self, path: Path = REF_SO):
        super().__init__(path)
        self.lib.tqref_last_error.restype = C.c_char_p
        self.lib.tqref_beta_cdf_aa.restype = C.c_double
        self.lib.tqref_beta_cdf_aa.argtypes = [C.c_double, C.c_double]

    def beta_cdf_aa(self, a, t):
        return self.lib.tqref_beta_cdf_aa(a, t)

    def max_threads(self) -> int:
        return int(self.lib.tqref_max_threads())

    def set_threads(self, n: int) -> None:
        self.lib.tqref_set_threads(C.c_int(n))


class ReferenceIndex:
    """The reference's flat CPU path (fit_calibration + encode + repack at
    creation, search_flat per query batch) under the pinned AVX2 backend."""

    def __init__(self, ref: Reference, x, bits, calib_rows=None, native_backend=False):
        self.ref = ref
        x = np.ascontiguousarray(x, np.float32)
        self.n, self.dim = x.shape
        self.bits = bits
        h = _P()
        cal = None if calib_rows is None else np.ascontiguousarray(calib_rows, np.float32)
        rc = ref.lib.tqref_index_create(_p(x), _SZ(self.n), _SZ(self.dim), _SZ(bits), _p(cal),
                                        _SZ(0 if cal is None else cal.shape[0]), C.c_int(int(native_backend)),
                                        C.byref(h))
        if rc != 0:
            raise RuntimeError(ref.lib.tqref_last_error().decode())
        self.h = h

    def search(self, q, k):
        q = np.ascontiguousarray(q, np.float32)
        nq = q.shape[0]
        s = np.zeros(max(nq * k, 1), np.float32)
        i = np.zeros(max(nq * k, 1), np.uint64)
        ke = _SZ(0)
        rc = self.ref.lib.tqref_index_search(self.h, _p(q), _SZ(nq), _SZ(k), _p(s), _p(i), C.byref(ke))
        if rc != 0:
            raise RuntimeError(self.ref.lib.tqref_last_error().decode())
        kk = ke.value
        return s[: nq * kk].reshape(nq, kk), i[: nq * kk].reshape(nq, kk)

    def packed(self):
        """The reference's encode output for the index rows: bit-plane codes
        (n x bits*dim/8) and alpha (n)."""
        packed = np.zeros((self.n, self.bits * self.dim // 8), np.uint8)
        alpha = np.zeros(self.n, np.float32)
        rc = self.ref.lib.tqref_index_packed(self.h, _p(packed), _p(alpha))
        if rc != 0:
            raise RuntimeError(self.ref.lib.tqref_last_error().decode())
        return packed, alpha

    def calibration(self):
        """The reference's TQ+ shift / scale (raises if not calibrated)."""
        sh = np.zeros(self.dim, np.float32)
        sc = np.zeros(self.dim, np.float32)
        rc = self.ref.lib.tqref_index_calibration(self.h, _p(sh), _p(sc))
        if rc != 0:
            raise RuntimeError(self.ref.lib.tqref_last_error().decode())
        return sh, sc

    def close(self):
        if self.h:
            self.ref.lib.tqref_index_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def _float_rescore(lib, fn, queries, corpus, ids, scores_init=None):
    q = np.ascontiguousarray(queries, np.float32)
    c = np.ascontiguousarray(corpus, np.float32)
    ids = np.ascontiguousarray(ids, np.uint64).copy()
    nq, k = ids.shape
    s = np.zeros((nq, k), np.float32)
    rc = getattr(lib, fn)(_p(q), _SZ(nq), _SZ(q.shape[1]), _p(c), _SZ(c.shape[0]), _SZ(k), _p(s), _p(ids))
    assert rc in (0, None)
    return s, ids


def oracle_float_rescore(orc: "Oracle", queries, corpus, ids):
    """Exact float re-rank of candidate ids (the C restatement)."""
    return _float_rescore(orc.lib, "tqo_float_rescore", queries, corpus, ids)


def reference_float_rescore(ref: "Reference", queries, corpus, ids):
    """The reference's own float_rescore_topk on the same candidate ids."""
    return _float_rescore(ref.lib, "tqref_float_rescore", queries, corpus, ids)


class ReferenceGpuIndex:
    """The reference's own GPU flat index (gpu::FlatIndex: add, prepare,
    search with host buffers; oracle/_ref/libtqrefgpu.so). Timed as the GPU
    bar to beat; its top-k is approximate (a few candidates per thread), so
    it is judged by recall, not compared bit for bit."""

    def __init__(self, dim: int, bits: int, path: Path = REF_GPU_SO):
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (make -C oracle refgpu REF=<reference tree>)")
        self.h = None
        self.lib = C.CDLL(str(path))
        self.lib.tqrefgpu_last_error.restype = C.c_char_p
        self.dim = dim
        h = _P()
        self._check(self.lib.tqrefgpu_create(_SZ(dim), _SZ(bits), C.byref(h)))
        self.h = h

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib.tqrefgpu_last_error().decode())

    def add(self, x):
        x = np.ascontiguousarray(x, np.float32)
        self._check(self.lib.tqrefgpu_add(self.h, _p(x), _SZ(x.shape[0])))

    def prepare(self):
        self._check(self.lib.tqrefgpu_prepare(self.h))

    def search(self, q, k):
        q = np.ascontiguousarray(q, np.float32)
        nq = q.shape[0]
        s = np.zeros(max(nq * k, 1), np.float32)
        i = np.zeros(max(nq * k, 1), np.uint64)
        ke = _SZ(0)
        self._check(self.lib.tqrefgpu_search(self.h, _p(q), _SZ(nq), _SZ(k), _p(s), _p(i), C.byref(ke)))
        kk = ke.value
        return s[: nq * kk].reshape(nq, kk), i[: nq * kk].reshape(nq, kk)

    def close(self):
        if self.h:
            self.lib.tqrefgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()
