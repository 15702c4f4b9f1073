// Test infrastructure only — not part of the product.
//
// C-ABI shim over the reference's OWN CPU implementation of the flat TurboQuant
// path (nishadtardalkar/vectorcache, compiled in place from its src/ tree by
// oracle/Makefile into oracle/_ref/libtqref.so). The parity tests, the golden
// fixture generator and bench.py's reference arm call these entry points; the
// product library never links or loads this file.
//
// Every function pins the reference's search backend to the AVX2 PERM0 uint8
// LUT scan by setting TURBOVEC_NO_VECTOR_MAJOR=1 (pack.cpp:214-220) unless the
// caller asks for the host's default backend explicitly (`native_backend`).
//
// Reference entry points wrapped (paths inside the reference project):
//   codebook()                 src/quantize/codebook.cpp:203
//   Rotation                   src/transform/rotation.cpp:139, :185
//   row_norm                   src/encode/encode.cpp:290
//   fit_calibration            src/encode/encode.cpp:327
//   encode                     src/encode/encode.cpp:294
//   codes_flat_from_packed     src/pack/pack.cpp:352
//   repack                     src/pack/pack.cpp:366
//   prepare_queries            src/search/search.cpp:762
//   score_prepared/search_flat src/search/search.cpp:1072, :1293
//   score_prepared_into        src/search/search.cpp:1156 (IVF residual scoring)
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <limits>
#include <memory>
#include <span>
#include <string>
#include <vector>

#include "vectorcache/encode/encode.hpp"
#include "vectorcache/pack/pack.hpp"
#include "vectorcache/quantize/codebook.hpp"
#include "vectorcache/search/float_rescore.hpp"
#include "vectorcache/search/search.hpp"
#include "vectorcache/transform/rotation.hpp"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

thread_local std::string g_err;

void pin_backend(int native_backend) {
  if (native_backend) {
    unsetenv("TURBOVEC_NO_VECTOR_MAJOR");
  } else {
    setenv("TURBOVEC_NO_VECTOR_MAJOR", "1", 1);
  }
}

template <typename F>
int guarded(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  } catch (...) {
    g_err = "unknown exception";
    return 1;
  }
}

struct RefIndex {
  std::size_t dim = 0, bits = 0, n = 0;
  std::unique_ptr<vectorcache::Rotation> rot;
  std::vector<float> boundaries, centroids;
  vectorcache::Calibration calib;
  bool has_calib = false;
  std::vector<std::uint8_t> packed;
  std::vector<float> alpha;
  std::vector<std::uint8_t> blocked;
  std::size_t n_blocks = 0;
  int native_backend = 0;  // the code layout from repack() depends on the backend
};

}  // namespace

extern "C" {

const char* tqref_last_error() { return g_err.c_str(); }

int tqref_max_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void tqref_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

// Beta(a, a) CDF used by the TQ+ anchor quantiles (encode.hpp:40).
double tqref_beta_cdf_aa(double a, double t) { return vectorcache::beta_cdf_aa(a, t); }

int tqref_codebook(std::size_t bits, std::size_t dim, float* boundaries, float* centroids) {
  return guarded([&] {
    auto [b, c] = vectorcache::codebook(bits, dim);
    std::memcpy(boundaries, b.data(), b.size() * sizeof(float));
    std::memcpy(centroids, c.data(), c.size() * sizeof(float));
  });
}

int tqref_rotation(std::size_t dim, float* signs, std::uint32_t* perm) {
  return guarded([&] {
    vectorcache::Rotation r(dim);
    auto s = r.signs(0);
    auto p = r.perm(0);
    std::memcpy(signs, s.data(), dim * sizeof(float));
    std::memcpy(perm, p.data(), dim * sizeof(std::uint32_t));
  });
}

// Normalize + rotate rows exactly as encode()/prepare_queries() do.
int tqref_rotate(const float* x, std::size_t n, std::size_t dim, float* rot_out, float* norms) {
  return guarded([&] {
    vectorcache::Rotation r(dim);
    std::vector<float> scratch(dim);
    for (std::size_t i = 0; i < n; ++i) {
      std::span<const float> src(x + i * dim, dim);
      const float nv = vectorcache::row_norm(src);
      norms[i] = nv;
      const float inv = (nv > vectorcache::kMinInputNorm) ? (1.f / nv) : 0.f;
      r.apply_scaled_into(src, inv, std::span<float>(rot_out + i * dim, dim), scratch);
    }
  });
}

int tqref_fit_calibration(const float* x, std::size_t n, std::size_t dim, std::size_t bits,
                          float* shift, float* scale) {
  return guarded([&] {
    vectorcache::Rotation r(dim);
    auto cb = vectorcache::codebook(bits, dim);
    std::vector<float> scratch;
    auto cal = vectorcache::fit_calibration(std::span<const float>(x, n * dim), n, dim, r,
                                            cb.second, scratch);
    std::memcpy(shift, cal.shift.data(), dim * sizeof(float));
    std::memcpy(scale, cal.scale_tq.data(), dim * sizeof(float));
  });
}

// packed_out: n * bits * dim/8 bytes (bit-plane rows); alpha: n floats.
int tqref_encode(const float* x, std::size_t n, std::size_t dim, std::size_t bits,
                 const float* shift, const float* scale, std::uint8_t* packed_out, float* alpha) {
  return guarded([&] {
    vectorcache::Rotation r(dim);
    auto cb = vectorcache::codebook(bits, dim);
    vectorcache::Calibration cal;
    if (shift) {
      cal.shift.assign(shift, shift + dim);
      cal.scale_tq.assign(scale, scale + dim);
    }
    std::vector<float> scratch;
    std::vector<std::uint8_t> packed;
    std::vector<float> scales;
    vectorcache::encode(std::span<const float>(x, n * dim), n, dim, r, cb.first, cb.second, bits,
                        shift ? &cal : nullptr, scratch, packed, scales);
    std::memcpy(packed_out, packed.data(), packed.size());
    std::memcpy(alpha, scales.data(), n * sizeof(float));
  });
}

int tqref_codes_flat(const std::uint8_t* packed, std::size_t n, std::size_t bits, std::size_t dim,
                     std::uint8_t* out) {
  return guarded([&] {
    const std::size_t bytes = n * bits * (dim / 8);
    auto flat = vectorcache::codes_flat_from_packed(std::span<const std::uint8_t>(packed, bytes), n,
                                                    bits, dim);
    std::memcpy(out, flat.data(), flat.size());
  });
}

// LUT bytes (nq * nbg * 32), scale, bias, bias_corr and q_rot for the pinned
// AVX2 backend.
int tqref_prepare_queries(const float* q, std::size_t nq, std::size_t dim, std::size_t bits,
                          const float* shift, const float* scale, float* q_rot, float* bias_corr,
                          std::uint8_t* luts, float* lut_scale, float* lut_bias) {
  return guarded([&] {
    pin_backend(0);
    vectorcache::Rotation r(dim);
    auto cb = vectorcache::codebook(bits, dim);
    std::span<const float> sh, sc;
    if (shift) {
      sh = std::span<const float>(shift, dim);
      sc = std::span<const float>(scale, dim);
    }
    auto prep = vectorcache::prepare_queries(std::span<const float>(q, nq * dim), nq, dim, r,
                                             cb.second, bits, sh, sc);
    if (prep.backend != vectorcache::SearchBackendKind::Avx2) {
      throw std::runtime_error("reference backend is not avx2_perm0");
    }
    const std::size_t nbg = prep.n_byte_groups;
    std::memcpy(q_rot, prep.q_rot.data(), nq * dim * sizeof(float));
    std::memcpy(bias_corr, prep.bias_corrs.data(), nq * sizeof(float));
    for (std::size_t i = 0; i < nq; ++i) {
      std::memcpy(luts + i * nbg * 32, prep.luts[i].uint8_luts.data(), nbg * 32);
      lut_scale[i] = prep.luts[i].scale;
      lut_bias[i] = prep.luts[i].bias;
    }
  });
}

// Exact float re-rank of given top-k ids (float_rescore_topk,
// src/search/float_rescore.cpp:80-164); scores/ids are nq x k, in place.
int tqref_float_rescore(const float* q, std::size_t nq, std::size_t dim, const float* corpus,
                        std::size_t n_corpus, std::size_t k, float* scores, std::uint64_t* ids) {
  return guarded([&] {
    vectorcache::SearchResults res;
    res.nq = nq;
    res.k = k;
    res.scores.assign(nq * k, 0.f);
    res.ids.resize_uninitialized(nq * k);
    std::memcpy(res.ids.data(), ids, nq * k * sizeof(std::uint64_t));
    vectorcache::float_rescore_topk(res, std::span<const float>(q, nq * dim),
                                    std::span<const float>(corpus, n_corpus * dim), dim);
    std::memcpy(scores, res.scores.data(), nq * k * sizeof(float));
    std::memcpy(ids, res.ids.data(), nq * k * sizeof(std::uint64_t));
  });
}

// ---- prepared reference index (for timing and search parity) -------------

int tqref_index_create(const float* x, std::size_t n, std::size_t dim, std::size_t bits,
                       const float* calib_rows, std::size_t n_calib, int native_backend,
                       void** out) {
  return guarded([&] {
    pin_backend(native_backend);
    auto h = std::make_unique<RefIndex>();
    h->dim = dim;
    h->bits = bits;
    h->n = n;
    h->native_backend = native_backend;
    h->rot = std::make_unique<vectorcache::Rotation>(dim);
    auto cb = vectorcache::codebook(bits, dim);
    h->boundaries = cb.first;
    h->centroids = cb.second;
    std::vector<float> scratch;
    if (calib_rows && n_calib > 0) {
      h->calib = vectorcache::fit_calibration(std::span<const float>(calib_rows, n_calib * dim),
                                              n_calib, dim, *h->rot, h->centroids, scratch);
      h->has_calib = true;
    }
    vectorcache::encode(std::span<const float>(x, n * dim), n, dim, *h->rot, h->boundaries,
                        h->centroids, bits, h->has_calib ? &h->calib : nullptr, scratch,
                        h->packed, h->alpha);
    auto [blocked, nb] = vectorcache::repack(h->packed, n, bits, dim);
    h->blocked = std::move(blocked);
    h->n_blocks = nb;
    *out = h.release();
  });
}

int tqref_index_destroy(void* h) {
  delete static_cast<RefIndex*>(h);
  return 0;
}

int tqref_index_calibration(void* hv, float* shift, float* scale) {
  return guarded([&] {
    auto* h = static_cast<RefIndex*>(hv);
    if (!h->has_calib) throw std::runtime_error("index has no calibration");
    std::memcpy(shift, h->calib.shift.data(), h->dim * sizeof(float));
    std::memcpy(scale, h->calib.scale_tq.data(), h->dim * sizeof(float));
  });
}

int tqref_index_packed(void* hv, std::uint8_t* packed, float* alpha) {
  return guarded([&] {
    auto* h = static_cast<RefIndex*>(hv);
    std::memcpy(packed, h->packed.data(), h->packed.size());
    std::memcpy(alpha, h->alpha.data(), h->n * sizeof(float));
  });
}

// scores/ids: nq * k capacity; rows written with stride *k_eff = min(k, n).
int tqref_index_search(void* hv, const float* q, std::size_t nq, std::size_t k, float* scores,
                       std::uint64_t* ids, std::size_t* k_eff) {
  return guarded([&] {
    auto* h = static_cast<RefIndex*>(hv);
    pin_backend(h->native_backend);
    std::span<const float> sh, sc;
    if (h->has_calib) {
      sh = h->calib.shift;
      sc = h->calib.scale_tq;
    }
    auto res = vectorcache::search_flat(std::span<const float>(q, nq * h->dim), nq, h->dim, k,
                                        *h->rot, h->centroids, h->bits, h->blocked, h->n_blocks,
                                        h->alpha, sh, sc);
    *k_eff = res.k;
    if (res.k > 0) {
      std::memcpy(scores, res.scores.data(), nq * res.k * sizeof(float));
      std::memcpy(ids, res.ids.data(), nq * res.k * sizeof(std::uint64_t));
    }
  });
}

// ---- IVF residual scoring (bucketed index parity) --------------------------
//
// The reference's building block for its IVF index: score_prepared_into
// (src/search/search.cpp:1156-1264) scores one bucket's codes into existing
// per-query top-k heaps, remapping local ids through the bucket's id map and
// adding a per-query score offset <q_hat, encode_c> after alpha * LUT score.
// This driver encodes every bucket's residual rows with the reference's own
// encode + repack, builds the query LUTs once (prepare_queries), then visits
// each query's probed buckets in the given order, one score_prepared_into call
// per (query, bucket), and sorts the heaps (heaps_to_search_results).
// residuals: n_slots x dim rows, bucket b at rows [start[b], start[b]+size[b]);
// ids: the original id of every slot; probes/offsets: nq x max_probe, the
// first n_probe[q] entries valid.
int tqref_ivf_search(const float* q, std::size_t nq, std::size_t dim, std::size_t bits,
                     const float* shift, const float* scale, const float* residuals,
                     const std::uint64_t* ids, const std::uint64_t* bucket_start,
                     const std::uint64_t* bucket_size, std::size_t n_buckets,
                     const std::uint32_t* probes, const std::uint32_t* n_probe,
                     std::size_t max_probe, const float* offsets, std::size_t k,
                     float* out_scores, std::uint64_t* out_ids) {
  return guarded([&] {
    pin_backend(0);
    vectorcache::Rotation r(dim);
    auto cb = vectorcache::codebook(bits, dim);
    vectorcache::Calibration calib;
    std::span<const float> sh, sc;
    if (shift) {
      calib.shift.assign(shift, shift + dim);
      calib.scale_tq.assign(scale, scale + dim);
      sh = calib.shift;
      sc = calib.scale_tq;
    }
    struct Bucket {
      std::vector<std::uint8_t> blocked;
      std::size_t n_blocks = 0;
      std::vector<float> alpha;
      std::vector<std::uint64_t> ids;
    };
    std::vector<Bucket> buckets(n_buckets);
    std::vector<float> scratch;
    for (std::size_t b = 0; b < n_buckets; ++b) {
      const std::size_t n = bucket_size[b];
      if (n == 0) continue;
      std::vector<std::uint8_t> packed;
      vectorcache::encode(std::span<const float>(residuals + bucket_start[b] * dim, n * dim), n, dim,
                          r, cb.first, cb.second, bits, shift ? &calib : nullptr, scratch, packed,
                          buckets[b].alpha);
      auto [blocked, nbl] = vectorcache::repack(packed, n, bits, dim);
      buckets[b].blocked = std::move(blocked);
      buckets[b].n_blocks = nbl;
      buckets[b].ids.assign(ids + bucket_start[b], ids + bucket_start[b] + n);
    }
    auto prep = vectorcache::prepare_queries(std::span<const float>(q, nq * dim), nq, dim, r,
                                             cb.second, bits, sh, sc);
    if (prep.backend != vectorcache::SearchBackendKind::Avx2) {
      throw std::runtime_error("reference backend is not avx2_perm0");
    }
    std::vector<float> heap_s(nq * k), heap_min(nq, -std::numeric_limits<float>::infinity());
    std::vector<std::uint64_t> heap_i(nq * k);
    std::vector<std::size_t> heap_sz(nq, 0), heap_mi(nq, 0);
    std::vector<float> offs(nq, 0.f);
    for (std::size_t qi = 0; qi < nq; ++qi) {
      const std::size_t one[1] = {qi};
      for (std::size_t j = 0; j < n_probe[qi]; ++j) {
        const Bucket& bk = buckets[probes[qi * max_probe + j]];
        if (bk.alpha.empty()) continue;
        offs[qi] = offsets[qi * max_probe + j];
        vectorcache::score_prepared_into(prep, k, bk.blocked, bk.n_blocks, bk.alpha, bk.ids,
                                         std::span<const std::size_t>(one, 1), heap_s.data(),
                                         heap_i.data(), heap_sz.data(), heap_min.data(),
                                         heap_mi.data(), offs.data());
      }
    }
    vectorcache::SearchResults res;
    vectorcache::heaps_to_search_results(res, nq, k, heap_s.data(), heap_i.data(), heap_sz.data());
    std::memcpy(out_scores, res.scores.data(), nq * k * sizeof(float));
    std::memcpy(out_ids, res.ids.data(), nq * k * sizeof(std::uint64_t));
  });
}

}  // extern "C"
