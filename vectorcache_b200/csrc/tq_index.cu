// Host side of the flat TurboQuant index and its C ABI (include/vectorcache_b200.h).
//
// The index owns its device memory and one CUDA stream. Lifecycle mirrors the
// reference's gpu::FlatIndex (src/gpu/flat_index.cpp:82-242) and the flat free
// functions (encode.cpp, pack.cpp, search.cpp): calibrate (optional TQ+) ->
// add -> prepare -> search.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/vectorcache_b200.h"
#include "tq_abi.h"
#include "tq_host_math.h"
#include "tq_index_impl.h"
#include "tq_kernels.h"

namespace vcb {

thread_local std::string g_last_error;

bool& dry_run_flag() {
  static thread_local bool flag = false;
  return flag;
}

void calibrate_index(tq_index* h, const float* d_sample, size_t n, cudaStream_t s) {
  require(n >= 2, TQ_ERR_INVALID_ARGUMENT, "calibration needs at least 2 rows");
  require(!h->prepared && h->n == 0, TQ_ERR_STATE, "calibrate must precede prepare()");
  DeviceBuffer yt, qlo;
  yt.reserve(n * h->dim * sizeof(float));
  qlo.reserve(2 * h->dim * sizeof(float));
  RotateArgs r{};
  r.x = d_sample;
  r.n = static_cast<long long>(n);
  r.dim = static_cast<int>(h->dim);
  r.block = static_cast<int>(h->block);
  r.inv_sqrt_block = h->inv_sqrt_block;
  r.perm_sign = h->d_perm_sign.as<uint32_t>();
  r.out_t = yt.as<float>();
  check(launch_rotate_rows_t(r, h->sms, s), "rotate kernel");
  const TqplusAnchor anc = tqplus_anchor(n, h->bits, h->dim);
  check(launch_order_stats(yt.as<float>(), static_cast<long long>(n), static_cast<int>(h->dim),
                                     static_cast<long long>(anc.lo_idx),
                                     static_cast<long long>(anc.hi_idx), qlo.as<float>(),
                                     qlo.as<float>() + h->dim, s),
             "order statistics kernel");
  std::vector<float> q(2 * h->dim);
  check(cudaMemcpyAsync(q.data(), qlo.get(), q.size() * 4, cudaMemcpyDeviceToHost, s), "D2H");
  check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  // Shift and scale per dimension (encode.cpp:277-283).
  h->shift.assign(h->dim, 0.f);
  h->scale.assign(h->dim, 1.f);
  for (size_t d = 0; d < h->dim; ++d) {
    const float q_lo = q[d], q_hi = q[h->dim + d];
    const float span = q_hi - q_lo;
    if (!(span > 1e-12f) || !(anc.qc_span > 0.f)) continue;
    const float sc = anc.qc_span / span;
    h->scale[d] = sc;
    h->shift[d] = anc.qc_lo / sc - q_lo;
  }
  std::vector<float> inv(h->dim);
  for (size_t d = 0; d < h->dim; ++d) inv[d] = 1.f / h->scale[d];
  h->d_shift.reserve(h->dim * 4);
  h->d_scale.reserve(h->dim * 4);
  h->d_inv_scale.reserve(h->dim * 4);
  h->upload(h->d_shift.get(), h->shift.data(), h->dim * 4);
  h->upload(h->d_scale.get(), h->scale.data(), h->dim * 4);
  h->upload(h->d_inv_scale.get(), inv.data(), h->dim * 4);
  h->sync();
  h->calibrated = true;
}

}  // namespace vcb

namespace {

using vcb::require;

void check_aligned(const void* p, const char* what) {
  if (reinterpret_cast<uintptr_t>(p) % 16 != 0) {
    vcb::fail(TQ_ERR_INVALID_ARGUMENT, std::string(what) + " must be 16-byte aligned");
  }
}


void do_add_device(tq_index* h, const float* d_x, size_t n, cudaStream_t s) {
  if (n == 0) return;
  check_aligned(d_x, "vectors");
  if (h->prepared) {
    h->encode_append(d_x, n, s);
    return;
  }
  // Stage on the device until prepare(), like gpu::FlatIndex::add.
  const size_t need = (h->staged_n + n) * h->dim * sizeof(float);
  if (need > h->d_staged.bytes()) {
    vcb::DeviceBuffer grown;
    grown.reserve(std::max(need, h->d_staged.bytes() + h->d_staged.bytes() / 2));
    if (h->staged_n) {
      vcb::check(cudaMemcpyAsync(grown.get(), h->d_staged.get(), h->staged_n * h->dim * sizeof(float),
                                 cudaMemcpyDeviceToDevice, s),
                 "cudaMemcpyAsync D2D");
    }
    vcb::check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    grown.swap(h->d_staged);
  }
  vcb::check(cudaMemcpyAsync(h->d_staged.as<float>() + h->staged_n * h->dim, d_x, n * h->dim * sizeof(float),
                             cudaMemcpyDeviceToDevice, s),
             "cudaMemcpyAsync D2D");
  h->staged_n += n;
}

// Bit-plane rows from row-major byte-group codes (encode.cpp:147-153).
void flat_to_planes(const uint8_t* flat, size_t n, size_t bits, size_t dim, uint8_t* out) {
  const size_t cpb = 8 / bits, field = (bits == 3) ? 4 : bits, nbg = dim / cpb, bpp = dim / 8;
  std::memset(out, 0, n * bits * bpp);
  for (size_t v = 0; v < n; ++v) {
    const uint8_t* row = flat + v * nbg;
    uint8_t* o = out + v * bits * bpp;
    for (size_t j = 0; j < dim; ++j) {
      const size_t g = j / cpb, sh = (cpb - 1 - j % cpb) * field;
      const unsigned code = (row[g] >> sh) & ((1u << field) - 1u);
      for (size_t p = 0; p < bits; ++p) {
        o[p * bpp + j / 8] |= static_cast<uint8_t>(((code >> p) & 1u) << (7 - j % 8));
      }
    }
  }
}

}  // namespace

extern "C" {

const char* tq_last_error(void) { return vcb::g_last_error.c_str(); }

const char* tq_version(void) { return "vectorcache_b200 0.1.0 (sm_100a)"; }

int tq_codebook(size_t bits, size_t dim, float* boundaries, float* centroids) {
  return vcb::guarded([&] {
    require(vcb::bits_supported(bits), TQ_ERR_INVALID_ARGUMENT, "bits must be 2, 3, or 4");
    require(dim >= 2, TQ_ERR_INVALID_ARGUMENT, "dim must be >= 2");
    const vcb::Codebook& cb = vcb::codebook(bits, dim);
    std::memcpy(boundaries, cb.boundaries.data(), cb.boundaries.size() * 4);
    std::memcpy(centroids, cb.centroids.data(), cb.centroids.size() * 4);
  });
}

int tq_rotation_tables(size_t dim, float* signs, uint32_t* perm) {
  return vcb::guarded([&] {
    require(vcb::dim_supported(dim), TQ_ERR_INVALID_ARGUMENT,
            "dim must be a positive multiple of 8, <= 16384");
    const vcb::RotationTables t = vcb::make_rotation(dim);
    std::memcpy(signs, t.signs.data(), dim * 4);
    std::memcpy(perm, t.perm.data(), dim * 4);
  });
}

int tq_index_create(size_t dim, size_t bits, uint32_t flags, int device, tq_index** out) {
  return vcb::guarded([&] {
    require(out != nullptr, TQ_ERR_INVALID_ARGUMENT, "out must not be NULL");
    *out = nullptr;
    require(vcb::dim_supported(dim), TQ_ERR_INVALID_ARGUMENT,
            "dim must be a positive multiple of 8, <= 16384");
    require(vcb::bits_supported(bits), TQ_ERR_INVALID_ARGUMENT, "bits must be 2, 3, or 4");
    require(flags == 0, TQ_ERR_INVALID_ARGUMENT, "flags must be 0");
    require(vcb::encode_dim_supported(static_cast<int>(dim)), TQ_ERR_UNSUPPORTED,
            "dim is not supported by the device kernels");
    int count = 0;
    vcb::check(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
    require(device >= 0 && device < count, TQ_ERR_INVALID_ARGUMENT, "no such CUDA device");
    vcb::DeviceGuard g(device);
    auto h = std::make_unique<tq_index>();
    h->device = device;
    vcb::check(cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, device), "attribute");
    vcb::check(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    h->dim = dim;
    h->bits = bits;
    h->nbg = vcb::byte_groups(bits, dim);
    h->block = vcb::wht_block(dim);
    h->inv_sqrt_block = 1.f / std::sqrt(static_cast<float>(h->block));
    h->cb = vcb::codebook(bits, dim);
    const vcb::RotationTables rot = vcb::make_rotation(dim);
    std::vector<uint32_t> ps(dim);
    for (size_t i = 0; i < dim; ++i) ps[i] = rot.perm[i] | (rot.signs[i] < 0.f ? 0x80000000u : 0u);
    std::vector<float> bnd(16, 0.f), cen(16, 0.f);
    std::copy(h->cb.boundaries.begin(), h->cb.boundaries.end(), bnd.begin());
    std::copy(h->cb.centroids.begin(), h->cb.centroids.end(), cen.begin());
    h->d_perm_sign.reserve(dim * 4);
    h->d_bnd.reserve(64);
    h->d_cen.reserve(64);
    h->d_counter.reserve(8);
    h->upload(h->d_perm_sign.get(), ps.data(), dim * 4);
    h->upload(h->d_bnd.get(), bnd.data(), 64);
    h->upload(h->d_cen.get(), cen.data(), 64);
    if (vcb::make_code_grid(h->cb.boundaries, &h->grid)) {
      std::vector<uint32_t> cells(2 * vcb::CodeGrid::kCells);
      for (int j = 0; j < vcb::CodeGrid::kCells; ++j) {
        cells[2 * j] = h->grid.base[j];
        std::memcpy(&cells[2 * j + 1], &h->grid.inner[j], 4);
      }
      h->d_grid.reserve(cells.size() * 4);
      h->upload(h->d_grid.get(), cells.data(), cells.size() * 4);
      h->has_grid = true;
    }
    vcb::check(cudaMemsetAsync(h->d_counter.get(), 0, 8, h->stream), "cudaMemsetAsync");
    h->sync();
    *out = h.release();
  });
}

int tq_index_destroy(tq_index* h) {
  return vcb::guarded([&] {
    if (!h) return;
    vcb::DeviceGuard g(h->device);
    delete h;
  });
}

int tq_index_calibrate(tq_index* h, const float* sample, size_t n) {
  return vcb::guarded([&] {
    require(h && sample, TQ_ERR_INVALID_ARGUMENT, "null argument");
    require(n >= 2, TQ_ERR_INVALID_ARGUMENT, "calibration needs at least 2 rows");
    vcb::DeviceGuard g(h->device);
    vcb::DeviceBuffer d;
    d.reserve(n * h->dim * 4);
    h->upload(d.get(), sample, n * h->dim * 4);
    vcb::calibrate_index(h, d.as<float>(), n, h->stream);
  });
}

int tq_index_calibrate_device(tq_index* h, const float* d_sample, size_t n, void* stream) {
  return vcb::guarded([&] {
    require(h && d_sample, TQ_ERR_INVALID_ARGUMENT, "null argument");
    check_aligned(d_sample, "sample");
    vcb::DeviceGuard g(h->device);
    vcb::calibrate_index(h, d_sample, n, h->pick(stream));
  });
}

int tq_index_add(tq_index* h, const float* vectors, size_t n) {
  return vcb::guarded([&] {
    require(h != nullptr, TQ_ERR_INVALID_ARGUMENT, "null index");
    if (n == 0) return;
    require(vectors != nullptr, TQ_ERR_INVALID_ARGUMENT, "null vectors");
    vcb::DeviceGuard g(h->device);
    vcb::DeviceBuffer d;
    d.reserve(n * h->dim * 4);
    h->upload(d.get(), vectors, n * h->dim * 4);
    do_add_device(h, d.as<float>(), n, h->stream);
    h->sync();
  });
}

int tq_index_add_device(tq_index* h, const float* d_vectors, size_t n, void* stream) {
  return vcb::guarded([&] {
    require(h != nullptr, TQ_ERR_INVALID_ARGUMENT, "null index");
    if (n == 0) return;
    require(d_vectors != nullptr, TQ_ERR_INVALID_ARGUMENT, "null vectors");
    vcb::DeviceGuard g(h->device);
    cudaStream_t s = h->pick(stream);
    if (s != h->stream) vcb::check(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    do_add_device(h, d_vectors, n, s);
    vcb::check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  });
}

int tq_index_prepare(tq_index* h) {
  return vcb::guarded([&] {
    require(h != nullptr, TQ_ERR_INVALID_ARGUMENT, "null index");
    if (h->prepared) return;
    require(h->staged_n > 0, TQ_ERR_STATE, "prepare with empty index");
    vcb::DeviceGuard g(h->device);
    h->encode_append(h->d_staged.as<float>(), h->staged_n, h->stream);
    h->sync();
    h->staged_n = 0;
    h->d_staged.release();
    h->d_flat.release();
    h->prepared = true;
  });
}

int tq_index_search_device(tq_index* h, const float* d_queries, size_t nq, size_t k, float* d_scores,
                           uint64_t* d_ids, size_t* k_eff, void* stream) {
  return vcb::guarded([&] {
    require(h != nullptr, TQ_ERR_INVALID_ARGUMENT, "null index");
    require(h->prepared, TQ_ERR_STATE, "search before prepare");
    require(k <= static_cast<size_t>(vcb::kMaxK), TQ_ERR_UNSUPPORTED, "k must be <= 256");
    const size_t ke = std::min(k, h->n);
    if (k_eff) *k_eff = ke;
    if (nq == 0 || ke == 0) return;
    require(d_queries && d_scores && d_ids, TQ_ERR_INVALID_ARGUMENT, "null buffer");
    check_aligned(d_queries, "queries");
    vcb::DeviceGuard g(h->device);
    h->search_device(d_queries, nq, k, d_scores, d_ids, ke, h->pick(stream));
  });
}

int tq_index_search(tq_index* h, const float* queries, size_t nq, size_t k, float* scores,
                    uint64_t* ids, size_t* k_eff) {
  return vcb::guarded([&] {
    require(h != nullptr, TQ_ERR_INVALID_ARGUMENT, "null index");
    require(h->prepared, TQ_ERR_STATE, "search before prepare");
    require(k <= static_cast<size_t>(vcb::kMaxK), TQ_ERR_UNSUPPORTED, "k must be <= 256");
    const size_t ke = std::min(k, h->n);
    if (k_eff) *k_eff = ke;
    if (nq == 0 || ke == 0) return;
    require(queries && scores && ids, TQ_ERR_INVALID_ARGUMENT, "null buffer");
    vcb::DeviceGuard g(h->device);
    h->d_queries.reserve(nq * h->dim * 4);
    h->d_out_s.reserve(nq * ke * 4);
    h->d_out_i.reserve(nq * ke * 8);
    h->upload(h->d_queries.get(), queries, nq * h->dim * 4);
    h->search_device(h->d_queries.as<float>(), nq, k, h->d_out_s.as<float>(), h->d_out_i.as<uint64_t>(),
                     ke, h->stream);
    vcb::check(cudaMemcpyAsync(scores, h->d_out_s.get(), nq * ke * 4, cudaMemcpyDeviceToHost, h->stream),
               "D2H");
    vcb::check(cudaMemcpyAsync(ids, h->d_out_i.get(), nq * ke * 8, cudaMemcpyDeviceToHost, h->stream), "D2H");
    h->sync();
  });
}

int tq_index_synchronize(tq_index* h) {
  return vcb::guarded([&] {
    require(h != nullptr, TQ_ERR_INVALID_ARGUMENT, "null index");
    vcb::DeviceGuard g(h->device);
    h->sync();
  });
}

int tq_index_info(const tq_index* h, size_t* dim, size_t* bits, size_t* n, int* prepared, int* calibrated) {
  return vcb::guarded([&] {
    require(h != nullptr, TQ_ERR_INVALID_ARGUMENT, "null index");
    if (dim) *dim = h->dim;
    if (bits) *bits = h->bits;
    if (n) *n = h->n + h->staged_n;
    if (prepared) *prepared = h->prepared ? 1 : 0;
    if (calibrated) *calibrated = h->calibrated ? 1 : 0;
  });
}

int tq_index_export_codes_flat(tq_index* h, uint8_t* out) {
  return vcb::guarded([&] {
    require(h && out, TQ_ERR_INVALID_ARGUMENT, "null argument");
    require(h->prepared, TQ_ERR_STATE, "export before prepare");
    vcb::DeviceGuard g(h->device);
    vcb::DeviceBuffer d;
    d.reserve(h->n * h->nbg);
    vcb::check(vcb::launch_export_flat(h->d_codes.as<uint32_t>(), static_cast<long long>(h->n),
                                       static_cast<int>(h->nbg), d.as<uint8_t>(), h->stream),
               "export kernel");
    vcb::check(cudaMemcpyAsync(out, d.get(), h->n * h->nbg, cudaMemcpyDeviceToHost, h->stream), "D2H");
    h->sync();
  });
}

int tq_index_export_packed(tq_index* h, uint8_t* out) {
  return vcb::guarded([&] {
    require(h && out, TQ_ERR_INVALID_ARGUMENT, "null argument");
    std::vector<uint8_t> flat(h->n * h->nbg);
    const int rc = tq_index_export_codes_flat(h, flat.data());
    if (rc != TQ_OK) vcb::fail(rc, vcb::g_last_error);
    flat_to_planes(flat.data(), h->n, h->bits, h->dim, out);
  });
}

int tq_index_export_alpha(tq_index* h, float* out) {
  return vcb::guarded([&] {
    require(h && out, TQ_ERR_INVALID_ARGUMENT, "null argument");
    require(h->prepared, TQ_ERR_STATE, "export before prepare");
    vcb::DeviceGuard g(h->device);
    vcb::check(cudaMemcpyAsync(out, h->d_alpha.get(), h->n * 4, cudaMemcpyDeviceToHost, h->stream), "D2H");
    h->sync();
  });
}

int tq_index_export_calibration(tq_index* h, float* shift, float* scale) {
  return vcb::guarded([&] {
    require(h && shift && scale, TQ_ERR_INVALID_ARGUMENT, "null argument");
    require(h->calibrated, TQ_ERR_STATE, "index is not calibrated");
    std::memcpy(shift, h->shift.data(), h->dim * 4);
    std::memcpy(scale, h->scale.data(), h->dim * 4);
  });
}

int tq_index_prepare_queries(tq_index* h, const float* queries, size_t nq, float* q_rot, float* bias_corr,
                             uint8_t* luts, float* lut_scale, float* lut_bias) {
  return vcb::guarded([&] {
    require(h && queries, TQ_ERR_INVALID_ARGUMENT, "null argument");
    if (nq == 0) return;
    vcb::DeviceGuard g(h->device);
    h->d_queries.reserve(nq * h->dim * 4);
    h->d_qrot.reserve(nq * h->dim * 4);
    h->upload(h->d_queries.get(), queries, nq * h->dim * 4);
    h->prep_queries(h->d_queries.as<float>(), nq, h->stream, h->d_qrot.as<float>());
    const float* qf = h->d_qf.as<float>();
    auto d2h = [&](void* dst, const void* src, size_t bytes) {
      if (dst) vcb::check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, h->stream), "D2H");
    };
    d2h(q_rot, h->d_qrot.get(), nq * h->dim * 4);
    d2h(luts, h->d_luts.get(), nq * h->nbg * 32);
    d2h(lut_scale, qf, nq * 4);
    d2h(lut_bias, qf + nq, nq * 4);
    d2h(bias_corr, qf + 2 * nq, nq * 4);
    h->sync();
  });
}

int tq_index_dense_scores(tq_index* h, const float* queries, size_t nq, uint32_t* int_scores, float* scores) {
  return vcb::guarded([&] {
    require(h && queries, TQ_ERR_INVALID_ARGUMENT, "null argument");
    require(h->prepared, TQ_ERR_STATE, "scores before prepare");
    if (nq == 0 || h->n == 0) return;
    vcb::DeviceGuard g(h->device);
    h->d_queries.reserve(nq * h->dim * 4);
    h->upload(h->d_queries.get(), queries, nq * h->dim * 4);
    h->prep_queries(h->d_queries.as<float>(), nq, h->stream, nullptr);
    vcb::DeviceBuffer di, ds;
    di.reserve(nq * h->n * 4);
    ds.reserve(nq * h->n * 4);
    const float* qf = h->d_qf.as<float>();
    vcb::check(vcb::launch_dense_scores(h->d_codes.as<uint32_t>(), h->d_alpha.as<float>(),
                                        h->d_luts.as<uint8_t>(), qf, qf + 3 * nq, static_cast<long long>(h->n),
                                        static_cast<int>(h->nbg), static_cast<long long>(nq),
                                        di.as<uint32_t>(), ds.as<float>(), h->stream),
               "dense scores kernel");
    if (int_scores) {
      vcb::check(cudaMemcpyAsync(int_scores, di.get(), nq * h->n * 4, cudaMemcpyDeviceToHost, h->stream), "D2H");
    }
    if (scores) {
      vcb::check(cudaMemcpyAsync(scores, ds.get(), nq * h->n * 4, cudaMemcpyDeviceToHost, h->stream), "D2H");
    }
    h->sync();
  });
}

int tq_index_replay_count(const tq_index* h, uint64_t* count) {
  return vcb::guarded([&] {
    require(h && count, TQ_ERR_INVALID_ARGUMENT, "null argument");
    vcb::DeviceGuard g(h->device);
    unsigned long long c = 0;
    vcb::check(cudaMemcpy(&c, h->d_counter.get(), 8, cudaMemcpyDeviceToHost), "D2H");
    *count = c;
  });
}

int tq_index_scan_plan(const tq_index* h, size_t nq, size_t k, int* q_per_cta, int* n_ranges,
                       uint64_t* range_vectors, int* split_batches, int* stages) {
  return vcb::guarded([&] {
    require(h != nullptr, TQ_ERR_INVALID_ARGUMENT, "null index");
    require(h->prepared, TQ_ERR_STATE, "scan plan before prepare");
    require(k >= 1 && k <= static_cast<size_t>(vcb::kMaxK), TQ_ERR_UNSUPPORTED, "k must be in [1, 256]");
    require(nq >= 1, TQ_ERR_INVALID_ARGUMENT, "nq must be >= 1");
    // search_device plans each pass of at most 65,536 queries.
    const size_t m = std::min<size_t>(nq, size_t{1} << 16);
    vcb::ScanPlan plan;
    if (!vcb::plan_scan(static_cast<long long>(h->n), static_cast<long long>(m), static_cast<int>(h->nbg),
                        static_cast<int>(std::min(k, h->n)), h->sms, &plan, 0, static_cast<int>(h->bits))) {
      vcb::fail(TQ_ERR_UNSUPPORTED, "no scan configuration fits shared memory for this dim / k");
    }
    if (q_per_cta) *q_per_cta = plan.q_per_cta;
    if (n_ranges) *n_ranges = plan.n_ranges;
    if (range_vectors) *range_vectors = static_cast<uint64_t>(plan.range_vectors);
    if (split_batches) *split_batches = std::max(1, plan.split_batches);
    if (stages) *stages = plan.stages;
  });
}

int tq_scan_plan_shape(uint64_t n, size_t nq, size_t dim, size_t bits, size_t k, int sms, int* q_per_cta,
                       int* n_ranges, uint64_t* range_vectors, int* split_batches, int* stages,
                       int* split_ctas_per_sm) {
  return vcb::guarded([&] {
    require(n >= 1 && nq >= 1, TQ_ERR_INVALID_ARGUMENT, "n and nq must be >= 1");
    require(dim >= 8 && dim <= 16384 && dim % 8 == 0, TQ_ERR_INVALID_ARGUMENT,
            "dim must be a positive multiple of 8, at most 16384");
    require(bits >= 2 && bits <= 4, TQ_ERR_INVALID_ARGUMENT, "bits must be 2, 3 or 4");
    require(k >= 1 && k <= static_cast<size_t>(vcb::kMaxK), TQ_ERR_UNSUPPORTED, "k must be in [1, 256]");
    require(sms >= 1, TQ_ERR_INVALID_ARGUMENT, "sms must be >= 1");
    const size_t nbg = dim / (8 / bits);  // byte groups: dim / 2 at 3 and 4 bits, dim / 4 at 2 bits
    // search_device plans each pass of at most 65,536 queries.
    const size_t m = std::min<size_t>(nq, size_t{1} << 16);
    vcb::ScanPlan plan;
    if (!vcb::plan_scan(static_cast<long long>(n), static_cast<long long>(m), static_cast<int>(nbg),
                        static_cast<int>(std::min<uint64_t>(k, n)), sms, &plan, 0, static_cast<int>(bits))) {
      vcb::fail(TQ_ERR_UNSUPPORTED, "no scan configuration fits shared memory for this dim / k");
    }
    if (q_per_cta) *q_per_cta = plan.q_per_cta;
    if (n_ranges) *n_ranges = plan.n_ranges;
    if (range_vectors) *range_vectors = static_cast<uint64_t>(plan.range_vectors);
    if (split_batches) *split_batches = std::max(1, plan.split_batches);
    if (stages) *stages = plan.stages;
    if (split_ctas_per_sm) *split_ctas_per_sm = plan.split_batches > 1 ? plan.split_ctas_per_sm : 0;
  });
}

}  // extern "C"

extern "C" {

int tq_index_get_stream(tq_index* h, void** stream) {
  return vcb::guarded([&] {
    require(h && stream, TQ_ERR_INVALID_ARGUMENT, "null argument");
    *stream = static_cast<void*>(h->stream);
  });
}

int tq_index_set_profiling(tq_index* h, int enabled) {
  return vcb::guarded([&] {
    require(h != nullptr, TQ_ERR_INVALID_ARGUMENT, "null index");
    h->profiling = enabled != 0;
  });
}

int tq_index_read_profile(tq_index* h, tq_profile* out) {
  return vcb::guarded([&] {
    require(h && out, TQ_ERR_INVALID_ARGUMENT, "null argument");
    vcb::DeviceGuard g(h->device);
    tq_profile p{};
    double* ms[4] = {&p.prep_ms, &p.scan_ms, &p.merge_ms, &p.encode_ms};
    h->last_by_name.clear();
    for (auto& t : h->timed_launches) {
      vcb::check(cudaEventSynchronize(t.stop), "cudaEventSynchronize");
      float e = 0.f;
      vcb::check(cudaEventElapsedTime(&e, t.start, t.stop), "cudaEventElapsedTime");
      *ms[t.kind] += e;
      auto named = std::find_if(h->last_by_name.begin(), h->last_by_name.end(),
                                [&](const tq_index::NamedTime& n) { return n.what == t.what; });
      if (named == h->last_by_name.end()) {
        h->last_by_name.push_back({t.what, 0.0, 0});
        named = h->last_by_name.end() - 1;
      }
      named->ms += e;
      ++named->launches;
      h->event_pool.push_back(t.start);
      h->event_pool.push_back(t.stop);
    }
    h->timed_launches.clear();
    p.prep_launches = h->launches[tq_index::kPrep];
    p.scan_launches = h->launches[tq_index::kScan];
    p.merge_launches = h->launches[tq_index::kMerge];
    p.encode_launches = h->launches[tq_index::kEncode];
    p.scan_stream_bytes = h->scan_stream_bytes;
    p.scan_queries = h->scan_queries;
    for (auto& c : h->launches) c = 0;
    h->scan_stream_bytes = 0;
    h->scan_queries = 0;
    *out = p;
  });
}

int tq_index_profile_entries(const tq_index* h, size_t* n) {
  return vcb::guarded([&] {
    require(h && n, TQ_ERR_INVALID_ARGUMENT, "null argument");
    *n = h->last_by_name.size();
  });
}

int tq_index_profile_entry(const tq_index* h, size_t i, char* name, size_t name_cap, double* ms,
                           uint64_t* launches) {
  return vcb::guarded([&] {
    require(h && name && ms && launches && name_cap > 0, TQ_ERR_INVALID_ARGUMENT, "null argument");
    require(i < h->last_by_name.size(), TQ_ERR_INVALID_ARGUMENT, "profile entry out of range");
    const auto& e = h->last_by_name[i];
    const size_t len = std::min(e.what.size(), name_cap - 1);
    std::memcpy(name, e.what.data(), len);
    name[len] = '\0';
    *ms = e.ms;
    *launches = e.launches;
  });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Search without device allocation (tq_index_search_device_noalloc).
//
// Callers that may not allocate device memory while serving (a server that
// reserved all free HBM for its own pool, a loop that cannot take cudaMalloc's
// implicit synchronization) get the same search with its temporaries placed in
// one fixed array compiled into the library. Every GPU that loads the library
// holds this array until the process exits.
namespace {

constexpr size_t kNoAllocScratchBytes = size_t{16} << 20;  // 16 MiB
constexpr int kNoAllocMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_addr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_scratch on `device` (which must be current).
// In host code the symbol's name is only a host-side handle, so the address is
// looked up once per device and cached.
unsigned char* noalloc_scratch(int device) {
  if (device < 0 || device >= kNoAllocMaxDevices) {
    vcb::fail(TQ_ERR_UNSUPPORTED, "device ordinal out of range for the no-alloc scratch table");
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (g_noalloc_addr[device] == nullptr) {
    void* p = nullptr;
    vcb::check(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(no-alloc scratch)");
    g_noalloc_addr[device] = p;
  }
  return static_cast<unsigned char*>(g_noalloc_addr[device]);
}

size_t align256(size_t v) { return (v + 255) / 256 * 256; }

}  // namespace

extern "C" int tq_index_search_device_noalloc(tq_index* h, const float* d_queries, size_t nq, size_t k,
                                              float* d_scores, uint64_t* d_ids, size_t* k_eff,
                                              void* stream) {
  return vcb::guarded([&] {
    require(h != nullptr, TQ_ERR_INVALID_ARGUMENT, "null index");
    require(h->prepared, TQ_ERR_STATE, "search before prepare");
    require(k <= static_cast<size_t>(vcb::kMaxK), TQ_ERR_UNSUPPORTED, "k must be <= 256");
    const size_t ke = std::min(k, h->n);
    if (k_eff) *k_eff = ke;
    if (nq == 0 || ke == 0) return;
    require(d_queries && d_scores && d_ids, TQ_ERR_INVALID_ARGUMENT, "null buffer");
    check_aligned(d_queries, "queries");

    // Carve the fixed array: LUTs, per-query constants, candidate lists. The
    // query count is bounded first so that the byte counts below cannot wrap.
    if (nq > kNoAllocScratchBytes / (h->nbg * 32)) {
      vcb::fail(TQ_ERR_INVALID_ARGUMENT,
                "request of " + std::to_string(nq) + " queries does not fit the no-alloc scratch (" +
                    std::to_string(kNoAllocScratchBytes) + " bytes; at most " +
                    std::to_string(kNoAllocScratchBytes / (h->nbg * 32)) + " queries of LUTs at this dim)");
    }
    const size_t lut_bytes = align256(nq * h->nbg * 32);
    const size_t qf_bytes = align256(nq * 4 * sizeof(float));
    const size_t per_list = nq * ke * (sizeof(float) + sizeof(uint32_t));
    if (lut_bytes + qf_bytes + 8 * per_list > kNoAllocScratchBytes) {
      vcb::fail(TQ_ERR_INVALID_ARGUMENT,
                "request needs " + std::to_string(lut_bytes + qf_bytes + 8 * per_list) +
                    " bytes of no-alloc scratch; the fixed array holds " +
                    std::to_string(kNoAllocScratchBytes) + " bytes (search fewer queries per call)");
    }
    vcb::ScanPlan plan;
    if (!vcb::plan_scan(static_cast<long long>(h->n), static_cast<long long>(nq), static_cast<int>(h->nbg),
                        static_cast<int>(ke), h->sms, &plan, 0, static_cast<int>(h->bits))) {
      vcb::fail(TQ_ERR_UNSUPPORTED, "no scan configuration fits shared memory for this dim / k");
    }
    // Fewer vector ranges if their candidate lists would not fit.
    const size_t max_lists = (kNoAllocScratchBytes - lut_bytes - qf_bytes) / per_list;
    const size_t per_range = static_cast<size_t>(plan.lists_per_range);
    if (static_cast<size_t>(plan.n_ranges) * per_range > max_lists) {
      const long long blocks = (static_cast<long long>(h->n) + vcb::kScanBlockVectors - 1) / vcb::kScanBlockVectors;
      long long ranges = static_cast<long long>(max_lists / per_range);
      const long long blocks_each = (blocks + ranges - 1) / ranges;
      ranges = (blocks + blocks_each - 1) / blocks_each;
      plan.n_ranges = static_cast<int>(ranges);
      plan.range_vectors = blocks_each * vcb::kScanBlockVectors;
    }
    const size_t lists = static_cast<size_t>(plan.n_ranges) * per_range;

    vcb::DeviceGuard g(h->device);
    unsigned char* base = noalloc_scratch(h->device);
    uint8_t* luts = base;
    float* qf = reinterpret_cast<float*>(base + lut_bytes);
    float* cand_s = reinterpret_cast<float*>(base + lut_bytes + qf_bytes);
    uint32_t* cand_i = reinterpret_cast<uint32_t*>(cand_s + nq * lists * ke);
    cudaStream_t s = h->pick(stream);

    vcb::QueryPrepArgs p{};
    p.q = d_queries;
    p.nq = static_cast<long long>(nq);
    p.dim = static_cast<int>(h->dim);
    p.bits = static_cast<int>(h->bits);
    p.block = static_cast<int>(h->block);
    p.nbg = static_cast<int>(h->nbg);
    p.inv_sqrt_block = h->inv_sqrt_block;
    p.perm_sign = h->d_perm_sign.as<uint32_t>();
    p.centroids = h->d_cen.as<float>();
    p.tqplus = h->calibrated;
    p.shift = h->d_shift.as<float>();
    p.scale = h->d_scale.as<float>();
    p.luts = luts;
    p.lut_scale = qf;
    p.lut_bias = qf + nq;
    p.bias_corr = qf + 2 * nq;
    p.fa_init = qf + 3 * nq;
    p.q_rot = nullptr;
    p.replay_count = h->d_counter.as<unsigned long long>();
    h->launch(tq_index::kPrep, s, "query prep kernel", [&] { return vcb::launch_query_prep(p, h->sms, s); });

    vcb::ScanArgs a{};
    a.codes = h->d_codes.as<uint32_t>();
    a.alpha = h->d_alpha.as<float>();
    a.luts = luts;
    a.lut_scale = qf;
    a.fa_init = qf + 3 * nq;
    a.n = static_cast<long long>(h->n);
    a.nbg = static_cast<int>(h->nbg);
    a.nq = static_cast<long long>(nq);
    a.k = static_cast<int>(ke);
    a.q_per_cta = plan.q_per_cta;
    a.range_vectors = plan.range_vectors;
    a.n_ranges = plan.n_ranges;
    a.lut_chunk_groups = plan.lut_chunk_groups;
    a.bits = static_cast<int>(h->bits);
    a.cand_score = cand_s;
    a.cand_id = cand_i;
    h->launch(tq_index::kScan, s, "scan kernel", [&] { return vcb::launch_scan(a, plan, s); });
    h->scan_stream_bytes += static_cast<uint64_t>((nq + plan.q_per_cta - 1) / plan.q_per_cta) * h->n * (h->nbg + 4);
    h->scan_queries += nq;

    vcb::MergeArgs m{};
    m.cand_score = cand_s;
    m.cand_id = cand_i;
    m.nq = static_cast<long long>(nq);
    m.n_lists = static_cast<int>(lists);
    m.k = static_cast<int>(ke);
    m.k_out = static_cast<int>(ke);
    m.out_score = d_scores;
    m.out_id = d_ids;
    h->launch(tq_index::kMerge, s, "merge kernel", [&] { return vcb::launch_merge(m, s); });
  });
}

// ---------------------------------------------------------------------------
// Index persistence (the reference has none). File layout, little-endian:
//   "VCBTQIX1", u32 version = 1, u32 dim, u32 bits, u32 flags (bit 0: TQ+),
//   u64 n, [f32 shift[dim], f32 scale[dim] when TQ+], u8 codes_flat[n * nbg],
//   f32 alpha[n], u64 FNV-1a of every byte after the magic.
namespace {

constexpr char kIndexMagic[8] = {'V', 'C', 'B', 'T', 'Q', 'I', 'X', '1'};

struct Fnv1a {
  uint64_t h = 1469598103934665603ull;
  void add(const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
  }
};

}  // namespace

extern "C" int tq_index_save(tq_index* h, const char* path) {
  return vcb::guarded([&] {
    require(h && path, TQ_ERR_INVALID_ARGUMENT, "null argument");
    require(h->prepared, TQ_ERR_STATE, "save before prepare");
    std::vector<uint8_t> flat(h->n * h->nbg);
    std::vector<float> alpha(h->n);
    if (h->n) {
      int rc = tq_index_export_codes_flat(h, flat.data());
      if (rc != TQ_OK) vcb::fail(rc, vcb::g_last_error);
      rc = tq_index_export_alpha(h, alpha.data());
      if (rc != TQ_OK) vcb::fail(rc, vcb::g_last_error);
    }
    const std::string tmp = std::string(path) + ".tmp";
    FILE* f = std::fopen(tmp.c_str(), "wb");
    require(f != nullptr, TQ_ERR_INVALID_ARGUMENT, "cannot create index file");
    Fnv1a sum;
    bool ok = std::fwrite(kIndexMagic, 1, 8, f) == 8;
    auto put = [&](const void* p, size_t n) {
      if (n == 0 || !ok) return;
      ok = std::fwrite(p, 1, n, f) == n;
      sum.add(p, n);
    };
    const uint32_t hdr[4] = {1u, static_cast<uint32_t>(h->dim), static_cast<uint32_t>(h->bits),
                             h->calibrated ? 1u : 0u};
    const uint64_t n64 = h->n;
    put(hdr, sizeof(hdr));
    put(&n64, sizeof(n64));
    if (h->calibrated) {
      put(h->shift.data(), h->dim * 4);
      put(h->scale.data(), h->dim * 4);
    }
    put(flat.data(), flat.size());
    put(alpha.data(), alpha.size() * 4);
    if (ok) ok = std::fwrite(&sum.h, 1, 8, f) == 8;
    ok = (std::fclose(f) == 0) && ok;
    require(ok, TQ_ERR_INVALID_ARGUMENT, "write failed");
    require(std::rename(tmp.c_str(), path) == 0, TQ_ERR_INVALID_ARGUMENT, "rename failed");
  });
}

extern "C" int tq_index_load(const char* path, int device, tq_index** out) {
  return vcb::guarded([&] {
    require(path && out, TQ_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    FILE* f = std::fopen(path, "rb");
    require(f != nullptr, TQ_ERR_INVALID_ARGUMENT, "cannot open index file");
    struct Closer {
      FILE* f;
      ~Closer() { std::fclose(f); }
    } closer{f};
    Fnv1a sum;
    auto get = [&](void* p, size_t n) {
      if (n == 0) return;
      require(std::fread(p, 1, n, f) == n, TQ_ERR_INVALID_ARGUMENT, "truncated index file");
      sum.add(p, n);
    };
    char magic[8];
    require(std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kIndexMagic, 8) == 0, TQ_ERR_INVALID_ARGUMENT,
            "not a vectorcache_b200 index file");
    uint32_t hdr[4];
    uint64_t n64 = 0;
    get(hdr, sizeof(hdr));
    require(hdr[0] == 1u, TQ_ERR_INVALID_ARGUMENT, "unsupported index file version");
    get(&n64, sizeof(n64));
    const size_t dim = hdr[1], bits = hdr[2];
    require(vcb::dim_supported(dim) && vcb::bits_supported(bits), TQ_ERR_INVALID_ARGUMENT, "corrupt index header");
    const size_t nbg = vcb::byte_groups(bits, dim);
    std::vector<float> shift, scale;
    if (hdr[3] & 1u) {
      shift.resize(dim);
      scale.resize(dim);
      get(shift.data(), dim * 4);
      get(scale.data(), dim * 4);
    }
    std::vector<uint8_t> flat(static_cast<size_t>(n64) * nbg);
    std::vector<float> alpha(static_cast<size_t>(n64));
    get(flat.data(), flat.size());
    get(alpha.data(), alpha.size() * 4);
    uint64_t stored = 0;
    require(std::fread(&stored, 1, 8, f) == 8, TQ_ERR_INVALID_ARGUMENT, "truncated index file");
    require(stored == sum.h, TQ_ERR_INVALID_ARGUMENT, "index file checksum mismatch");

    tq_index* raw = nullptr;
    int rc = tq_index_create(dim, bits, 0, device, &raw);
    if (rc != TQ_OK) vcb::fail(rc, vcb::g_last_error);
    std::unique_ptr<tq_index, int (*)(tq_index*)> h(raw, tq_index_destroy);
    vcb::DeviceGuard g(device);
    if (!shift.empty()) {
      h->shift = shift;
      h->scale = scale;
      std::vector<float> inv(dim);
      for (size_t d = 0; d < dim; ++d) inv[d] = 1.f / scale[d];
      h->d_shift.reserve(dim * 4);
      h->d_scale.reserve(dim * 4);
      h->d_inv_scale.reserve(dim * 4);
      h->upload(h->d_shift.get(), shift.data(), dim * 4);
      h->upload(h->d_scale.get(), scale.data(), dim * 4);
      h->upload(h->d_inv_scale.get(), inv.data(), dim * 4);
      h->calibrated = true;
    }
    const size_t n = static_cast<size_t>(n64);
    if (n > 0) {
      h->ensure_capacity(n);
      const size_t stride = h->flat_stride();
      std::vector<uint8_t> padded(n * stride, 0);
      for (size_t v = 0; v < n; ++v) std::memcpy(padded.data() + v * stride, flat.data() + v * nbg, nbg);
      h->d_flat.reserve(padded.size());
      h->upload(h->d_flat.get(), padded.data(), padded.size());
      h->upload(h->d_alpha.get(), alpha.data(), n * 4);
      vcb::RelayoutArgs r{};
      r.flat = h->d_flat.as<uint8_t>();
      r.src_first = 0;
      r.src_n = static_cast<long long>(n);
      r.flat_stride = static_cast<int>(stride);
      r.keep_below = 0;
      r.n_total = static_cast<long long>(n);
      r.nbg = static_cast<int>(nbg);
      r.bits = static_cast<int>(bits);
      r.codes = h->d_codes.as<uint32_t>();
      vcb::check(vcb::launch_relayout(r, h->stream), "relayout kernel");
      h->sync();
      h->d_flat.release();
      h->n = n;
    }
    h->prepared = true;
    *out = h.release();
  });
}

// Append the rows of a float32 .npy matrix (rows, dim), streamed in chunks
// (the reference's NpyReader::copy_rows_into, src/datasets/npy.cpp).
extern "C" int tq_npy_f32_info(const char* path, size_t* rows, size_t* cols);
extern "C" int tq_npy_f32_read(const char* path, size_t row0, size_t nrows, float* out);

extern "C" int tq_index_add_npy(tq_index* h, const char* path) {
  return vcb::guarded([&] {
    require(h && path, TQ_ERR_INVALID_ARGUMENT, "null argument");
    size_t rows = 0, cols = 0;
    int rc = tq_npy_f32_info(path, &rows, &cols);
    if (rc != TQ_OK) vcb::fail(rc, vcb::g_last_error);
    require(cols == h->dim, TQ_ERR_INVALID_ARGUMENT, ".npy column count differs from the index dim");
    const size_t chunk = std::max<size_t>(1, (size_t{256} << 20) / (cols * 4));
    std::vector<float> buf(std::min(rows, chunk) * cols);
    for (size_t r0 = 0; r0 < rows; r0 += chunk) {
      const size_t m = std::min(chunk, rows - r0);
      rc = tq_npy_f32_read(path, r0, m, buf.data());
      if (rc != TQ_OK) vcb::fail(rc, vcb::g_last_error);
      rc = tq_index_add(h, buf.data(), m);
      if (rc != TQ_OK) vcb::fail(rc, vcb::g_last_error);
    }
  });
}

// ---------------------------------------------------------------------------
// Exact float re-rank of a top-k (float_rescore_topk, src/search/float_rescore.cpp:80-164).
extern "C" int tq_rescore_device(const float* d_queries, size_t nq, size_t dim, const float* d_corpus,
                                 size_t n_corpus, size_t k, float* d_scores, uint64_t* d_ids, void* stream) {
  return vcb::guarded([&] {
    if (nq == 0 || k == 0 || dim == 0) return;
    require(d_queries && d_scores && d_ids, TQ_ERR_INVALID_ARGUMENT, "null buffer");
    require(n_corpus == 0 || d_corpus != nullptr, TQ_ERR_INVALID_ARGUMENT, "null corpus");
    require(k <= 4096, TQ_ERR_UNSUPPORTED, "rescore k must be <= 4096");
    vcb::check(vcb::launch_rescore(d_queries, static_cast<long long>(nq), static_cast<int>(dim), d_corpus,
                                   static_cast<long long>(n_corpus), static_cast<int>(k), d_scores, d_ids,
                                   static_cast<cudaStream_t>(stream)),
               "rescore kernel");
  });
}

extern "C" int tq_rescore(const float* queries, size_t nq, size_t dim, const float* corpus, size_t n_corpus,
                          size_t k, float* scores, uint64_t* ids, int device) {
  return vcb::guarded([&] {
    if (nq == 0 || k == 0 || dim == 0) return;
    require(queries && scores && ids, TQ_ERR_INVALID_ARGUMENT, "null buffer");
    require(n_corpus == 0 || corpus != nullptr, TQ_ERR_INVALID_ARGUMENT, "null corpus");
    require(k <= 4096, TQ_ERR_UNSUPPORTED, "rescore k must be <= 4096");
    vcb::DeviceGuard g(device);
    cudaStream_t s = nullptr;
    vcb::check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
    struct StreamGuard {
      cudaStream_t s;
      ~StreamGuard() { cudaStreamDestroy(s); }
    } sg{s};
    vcb::DeviceBuffer dq, dc, ds, di;
    dq.reserve(nq * dim * 4);
    dc.reserve(std::max<size_t>(n_corpus, 1) * dim * 4);
    ds.reserve(nq * k * 4);
    di.reserve(nq * k * 8);
    vcb::check(cudaMemcpyAsync(dq.get(), queries, nq * dim * 4, cudaMemcpyHostToDevice, s), "H2D");
    if (n_corpus) vcb::check(cudaMemcpyAsync(dc.get(), corpus, n_corpus * dim * 4, cudaMemcpyHostToDevice, s), "H2D");
    vcb::check(cudaMemcpyAsync(di.get(), ids, nq * k * 8, cudaMemcpyHostToDevice, s), "H2D");
    vcb::check(vcb::launch_rescore(dq.as<float>(), static_cast<long long>(nq), static_cast<int>(dim), dc.as<float>(),
                                   static_cast<long long>(n_corpus), static_cast<int>(k), ds.as<float>(),
                                   di.as<uint64_t>(), s),
               "rescore kernel");
    vcb::check(cudaMemcpyAsync(scores, ds.get(), nq * k * 4, cudaMemcpyDeviceToHost, s), "D2H");
    vcb::check(cudaMemcpyAsync(ids, di.get(), nq * k * 8, cudaMemcpyDeviceToHost, s), "D2H");
    vcb::check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  });
}
