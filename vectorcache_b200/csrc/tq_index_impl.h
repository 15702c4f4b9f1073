// The flat TurboQuant index object shared by the C ABI translation units:
// tq_index.cu (flat index entry points) and tq_bucketed.cu, which uses one
// flat index as its encoder and query-LUT engine over bucket-ordered slots.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/vectorcache_b200.h"
#include "tq_abi.h"
#include "tq_host_math.h"
#include "tq_kernels.h"

namespace vcb {

inline void check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  const int code = (e == cudaErrorMemoryAllocation) ? TQ_ERR_OUT_OF_MEMORY : TQ_ERR_CUDA;
  throw Error(code, std::string(what) + ": " + cudaGetErrorString(e));
}

// Sizing pass of a search (serving admission): while set on the calling
// thread, tq_index::launch and the other device calls of the search paths do
// nothing, and scratch buffers bound to a measuring arena only count bytes.
bool& dry_run_flag();

// A region of device memory that scratch buffers bound to it draw from in
// order (bump allocation; a buffer that grows abandons its old piece). In
// measure mode it hands out placeholder addresses that nothing dereferences
// and only counts the bytes, so a dry run of a search through the same host
// code yields exactly the region size the real run needs.
struct ScratchArena {
  static constexpr size_t kAlign = 256;
  unsigned char* base = nullptr;
  size_t size = 0, used = 0;
  bool measure = false;

  static size_t piece(size_t bytes) { return (std::max<size_t>(bytes, 16) + kAlign - 1) / kAlign * kAlign; }
  void* take(size_t bytes) {
    const size_t b = piece(bytes);
    if (!measure && used + b > size) {
      throw Error(TQ_ERR_OUT_OF_MEMORY, "serving scratch region exhausted (" + std::to_string(used + b) +
                                            " of " + std::to_string(size) + " bytes)");
    }
    void* p = measure ? reinterpret_cast<void*>(kPlaceholder + used) : static_cast<void*>(base + used);
    used += b;
    return p;
  }
  void reset(unsigned char* b, size_t n, bool m) {
    base = b;
    size = n;
    used = 0;
    measure = m;
  }

 private:
  static constexpr uintptr_t kPlaceholder = uintptr_t{1} << 44;
};

// Grow-only device allocation: cudaMalloc, or a piece of a bound ScratchArena.
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  ~DeviceBuffer() { release(); }

  void* reserve(size_t bytes) {
    if (bytes <= bytes_ && ptr_) return ptr_;
    release();
    if (bytes == 0) bytes = 16;
    if (arena_) {
      ptr_ = arena_->take(bytes);
    } else {
      check(cudaMalloc(&ptr_, bytes), "cudaMalloc");
    }
    bytes_ = bytes;
    return ptr_;
  }
  void release() {
    if (ptr_ && !arena_) cudaFree(ptr_);
    ptr_ = nullptr;
    bytes_ = 0;
  }
  // Later reserves draw from `a` (nullptr: cudaMalloc again); drops the current storage.
  void bind(ScratchArena* a) {
    release();
    arena_ = a;
  }
  void swap(DeviceBuffer& o) noexcept {
    std::swap(ptr_, o.ptr_);
    std::swap(bytes_, o.bytes_);
    std::swap(arena_, o.arena_);
  }
  void* get() const { return ptr_; }
  size_t bytes() const { return bytes_; }
  template <typename T>
  T* as() const {
    return static_cast<T*>(ptr_);
  }

 private:
  void* ptr_ = nullptr;
  size_t bytes_ = 0;
  ScratchArena* arena_ = nullptr;
};

class DeviceGuard {
 public:
  explicit DeviceGuard(int device) {
    check(cudaGetDevice(&prev_), "cudaGetDevice");
    if (prev_ != device) check(cudaSetDevice(device), "cudaSetDevice");
    restore_ = prev_ != device;
  }
  ~DeviceGuard() {
    if (restore_) cudaSetDevice(prev_);
  }

 private:
  int prev_ = 0;
  bool restore_ = false;
};

inline size_t round_up(size_t v, size_t m) { return (v + m - 1) / m * m; }

// Device scratch of one flat search: query LUTs, per-query constants and
// candidate lists, and (optional) the batch-split scan's integer sums. Grown
// on demand by the search.
struct FlatScratch {
  DeviceBuffer* luts;
  DeviceBuffer* qf;
  DeviceBuffer* cand_s;
  DeviceBuffer* cand_i;
  DeviceBuffer* partial = nullptr;  // nullptr: the scan does not split
  long long range_cap = 0;          // > 0: at most this many vectors per scan CTA
};

// Owning variant for callers that run searches concurrently (one per stream).
struct FlatScratchStore {
  DeviceBuffer luts, qf, cand_s, cand_i, partial;
  long long range_cap = 0;  // see FlatScratch::range_cap
  FlatScratch ref() { return {&luts, &qf, &cand_s, &cand_i, &partial, range_cap}; }
  void bind(ScratchArena* a) {
    for (DeviceBuffer* b : {&luts, &qf, &cand_s, &cand_i, &partial}) b->bind(a);
  }
};

}  // namespace vcb

struct tq_index;

namespace vcb {
// TQ+ fit (encode.cpp:242-286, 327-335) from n device rows; defined in tq_index.cu.
void calibrate_index(tq_index* h, const float* d_sample, size_t n, cudaStream_t s);
}  // namespace vcb

struct tq_index {
  int device = 0;
  int sms = 148;
  cudaStream_t stream = nullptr;
  size_t dim = 0, bits = 0, nbg = 0, block = 0;
  float inv_sqrt_block = 0.f;
  vcb::Codebook cb;
  vcb::CodeGrid grid;     // the codebook's code grid (encode), when has_grid
  bool has_grid = false;
  bool calibrated = false;
  std::vector<float> shift, scale;
  bool prepared = false;
  size_t n = 0;          // encoded vectors
  size_t staged_n = 0;   // rows waiting for prepare()
  size_t cap = 0;        // layout capacity in vectors (multiple of kScanBlockVectors)

  vcb::DeviceBuffer d_perm_sign, d_bnd, d_cen, d_grid, d_shift, d_scale, d_inv_scale;
  vcb::DeviceBuffer d_codes, d_alpha, d_staged, d_flat, d_counter;
  // search scratch
  vcb::DeviceBuffer d_queries, d_luts, d_qf, d_cand_s, d_cand_i, d_out_s, d_out_i, d_qrot, d_partial;

  // Optional per-launch timing (tq_index_set_profiling).
  enum Kind { kPrep = 0, kScan = 1, kMerge = 2, kEncode = 3 };
  struct Timed {
    int kind;
    const char* what;  // a string literal naming the launch
    cudaEvent_t start, stop;
  };
  struct NamedTime {
    std::string what;
    double ms;
    uint64_t launches;
  };
  bool profiling = false;
  std::vector<cudaEvent_t> event_pool;
  std::vector<Timed> timed_launches;
  std::vector<NamedTime> last_by_name;  // per launch name, as of the last read
  uint64_t launches[4] = {0, 0, 0, 0};
  uint64_t scan_stream_bytes = 0, scan_queries = 0;

  ~tq_index() {
    if (stream) {
      cudaStreamSynchronize(stream);
      cudaStreamDestroy(stream);
    }
    for (auto& t : timed_launches) {
      cudaEventDestroy(t.start);
      cudaEventDestroy(t.stop);
    }
    for (auto e : event_pool) cudaEventDestroy(e);
  }

  cudaEvent_t take_event() {
    if (!event_pool.empty()) {
      cudaEvent_t e = event_pool.back();
      event_pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    vcb::check(cudaEventCreate(&e), "cudaEventCreate");
    return e;
  }

  // Runs one kernel launch, bracketed by events when profiling is on; a
  // sizing pass (vcb::dry_run_flag) launches nothing.
  template <typename F>
  void launch(int kind, cudaStream_t s, const char* what, F&& fn) {
    if (vcb::dry_run_flag()) return;
    ++launches[kind];
    if (!profiling) {
      vcb::check(fn(), what);
      return;
    }
    Timed t{kind, what, take_event(), take_event()};
    vcb::check(cudaEventRecord(t.start, s), "cudaEventRecord");
    vcb::check(fn(), what);
    vcb::check(cudaEventRecord(t.stop, s), "cudaEventRecord");
    timed_launches.push_back(t);
  }

  void sync() { vcb::check(cudaStreamSynchronize(stream), "cudaStreamSynchronize"); }

  cudaStream_t pick(void* s) const { return s ? static_cast<cudaStream_t>(s) : stream; }

  size_t flat_stride() const { return vcb::round_up(nbg, 32); }

  void upload(void* dst, const void* src, size_t bytes) {
    vcb::check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream), "cudaMemcpyAsync H2D");
  }

  // Grow the scan layout and alpha buffers to hold `want` vectors.
  void ensure_capacity(size_t want) {
    if (want <= cap) return;
    size_t new_cap = std::max(want, cap + cap / 2);
    new_cap = vcb::round_up(new_cap, vcb::kScanBlockVectors);
    const size_t code_bytes = (new_cap / vcb::kTileVectors) * nbg * vcb::kTileWords * 4;
    vcb::DeviceBuffer codes, alpha;
    codes.reserve(code_bytes);
    alpha.reserve(new_cap * 4);
    vcb::check(cudaMemsetAsync(codes.get(), 0, code_bytes, stream), "cudaMemsetAsync");
    vcb::check(cudaMemsetAsync(alpha.get(), 0, new_cap * 4, stream), "cudaMemsetAsync");
    if (cap > 0) {
      // Tiles are self-contained, so the old layout is a prefix of the new one.
      const size_t old_code_bytes = (cap / vcb::kTileVectors) * nbg * vcb::kTileWords * 4;
      vcb::check(cudaMemcpyAsync(codes.get(), d_codes.get(), old_code_bytes, cudaMemcpyDeviceToDevice, stream),
                 "cudaMemcpyAsync D2D");
      vcb::check(cudaMemcpyAsync(alpha.get(), d_alpha.get(), cap * 4, cudaMemcpyDeviceToDevice, stream),
                 "cudaMemcpyAsync D2D");
    }
    sync();
    codes.swap(d_codes);
    alpha.swap(d_alpha);
    cap = new_cap;
  }

  // Encode `count` rows at device pointer x and append them after the current n.
  void encode_append(const float* x, size_t count, cudaStream_t s) {
    if (count == 0) return;
    ensure_capacity(n + count);
    const size_t stride = flat_stride();
    const size_t chunk = std::max<size_t>(1, std::min<size_t>(count, (size_t{512} << 20) / stride));
    d_flat.reserve(chunk * stride);
    for (size_t done = 0; done < count; done += chunk) {
      const size_t m = std::min(chunk, count - done);
      vcb::EncodeArgs a{};
      a.x = x + done * dim;
      a.n = static_cast<long long>(m);
      a.dim = static_cast<int>(dim);
      a.bits = static_cast<int>(bits);
      a.block = static_cast<int>(block);
      a.inv_sqrt_block = inv_sqrt_block;
      a.perm_sign = d_perm_sign.as<uint32_t>();
      a.boundaries = d_bnd.as<float>();
      a.centroids = d_cen.as<float>();
      a.tqplus = calibrated;
      a.shift = d_shift.as<float>();
      a.scale = d_scale.as<float>();
      a.inv_scale = d_inv_scale.as<float>();
      a.out_flat = d_flat.as<uint8_t>();
      a.flat_stride = static_cast<int>(stride);
      a.out_alpha = d_alpha.as<float>() + n + done;
      a.replay_count = d_counter.as<unsigned long long>();
      if (has_grid) {
        a.grid = d_grid.as<uint2>();
        a.grid_lo = grid.lo;
        a.grid_hi = grid.hi;
        a.grid_a = grid.a;
        a.grid_k = grid.k;
      }
      launch(kEncode, s, "encode kernel", [&] { return vcb::launch_encode(a, sms, s); });
      vcb::RelayoutArgs r{};
      r.flat = d_flat.as<uint8_t>();
      r.src_first = static_cast<long long>(n + done);
      r.src_n = static_cast<long long>(m);
      r.flat_stride = static_cast<int>(stride);
      r.keep_below = static_cast<long long>(n + done);
      r.n_total = static_cast<long long>(n + done + m);
      r.nbg = static_cast<int>(nbg);
      r.bits = static_cast<int>(bits);
      r.codes = d_codes.as<uint32_t>();
      launch(kEncode, s, "relayout kernel", [&] { return vcb::launch_relayout(r, s); });
    }
    n += count;
  }

  // The index's own search scratch (one search at a time on one stream).
  vcb::FlatScratch own_scratch() { return {&d_luts, &d_qf, &d_cand_s, &d_cand_i, &d_partial}; }

  // LUTs and per-query constants for nq device rows.
  void prep_queries(const float* d_q, size_t nq, cudaStream_t s, float* q_rot_out) {
    prep_queries(d_q, nq, s, q_rot_out, own_scratch());
  }
  void prep_queries(const float* d_q, size_t nq, cudaStream_t s, float* q_rot_out, vcb::FlatScratch sc) {
    sc.luts->reserve(nq * nbg * 32);
    sc.qf->reserve(nq * 4 * sizeof(float));
    float* qf = sc.qf->as<float>();
    vcb::QueryPrepArgs a{};
    a.q = d_q;
    a.nq = static_cast<long long>(nq);
    a.dim = static_cast<int>(dim);
    a.bits = static_cast<int>(bits);
    a.block = static_cast<int>(block);
    a.nbg = static_cast<int>(nbg);
    a.inv_sqrt_block = inv_sqrt_block;
    a.perm_sign = d_perm_sign.as<uint32_t>();
    a.centroids = d_cen.as<float>();
    a.tqplus = calibrated;
    a.shift = d_shift.as<float>();
    a.scale = d_scale.as<float>();
    a.luts = sc.luts->as<uint8_t>();
    a.lut_scale = qf;
    a.lut_bias = qf + nq;
    a.bias_corr = qf + 2 * nq;
    a.fa_init = qf + 3 * nq;
    a.q_rot = q_rot_out;
    a.replay_count = d_counter.as<unsigned long long>();
    launch(kPrep, s, "query prep kernel", [&] { return vcb::launch_query_prep(a, sms, s); });
  }

  // Full device search of nq rows at d_q into d_scores/d_ids (stride k_eff).
  void search_device(const float* d_q, size_t nq, size_t k, float* d_scores, uint64_t* d_ids,
                     size_t k_eff, cudaStream_t s) {
    search_device(d_q, nq, k, d_scores, d_ids, k_eff, s, own_scratch());
  }
  // Same with caller-owned scratch: searches with distinct scratch may run
  // concurrently on distinct streams (the index data is only read).
  void search_device(const float* d_q, size_t nq, size_t k, float* d_scores, uint64_t* d_ids,
                     size_t k_eff, cudaStream_t s, vcb::FlatScratch sc) {
    if (nq == 0 || k_eff == 0) return;
    // Bound the scratch per pass: LUTs + candidate lists.
    const size_t max_pass = 1 << 16;
    for (size_t q0 = 0; q0 < nq; q0 += max_pass) {
      const size_t m = std::min(max_pass, nq - q0);
      prep_queries(d_q + q0 * dim, m, s, nullptr, sc);
      vcb::ScanPlan plan;
      if (!vcb::plan_scan(static_cast<long long>(n), static_cast<long long>(m), static_cast<int>(nbg),
                          static_cast<int>(k_eff), sms, &plan, sc.range_cap, static_cast<int>(bits))) {
        vcb::fail(TQ_ERR_UNSUPPORTED, "no scan configuration fits shared memory for this dim / k");
      }
      const size_t lists = static_cast<size_t>(plan.n_ranges) * plan.lists_per_range;
      sc.cand_s->reserve(m * lists * k_eff * 4);
      sc.cand_i->reserve(m * lists * k_eff * 4);
      const float* qf = sc.qf->as<float>();
      vcb::ScanArgs a{};
      a.codes = d_codes.as<uint32_t>();
      a.alpha = d_alpha.as<float>();
      a.luts = sc.luts->as<uint8_t>();
      a.lut_scale = qf;
      a.fa_init = qf + 3 * m;
      a.n = static_cast<long long>(n);
      a.nbg = static_cast<int>(nbg);
      a.nq = static_cast<long long>(m);
      a.k = static_cast<int>(k_eff);
      a.q_per_cta = plan.q_per_cta;
      a.range_vectors = plan.range_vectors;
      a.n_ranges = plan.n_ranges;
      a.lut_chunk_groups = plan.lut_chunk_groups;
      a.bits = static_cast<int>(bits);
      a.cand_score = sc.cand_s->as<float>();
      a.cand_id = sc.cand_i->as<uint32_t>();
      if (plan.split_batches > 1 && sc.partial) {
        // Batch sums, then one arrival counter per (query group, block),
        // zeroed for this launch.
        const size_t sums = m * static_cast<size_t>(plan.split_batches) * cap;
        const size_t counters = static_cast<size_t>((m + plan.q_per_cta - 1) / plan.q_per_cta) *
                                ((n + vcb::kScanBlockVectors - 1) / vcb::kScanBlockVectors);
        sc.partial->reserve((sums + counters) * 4);
        a.partial = sc.partial->as<uint32_t>();
        a.partial_stride = static_cast<long long>(cap);
        a.partial_batches = plan.split_batches;
        a.arrive = a.partial + sums;
        if (!vcb::dry_run_flag()) {
          vcb::check(cudaMemsetAsync(a.arrive, 0, counters * 4, s), "cudaMemsetAsync");
        }
      }
      launch(kScan, s, "scan kernel", [&] { return vcb::launch_scan(a, plan, s); });
      if (!vcb::dry_run_flag()) {
        scan_stream_bytes += static_cast<uint64_t>((m + plan.q_per_cta - 1) / plan.q_per_cta) * n * (nbg + 4);
        scan_queries += m;
      }
      vcb::MergeArgs mg{};
      mg.cand_score = a.cand_score;
      mg.cand_id = a.cand_id;
      mg.nq = static_cast<long long>(m);
      mg.n_lists = static_cast<int>(lists);
      mg.k = static_cast<int>(k_eff);
      mg.k_out = static_cast<int>(k_eff);
      mg.out_score = d_scores + q0 * k_eff;
      mg.out_id = d_ids + q0 * k_eff;
      launch(kMerge, s, "merge kernel", [&] { return vcb::launch_merge(mg, s); });
    }
    (void)k;
  }
};

