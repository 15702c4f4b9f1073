// vectorcache_b200.hpp — header-only C++20 host API over the C ABI in
// vectorcache_b200.h, shaped like the reference's flat index
// (nishadtardalkar/vectorcache README.md:100-121, gpu::FlatIndex in
// include/vectorcache/gpu/flat_index.hpp:19-73).
//
//   vcb::TurboQuantIndex index(/*dim=*/1536, /*bits=*/4);
//   index.calibrate(sample, n_sample);   // optional TQ+
//   index.add(database, n);              // float[n * dim], host memory
//   index.prepare();
//   vcb::SearchResults res = index.search(queries, nq, /*k=*/10);
//
// Errors surface as the reference's exception types: std::invalid_argument for
// bad shapes or parameters, std::runtime_error for call-order and device
// errors (std::bad_alloc for device out-of-memory).
#pragma once

#include <cstddef>
#include <cstdint>
#include <new>
#include <span>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "vectorcache_b200.h"

namespace vcb {

inline void throw_on_error(int rc) {
  if (rc == TQ_OK) return;
  const std::string msg = tq_last_error();
  switch (rc) {
    case TQ_ERR_INVALID_ARGUMENT:
      throw std::invalid_argument(msg);
    case TQ_ERR_OUT_OF_MEMORY:
      throw std::bad_alloc();
    default:
      throw std::runtime_error(msg);
  }
}

// Row-major top-k like vectorcache::SearchResults (search.hpp:77-84).
struct SearchResults {
  std::vector<float> scores;      // nq * k
  std::vector<std::uint64_t> ids; // nq * k
  std::size_t k = 0;
  std::size_t nq = 0;
};

class TurboQuantIndex {
 public:
  TurboQuantIndex(std::size_t dim, std::size_t bits, int device = 0) : dim_(dim), bits_(bits) {
    throw_on_error(tq_index_create(dim, bits, 0, device, &h_));
  }
  ~TurboQuantIndex() {
    if (h_) tq_index_destroy(h_);
  }
  TurboQuantIndex(const TurboQuantIndex&) = delete;
  TurboQuantIndex& operator=(const TurboQuantIndex&) = delete;
  TurboQuantIndex(TurboQuantIndex&& o) noexcept : h_(std::exchange(o.h_, nullptr)), dim_(o.dim_), bits_(o.bits_) {}
  TurboQuantIndex& operator=(TurboQuantIndex&& o) noexcept {
    if (this != &o) {
      if (h_) tq_index_destroy(h_);
      h_ = std::exchange(o.h_, nullptr);
      dim_ = o.dim_;
      bits_ = o.bits_;
    }
    return *this;
  }

  std::size_t dim() const { return dim_; }
  std::size_t bits() const { return bits_; }
  std::size_t size() const {
    std::size_t n = 0;
    throw_on_error(tq_index_info(h_, nullptr, nullptr, &n, nullptr, nullptr));
    return n;
  }

  void calibrate(std::span<const float> sample) {
    check_rows(sample.size());
    throw_on_error(tq_index_calibrate(h_, sample.data(), sample.size() / dim_));
  }
  void add(std::span<const float> vectors) {
    check_rows(vectors.size());
    throw_on_error(tq_index_add(h_, vectors.data(), vectors.size() / dim_));
  }
  void prepare() { throw_on_error(tq_index_prepare(h_)); }

  SearchResults search(std::span<const float> queries, std::size_t k) const {
    check_rows(queries.size());
    SearchResults out;
    out.nq = queries.size() / dim_;
    out.scores.resize(out.nq * k);
    out.ids.resize(out.nq * k);
    std::size_t k_eff = 0;
    throw_on_error(tq_index_search(h_, queries.data(), out.nq, k, out.scores.data(), out.ids.data(), &k_eff));
    out.k = k_eff;
    out.scores.resize(out.nq * k_eff);
    out.ids.resize(out.nq * k_eff);
    return out;
  }

  tq_index* handle() const { return h_; }

 private:
  void check_rows(std::size_t floats) const {
    if (floats % dim_ != 0) throw std::invalid_argument("vectors size must be multiple of dim");
  }

  tq_index* h_ = nullptr;
  std::size_t dim_ = 0;
  std::size_t bits_ = 0;
};

}  // namespace vcb
