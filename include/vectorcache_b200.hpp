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

// BucketParams of the reference README (README.md:113-120), plus rerank_k.
struct BucketParams {
  std::uint32_t n_probe = 64;
  std::uint32_t max_bucket_size = 800;
  std::uint32_t energy_soft = 400;
  std::uint64_t expected_n = 0;  // corpus size the partition is sized for (0: rows at prepare)
  std::uint32_t kmeans_iters = 4;
  std::uint32_t rerank_k = 0;    // > k: exact float re-rank of the scan's top rerank_k
  std::uint64_t seed = 0x5eed5eedull;

  tq_bucket_params c() const {
    tq_bucket_params p;
    tq_bucket_params_init(&p);
    p.n_probe = n_probe;
    p.max_bucket_size = max_bucket_size;
    p.energy_soft = energy_soft;
    p.expected_n = expected_n;
    p.kmeans_iters = kmeans_iters;
    p.rerank_k = rerank_k;
    p.seed = seed;
    return p;
  }
};

// BucketedTurboQuantIndex of the reference README (README.md:56, :113-120):
//   vcb::BucketParams p; p.expected_n = N;
//   vcb::BucketedTurboQuantIndex bindex(dim, bits, p);
//   bindex.calibrate(sample); bindex.add(database); bindex.prepare();
//   auto bres = bindex.search(queries, k);
class BucketedTurboQuantIndex {
 public:
  BucketedTurboQuantIndex(std::size_t dim, std::size_t bits, const BucketParams& p = {}, int device = 0)
      : dim_(dim) {
    const tq_bucket_params cp = p.c();
    throw_on_error(tq_bucketed_create(dim, bits, &cp, device, &h_));
  }
  ~BucketedTurboQuantIndex() {
    if (h_) tq_bucketed_destroy(h_);
  }
  BucketedTurboQuantIndex(const BucketedTurboQuantIndex&) = delete;
  BucketedTurboQuantIndex& operator=(const BucketedTurboQuantIndex&) = delete;
  BucketedTurboQuantIndex(BucketedTurboQuantIndex&& o) noexcept
      : h_(std::exchange(o.h_, nullptr)), dim_(o.dim_) {}
  BucketedTurboQuantIndex& operator=(BucketedTurboQuantIndex&& o) noexcept {
    if (this != &o) {
      if (h_) tq_bucketed_destroy(h_);
      h_ = std::exchange(o.h_, nullptr);
      dim_ = o.dim_;
    }
    return *this;
  }

  std::size_t dim() const { return dim_; }
  std::size_t n_buckets() const {
    std::size_t nb = 0;
    throw_on_error(tq_bucketed_info(h_, nullptr, nullptr, nullptr, nullptr, &nb, nullptr, nullptr));
    return nb;
  }
  void calibrate(std::span<const float> sample) {
    check_rows(sample.size());
    throw_on_error(tq_bucketed_calibrate(h_, sample.data(), sample.size() / dim_));
  }
  void add(std::span<const float> vectors) {
    check_rows(vectors.size());
    throw_on_error(tq_bucketed_add(h_, vectors.data(), vectors.size() / dim_));
  }
  void prepare() { throw_on_error(tq_bucketed_prepare(h_)); }
  // n_probe = 0: the index's BucketParams::n_probe; n_probe_per_query (optional,
  // one entry per query, each <= n_probe): the learned predictor's output.
  SearchResults search(std::span<const float> queries, std::size_t k, std::size_t n_probe = 0,
                       std::span<const std::uint32_t> n_probe_per_query = {}) const {
    check_rows(queries.size());
    SearchResults out;
    out.nq = queries.size() / dim_;
    out.scores.resize(out.nq * k);
    out.ids.resize(out.nq * k);
    std::size_t k_eff = 0;
    throw_on_error(tq_bucketed_search(h_, queries.data(), out.nq, k, n_probe,
                                      n_probe_per_query.empty() ? nullptr : n_probe_per_query.data(),
                                      out.scores.data(), out.ids.data(), &k_eff));
    out.k = k_eff;
    out.scores.resize(out.nq * k_eff);
    out.ids.resize(out.nq * k_eff);
    return out;
  }
  tq_bucketed* handle() const { return h_; }

 private:
  void check_rows(std::size_t floats) const {
    if (floats % dim_ != 0) throw std::invalid_argument("vectors size must be multiple of dim");
  }
  tq_bucketed* h_ = nullptr;
  std::size_t dim_ = 0;
};

// The learned n_probe predictor (BF16 MLP trained on the GPU).
class ProbeMLP {
 public:
  ProbeMLP(std::span<const std::uint32_t> classes, std::size_t hidden = 128, std::size_t layers = 2,
           std::uint64_t seed = 1, int device = 0, int objective = TQ_PROBE_OBJECTIVE_CLASSES) {
    throw_on_error(tq_probe_mlp_create(hidden, layers, classes.data(), classes.size(), seed, device, &h_));
    const int rc = tq_probe_mlp_set_objective(h_, objective);
    if (rc != TQ_OK) {
      tq_probe_mlp_destroy(h_);
      h_ = nullptr;
      throw_on_error(rc);
    }
  }
  ~ProbeMLP() {
    if (h_) tq_probe_mlp_destroy(h_);
  }
  ProbeMLP(const ProbeMLP&) = delete;
  ProbeMLP& operator=(const ProbeMLP&) = delete;
  tq_probe_mlp* handle() const { return h_; }

 private:
  tq_probe_mlp* h_ = nullptr;
};

// Continuous-batching server over prepared indexes.
class Server {
 public:
  Server(int device, std::size_t hbm_budget_bytes, std::size_t max_slots, std::size_t max_batch) {
    throw_on_error(tq_server_create(device, hbm_budget_bytes, max_slots, max_batch, &h_));
  }
  ~Server() {
    if (h_) tq_server_destroy(h_);
  }
  Server(const Server&) = delete;
  Server& operator=(const Server&) = delete;
  int add(const TurboQuantIndex& index, std::size_t max_k) {
    int t = -1;
    throw_on_error(tq_server_add_flat(h_, index.handle(), max_k, &t));
    return t;
  }
  int add(const BucketedTurboQuantIndex& index, std::size_t max_k, std::size_t max_probe,
          const ProbeMLP* mlp = nullptr, float coverage = 0.9f, float min_confidence = 0.f) {
    int t = -1;
    throw_on_error(tq_server_add_bucketed(h_, index.handle(), max_k, max_probe, mlp ? mlp->handle() : nullptr,
                                          coverage, min_confidence, &t));
    return t;
  }
  void start() { throw_on_error(tq_server_start(h_)); }
  // Queues a request; `queries` and the result vectors of the returned
  // request must stay alive until wait().
  struct Request {
    std::uint64_t id = 0;
    std::size_t nq = 0, k = 0;
    std::vector<float> scores;
    std::vector<std::uint64_t> ids;
  };
  void submit(int target, std::span<const float> queries, std::size_t nq, std::size_t k, std::size_t n_probe,
              Request& r) {
    r.nq = nq;
    r.k = k;
    r.scores.resize(nq * k);
    r.ids.resize(nq * k);
    throw_on_error(tq_server_submit(h_, target, queries.data(), nq, k, n_probe, r.scores.data(), r.ids.data(),
                                    &r.id));
  }
  // Blocks until the request is done; returns its latency in microseconds.
  double wait(Request& r) {
    std::size_t k_eff = 0;
    double lat = 0.0;
    throw_on_error(tq_server_wait(h_, r.id, &k_eff, &lat));
    r.k = k_eff;
    r.scores.resize(r.nq * k_eff);
    r.ids.resize(r.nq * k_eff);
    return lat;
  }

 private:
  tq_server* h_ = nullptr;
};

}  // namespace vcb
