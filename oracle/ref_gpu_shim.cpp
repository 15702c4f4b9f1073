// Test infrastructure only: a C entry point to the reference's own GPU flat
// index (vectorcache::gpu::FlatIndex, src/gpu/flat_index.cpp:82-242, kernels
// in src/gpu/kernels.cu:69-516), built by `make -C oracle refgpu` from the
// reference sources with the one cast kernels.cu:719 needs to compile
// (uint64_t* -> unsigned long long*). bench.py times it on the same B200 as
// the bar to beat: its scan is a float-ADC scan without TQ+ whose top-k keeps
// a few candidates per thread, so its results are approximate and are judged
// by recall, never used as a parity reference.
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <exception>
#include <span>
#include <string>

#include "vectorcache/gpu/flat_index.hpp"

namespace {
thread_local std::string g_err;

template <typename F>
int guarded(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  } catch (...) {
    g_err = "unknown error";
    return 1;
  }
}
}  // namespace

extern "C" {

const char* tqrefgpu_last_error() { return g_err.c_str(); }

int tqrefgpu_create(std::size_t dim, std::size_t bits, void** out) {
  return guarded([&] { *out = new vectorcache::gpu::FlatIndex(dim, bits); });
}

int tqrefgpu_destroy(void* h) {
  delete static_cast<vectorcache::gpu::FlatIndex*>(h);
  return 0;
}

int tqrefgpu_add(void* h, const float* x, std::size_t n) {
  return guarded([&] {
    auto* idx = static_cast<vectorcache::gpu::FlatIndex*>(h);
    idx->add(std::span<const float>(x, n * idx->dim()));
  });
}

int tqrefgpu_prepare(void* h) {
  return guarded([&] { static_cast<vectorcache::gpu::FlatIndex*>(h)->prepare(); });
}

// scores/ids: nq * k entries, rows of stride k_eff = min(k, size).
int tqrefgpu_search(void* h, const float* q, std::size_t nq, std::size_t k, float* scores,
                    std::uint64_t* ids, std::size_t* k_eff) {
  return guarded([&] {
    auto* idx = static_cast<vectorcache::gpu::FlatIndex*>(h);
    auto res = idx->search(std::span<const float>(q, nq * idx->dim()), k);
    *k_eff = res.k;
    if (res.k > 0) {
      std::memcpy(scores, res.scores.data(), nq * res.k * sizeof(float));
      std::memcpy(ids, res.ids.data(), nq * res.k * sizeof(std::uint64_t));
    }
  });
}

}  // extern "C"
