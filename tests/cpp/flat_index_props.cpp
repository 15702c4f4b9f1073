// C++20 host program over include/vectorcache_b200.hpp, restating the
// properties the reference's index tests check (tests/test_index.cpp):
//   - ids in range, scores sorted descending (:11-38)
//   - a database vector queried against the index finds itself first (:40-55)
//   - a batch search equals one-query-at-a-time searches (:86-113)
// plus the error types the reference throws for bad arguments and call order.
// Prints "OK <n> <dim> <bits>" and exits 0 when every property holds.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <span>
#include <stdexcept>
#include <vector>

#include "vectorcache_b200.hpp"

#define CHECK(cond)                                                   \
  do {                                                                \
    if (!(cond)) {                                                    \
      std::fprintf(stderr, "FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond); \
      return 1;                                                       \
    }                                                                 \
  } while (0)

int main() {
  const std::size_t dim = 256, bits = 4, n = 5000, nq = 16, k = 10;
  std::mt19937 rng(42);
  std::normal_distribution<float> nd(0.f, 1.f);
  std::vector<float> base(n * dim), queries(nq * dim);
  for (auto& v : base) v = nd(rng);
  for (std::size_t q = 0; q < nq; ++q) {
    for (std::size_t d = 0; d < dim; ++d) queries[q * dim + d] = base[(q * 97) * dim + d];
  }

  // Reference-style argument checks (rotation.cpp:140-145, flat_index.cpp:92-98).
  bool threw = false;
  try {
    vcb::TurboQuantIndex bad(100, 4);
  } catch (const std::invalid_argument&) {
    threw = true;
  }
  CHECK(threw);

  vcb::TurboQuantIndex index(dim, bits);
  threw = false;
  try {
    index.prepare();  // empty index (flat_index.cpp:149-151)
  } catch (const std::runtime_error&) {
    threw = true;
  }
  CHECK(threw);

  index.calibrate(std::span<const float>(base.data(), 1000 * dim));
  index.add(std::span<const float>(base.data(), base.size()));
  index.prepare();
  CHECK(index.size() == n);

  const vcb::SearchResults batch = index.search(std::span<const float>(queries.data(), queries.size()), k);
  CHECK(batch.k == k && batch.nq == nq);
  for (std::size_t q = 0; q < nq; ++q) {
    for (std::size_t j = 0; j < k; ++j) {
      CHECK(batch.ids[q * k + j] < n);
      if (j > 0) CHECK(batch.scores[q * k + j - 1] >= batch.scores[q * k + j]);
    }
    CHECK(batch.ids[q * k] == q * 97);  // self-query
    const vcb::SearchResults one =
        index.search(std::span<const float>(queries.data() + q * dim, dim), k);
    for (std::size_t j = 0; j < k; ++j) {
      CHECK(one.ids[j] == batch.ids[q * k + j]);
      CHECK(one.scores[j] == batch.scores[q * k + j]);
    }
  }
  std::printf("OK %zu %zu %zu\n", n, dim, bits);
  return 0;
}
