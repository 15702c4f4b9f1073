// C++20 host program over include/vectorcache_b200.hpp for the bucketed index
// and the serving loop:
//   - ids in range, scores sorted descending, a database row finds itself first
//     with every bucket probed;
//   - per-query probe counts: a query scanned with n_probe_per_query[q] = p gets
//     the same top-k as a search at n_probe = p;
//   - a request served by vcb::Server returns the direct search's results.
// Prints "OK <n_buckets>" and exits 0 when every property holds.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <span>
#include <vector>

#include "vectorcache_b200.hpp"

#define CHECK(cond)                                                          \
  do {                                                                       \
    if (!(cond)) {                                                           \
      std::fprintf(stderr, "FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond); \
      return 1;                                                              \
    }                                                                        \
  } while (0)

int main() {
  const std::size_t dim = 100, n = 20000, nq = 32, k = 10;
  std::mt19937 rng(7);
  std::normal_distribution<float> nd(0.f, 1.f);
  std::vector<float> centers(40 * dim);
  for (float& v : centers) v = nd(rng);
  std::vector<float> base(n * dim);
  for (std::size_t i = 0; i < n; ++i) {
    const std::size_t c = rng() % 40;
    for (std::size_t d = 0; d < dim; ++d) base[i * dim + d] = centers[c * dim + d] + 0.4f * nd(rng);
  }
  vcb::BucketParams p;
  p.max_bucket_size = 300;
  p.energy_soft = 150;
  p.n_probe = 16;
  vcb::BucketedTurboQuantIndex index(dim, 4, p);
  index.add(base);
  index.prepare();
  const std::size_t nb = index.n_buckets();
  CHECK(nb >= 20);

  std::vector<float> queries(base.begin(), base.begin() + nq * dim);
  const vcb::SearchResults all = index.search(queries, k, std::min<std::size_t>(nb, 256));
  CHECK(all.nq == nq && all.k == k);
  for (std::size_t q = 0; q < nq; ++q) {
    for (std::size_t j = 0; j < k; ++j) {
      CHECK(all.ids[q * k + j] < n);
      if (j > 0) CHECK(all.scores[q * k + j - 1] >= all.scores[q * k + j]);
    }
    CHECK(all.ids[q * k] == q);  // a database row finds itself first
  }

  std::vector<std::uint32_t> per(nq);
  for (std::size_t q = 0; q < nq; ++q) per[q] = 1 + static_cast<std::uint32_t>(q % 8);
  const vcb::SearchResults mixed = index.search(queries, k, 8, per);
  for (std::uint32_t c = 1; c <= 8; ++c) {
    std::vector<float> sub;
    std::vector<std::size_t> rows;
    for (std::size_t q = 0; q < nq; ++q) {
      if (per[q] == c) {
        rows.push_back(q);
        sub.insert(sub.end(), queries.begin() + q * dim, queries.begin() + (q + 1) * dim);
      }
    }
    const vcb::SearchResults alone = index.search(sub, k, c);
    for (std::size_t r = 0; r < rows.size(); ++r) {
      for (std::size_t j = 0; j < k; ++j) CHECK(alone.ids[r * k + j] == mixed.ids[rows[r] * k + j]);
    }
  }

  vcb::Server server(0, std::size_t{64} << 30, 2, 256);
  const int target = server.add(index, 64, 16);
  server.start();
  vcb::Server::Request req;
  server.submit(target, queries, nq, k, 16, req);
  const double lat = server.wait(req);
  const vcb::SearchResults direct = index.search(queries, k, 16);
  CHECK(lat > 0.0);
  CHECK(req.ids == direct.ids);
  CHECK(req.scores == direct.scores);

  std::printf("OK %zu\n", nb);
  return 0;
}
