// Host side of the bucketed (IVF) TurboQuant index and its C ABI
// (include/vectorcache_b200.h, "bucketed index").
//
// The reference documents BucketedTurboQuantIndex / BucketParams (README.md:56,
// :91-98, :113-120) but ships no implementation of them; the per-bucket scoring
// it composes is score_prepared_into (src/search/search.cpp:1156-1264), whose
// arithmetic the bucket scan reproduces bit for bit. The partition itself is
// this library's own design:
//
//   * rows are L2-normalized (and zero-padded to a multiple of 8 coordinates);
//   * initial partition: ceil(expected_n / energy_soft) seeds drawn without
//     replacement (mt19937_64(seed)), then `kmeans_iters` rounds of spherical
//     k-means (fp32 routing contraction, argmax with ties to the lower bucket,
//     centroids from exact fixed-point sums, so the build is deterministic);
//   * hard fission: every bucket above max_bucket_size is split by one 2-means
//     round (tq_bucket.h: launch_split) until none is;
//   * encode centroid = mean of the bucket's members when the bucket is formed
//     (frozen afterwards), routing centroid = normalized current mean;
//   * residuals x_hat - encode_c are encoded by the flat TurboQuant encoder (TQ+
//     fitted on residuals of the calibration sample), laid out bucket by bucket
//     at 256-slot boundaries of the flat scan layout;
//   * search: query LUTs built once on q_hat; routing scores q_hat . route^T;
//     the top n_probe buckets are scanned with score (fa * alpha) + <q_hat,
//     encode_c>; results are the top-k in (score desc, id asc) order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "../../include/vectorcache_b200.h"
#include "tq_abi.h"
#include "tq_bucket.h"
#include "tq_index_impl.h"
#include "tq_kernels.h"
#include "tq_probe.h"
#include "tq_serving_hooks.h"

namespace vcb {
// Device scratch of one bucketed search (routing, probe pairs, candidate
// lists, re-rank) plus the flat engine's query scratch.
struct BucketScratch {
  DeviceBuffer qh, route, top_s, top_i, counts, fill, pstart, istart, pairs, off, items, nitems, cand_s,
      cand_i, rr_s, rr_i, np, floor, acount, encs;
  FlatScratchStore flat;
  ProbeScratch probe;
  void bind(ScratchArena* a) {
    for (DeviceBuffer* b : {&qh, &route, &top_s, &top_i, &counts, &fill, &pstart, &istart, &pairs, &off, &items,
                            &nitems, &cand_s, &cand_i, &rr_s, &rr_i, &np, &floor, &acount, &encs}) {
      b->bind(a);
    }
    flat.bind(a);
    probe.bind(a);
  }
};
}  // namespace vcb

struct tq_bucketed {
  int device = 0;
  size_t dim_in = 0, dim = 0, bits = 0, nbg = 0;
  tq_bucket_params p{};
  tq_index* eng = nullptr;  // encoder / LUT engine; its codes and alpha are the slot layout

  vcb::DeviceBuffer d_x;    // n x dim normalized rows
  size_t n = 0, cap_rows = 0, n_built = 0;
  vcb::DeviceBuffer d_label;
  int nb = 0;
  size_t cap_b = 0;
  vcb::DeviceBuffer d_enc, d_route, d_tmp_enc, d_tmp_route;
  vcb::DeviceBuffer d_counts, d_starts, d_fill, d_members, d_acc;
  std::vector<uint32_t> h_size;
  std::vector<uint64_t> h_slot_start;
  vcb::DeviceBuffer d_bucket_size, d_slot_start, d_slot_ids;
  size_t n_slots = 0;
  vcb::DeviceBuffer d_calib;
  size_t n_calib = 0;
  bool prepared = false, built_once = false;

  // search scratch
  vcb::DeviceBuffer s_q, s_out_s, s_out_i, s_np;  // host-API staging
  vcb::BucketScratch own;                             // the index's own search scratch

  ~tq_bucketed() {
    if (eng) tq_index_destroy(eng);
  }

  cudaStream_t stream() const { return eng->stream; }
  void sync() { eng->sync(); }

  template <typename F>
  void run(const char* what, F&& fn) {
    vcb::check(fn(), what);
  }

  // Append n_new rows (dim_in floats each, device) as normalized padded rows.
  void add_rows(const float* d_src, size_t n_new, cudaStream_t s) {
    if (n_new == 0) return;
    if (n + n_new > cap_rows) {
      const size_t cap = std::max(n + n_new, cap_rows + cap_rows / 2);
      vcb::DeviceBuffer grown;
      grown.reserve(cap * dim * 4);
      if (n) {
        vcb::check(cudaMemcpyAsync(grown.get(), d_x.get(), n * dim * 4, cudaMemcpyDeviceToDevice, s), "D2D");
      }
      vcb::check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
      grown.swap(d_x);
      cap_rows = cap;
    }
    run("normalize kernel", [&] {
      return vcb::launch_normalize_rows(d_src, static_cast<long long>(n_new), static_cast<int>(dim_in),
                                        static_cast<int>(dim), d_x.as<float>() + n * dim, s);
    });
    n += n_new;
  }

  // Grows the per-bucket buffers; returns true when they were reallocated, in
  // which case the grouping buffers (counts, starts) hold no data any more.
  bool ensure_buckets(size_t want) {
    if (want <= cap_b) return false;
    const size_t cap = std::max(want, cap_b * 2);
    vcb::DeviceBuffer e, r;
    e.reserve(cap * dim * 4);
    r.reserve(cap * dim * 4);
    if (nb) {
      vcb::check(cudaMemcpyAsync(e.get(), d_enc.get(), nb * dim * 4, cudaMemcpyDeviceToDevice, stream()), "D2D");
      vcb::check(cudaMemcpyAsync(r.get(), d_route.get(), nb * dim * 4, cudaMemcpyDeviceToDevice, stream()), "D2D");
    }
    sync();
    e.swap(d_enc);
    r.swap(d_route);
    d_tmp_enc.reserve(cap * dim * 4);
    d_tmp_route.reserve(cap * dim * 4);
    d_counts.reserve(cap * 4);
    d_fill.reserve(cap * 4);
    d_starts.reserve((cap + 1) * 8);
    d_acc.reserve(cap * dim * 8);
    cap_b = cap;
    return true;
  }

  // Counting sort of the current labels; fills h_size.
  void group() {
    d_members.reserve(std::max<size_t>(n, 1) * 4);
    run("group kernels", [&] {
      return vcb::launch_group_by_label(d_label.as<uint32_t>(), static_cast<long long>(n), nb,
                                        d_counts.as<uint32_t>(), d_starts.as<unsigned long long>(),
                                        d_fill.as<uint32_t>(), d_members.as<uint32_t>(), stream());
    });
    h_size.resize(nb);
    vcb::check(cudaMemcpyAsync(h_size.data(), d_counts.get(), nb * 4, cudaMemcpyDeviceToHost, stream()), "D2H");
    sync();
  }

  void centroids_into(float* enc, float* route) {
    run("centroid kernels", [&] {
      return vcb::launch_centroids(d_x.as<float>(), static_cast<int>(dim), d_starts.as<unsigned long long>(),
                                   d_members.as<uint32_t>(), nb, d_acc.as<long long>(), enc, route, stream());
    });
  }

  void initial_partition() {
    const uint64_t target = p.expected_n ? std::max<uint64_t>(p.expected_n, n) : n;
    size_t k0 = static_cast<size_t>((target + p.energy_soft - 1) / std::max<uint32_t>(p.energy_soft, 1));
    k0 = std::max<size_t>(1, std::min(k0, n));
    // k0 distinct seed rows: partial Fisher-Yates over the row ids.
    std::vector<uint32_t> ids(n);
    std::iota(ids.begin(), ids.end(), 0u);
    std::mt19937_64 rng(p.seed);
    for (size_t i = 0; i < k0; ++i) {
      std::uniform_int_distribution<size_t> pick(i, n - 1);
      std::swap(ids[i], ids[pick(rng)]);
    }
    std::sort(ids.begin(), ids.begin() + static_cast<long>(k0));
    ensure_buckets(k0);
    vcb::DeviceBuffer d_ids;
    d_ids.reserve(k0 * 4);
    eng->upload(d_ids.get(), ids.data(), k0 * 4);
    run("gather kernel", [&] {
      return vcb::launch_gather_rows(d_x.as<float>(), d_ids.as<uint32_t>(), static_cast<long long>(k0),
                                     static_cast<int>(dim), d_route.as<float>(), stream());
    });
    vcb::check(cudaMemcpyAsync(d_enc.get(), d_route.get(), k0 * dim * 4, cudaMemcpyDeviceToDevice, stream()), "D2D");
    nb = static_cast<int>(k0);
    const uint32_t iters = std::max<uint32_t>(p.kmeans_iters, 1);
    for (uint32_t it = 0; it < iters; ++it) {
      run("assign kernel", [&] {
        return vcb::launch_assign(d_x.as<float>(), static_cast<long long>(n), d_route.as<float>(), nb,
                                  static_cast<int>(dim), d_label.as<uint32_t>(), nullptr, stream());
      });
      group();
      centroids_into(d_enc.as<float>(), d_route.as<float>());
    }
    sync();
    sync();
    d_ids.release();
  }

  // Split every bucket above max_bucket_size until none is. Buckets formed here
  // (and all buckets on the first build) get fresh encode centroids; the
  // routing centroids of all buckets follow their current means.
  void fission(std::vector<char>& fresh) {
    // 2-means splits for this many levels; deeper, a bucket still above the cap
    // (outlier-peeling splits) is halved by id bits so the loop always ends.
    constexpr int kGeometricLevels = 24;
    for (int level = 0; level < kGeometricLevels + 40; ++level) {
      group();
      centroids_into(d_tmp_enc.as<float>(), d_tmp_route.as<float>());
      std::vector<uint32_t> rows_fresh, rows_all;
      for (int b = 0; b < nb; ++b) {
        if (h_size[b] == 0) continue;  // empty buckets keep their centroids
        rows_all.push_back(static_cast<uint32_t>(b));
        if (fresh[b]) rows_fresh.push_back(static_cast<uint32_t>(b));
      }
      copy_rows(d_tmp_route.as<float>(), d_route.as<float>(), rows_all);
      copy_rows(d_tmp_enc.as<float>(), d_enc.as<float>(), rows_fresh);
      std::vector<uint32_t> over, fresh_ids;
      for (int b = 0; b < nb; ++b) {
        if (h_size[b] > p.max_bucket_size) over.push_back(static_cast<uint32_t>(b));
      }
      if (over.empty()) return;
      if (ensure_buckets(nb + over.size())) group();  // starts/members for the split below
      std::vector<uint32_t> newl(over.size());
      for (size_t t = 0; t < over.size(); ++t) newl[t] = static_cast<uint32_t>(nb + t);
      vcb::DeviceBuffer d_groups, d_new;
      d_groups.reserve(over.size() * 4);
      d_new.reserve(over.size() * 4);
      eng->upload(d_groups.get(), over.data(), over.size() * 4);
      eng->upload(d_new.get(), newl.data(), newl.size() * 4);
      run("split kernel", [&] {
        return vcb::launch_split(d_x.as<float>(), static_cast<int>(dim), d_starts.as<unsigned long long>(),
                                 d_members.as<uint32_t>(), d_groups.as<uint32_t>(), d_new.as<uint32_t>(),
                                 static_cast<int>(over.size()), d_route.as<float>(), d_label.as<uint32_t>(),
                                 level >= kGeometricLevels, stream());
      });
      fresh.resize(nb + over.size(), 1);
      for (uint32_t b : over) fresh[b] = 1;
      nb += static_cast<int>(over.size());
      sync();
    }
    vcb::fail(TQ_ERR_STATE, "bucket fission did not converge");
  }

  void copy_rows(const float* src, float* dst, const std::vector<uint32_t>& rows) {
    if (rows.empty()) return;
    // dst[rows[r]] = src[rows[r]]: gather into a packed buffer, then scatter
    // row by row in runs of consecutive ids.
    size_t i = 0;
    while (i < rows.size()) {
      size_t j = i + 1;
      while (j < rows.size() && rows[j] == rows[j - 1] + 1) ++j;
      vcb::check(cudaMemcpyAsync(dst + static_cast<size_t>(rows[i]) * dim, src + static_cast<size_t>(rows[i]) * dim,
                                 (j - i) * dim * 4, cudaMemcpyDeviceToDevice, stream()),
                 "D2D");
      i = j;
    }
  }

  // Drop empty buckets (relabel rows, compact centroid rows).
  void compact() {
    group();
    std::vector<uint32_t> remap(nb, 0xffffffffu), keep;
    for (int b = 0; b < nb; ++b) {
      if (h_size[b] > 0) {
        remap[b] = static_cast<uint32_t>(keep.size());
        keep.push_back(static_cast<uint32_t>(b));
      }
    }
    if (static_cast<int>(keep.size()) == nb) return;
    vcb::DeviceBuffer d_remap, d_keep;
    d_remap.reserve(remap.size() * 4);
    d_keep.reserve(keep.size() * 4);
    eng->upload(d_remap.get(), remap.data(), remap.size() * 4);
    eng->upload(d_keep.get(), keep.data(), keep.size() * 4);
    run("relabel kernel", [&] {
      return vcb::launch_relabel(d_label.as<uint32_t>(), static_cast<long long>(n), d_remap.as<uint32_t>(), stream());
    });
    run("gather kernel", [&] {
      return vcb::launch_gather_rows(d_enc.as<float>(), d_keep.as<uint32_t>(), static_cast<long long>(keep.size()),
                                     static_cast<int>(dim), d_tmp_enc.as<float>(), stream());
    });
    run("gather kernel", [&] {
      return vcb::launch_gather_rows(d_route.as<float>(), d_keep.as<uint32_t>(), static_cast<long long>(keep.size()),
                                     static_cast<int>(dim), d_tmp_route.as<float>(), stream());
    });
    vcb::check(cudaMemcpyAsync(d_enc.get(), d_tmp_enc.get(), keep.size() * dim * 4, cudaMemcpyDeviceToDevice,
                               stream()), "D2D");
    vcb::check(cudaMemcpyAsync(d_route.get(), d_tmp_route.get(), keep.size() * dim * 4, cudaMemcpyDeviceToDevice,
                               stream()), "D2D");
    nb = static_cast<int>(keep.size());
    sync();
  }

  void build() {
    d_label.reserve(std::max<size_t>(cap_rows, n) * 4);
    std::vector<char> fresh;
    if (!built_once) {
      initial_partition();
      fresh.assign(nb, 1);
    } else {
      // New rows go to their nearest routing centroid.
      const size_t m = n - n_built;
      if (m > 0) {
        vcb::DeviceBuffer grown;
        grown.reserve(n * 4);
        vcb::check(cudaMemcpyAsync(grown.get(), d_label.get(), n_built * 4, cudaMemcpyDeviceToDevice, stream()),
                   "D2D");
        sync();
        grown.swap(d_label);
        run("assign kernel", [&] {
          return vcb::launch_assign(d_x.as<float>() + n_built * dim, static_cast<long long>(m), d_route.as<float>(),
                                    nb, static_cast<int>(dim), d_label.as<uint32_t>() + n_built, nullptr, stream());
        });
      }
      fresh.assign(nb, 0);
    }
    fission(fresh);
    compact();
    layout();
    n_built = n;
    built_once = true;
  }

  void layout() {
    group();
    uint32_t max_size = 1;
    for (int b = 0; b < nb; ++b) max_size = std::max(max_size, h_size[b]);
    run("sort kernel", [&] {
      return vcb::launch_sort_groups(d_starts.as<unsigned long long>(), nb, static_cast<int>(max_size),
                                     d_members.as<uint32_t>(), stream());
    });
    h_slot_start.assign(nb + 1, 0);
    for (int b = 0; b < nb; ++b) {
      h_slot_start[b + 1] =
          h_slot_start[b] + vcb::round_up(h_size[b], static_cast<size_t>(vcb::kBucketSlotAlign));
    }
    n_slots = h_slot_start[nb];
    d_slot_start.reserve((nb + 1) * 8);
    d_bucket_size.reserve(std::max(nb, 1) * 4);
    eng->upload(d_slot_start.get(), h_slot_start.data(), (nb + 1) * 8);
    eng->upload(d_bucket_size.get(), h_size.data(), nb * 4);
    d_slot_ids.reserve(vcb::round_up(n_slots, vcb::kScanBlockVectors) * 4);
    vcb::DeviceBuffer R;
    R.reserve(n_slots * dim * 4);
    run("residual kernel", [&] {
      return vcb::launch_build_residuals(d_x.as<float>(), static_cast<int>(dim), d_starts.as<unsigned long long>(),
                                         d_members.as<uint32_t>(), nb, d_slot_start.as<unsigned long long>(),
                                         d_enc.as<float>(), static_cast<long long>(n_slots), R.as<float>(),
                                         d_slot_ids.as<uint32_t>(), stream());
    });
    // Re-encode every slot with the flat encoder.
    eng->n = 0;
    eng->prepared = false;
    if (n_calib > 0 && !eng->calibrated) {
      vcb::DeviceBuffer lab, rc;
      lab.reserve(n_calib * 4);
      rc.reserve(n_calib * dim * 4);
      run("assign kernel", [&] {
        return vcb::launch_assign(d_calib.as<float>(), static_cast<long long>(n_calib), d_route.as<float>(), nb,
                                  static_cast<int>(dim), lab.as<uint32_t>(), nullptr, stream());
      });
      run("residual kernel", [&] {
        return vcb::launch_residual_rows(d_calib.as<float>(), static_cast<long long>(n_calib),
                                         static_cast<int>(dim), lab.as<uint32_t>(), d_enc.as<float>(),
                                         rc.as<float>(), stream());
      });
      vcb::calibrate_index(eng, rc.as<float>(), n_calib, stream());
    }
    eng->encode_append(R.as<float>(), n_slots, stream());
    sync();
    eng->d_flat.release();
    eng->prepared = true;
    prepared = true;
  }

  // Routing of m normalized queries: scores (m x nb) and the top p per query.
  void route(const float* qh, size_t m, int ptop, cudaStream_t s, vcb::BucketScratch& sc) {
    sc.route.reserve(m * nb * 4);
    sc.top_s.reserve(m * ptop * 4);
    sc.top_i.reserve(m * ptop * 4);
    eng->launch(tq_index::kPrep, s, "routing kernel", [&] {
      return vcb::launch_gemm_nt(qh, static_cast<long long>(m), d_route.as<float>(), nb, static_cast<int>(dim),
                                 sc.route.as<float>(), nb, s);
    });
    eng->launch(tq_index::kPrep, s, "select kernel", [&] {
      return vcb::launch_select_top(sc.route.as<float>(), static_cast<long long>(m), nb, nb, ptop, sc.top_s.as<float>(),
                                    sc.top_i.as<uint32_t>(), s);
    });
  }

  // Queries per pass: routing scores (nb floats per query) within 256 MiB and
  // candidate lists (max_probe lists of kscan (score, id) per query) within
  // 8 GiB — 13,981 queries at 768 probes and a re-rank of 100. Every pass
  // repeats the routing, pair and floor launches on a smaller grid: at 1 GiB
  // with two lists per probe the same search ran in 8 passes and took 1.7x
  // as long for 64 probes per query under a 512-probe cap.
  size_t pass_queries(size_t max_probe = 1, size_t kscan = 1) const {
    const size_t by_route = std::max<size_t>(1, (size_t{256} << 20) / (static_cast<size_t>(nb) * 4));
    const size_t by_cand =
        std::max<size_t>(1, (size_t{8} << 30) / (max_probe * vcb::kBsListsPerProbe * kscan * 8));
    return std::min<size_t>({16384, by_route, by_cand});
  }

  // Device search: nq raw queries (dim_in floats) -> top k_eff per query.
  void search_device(const float* d_q, size_t nq, size_t ke, int max_probe, const uint32_t* d_np, float* d_scores,
                     uint64_t* d_ids, cudaStream_t s, float* trace_off = nullptr, uint32_t* trace_probe = nullptr,
                     float* trace_qh = nullptr) {
    search_device(d_q, nq, ke, max_probe, d_np, d_scores, d_ids, s, own, trace_off, trace_probe, trace_qh);
  }
  // Same with caller-owned scratch: searches with distinct scratch may run
  // concurrently on distinct streams (the index data is only read).
  void search_device(const float* d_q, size_t nq, size_t ke, int max_probe, const uint32_t* d_np, float* d_scores,
                     uint64_t* d_ids, cudaStream_t s, vcb::BucketScratch& sc, float* trace_off = nullptr,
                     uint32_t* trace_probe = nullptr, float* trace_qh = nullptr,
                     const vcb::LearnedProbe* lp = nullptr) {
    // With the learned probe, one routing pass serves both the network's
    // features (top 256 scores) and the probes (top max_probe buckets).
    const int ptop = lp ? std::max(max_probe, 256) : max_probe;
    const bool rerank = p.rerank_k > ke;
    // With re-ranking the scan keeps kscan candidates per query.
    const size_t kscan = rerank ? std::min<size_t>({static_cast<size_t>(p.rerank_k), n, 256}) : ke;
    const size_t pass = pass_queries(static_cast<size_t>(max_probe), kscan);
    for (size_t q0 = 0; q0 < nq; q0 += pass) {
      const size_t m = std::min(pass, nq - q0);
      sc.qh.reserve(m * dim * 4);
      float* qh = sc.qh.as<float>();
      eng->launch(tq_index::kPrep, s, "normalize kernel", [&] {
        return vcb::launch_normalize_rows(d_q + q0 * dim_in, static_cast<long long>(m), static_cast<int>(dim_in),
                                          static_cast<int>(dim), qh, s);
      });
      route(qh, m, ptop, s, sc);
      const uint32_t* np_pass = d_np ? d_np + q0 : nullptr;
      if (lp) {
        sc.np.reserve(m * 4);
        vcb::probe_reserve(lp->mlp, m, sc.probe);
        eng->launch(tq_index::kPrep, s, "probe network", [&] {
          vcb::probe_predict(lp->mlp, sc.top_s.as<float>(), m, ptop, lp->coverage, lp->min_confidence,
                             static_cast<uint32_t>(max_probe), sc.np.as<uint32_t>(), s, sc.probe);
          return cudaGetLastError();
        });
        np_pass = sc.np.as<uint32_t>();
      }
      eng->prep_queries(qh, m, s, nullptr, sc.flat.ref());
      // Pairs and work items.
      const long long items = vcb::max_items(static_cast<long long>(m), max_probe, nb);
      sc.counts.reserve(nb * 4);
      sc.fill.reserve(nb * 4);
      sc.pstart.reserve((nb + 1) * 8);
      sc.istart.reserve((nb + 1) * 8);
      sc.pairs.reserve(m * max_probe * 4);
      sc.off.reserve(m * max_probe * 4);
      sc.items.reserve(static_cast<size_t>(items) * 16);
      sc.nitems.reserve(16);  // item count, then the scan's work counter
      vcb::PairArgs pa{};
      pa.probes = sc.top_i.as<uint32_t>();
      pa.probe_stride = ptop;
      pa.n_probe = np_pass;
      pa.fixed_probe = max_probe;
      pa.max_probe = max_probe;
      pa.nq = static_cast<long long>(m);
      pa.nb = nb;
      pa.counts = sc.counts.as<uint32_t>();
      pa.pair_start = sc.pstart.as<unsigned long long>();
      pa.item_start = sc.istart.as<unsigned long long>();
      pa.fill = sc.fill.as<uint32_t>();
      pa.pairs = sc.pairs.as<uint32_t>();
      pa.offsets = sc.off.as<float>();
      pa.items = sc.items.as<uint4>();
      pa.n_items = sc.nitems.as<unsigned long long>();
      // Offsets <q_hat, encode_c> of every probed bucket: one q_hat . enc^T
      // product per pass, gathered per pair.
      sc.encs.reserve(m * nb * 4);
      eng->launch(tq_index::kPrep, s, "offset kernel", [&] {
        return vcb::launch_gemm_nt(qh, static_cast<long long>(m), d_enc.as<float>(), nb, static_cast<int>(dim),
                                   sc.encs.as<float>(), nb, s);
      });
      pa.enc_scores = sc.encs.as<float>();
      pa.enc_ld = nb;
      const size_t lists = m * max_probe * vcb::kBsListsPerProbe;
      sc.cand_s.reserve(lists * kscan * 4);
      sc.cand_i.reserve(lists * kscan * 4);
      sc.floor.reserve(m * 4);
      const float* qf = sc.flat.qf.as<float>();
      vcb::BucketScanArgs ba{};
      ba.codes = eng->d_codes.as<uint32_t>();
      ba.alpha = eng->d_alpha.as<float>();
      ba.slot_ids = d_slot_ids.as<uint32_t>();
      ba.slot_start = d_slot_start.as<unsigned long long>();
      ba.bucket_size = d_bucket_size.as<uint32_t>();
      ba.luts = sc.flat.luts.as<uint8_t>();
      ba.lut_scale = qf;
      ba.fa_init = qf + 3 * m;
      ba.pairs = pa.pairs;
      ba.offsets = pa.offsets;
      ba.items = pa.items;
      ba.n_items = pa.n_items;
      ba.next_item = pa.n_items + 1;
      ba.nbg = static_cast<int>(nbg);
      ba.bits = static_cast<int>(bits);
      ba.k = static_cast<int>(kscan);
      ba.max_probe = max_probe;
      ba.cand_score = sc.cand_s.as<float>();
      ba.cand_id = sc.cand_i.as<uint32_t>();
      // Every (query, probe, tile set) appends its kept candidates to the
      // query's region; the merges read exactly those.
      sc.acount.reserve(m * 4);
      if (!vcb::dry_run_flag()) vcb::check(cudaMemsetAsync(sc.acount.get(), 0, m * 4, s), "cudaMemsetAsync");
      ba.append_count = sc.acount.as<uint32_t>();
      // The best-routed buckets first: the k-th best score over a query's
      // first 8 (32 from 128 probes) probes is a lower bound of its k-th best over all
      // probes, so the scan of the remaining probes keeps only scores at or
      // above it (few insertions, few candidates for the merge). The kept top
      // k is the same. The first-probe count follows each query's own n_probe
      // (per-query counts: a query with 64 probes spends 8 of them without
      // the full floor, as a fixed n_probe of 64 does, not 32).
      const bool mid_floor = static_cast<long long>(m) >= vcb::kMidFloorMinQueries;
      pa.wide_from = mid_floor ? vcb::kFloorWideFrom : vcb::kFloorWideFromSmall;
      const int first =
          std::min(max_probe >= pa.wide_from ? vcb::kFloorProbesWide : vcb::kFloorProbes, max_probe);
      const bool two_phase = max_probe > vcb::kFloorProbes;
      if (two_phase) {
        // a query's candidate region: max_probe lists of kscan entries
        const long long region = static_cast<long long>(max_probe) * vcb::kBsListsPerProbe * kscan;
        // Probe 0 alone, then probes 1..first-1 above probe 0's floor (the
        // first probes cost most without a floor), then the floor of all
        // first probes for the rest. Each floor is the k-th best of the
        // candidates appended so far, a lower bound of the final k-th best.
        // The scan grid of a step is its own item bound (pairs / 8 + buckets):
        // one probe per query, then at most first - 1 (a query's first count
        // never exceeds the one of max_probe), then at most max_probe - 1.
        // With 32 first probes, a floor after the first 8 as well: probes 8..31
        // then scan above the k-th best of 8 probes instead of probe 0's.
        int steps[4] = {0, 1, first, 0};
        int n_steps = 2;
        if (mid_floor && first > vcb::kFloorProbes) {
          steps[2] = vcb::kFloorProbes;
          steps[3] = first;
          n_steps = 3;
          // The steps are fixed now, so every query with more than 32 probes
          // (per-query counts below the wide threshold included) takes 32
          // first probes: its far probes then scan above the k-th best of 32
          // probes instead of 8, at no extra launch.
          pa.wide_from = vcb::kFloorProbesWide + 1;
        }
        for (int st = 0; st < n_steps; ++st) {
          pa.probe_begin = steps[st];
          // the last first-probe step ends at the query's own first count
          pa.probe_end = st == 0 ? 1 : (st + 1 == n_steps ? max_probe : steps[st + 1]);
          pa.first_split = st == 0 ? 0 : 1;
          const long long step_items =
              vcb::max_items(static_cast<long long>(m), steps[st + 1] - steps[st], nb);
          eng->launch(tq_index::kPrep, s, "pair kernels (first probes)",
                      [&] { return vcb::launch_build_pairs(pa, s); });
          eng->launch(tq_index::kScan, s, "bucket scan kernel (first probes)",
                      [&] { return vcb::launch_bucket_scan(ba, std::min(items, step_items), s); });
          eng->launch(tq_index::kPrep, s, "floor kernel", [&] {
            return vcb::launch_kth_floor(ba.cand_score, region, ba.append_count, static_cast<long long>(m),
                                         static_cast<int>(kscan), sc.floor.as<float>(), s);
          });
          ba.floor = sc.floor.as<float>();
        }
        pa.probe_begin = 0;
        pa.probe_end = max_probe;
        pa.first_split = 2;  // from the query's first count on
      }
      const long long last_items =
          two_phase ? std::min(items, vcb::max_items(static_cast<long long>(m), max_probe - 1, nb)) : items;
      eng->launch(tq_index::kPrep, s, "pair kernels", [&] { return vcb::launch_build_pairs(pa, s); });
      eng->launch(tq_index::kScan, s, "bucket scan kernel",
                  [&] { return vcb::launch_bucket_scan(ba, last_items, s); });
      vcb::MergeArgs mg{};
      mg.cand_score = ba.cand_score;
      mg.cand_id = ba.cand_id;
      mg.nq = static_cast<long long>(m);
      mg.n_lists = max_probe * vcb::kBsListsPerProbe;
      mg.k = static_cast<int>(kscan);
      mg.k_out = static_cast<int>(kscan);
      mg.out_score = d_scores + q0 * ke;
      mg.out_id = d_ids + q0 * ke;
      mg.entry_count = ba.append_count;
      if (rerank) {
        sc.rr_s.reserve(m * kscan * 4);
        sc.rr_i.reserve(m * kscan * 8);
        mg.out_score = sc.rr_s.as<float>();
        mg.out_id = sc.rr_i.as<uint64_t>();
        mg.pad_id = ~0ull;  // unfilled slots score -inf in the re-rank
      }
      eng->launch(tq_index::kMerge, s, "merge kernel", [&] { return vcb::launch_merge(mg, s); });
      if (rerank) {
        eng->launch(tq_index::kMerge, s, "rescore kernel", [&] {
          return vcb::launch_rescore(qh, static_cast<long long>(m), static_cast<int>(dim), d_x.as<float>(),
                                     static_cast<long long>(n), static_cast<int>(kscan), sc.rr_s.as<float>(),
                                     sc.rr_i.as<uint64_t>(), s);
        });
        eng->launch(tq_index::kMerge, s, "take kernel", [&] {
          return vcb::launch_take_columns(sc.rr_s.as<float>(), sc.rr_i.as<uint64_t>(), static_cast<long long>(m),
                                          static_cast<int>(kscan), static_cast<int>(ke), n, d_scores + q0 * ke,
                                          d_ids + q0 * ke, s);
        });
      }
      if (!vcb::dry_run_flag()) eng->scan_queries += m;
      if (trace_off) {
        vcb::check(cudaMemcpyAsync(trace_off + q0 * max_probe, sc.off.get(), m * max_probe * 4,
                                   cudaMemcpyDeviceToHost, s), "D2H");
        vcb::check(cudaMemcpyAsync(trace_probe + q0 * max_probe, sc.top_i.get(), m * max_probe * 4,
                                   cudaMemcpyDeviceToHost, s), "D2H");
        vcb::check(cudaMemcpyAsync(trace_qh + q0 * dim, sc.qh.get(), m * dim * 4, cudaMemcpyDeviceToHost, s), "D2H");
        vcb::check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
      }
    }
  }
};

namespace {

using vcb::require;

void check_params(const tq_bucket_params& p) {
  require(p.n_probe >= 1 && p.n_probe <= vcb::kMaxProbe, TQ_ERR_INVALID_ARGUMENT, "n_probe must be in [1, 2048]");
  require(p.max_bucket_size >= 2 && p.max_bucket_size <= 8192, TQ_ERR_INVALID_ARGUMENT,
          "max_bucket_size must be in [2, 8192]");
  require(p.energy_soft >= 1, TQ_ERR_INVALID_ARGUMENT, "energy_soft must be >= 1");
  require(p.rerank_k <= 256, TQ_ERR_INVALID_ARGUMENT, "rerank_k must be <= 256");
}

tq_bucketed* checked(tq_bucketed* h) {
  require(h != nullptr, TQ_ERR_INVALID_ARGUMENT, "null index");
  return h;
}

}  // namespace

extern "C" {

void tq_bucket_params_init(tq_bucket_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->n_probe = 64;
  p->max_bucket_size = 800;
  p->energy_soft = 400;
  p->kmeans_iters = 4;
  p->rerank_k = 0;
  p->reserved = 0;
  p->expected_n = 0;
  p->seed = 0x5eed5eedull;
}

int tq_bucketed_create(size_t dim, size_t bits, const tq_bucket_params* params, int device, tq_bucketed** out) {
  return vcb::guarded([&] {
    require(out != nullptr, TQ_ERR_INVALID_ARGUMENT, "out must not be NULL");
    *out = nullptr;
    require(dim >= 1 && dim <= 2048, TQ_ERR_INVALID_ARGUMENT, "dim must be in [1, 2048]");
    auto h = std::make_unique<tq_bucketed>();
    if (params) {
      h->p = *params;
    } else {
      tq_bucket_params_init(&h->p);
    }
    check_params(h->p);
    h->dim_in = dim;
    h->dim = vcb::round_up(dim, 8);  // the rotation needs a multiple of 8 coordinates
    h->bits = bits;
    tq_index* eng = nullptr;
    const int rc = tq_index_create(h->dim, bits, 0, device, &eng);
    if (rc != TQ_OK) vcb::fail(rc, tq_last_error());
    h->eng = eng;
    h->device = device;
    h->nbg = eng->nbg;
    *out = h.release();
  });
}

int tq_bucketed_destroy(tq_bucketed* h) {
  return vcb::guarded([&] {
    if (!h) return;
    vcb::DeviceGuard g(h->device);
    delete h;
  });
}

int tq_bucketed_calibrate(tq_bucketed* h, const float* sample, size_t n) {
  return vcb::guarded([&] {
    checked(h);
    require(sample != nullptr, TQ_ERR_INVALID_ARGUMENT, "null sample");
    require(n >= 2, TQ_ERR_INVALID_ARGUMENT, "calibration needs at least 2 rows");
    require(!h->built_once, TQ_ERR_STATE, "calibrate must precede prepare()");
    vcb::DeviceGuard g(h->device);
    vcb::DeviceBuffer raw;
    raw.reserve(n * h->dim_in * 4);
    h->eng->upload(raw.get(), sample, n * h->dim_in * 4);
    h->d_calib.reserve(n * h->dim * 4);
    vcb::check(vcb::launch_normalize_rows(raw.as<float>(), static_cast<long long>(n), static_cast<int>(h->dim_in),
                                          static_cast<int>(h->dim), h->d_calib.as<float>(), h->stream()),
               "normalize kernel");
    h->sync();
    h->n_calib = n;
  });
}

int tq_bucketed_add(tq_bucketed* h, const float* x, size_t n) {
  return vcb::guarded([&] {
    checked(h);
    if (n == 0) return;
    require(x != nullptr, TQ_ERR_INVALID_ARGUMENT, "null vectors");
    require(h->n + n <= 0xfffffff0ull, TQ_ERR_UNSUPPORTED, "at most 2^32 - 16 rows");
    vcb::DeviceGuard g(h->device);
    const size_t chunk = std::max<size_t>(1, (size_t{256} << 20) / (h->dim_in * 4));
    vcb::DeviceBuffer raw;
    raw.reserve(std::min(n, chunk) * h->dim_in * 4);
    for (size_t s = 0; s < n; s += chunk) {
      const size_t m = std::min(chunk, n - s);
      h->eng->upload(raw.get(), x + s * h->dim_in, m * h->dim_in * 4);
      h->add_rows(raw.as<float>(), m, h->stream());
      h->sync();
    }
    h->prepared = false;
  });
}

int tq_bucketed_add_device(tq_bucketed* h, const float* d_x, size_t n, void* stream) {
  return vcb::guarded([&] {
    checked(h);
    if (n == 0) return;
    require(d_x != nullptr, TQ_ERR_INVALID_ARGUMENT, "null vectors");
    require(h->n + n <= 0xfffffff0ull, TQ_ERR_UNSUPPORTED, "at most 2^32 - 16 rows");
    vcb::DeviceGuard g(h->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->stream();
    if (s != h->stream()) h->sync();
    h->add_rows(d_x, n, s);
    vcb::check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    h->prepared = false;
  });
}

int tq_bucketed_prepare(tq_bucketed* h) {
  return vcb::guarded([&] {
    checked(h);
    if (h->prepared) return;
    require(h->n > 0, TQ_ERR_STATE, "prepare with empty index");
    vcb::DeviceGuard g(h->device);
    h->build();
  });
}

int tq_bucketed_search_device(tq_bucketed* h, const float* d_queries, size_t nq, size_t k, size_t n_probe,
                              const uint32_t* d_n_probe, float* d_scores, uint64_t* d_ids, size_t* k_eff,
                              void* stream) {
  return vcb::guarded([&] {
    checked(h);
    require(h->prepared, TQ_ERR_STATE, "search before prepare");
    require(k <= static_cast<size_t>(vcb::kMaxK), TQ_ERR_UNSUPPORTED, "k must be <= 256");
    const size_t ke = std::min(k, h->n);
    if (k_eff) *k_eff = ke;
    if (nq == 0 || ke == 0) return;
    require(d_queries && d_scores && d_ids, TQ_ERR_INVALID_ARGUMENT, "null buffer");
    const size_t np = n_probe ? n_probe : h->p.n_probe;
    require(np >= 1 && np <= static_cast<size_t>(vcb::kMaxProbe), TQ_ERR_INVALID_ARGUMENT, "n_probe must be in [1, 2048]");
    vcb::DeviceGuard g(h->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->stream();
    h->search_device(d_queries, nq, ke, static_cast<int>(std::min<size_t>(np, h->nb)), d_n_probe, d_scores, d_ids,
                     s);
  });
}

int tq_bucketed_search(tq_bucketed* h, const float* queries, size_t nq, size_t k, size_t n_probe,
                       const uint32_t* n_probe_per_query, float* scores, uint64_t* ids, size_t* k_eff) {
  return vcb::guarded([&] {
    checked(h);
    require(h->prepared, TQ_ERR_STATE, "search before prepare");
    require(k <= static_cast<size_t>(vcb::kMaxK), TQ_ERR_UNSUPPORTED, "k must be <= 256");
    const size_t ke = std::min(k, h->n);
    if (k_eff) *k_eff = ke;
    if (nq == 0 || ke == 0) return;
    require(queries && scores && ids, TQ_ERR_INVALID_ARGUMENT, "null buffer");
    const size_t np = n_probe ? n_probe : h->p.n_probe;
    require(np >= 1 && np <= static_cast<size_t>(vcb::kMaxProbe), TQ_ERR_INVALID_ARGUMENT, "n_probe must be in [1, 2048]");
    vcb::DeviceGuard g(h->device);
    h->s_q.reserve(nq * h->dim_in * 4);
    h->s_out_s.reserve(nq * ke * 4);
    h->s_out_i.reserve(nq * ke * 8);
    h->eng->upload(h->s_q.get(), queries, nq * h->dim_in * 4);
    const uint32_t* d_np = nullptr;
    if (n_probe_per_query) {
      h->s_np.reserve(nq * 4);
      h->eng->upload(h->s_np.get(), n_probe_per_query, nq * 4);
      d_np = h->s_np.as<uint32_t>();
    }
    h->search_device(h->s_q.as<float>(), nq, ke, static_cast<int>(std::min<size_t>(np, h->nb)), d_np,
                     h->s_out_s.as<float>(), h->s_out_i.as<uint64_t>(), h->stream());
    vcb::check(cudaMemcpyAsync(scores, h->s_out_s.get(), nq * ke * 4, cudaMemcpyDeviceToHost, h->stream()), "D2H");
    vcb::check(cudaMemcpyAsync(ids, h->s_out_i.get(), nq * ke * 8, cudaMemcpyDeviceToHost, h->stream()), "D2H");
    h->sync();
  });
}

int tq_bucketed_search_trace(tq_bucketed* h, const float* queries, size_t nq, size_t k, size_t n_probe,
                             const uint32_t* n_probe_per_query, float* scores, uint64_t* ids, size_t* k_eff,
                             uint32_t* probes, float* offsets, float* q_hat) {
  return vcb::guarded([&] {
    checked(h);
    require(h->prepared, TQ_ERR_STATE, "search before prepare");
    require(probes && offsets && q_hat, TQ_ERR_INVALID_ARGUMENT, "null trace buffer");
    const size_t ke = std::min(k, h->n);
    if (k_eff) *k_eff = ke;
    require(k >= 1 && k <= static_cast<size_t>(vcb::kMaxK), TQ_ERR_UNSUPPORTED, "k must be in [1, 256]");
    const size_t np = std::min<size_t>(n_probe ? n_probe : h->p.n_probe, h->nb);
    if (nq == 0) return;
    vcb::DeviceGuard g(h->device);
    h->s_q.reserve(nq * h->dim_in * 4);
    h->s_out_s.reserve(nq * ke * 4);
    h->s_out_i.reserve(nq * ke * 8);
    h->eng->upload(h->s_q.get(), queries, nq * h->dim_in * 4);
    const uint32_t* d_np = nullptr;
    if (n_probe_per_query) {
      h->s_np.reserve(nq * 4);
      h->eng->upload(h->s_np.get(), n_probe_per_query, nq * 4);
      d_np = h->s_np.as<uint32_t>();
    }
    h->search_device(h->s_q.as<float>(), nq, ke, static_cast<int>(np), d_np, h->s_out_s.as<float>(),
                     h->s_out_i.as<uint64_t>(), h->stream(), offsets, probes, q_hat);
    vcb::check(cudaMemcpyAsync(scores, h->s_out_s.get(), nq * ke * 4, cudaMemcpyDeviceToHost, h->stream()), "D2H");
    vcb::check(cudaMemcpyAsync(ids, h->s_out_i.get(), nq * ke * 8, cudaMemcpyDeviceToHost, h->stream()), "D2H");
    h->sync();
  });
}

int tq_bucketed_search_learned_device(tq_bucketed* h, const float* d_queries, size_t nq, size_t k,
                                      tq_probe_mlp* mlp, float coverage, float min_confidence,
                                      size_t fallback_n_probe, float* d_scores, uint64_t* d_ids, size_t* k_eff,
                                      void* stream) {
  return vcb::guarded([&] {
    checked(h);
    require(mlp != nullptr, TQ_ERR_INVALID_ARGUMENT, "null model");
    require(h->prepared, TQ_ERR_STATE, "search before prepare");
    require(k <= static_cast<size_t>(vcb::kMaxK), TQ_ERR_UNSUPPORTED, "k must be <= 256");
    const size_t ke = std::min(k, h->n);
    if (k_eff) *k_eff = ke;
    if (nq == 0 || ke == 0) return;
    require(d_queries && d_scores && d_ids, TQ_ERR_INVALID_ARGUMENT, "null buffer");
    const size_t np = fallback_n_probe ? fallback_n_probe : h->p.n_probe;
    require(np >= 1 && np <= static_cast<size_t>(vcb::kMaxProbe), TQ_ERR_INVALID_ARGUMENT,
            "fallback n_probe must be in [1, 2048]");
    vcb::DeviceGuard g(h->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->stream();
    const vcb::LearnedProbe lp{mlp, coverage, min_confidence};
    h->search_device(d_queries, nq, ke, static_cast<int>(std::min<size_t>(np, h->nb)), nullptr, d_scores, d_ids, s,
                     h->own, nullptr, nullptr, nullptr, &lp);
  });
}

int tq_select_top_device(const float* d_scores, size_t rows, size_t ld, size_t ncols, size_t p, float* d_top_scores,
                         uint32_t* d_top_ids, int device, void* stream) {
  return vcb::guarded([&] {
    require(p >= 1 && p <= static_cast<size_t>(vcb::kMaxProbe), TQ_ERR_INVALID_ARGUMENT, "p must be in [1, 2048]");
    require(ncols <= ld || rows <= 1, TQ_ERR_INVALID_ARGUMENT, "ncols must be <= ld");
    require(ncols <= 0x7fffffffu, TQ_ERR_INVALID_ARGUMENT, "ncols too large");
    if (rows == 0) return;
    require(d_scores && d_top_scores && d_top_ids, TQ_ERR_INVALID_ARGUMENT, "null buffer");
    vcb::DeviceGuard g(device);
    vcb::check(vcb::launch_select_top(d_scores, static_cast<long long>(rows), static_cast<long long>(ld),
                                      static_cast<int>(ncols), static_cast<int>(p), d_top_scores, d_top_ids,
                                      static_cast<cudaStream_t>(stream)),
               "select kernel");
  });
}

int tq_bucketed_route_device(tq_bucketed* h, const float* d_queries, size_t nq, size_t p, float* d_top_scores,
                             uint32_t* d_top_ids, void* stream) {
  return vcb::guarded([&] {
    checked(h);
    require(h->prepared, TQ_ERR_STATE, "route before prepare");
    require(p >= 1 && p <= static_cast<size_t>(vcb::kMaxProbe), TQ_ERR_INVALID_ARGUMENT, "p must be in [1, 2048]");
    if (nq == 0) return;
    require(d_queries && d_top_scores && d_top_ids, TQ_ERR_INVALID_ARGUMENT, "null buffer");
    vcb::DeviceGuard g(h->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->stream();
    const size_t pass = h->pass_queries();
    for (size_t q0 = 0; q0 < nq; q0 += pass) {
      const size_t m = std::min(pass, nq - q0);
      h->own.qh.reserve(m * h->dim * 4);
      vcb::check(vcb::launch_normalize_rows(d_queries + q0 * h->dim_in, static_cast<long long>(m),
                                            static_cast<int>(h->dim_in), static_cast<int>(h->dim),
                                            h->own.qh.as<float>(), s),
                 "normalize kernel");
      h->own.route.reserve(m * h->nb * 4);
      vcb::check(vcb::launch_gemm_nt(h->own.qh.as<float>(), static_cast<long long>(m), h->d_route.as<float>(), h->nb,
                                     static_cast<int>(h->dim), h->own.route.as<float>(), h->nb, s),
                 "routing kernel");
      vcb::check(vcb::launch_select_top(h->own.route.as<float>(), static_cast<long long>(m), h->nb, h->nb,
                                        static_cast<int>(p), d_top_scores + q0 * p, d_top_ids + q0 * p, s),
                 "select kernel");
    }
  });
}

int tq_bucketed_route(tq_bucketed* h, const float* queries, size_t nq, float* q_hat, float* scores) {
  return vcb::guarded([&] {
    checked(h);
    require(h->prepared, TQ_ERR_STATE, "route before prepare");
    if (nq == 0) return;
    require(queries != nullptr, TQ_ERR_INVALID_ARGUMENT, "null queries");
    vcb::DeviceGuard g(h->device);
    h->s_q.reserve(nq * h->dim_in * 4);
    h->own.qh.reserve(nq * h->dim * 4);
    h->own.route.reserve(nq * h->nb * 4);
    h->eng->upload(h->s_q.get(), queries, nq * h->dim_in * 4);
    vcb::check(vcb::launch_normalize_rows(h->s_q.as<float>(), static_cast<long long>(nq), static_cast<int>(h->dim_in),
                                          static_cast<int>(h->dim), h->own.qh.as<float>(), h->stream()),
               "normalize kernel");
    vcb::check(vcb::launch_gemm_nt(h->own.qh.as<float>(), static_cast<long long>(nq), h->d_route.as<float>(), h->nb,
                                   static_cast<int>(h->dim), h->own.route.as<float>(), h->nb, h->stream()),
               "routing kernel");
    if (q_hat) {
      vcb::check(cudaMemcpyAsync(q_hat, h->own.qh.get(), nq * h->dim * 4, cudaMemcpyDeviceToHost, h->stream()), "D2H");
    }
    if (scores) {
      vcb::check(cudaMemcpyAsync(scores, h->own.route.get(), nq * h->nb * 4, cudaMemcpyDeviceToHost, h->stream()),
                 "D2H");
    }
    h->sync();
  });
}

int tq_bucketed_info(const tq_bucketed* h, size_t* dim, size_t* dim_padded, size_t* bits, size_t* n,
                     size_t* n_buckets, size_t* n_slots, int* prepared) {
  return vcb::guarded([&] {
    require(h != nullptr, TQ_ERR_INVALID_ARGUMENT, "null index");
    if (dim) *dim = h->dim_in;
    if (dim_padded) *dim_padded = h->dim;
    if (bits) *bits = h->bits;
    if (n) *n = h->n;
    if (n_buckets) *n_buckets = static_cast<size_t>(h->nb);
    if (n_slots) *n_slots = h->n_slots;
    if (prepared) *prepared = h->prepared ? 1 : 0;
  });
}

int tq_bucketed_export_layout(tq_bucketed* h, uint64_t* slot_start, uint32_t* bucket_size, uint32_t* slot_ids,
                              uint32_t* labels) {
  return vcb::guarded([&] {
    checked(h);
    require(h->prepared, TQ_ERR_STATE, "export before prepare");
    vcb::DeviceGuard g(h->device);
    if (slot_start) std::memcpy(slot_start, h->h_slot_start.data(), (h->nb + 1) * 8);
    if (bucket_size) std::memcpy(bucket_size, h->h_size.data(), h->nb * 4);
    if (slot_ids) {
      vcb::check(cudaMemcpyAsync(slot_ids, h->d_slot_ids.get(), h->n_slots * 4, cudaMemcpyDeviceToHost, h->stream()),
                 "D2H");
    }
    if (labels) {
      vcb::check(cudaMemcpyAsync(labels, h->d_label.get(), h->n * 4, cudaMemcpyDeviceToHost, h->stream()), "D2H");
    }
    h->sync();
  });
}

int tq_bucketed_export_centroids(tq_bucketed* h, float* route, float* enc) {
  return vcb::guarded([&] {
    checked(h);
    require(h->prepared, TQ_ERR_STATE, "export before prepare");
    vcb::DeviceGuard g(h->device);
    if (route) {
      vcb::check(cudaMemcpyAsync(route, h->d_route.get(), h->nb * h->dim * 4, cudaMemcpyDeviceToHost, h->stream()),
                 "D2H");
    }
    if (enc) {
      vcb::check(cudaMemcpyAsync(enc, h->d_enc.get(), h->nb * h->dim * 4, cudaMemcpyDeviceToHost, h->stream()),
                 "D2H");
    }
    h->sync();
  });
}

int tq_bucketed_export_rows(tq_bucketed* h, float* x_hat) {
  return vcb::guarded([&] {
    checked(h);
    require(x_hat != nullptr, TQ_ERR_INVALID_ARGUMENT, "null output");
    vcb::DeviceGuard g(h->device);
    vcb::check(cudaMemcpyAsync(x_hat, h->d_x.get(), h->n * h->dim * 4, cudaMemcpyDeviceToHost, h->stream()), "D2H");
    h->sync();
  });
}

int tq_bucketed_engine(tq_bucketed* h, tq_index** engine) {
  return vcb::guarded([&] {
    checked(h);
    require(engine != nullptr, TQ_ERR_INVALID_ARGUMENT, "null output");
    *engine = h->eng;
  });
}

}  // extern "C"

// ---- hooks for the serving loop (tq_server.cu) ------------------------------
namespace vcb {

BucketScratch* bucket_scratch_new() { return new BucketScratch(); }
void bucket_scratch_delete(BucketScratch* sc) { delete sc; }
void bucket_scratch_bind(BucketScratch* sc, ScratchArena* a) { sc->bind(a); }

size_t bucketed_dim_in(const tq_bucketed* h) { return h->dim_in; }
size_t bucketed_size(const tq_bucketed* h) { return h->n; }
bool bucketed_prepared(const tq_bucketed* h) { return h->prepared; }

// One search of nq device queries with caller-owned scratch on stream s; the
// learned probe when lp is not null (n_probe is then its maximum / fallback).
size_t bucketed_search_with(tq_bucketed* h, const float* d_q, size_t nq, size_t k, size_t n_probe,
                            const LearnedProbe* lp, float* d_scores, uint64_t* d_ids, cudaStream_t s,
                            BucketScratch& sc) {
  const size_t ke = std::min(k, h->n);
  if (nq == 0 || ke == 0) return ke;
  const size_t np = std::min<size_t>(n_probe ? n_probe : h->p.n_probe, static_cast<size_t>(h->nb));
  h->search_device(d_q, nq, ke, static_cast<int>(np), nullptr, d_scores, d_ids, s, sc, nullptr, nullptr, nullptr, lp);
  return ke;
}

}  // namespace vcb
