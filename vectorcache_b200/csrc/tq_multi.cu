// Multi-index search: one persistent, CUDA-graph-captured scan launch serving
// many flat indexes of uneven n, dim and bits with uneven query batches. No
// counterpart in the reference (its flat search serves one index per call:
// search.cpp:1293-1302).
//
// A plan fixes the batch size and k of every index. Work items are (index,
// vector range, up to 8 of its queries); the persistent scan kernel
// (tq_bucket.cu: multi_scan_kernel) pulls them from a global counter, so large
// and small indexes share the GPU in one launch. The captured graph is: the
// query-LUT kernel of every index (each index has its own rotation and
// codebook), the counter reset, the one scan launch, and the merge of every
// index's candidate lists. Per query the arithmetic and the exact (score desc,
// id asc) top-k are those of the flat search, so results equal the per-index
// search bit for bit.
//
// The autotuner times candidates on the planned workload itself (CUDA events,
// one untimed and one timed run each), in three passes: the vector-range
// length of a work item, the resident CTAs per SM, and how many of the
// heaviest index batches run the single-index scan kernels (inside the same
// graph) instead of the persistent launch; then it captures the graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/vectorcache_b200.h"
#include "tq_abi.h"
#include "tq_bucket.h"
#include "tq_index_impl.h"
#include "tq_kernels.h"

struct tq_multi {
  int device = 0, sms = 148;
  cudaStream_t stream = nullptr;
  std::vector<tq_index*> idx;
  // plan
  std::vector<size_t> nq, k, ke;
  std::vector<char> direct;  // index runs the single-index kernels instead of the persistent launch
  size_t n_direct = 0;
  std::vector<std::unique_ptr<vcb::FlatScratchStore>> scratch;
  std::vector<std::unique_ptr<vcb::DeviceBuffer>> d_q, d_s, d_i;
  vcb::DeviceBuffer d_desc, d_items, d_counter;
  std::vector<vcb::MultiIndexDesc> descs;
  std::vector<vcb::MultiItem> items;
  long long range_vectors = 8192;
  int ctas = 0;
  size_t smem = 0;
  bool any3 = false, any24 = false;
  bool planned = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<double> tuned_ms;  // per candidate, for the report

  ~tq_multi() {
    if (stream) cudaStreamSynchronize(stream);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (stream) cudaStreamDestroy(stream);
  }

  // Items and descriptors for a range length; sizes the scratch.
  void build_items(long long rv) {
    range_vectors = rv;
    descs.clear();
    items.clear();
    int max_nbg = 1, max_k = 1;
    any3 = any24 = false;
    struct Cost {
      double cost;
      vcb::MultiItem it;
    };
    std::vector<Cost> all;
    for (size_t i = 0; i < idx.size(); ++i) {
      tq_index* h = idx[i];
      vcb::MultiIndexDesc d{};
      d.codes = h->d_codes.as<uint32_t>();
      d.alpha = h->d_alpha.as<float>();
      d.n = static_cast<long long>(h->n);
      d.range_vectors = rv;
      d.n_ranges = static_cast<int>((h->n + rv - 1) / rv);
      d.nbg = static_cast<int>(h->nbg);
      d.bits = static_cast<int>(h->bits);
      d.k = static_cast<int>(ke[i]);
      auto& sc = *scratch[i];
      sc.luts.reserve(std::max<size_t>(nq[i], 1) * h->nbg * 32);
      sc.qf.reserve(std::max<size_t>(nq[i], 1) * 4 * sizeof(float));
      const size_t lists = nq[i] * static_cast<size_t>(d.n_ranges) * 2;
      sc.cand_s.reserve(std::max<size_t>(lists * ke[i], 1) * 4);
      sc.cand_i.reserve(std::max<size_t>(lists * ke[i], 1) * 4);
      d.luts = sc.luts.as<uint8_t>();
      d.lut_scale = sc.qf.as<float>();
      d.fa_init = sc.qf.as<float>() + 3 * nq[i];
      d.cand_s = sc.cand_s.as<float>();
      d.cand_i = sc.cand_i.as<uint32_t>();
      descs.push_back(d);
      if (nq[i] == 0 || ke[i] == 0 || direct[i]) continue;
      max_nbg = std::max(max_nbg, d.nbg);
      max_k = std::max(max_k, d.k);
      (d.bits == 3 ? any3 : any24) = true;
      for (int r = 0; r < d.n_ranges; ++r) {
        const long long size = std::min<long long>(rv, d.n - static_cast<long long>(r) * rv);
        for (size_t q0 = 0; q0 < nq[i]; q0 += vcb::kItemQueries) {
          const int cnt = static_cast<int>(std::min<size_t>(vcb::kItemQueries, nq[i] - q0));
          // Cost: lookups of the item's busiest warp pair (queries in quads).
          const double cost = static_cast<double>(size) * d.nbg * ((cnt + 3) / 4);
          all.push_back({cost, vcb::MultiItem{static_cast<int>(i), r, static_cast<int>(q0), cnt}});
        }
      }
    }
    // Largest items first: the tail of the persistent launch is made of small ones.
    std::stable_sort(all.begin(), all.end(), [](const Cost& a, const Cost& b) { return a.cost > b.cost; });
    for (const Cost& c : all) items.push_back(c.it);
    smem = vcb::multi_scan_smem_bytes(max_nbg, max_k);
    d_desc.reserve(std::max<size_t>(descs.size(), 1) * sizeof(vcb::MultiIndexDesc));
    d_items.reserve(std::max<size_t>(items.size(), 1) * sizeof(vcb::MultiItem));
    vcb::check(cudaMemcpyAsync(d_desc.get(), descs.data(), descs.size() * sizeof(vcb::MultiIndexDesc),
                               cudaMemcpyHostToDevice, stream),
               "H2D");
    if (!items.empty()) {
      vcb::check(cudaMemcpyAsync(d_items.get(), items.data(), items.size() * sizeof(vcb::MultiItem),
                                 cudaMemcpyHostToDevice, stream),
                 "H2D");
    }
    vcb::check(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
  }

  // The whole multi-index search on stream s (what the graph captures):
  // indexes marked `direct` run the single-index scan kernels (best for the
  // heaviest index batches), all others share the one persistent launch.
  void run(cudaStream_t s) {
    for (size_t i = 0; i < idx.size(); ++i) {
      if (nq[i] == 0 || ke[i] == 0 || !direct[i]) continue;
      idx[i]->search_device(d_q[i]->as<float>(), nq[i], k[i], d_s[i]->as<float>(), d_i[i]->as<uint64_t>(), ke[i], s,
                            scratch[i]->ref());
    }
    for (size_t i = 0; i < idx.size(); ++i) {
      if (nq[i] == 0 || ke[i] == 0 || direct[i]) continue;
      idx[i]->prep_queries(d_q[i]->as<float>(), nq[i], s, nullptr, scratch[i]->ref());
    }
    vcb::check(cudaMemsetAsync(d_counter.get(), 0, 8, s), "cudaMemsetAsync");
    vcb::MultiScanArgs a{};
    a.indexes = d_desc.as<vcb::MultiIndexDesc>();
    a.items = d_items.as<vcb::MultiItem>();
    a.n_items = static_cast<long long>(items.size());
    a.next_item = d_counter.as<unsigned long long>();
    vcb::check(vcb::launch_multi_scan(a, ctas, smem, any3, any24, s), "multi scan kernel");
    for (size_t i = 0; i < idx.size(); ++i) {
      if (nq[i] == 0 || ke[i] == 0 || direct[i]) continue;
      vcb::MergeArgs mg{};
      mg.cand_score = descs[i].cand_s;
      mg.cand_id = descs[i].cand_i;
      mg.nq = static_cast<long long>(nq[i]);
      mg.n_lists = descs[i].n_ranges * 2;
      mg.k = static_cast<int>(ke[i]);
      mg.k_out = static_cast<int>(ke[i]);
      mg.out_score = d_s[i]->as<float>();
      mg.out_id = d_i[i]->as<uint64_t>();
      vcb::check(vcb::launch_merge(mg, s), "merge kernel");
    }
  }

  double time_ms(int reps) {
    cudaEvent_t e0, e1;
    vcb::check(cudaEventCreate(&e0), "cudaEventCreate");
    vcb::check(cudaEventCreate(&e1), "cudaEventCreate");
    std::vector<double> t;
    for (int r = 0; r < reps; ++r) {
      vcb::check(cudaEventRecord(e0, stream), "cudaEventRecord");
      run(stream);
      vcb::check(cudaEventRecord(e1, stream), "cudaEventRecord");
      vcb::check(cudaEventSynchronize(e1), "cudaEventSynchronize");
      float ms = 0.f;
      vcb::check(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
      t.push_back(ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::sort(t.begin(), t.end());
    return t[t.size() / 2];
  }

  void capture() {
    if (exec) {
      cudaGraphExecDestroy(exec);
      exec = nullptr;
    }
    if (graph) {
      cudaGraphDestroy(graph);
      graph = nullptr;
    }
    run(stream);  // grows every scratch buffer outside the capture
    vcb::check(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    vcb::check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    try {
      run(stream);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    vcb::check(cudaStreamEndCapture(stream, &graph), "cudaStreamEndCapture");
    vcb::check(cudaGraphInstantiate(&exec, graph, 0), "cudaGraphInstantiate");
  }
};

namespace {

using vcb::require;

tq_multi* checked(tq_multi* h) {
  require(h != nullptr, TQ_ERR_INVALID_ARGUMENT, "null multi-index handle");
  return h;
}

}  // namespace

extern "C" {

int tq_multi_create(tq_index* const* indexes, size_t n_indexes, tq_multi** out) {
  return vcb::guarded([&] {
    require(out != nullptr && indexes != nullptr, TQ_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    require(n_indexes >= 1, TQ_ERR_INVALID_ARGUMENT, "need at least one index");
    auto h = std::make_unique<tq_multi>();
    for (size_t i = 0; i < n_indexes; ++i) {
      tq_index* x = indexes[i];
      require(x != nullptr && x->prepared, TQ_ERR_STATE, "every index must be prepared");
      require(x->device == indexes[0]->device, TQ_ERR_INVALID_ARGUMENT, "indexes on different devices");
      require(x->n <= 0x7fffffffull, TQ_ERR_UNSUPPORTED, "index larger than 2^31 vectors");
      h->idx.push_back(x);
    }
    h->device = indexes[0]->device;
    vcb::DeviceGuard g(h->device);
    h->sms = indexes[0]->sms;
    vcb::check(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    h->d_counter.reserve(8);
    *out = h.release();
  });
}

int tq_multi_destroy(tq_multi* h) {
  return vcb::guarded([&] {
    if (!h) return;
    vcb::DeviceGuard g(h->device);
    delete h;
  });
}

int tq_multi_plan(tq_multi* h, const size_t* nq, const size_t* k, int autotune) {
  return vcb::guarded([&] {
    checked(h);
    require(nq != nullptr && k != nullptr, TQ_ERR_INVALID_ARGUMENT, "null argument");
    vcb::DeviceGuard g(h->device);
    const size_t m = h->idx.size();
    h->nq.assign(nq, nq + m);
    h->k.assign(k, k + m);
    h->ke.resize(m);
    h->direct.assign(m, 0);
    h->n_direct = 0;
    h->scratch.clear();
    h->d_q.clear();
    h->d_s.clear();
    h->d_i.clear();
    for (size_t i = 0; i < m; ++i) {
      require(k[i] >= 1 && k[i] <= static_cast<size_t>(vcb::kMaxK), TQ_ERR_INVALID_ARGUMENT, "k must be in [1, 256]");
      h->ke[i] = std::min(k[i], h->idx[i]->n);
      h->scratch.push_back(std::make_unique<vcb::FlatScratchStore>());
      h->d_q.push_back(std::make_unique<vcb::DeviceBuffer>());
      h->d_s.push_back(std::make_unique<vcb::DeviceBuffer>());
      h->d_i.push_back(std::make_unique<vcb::DeviceBuffer>());
      h->d_q[i]->reserve(std::max<size_t>(nq[i], 1) * h->idx[i]->dim * 4);
      h->d_s[i]->reserve(std::max<size_t>(nq[i] * h->ke[i], 1) * 4);
      h->d_i[i]->reserve(std::max<size_t>(nq[i] * h->ke[i], 1) * 8);
      vcb::check(cudaMemsetAsync(h->d_q[i]->get(), 0, std::max<size_t>(nq[i], 1) * h->idx[i]->dim * 4, h->stream),
                 "cudaMemsetAsync");
    }
    // Autotuner, two passes over the planned workload itself: the item range
    // length at the most resident CTAs, then the resident CTAs per SM at that
    // length. Each candidate: one untimed run (grows scratch, loads kernels),
    // one timed run (CUDA events).
    h->tuned_ms.clear();
    long long best_rv = 8192;
    if (autotune) {
      const long long ranges[] = {4096, 8192, 16384, 32768};
      double best = -1.0;
      for (long long rv : ranges) {
        h->build_items(rv);
        h->ctas = h->sms * std::max(1, vcb::multi_scan_ctas_per_sm(h->smem, h->any3));
        h->time_ms(1);
        const double ms = h->time_ms(1);
        h->tuned_ms.push_back(ms);
        if (best < 0 || ms < best) {
          best = ms;
          best_rv = rv;
        }
      }
    }
    h->build_items(best_rv);
    const int per_sm = std::max(1, vcb::multi_scan_ctas_per_sm(h->smem, h->any3));
    int best_c = per_sm;
    if (autotune && per_sm > 1) {
      double best = -1.0;
      for (int c = 1; c <= per_sm; ++c) {
        h->ctas = h->sms * c;
        const double ms = h->time_ms(1);
        h->tuned_ms.push_back(ms);
        if (best < 0 || ms < best) {
          best = ms;
          best_c = c;
        }
      }
    }
    h->ctas = h->sms * best_c;
    // Third pass: how many of the heaviest index batches (nq x n x byte groups)
    // go to the single-index kernels instead of the persistent launch.
    if (autotune) {
      std::vector<size_t> order(m);
      std::iota(order.begin(), order.end(), size_t{0});
      auto work = [&](size_t i) {
        return static_cast<double>(h->nq[i]) * static_cast<double>(h->idx[i]->n) * static_cast<double>(h->idx[i]->nbg);
      };
      std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return work(a) > work(b); });
      auto set_direct = [&](size_t d) {
        h->direct.assign(m, 0);
        for (size_t t = 0; t < d; ++t) h->direct[order[t]] = 1;
        h->n_direct = d;
        h->build_items(best_rv);
        const int ps = std::max(1, vcb::multi_scan_ctas_per_sm(h->smem, h->any3));
        h->ctas = h->sms * std::min(best_c, ps);
      };
      set_direct(0);
      double best = h->time_ms(1);
      size_t best_d = 0;
      for (size_t d : {size_t{1}, size_t{2}, size_t{4}, size_t{8}, size_t{16}, m}) {
        if (d > m || d == 0) continue;
        set_direct(d);
        h->time_ms(1);
        const double ms = h->time_ms(1);
        h->tuned_ms.push_back(ms);
        if (ms < best) {
          best = ms;
          best_d = d;
        }
        if (d == m) break;
      }
      set_direct(best_d);
    }
    h->capture();
    h->planned = true;
  });
}

int tq_multi_buffers(tq_multi* h, size_t i, float** d_queries, float** d_scores, uint64_t** d_ids, size_t* k_eff) {
  return vcb::guarded([&] {
    checked(h);
    require(h->planned, TQ_ERR_STATE, "plan() first");
    require(i < h->idx.size(), TQ_ERR_INVALID_ARGUMENT, "no such index");
    if (d_queries) *d_queries = h->d_q[i]->as<float>();
    if (d_scores) *d_scores = h->d_s[i]->as<float>();
    if (d_ids) *d_ids = h->d_i[i]->as<uint64_t>();
    if (k_eff) *k_eff = h->ke[i];
  });
}

int tq_multi_launch(tq_multi* h, void* stream) {
  return vcb::guarded([&] {
    checked(h);
    require(h->planned, TQ_ERR_STATE, "plan() first");
    vcb::DeviceGuard g(h->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->stream;
    vcb::check(cudaGraphLaunch(h->exec, s), "cudaGraphLaunch");
  });
}

int tq_multi_run_uncaptured(tq_multi* h, void* stream) {
  return vcb::guarded([&] {
    checked(h);
    require(h->planned, TQ_ERR_STATE, "plan() first");
    vcb::DeviceGuard g(h->device);
    h->run(stream ? static_cast<cudaStream_t>(stream) : h->stream);
  });
}

int tq_multi_synchronize(tq_multi* h) {
  return vcb::guarded([&] {
    checked(h);
    vcb::DeviceGuard g(h->device);
    vcb::check(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
  });
}

int tq_multi_config(tq_multi* h, long long* range_vectors, int* ctas, size_t* n_items, size_t* smem_bytes,
                    double* tuned_ms, size_t* n_tuned) {
  return vcb::guarded([&] {
    checked(h);
    require(h->planned, TQ_ERR_STATE, "plan() first");
    if (range_vectors) *range_vectors = h->range_vectors;
    if (ctas) *ctas = h->ctas;
    if (n_items) *n_items = h->items.size();
    if (smem_bytes) *smem_bytes = h->smem;
    if (n_tuned) {
      const size_t cap = *n_tuned;
      *n_tuned = h->tuned_ms.size();
      if (tuned_ms) std::copy_n(h->tuned_ms.begin(), std::min(cap, h->tuned_ms.size()), tuned_ms);
    }
  });
}

}  // extern "C"

extern "C" {

int tq_copy_to_device(void* d_dst, const void* src, size_t bytes) {
  return vcb::guarded([&] {
    require(d_dst != nullptr && (src != nullptr || bytes == 0), TQ_ERR_INVALID_ARGUMENT, "null argument");
    if (bytes) vcb::check(cudaMemcpy(d_dst, src, bytes, cudaMemcpyHostToDevice), "cudaMemcpy H2D");
  });
}

int tq_copy_to_host(void* dst, const void* d_src, size_t bytes) {
  return vcb::guarded([&] {
    require(dst != nullptr && (d_src != nullptr || bytes == 0), TQ_ERR_INVALID_ARGUMENT, "null argument");
    if (bytes) vcb::check(cudaMemcpy(dst, d_src, bytes, cudaMemcpyDeviceToHost), "cudaMemcpy D2H");
  });
}

}  // extern "C"

extern "C" int tq_multi_direct(tq_multi* h, size_t* n_direct, uint8_t* flags) {
  return vcb::guarded([&] {
    checked(h);
    require(h->planned, TQ_ERR_STATE, "plan() first");
    if (n_direct) *n_direct = h->n_direct;
    if (flags) {
      for (size_t i = 0; i < h->direct.size(); ++i) flags[i] = static_cast<uint8_t>(h->direct[i]);
    }
  });
}
