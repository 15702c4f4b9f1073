// Serving loop: continuous batching of search requests over resident flat and
// bucketed indexes on one GPU. No counterpart in the reference.
//
// A request (index, nq host queries, k, n_probe) waits in a FIFO queue. A
// worker thread owns S slots; each slot has its own CUDA stream, pinned host
// staging, device query / result buffers and search scratch, so batches in
// different slots run concurrently on the device. Whenever a slot is free the
// worker admits the oldest waiting request together with every later waiting
// request it can share a launch with (same index, k and n_probe) up to
// max_batch queries — requests that arrive while others run join the next
// launch — copies their queries into the slot, queues H2D copy, search and D2H
// copy on the slot's stream, and marks the completion time from a host
// callback queued after the copy. Slots are created at start() only while the
// device memory in use (resident indexes included) stays within the HBM
// budget; each slot's scratch is grown there, by one full-size warm-up search
// per index (and a two-query one for the batch-split scan of small flat
// batches), so serving itself allocates nothing.
//
// Every query's result is computed independently of the other queries of its
// batch (per-query LUTs and an exact top-k), so a result is the same whether
// the request ran alone or in a mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <random>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/vectorcache_b200.h"
#include "tq_abi.h"
#include "tq_index_impl.h"
#include "tq_serving_hooks.h"

namespace {

// Vectors per scan CTA of a served flat search: a 10M x 768 3-bit scan of 128
// queries then runs in CTAs of a few ms, so bucketed batches on the
// high-priority stream wait at most that long for an SM.
constexpr long long kServingRangeVectors = 65536;

int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

struct Target {
  tq_index* flat = nullptr;
  tq_bucketed* bkt = nullptr;
  tq_probe_mlp* mlp = nullptr;
  float coverage = 0.9f, min_conf = 0.f;
  size_t dim_in = 0, max_k = 0, max_probe = 0;
};

struct Request {
  uint64_t id = 0;
  int target = 0;
  const float* q = nullptr;
  size_t nq = 0, k = 0, n_probe = 0;
  float* out_s = nullptr;
  uint64_t* out_i = nullptr;
  int64_t t_arrive = 0, t_done = 0;
  size_t k_eff = 0;
  bool done = false;
  int status = TQ_OK;
  std::string error;
};

struct Slot {
  cudaStream_t stream = nullptr;     // flat batches (normal priority)
  cudaStream_t stream_hi = nullptr;  // bucketed batches (highest priority)
  cudaEvent_t done = nullptr;
  float* h_q = nullptr;
  float* h_s = nullptr;
  uint64_t* h_i = nullptr;
  vcb::DeviceBuffer d_q, d_s, d_i;
  vcb::FlatScratchStore flat;
  vcb::BucketScratch* bkt = nullptr;
  std::vector<Request*> batch;
  size_t k_eff = 0, nq = 0;
  bool busy = false;
  std::atomic<int64_t> done_ns{0};
  ~Slot() {
    if (stream) cudaStreamSynchronize(stream);
    if (stream_hi) cudaStreamSynchronize(stream_hi);
    if (h_q) cudaFreeHost(h_q);
    if (h_s) cudaFreeHost(h_s);
    if (h_i) cudaFreeHost(h_i);
    if (done) cudaEventDestroy(done);
    if (stream) cudaStreamDestroy(stream);
    if (stream_hi) cudaStreamDestroy(stream_hi);
    if (bkt) vcb::bucket_scratch_delete(bkt);
  }
};

void CUDART_CB mark_done(void* p) { static_cast<Slot*>(p)->done_ns.store(now_ns()); }

}  // namespace

struct tq_server {
  int device = 0;
  size_t budget = 0, max_slots = 0, max_batch = 0;
  std::vector<Target> targets;
  std::vector<std::unique_ptr<Slot>> slots;
  size_t max_dim = 0, max_k = 0;
  size_t slot_bytes = 0, resident_bytes = 0;

  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> pending;
  std::unordered_map<uint64_t, std::unique_ptr<Request>> requests;
  uint64_t next_id = 1;
  std::thread worker;
  bool started = false, stopping = false;
  std::string worker_error;
  // counters
  uint64_t batches = 0, queries = 0, completed = 0;
  size_t peak_inflight = 0;

  ~tq_server() { stop(); }

  void stop() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stopping = true;
    }
    cv_work.notify_all();
    if (worker.joinable()) worker.join();
  }

  // Runs one batch of the slot's requests (caller holds the lock).
  void launch(Slot& sl) {
    Request* r0 = sl.batch.front();
    const Target& t = targets[r0->target];
    size_t row = 0;
    for (Request* r : sl.batch) {
      std::memcpy(sl.h_q + row * t.dim_in, r->q, r->nq * t.dim_in * 4);
      row += r->nq;
    }
    sl.nq = row;
    // Flat scans are long (every vector for every query) and run on the slot's
    // normal-priority stream, in CTAs of bounded work; bucketed batches go to
    // its highest-priority stream, so the block scheduler starts their CTAs as
    // soon as running flat CTAs retire instead of after the whole flat scan.
    cudaStream_t s = t.flat ? sl.stream : sl.stream_hi;
    vcb::check(cudaMemcpyAsync(sl.d_q.get(), sl.h_q, row * t.dim_in * 4, cudaMemcpyHostToDevice, s), "H2D");
    size_t ke;
    if (t.flat) {
      ke = std::min(r0->k, t.flat->n);
      t.flat->search_device(sl.d_q.as<float>(), row, r0->k, sl.d_s.as<float>(), sl.d_i.as<uint64_t>(), ke, s,
                            sl.flat.ref());
    } else {
      const vcb::LearnedProbe lp{t.mlp, t.coverage, t.min_conf};
      ke = vcb::bucketed_search_with(t.bkt, sl.d_q.as<float>(), row, r0->k, r0->n_probe, t.mlp ? &lp : nullptr,
                                     sl.d_s.as<float>(), sl.d_i.as<uint64_t>(), s, *sl.bkt);
    }
    sl.k_eff = ke;
    vcb::check(cudaMemcpyAsync(sl.h_s, sl.d_s.get(), row * ke * 4, cudaMemcpyDeviceToHost, s), "D2H");
    vcb::check(cudaMemcpyAsync(sl.h_i, sl.d_i.get(), row * ke * 8, cudaMemcpyDeviceToHost, s), "D2H");
    vcb::check(cudaLaunchHostFunc(s, mark_done, &sl), "cudaLaunchHostFunc");
    vcb::check(cudaEventRecord(sl.done, s), "cudaEventRecord");
    sl.busy = true;
    ++batches;
    queries += row;
  }

  void retire(Slot& sl) {
    size_t row = 0;
    const int64_t t = sl.done_ns.load();
    for (Request* r : sl.batch) {
      if (r->out_s) std::memcpy(r->out_s, sl.h_s + row * sl.k_eff, r->nq * sl.k_eff * 4);
      if (r->out_i) std::memcpy(r->out_i, sl.h_i + row * sl.k_eff, r->nq * sl.k_eff * 8);
      r->k_eff = sl.k_eff;
      r->t_done = t;
      r->done = true;
      row += r->nq;
      ++completed;
    }
    sl.batch.clear();
    sl.busy = false;
  }

  // Oldest waiting request plus later compatible ones, up to max_batch queries.
  void take_batch(Slot& sl) {
    Request* r0 = pending.front();
    pending.pop_front();
    sl.batch.push_back(r0);
    size_t total = r0->nq;
    for (auto it = pending.begin(); it != pending.end();) {
      Request* r = *it;
      if (r->target == r0->target && r->k == r0->k && r->n_probe == r0->n_probe && total + r->nq <= max_batch) {
        sl.batch.push_back(r);
        total += r->nq;
        it = pending.erase(it);
      } else {
        ++it;
      }
    }
  }

  void run() {
    vcb::DeviceGuard g(device);
    std::unique_lock<std::mutex> lk(mu);
    while (true) {
      bool progress = false;
      size_t inflight = 0;
      for (auto& sp : slots) {
        Slot& sl = *sp;
        if (sl.busy) {
          const cudaError_t e = cudaEventQuery(sl.done);
          if (e == cudaSuccess) {
            retire(sl);
            progress = true;
          } else if (e != cudaErrorNotReady) {
            worker_error = cudaGetErrorString(e);
            for (Request* r : sl.batch) {
              r->status = TQ_ERR_CUDA;
              r->error = worker_error;
              r->done = true;
            }
            sl.batch.clear();
            sl.busy = false;
            progress = true;
          }
        }
      }
      if (progress) cv_done.notify_all();
      for (auto& sp : slots) {
        Slot& sl = *sp;
        if (!sl.busy && !pending.empty()) {
          take_batch(sl);
          try {
            launch(sl);
          } catch (const std::exception& ex) {
            for (Request* r : sl.batch) {
              r->status = TQ_ERR_CUDA;
              r->error = ex.what();
              r->done = true;
            }
            sl.batch.clear();
            cv_done.notify_all();
          }
          progress = true;
        }
        inflight += sl.busy ? 1 : 0;
      }
      peak_inflight = std::max(peak_inflight, inflight);
      if (stopping && pending.empty() && inflight == 0) break;
      if (!progress) {
        if (inflight == 0) {
          cv_work.wait(lk, [&] { return stopping || !pending.empty(); });
        } else {
          // Device work in flight: poll its completion every 20 us, or sooner
          // when a request arrives.
          cv_work.wait_for(lk, std::chrono::microseconds(20));
        }
      }
    }
  }

  void start() {
    vcb::DeviceGuard g(device);
    for (const Target& t : targets) {
      max_dim = std::max(max_dim, t.dim_in);
      max_k = std::max(max_k, t.max_k);
    }
    // Warm-up queries: a fixed pseudo-random batch.
    std::vector<float> warm(max_batch * max_dim);
    std::mt19937 rng(7);
    std::normal_distribution<float> nd;
    for (float& v : warm) v = nd(rng);
    {
      // One small search per index with throwaway scratch first: kernels are
      // loaded on their first launch, and that device memory must not be
      // counted as a slot's.
      vcb::DeviceBuffer q, sc_s, sc_i;
      vcb::FlatScratchStore fs;
      vcb::BucketScratch* bs = vcb::bucket_scratch_new();
      const size_t m = std::min<size_t>(max_batch, 64);
      q.reserve(m * max_dim * 4);
      sc_s.reserve(m * max_k * 4);
      sc_i.reserve(m * max_k * 8);
      vcb::check(cudaMemcpy(q.get(), warm.data(), m * max_dim * 4, cudaMemcpyHostToDevice), "H2D");
      for (const Target& t : targets) {
        if (t.flat) {
          t.flat->search_device(q.as<float>(), m, t.max_k, sc_s.as<float>(), sc_i.as<uint64_t>(),
                                std::min(t.max_k, t.flat->n), nullptr, fs.ref());
          // one- and two-query searches may take the batch-split scan kernels
          t.flat->search_device(q.as<float>(), std::min<size_t>(m, 2), t.max_k, sc_s.as<float>(),
                                sc_i.as<uint64_t>(), std::min(t.max_k, t.flat->n), nullptr, fs.ref());
        } else {
          const vcb::LearnedProbe lp{t.mlp, t.coverage, t.min_conf};
          vcb::bucketed_search_with(t.bkt, q.as<float>(), m, t.max_k, t.max_probe, t.mlp ? &lp : nullptr,
                                    sc_s.as<float>(), sc_i.as<uint64_t>(), nullptr, *bs);
        }
      }
      vcb::check(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
      vcb::bucket_scratch_delete(bs);
    }
    size_t free_b = 0, total_b = 0;
    vcb::check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    resident_bytes = total_b - free_b;
    for (size_t s = 0; s < max_slots; ++s) {
      auto sl = std::make_unique<Slot>();
      vcb::check(cudaStreamCreateWithFlags(&sl->stream, cudaStreamNonBlocking), "cudaStreamCreate");
      int least = 0, greatest = 0;
      vcb::check(cudaDeviceGetStreamPriorityRange(&least, &greatest), "cudaDeviceGetStreamPriorityRange");
      vcb::check(cudaStreamCreateWithPriority(&sl->stream_hi, cudaStreamNonBlocking, greatest),
                 "cudaStreamCreateWithPriority");
      sl->flat.range_cap = kServingRangeVectors;
      vcb::check(cudaEventCreateWithFlags(&sl->done, cudaEventDisableTiming), "cudaEventCreate");
      vcb::check(cudaMallocHost(&sl->h_q, max_batch * max_dim * 4), "cudaMallocHost");
      vcb::check(cudaMallocHost(&sl->h_s, max_batch * max_k * 4), "cudaMallocHost");
      vcb::check(cudaMallocHost(reinterpret_cast<void**>(&sl->h_i), max_batch * max_k * 8), "cudaMallocHost");
      sl->d_q.reserve(max_batch * max_dim * 4);
      sl->d_s.reserve(max_batch * max_k * 4);
      sl->d_i.reserve(max_batch * max_k * 8);
      sl->bkt = vcb::bucket_scratch_new();
      vcb::check(cudaMemcpy(sl->d_q.get(), warm.data(), warm.size() * 4, cudaMemcpyHostToDevice), "H2D");
      for (const Target& t : targets) {
        if (t.flat) {
          const size_t ke = std::min(t.max_k, t.flat->n);
          t.flat->search_device(sl->d_q.as<float>(), max_batch, t.max_k, sl->d_s.as<float>(), sl->d_i.as<uint64_t>(),
                                ke, sl->stream, sl->flat.ref());
          // grows the batch-split scratch that one- and two-query batches use
          t.flat->search_device(sl->d_q.as<float>(), std::min<size_t>(max_batch, 2), t.max_k, sl->d_s.as<float>(),
                                sl->d_i.as<uint64_t>(), ke, sl->stream, sl->flat.ref());
        } else {
          const vcb::LearnedProbe lp{t.mlp, t.coverage, t.min_conf};
          vcb::bucketed_search_with(t.bkt, sl->d_q.as<float>(), max_batch, t.max_k, t.max_probe,
                                    t.mlp ? &lp : nullptr, sl->d_s.as<float>(), sl->d_i.as<uint64_t>(), sl->stream,
                                    *sl->bkt);
        }
      }
      vcb::check(cudaStreamSynchronize(sl->stream), "cudaStreamSynchronize");
      vcb::check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
      const size_t used = total_b - free_b;
      if (s == 0) slot_bytes = used - resident_bytes;
      if (used > budget && !slots.empty()) break;  // this slot does not fit: drop it
      slots.push_back(std::move(sl));
      if (used + slot_bytes > budget) break;
    }
    vcb::require(!slots.empty() && total_b - free_b <= budget, TQ_ERR_OUT_OF_MEMORY,
                 "the HBM budget does not hold the resident indexes plus one serving slot");
    started = true;
    worker = std::thread([this] { run(); });
  }
};

namespace {

using vcb::require;

tq_server* checked(tq_server* h) {
  require(h != nullptr, TQ_ERR_INVALID_ARGUMENT, "null server");
  return h;
}

}  // namespace

extern "C" {

int tq_server_create(int device, size_t hbm_budget_bytes, size_t max_slots, size_t max_batch, tq_server** out) {
  return vcb::guarded([&] {
    require(out != nullptr, TQ_ERR_INVALID_ARGUMENT, "out must not be NULL");
    *out = nullptr;
    require(max_slots >= 1 && max_slots <= 64, TQ_ERR_INVALID_ARGUMENT, "max_slots must be in [1, 64]");
    require(max_batch >= 1 && max_batch <= 65536, TQ_ERR_INVALID_ARGUMENT, "max_batch must be in [1, 65536]");
    int count = 0;
    vcb::check(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
    require(device >= 0 && device < count, TQ_ERR_INVALID_ARGUMENT, "no such CUDA device");
    auto h = std::make_unique<tq_server>();
    h->device = device;
    h->budget = hbm_budget_bytes;
    h->max_slots = max_slots;
    h->max_batch = max_batch;
    *out = h.release();
  });
}

int tq_server_destroy(tq_server* h) {
  return vcb::guarded([&] {
    if (!h) return;
    vcb::DeviceGuard g(h->device);
    delete h;
  });
}

int tq_server_add_flat(tq_server* h, tq_index* index, size_t max_k, int* target) {
  return vcb::guarded([&] {
    checked(h);
    require(index != nullptr && target != nullptr, TQ_ERR_INVALID_ARGUMENT, "null argument");
    require(!h->started, TQ_ERR_STATE, "add indexes before start()");
    require(index->prepared, TQ_ERR_STATE, "index is not prepared");
    require(index->device == h->device, TQ_ERR_INVALID_ARGUMENT, "index lives on another device");
    require(max_k >= 1 && max_k <= 256, TQ_ERR_INVALID_ARGUMENT, "max_k must be in [1, 256]");
    Target t;
    t.flat = index;
    t.dim_in = index->dim;
    t.max_k = max_k;
    h->targets.push_back(t);
    *target = static_cast<int>(h->targets.size() - 1);
  });
}

int tq_server_add_bucketed(tq_server* h, tq_bucketed* index, size_t max_k, size_t max_probe, tq_probe_mlp* mlp,
                           float coverage, float min_confidence, int* target) {
  return vcb::guarded([&] {
    checked(h);
    require(index != nullptr && target != nullptr, TQ_ERR_INVALID_ARGUMENT, "null argument");
    require(!h->started, TQ_ERR_STATE, "add indexes before start()");
    require(vcb::bucketed_prepared(index), TQ_ERR_STATE, "index is not prepared");
    require(max_k >= 1 && max_k <= 256, TQ_ERR_INVALID_ARGUMENT, "max_k must be in [1, 256]");
    require(max_probe >= 1 && max_probe <= 2048, TQ_ERR_INVALID_ARGUMENT, "max_probe must be in [1, 2048]");
    Target t;
    t.bkt = index;
    t.mlp = mlp;
    t.coverage = coverage;
    t.min_conf = min_confidence;
    t.dim_in = vcb::bucketed_dim_in(index);
    t.max_k = max_k;
    t.max_probe = max_probe;
    h->targets.push_back(t);
    *target = static_cast<int>(h->targets.size() - 1);
  });
}

int tq_server_start(tq_server* h) {
  return vcb::guarded([&] {
    checked(h);
    require(!h->started, TQ_ERR_STATE, "already started");
    require(!h->targets.empty(), TQ_ERR_STATE, "no index to serve");
    h->start();
  });
}

int tq_server_info(tq_server* h, size_t* n_slots, size_t* slot_bytes, size_t* resident_bytes) {
  return vcb::guarded([&] {
    checked(h);
    if (n_slots) *n_slots = h->slots.size();
    if (slot_bytes) *slot_bytes = h->slot_bytes;
    if (resident_bytes) *resident_bytes = h->resident_bytes;
  });
}

int tq_server_submit(tq_server* h, int target, const float* queries, size_t nq, size_t k, size_t n_probe,
                     float* scores, uint64_t* ids, uint64_t* request) {
  return vcb::guarded([&] {
    checked(h);
    require(h->started, TQ_ERR_STATE, "start() the server first");
    require(target >= 0 && target < static_cast<int>(h->targets.size()), TQ_ERR_INVALID_ARGUMENT, "no such index");
    const Target& t = h->targets[target];
    require(queries != nullptr && request != nullptr, TQ_ERR_INVALID_ARGUMENT, "null argument");
    require(nq >= 1 && nq <= h->max_batch, TQ_ERR_INVALID_ARGUMENT, "nq must be in [1, max_batch]");
    require(k >= 1 && k <= t.max_k, TQ_ERR_INVALID_ARGUMENT, "k must be in [1, max_k of the index]");
    require(t.flat || (n_probe <= t.max_probe), TQ_ERR_INVALID_ARGUMENT, "n_probe above the index's max_probe");
    auto r = std::make_unique<Request>();
    r->target = target;
    r->q = queries;
    r->nq = nq;
    r->k = k;
    r->n_probe = t.flat ? 0 : (n_probe ? n_probe : t.max_probe);
    r->out_s = scores;
    r->out_i = ids;
    r->t_arrive = now_ns();
    {
      std::lock_guard<std::mutex> lk(h->mu);
      r->id = h->next_id++;
      *request = r->id;
      h->pending.push_back(r.get());
      h->requests.emplace(r->id, std::move(r));
    }
    h->cv_work.notify_one();
  });
}

int tq_server_wait(tq_server* h, uint64_t request, size_t* k_eff, double* latency_us) {
  return vcb::guarded([&] {
    checked(h);
    std::unique_lock<std::mutex> lk(h->mu);
    auto it = h->requests.find(request);
    require(it != h->requests.end(), TQ_ERR_INVALID_ARGUMENT, "unknown request");
    Request* r = it->second.get();
    h->cv_done.wait(lk, [&] { return r->done; });
    const int status = r->status;
    const std::string err = r->error;
    if (k_eff) *k_eff = r->k_eff;
    if (latency_us) *latency_us = static_cast<double>(r->t_done - r->t_arrive) / 1e3;
    h->requests.erase(it);
    if (status != TQ_OK) vcb::fail(status, err);
  });
}

int tq_server_stats(tq_server* h, uint64_t* batches, uint64_t* queries, uint64_t* completed, size_t* peak_inflight) {
  return vcb::guarded([&] {
    checked(h);
    std::lock_guard<std::mutex> lk(h->mu);
    if (batches) *batches = h->batches;
    if (queries) *queries = h->queries;
    if (completed) *completed = h->completed;
    if (peak_inflight) *peak_inflight = h->peak_inflight;
  });
}

int tq_server_replay(tq_server* h, const tq_replay_item* items, size_t n, double* latency_us, double* wall_s) {
  return vcb::guarded([&] {
    checked(h);
    require(items != nullptr || n == 0, TQ_ERR_INVALID_ARGUMENT, "null items");
    std::vector<uint64_t> ids(n);
    const int64_t t0 = now_ns();
    for (size_t i = 0; i < n; ++i) {
      const int64_t due = t0 + static_cast<int64_t>(items[i].arrival_us * 1e3);
      while (now_ns() < due) {
        const int64_t left = due - now_ns();
        if (left > 200000) std::this_thread::sleep_for(std::chrono::nanoseconds(left - 100000));
      }
      const int rc = tq_server_submit(h, items[i].target, items[i].queries, items[i].nq, items[i].k,
                                      items[i].n_probe, items[i].scores, items[i].ids, &ids[i]);
      if (rc != TQ_OK) vcb::fail(rc, tq_last_error());
      // Open-loop latency: measured from the scheduled arrival.
      std::lock_guard<std::mutex> lk(h->mu);
      h->requests[ids[i]]->t_arrive = due;
    }
    for (size_t i = 0; i < n; ++i) {
      double lat = 0.0;
      const int rc = tq_server_wait(h, ids[i], nullptr, &lat);
      if (rc != TQ_OK) vcb::fail(rc, tq_last_error());
      if (latency_us) latency_us[i] = lat;
    }
    if (wall_s) *wall_s = static_cast<double>(now_ns() - t0) / 1e9;
  });
}

}  // extern "C"
