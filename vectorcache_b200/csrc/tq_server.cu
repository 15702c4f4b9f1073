// Serving loop: continuous batching of search requests over resident flat and
// bucketed indexes on one GPU. No counterpart in the reference.
//
// A request (index, nq host queries, k, n_probe) waits in a FIFO queue. A
// worker thread owns S slots; each slot has its own CUDA streams, pinned host
// staging and device query / result buffers, so batches in different slots
// run concurrently on the device. Search scratch (query LUTs, routing scores,
// candidate lists, ...) comes from one device arena sized by the HBM budget:
// whenever a slot is free, the worker forms a batch from the oldest waiting
// request and every later waiting request it can share a launch with (same
// index, k and n_probe) up to max_batch queries, sizes the batch's scratch
// exactly by a dry run of the same search code (no device work), and takes
// that many bytes from the arena. A batch that does not fit waits — and the
// requests behind it with it — until running batches return their scratch;
// so requests are admitted as slots and memory free up. The launch queues the
// H2D copy, search and D2H copy on the slot's stream and marks the completion
// time from a host callback queued after the copy. Serving allocates no device
// memory: the arena, the slots' buffers and every kernel are set up at start().
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
#include <map>
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
  vcb::FlatScratchStore flat;          // bound to `region` per batch
  vcb::BucketScratch* bkt = nullptr;   // bound to `region` per batch
  vcb::ScratchArena region;            // this batch's piece of the server's arena
  size_t region_off = 0, region_bytes = 0;
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

// First-fit allocator of byte ranges of the scratch arena; freed ranges merge
// with their free neighbours.
class ArenaPool {
 public:
  void reset(size_t size) {
    free_.clear();
    if (size) free_[0] = size;
    used_ = 0;
  }
  bool take(size_t bytes, size_t* off) {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < bytes) continue;
      *off = it->first;
      const size_t rest = it->second - bytes, next_off = it->first + bytes;
      free_.erase(it);
      if (rest) free_[next_off] = rest;
      used_ += bytes;
      return true;
    }
    return false;
  }
  void give(size_t off, size_t bytes) {
    used_ -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t used() const { return used_; }

 private:
  std::map<size_t, size_t> free_;
  size_t used_ = 0;
};

}  // namespace

struct tq_server {
  int device = 0;
  size_t budget = 0, max_slots = 0, max_batch = 0;
  std::vector<Target> targets;
  std::vector<std::unique_ptr<Slot>> slots;
  size_t max_dim = 0, max_k = 0;
  size_t slot_bytes = 0, resident_bytes = 0;
  // Scratch arena: every batch's scratch is a range of it, sized by a dry run.
  vcb::DeviceBuffer arena;
  size_t arena_bytes = 0, arena_peak = 0, max_need = 0;
  ArenaPool pool;
  vcb::ScratchArena sizer;            // measure-mode arena of the dry runs
  vcb::FlatScratchStore sizer_flat;   // scratch the dry runs size
  vcb::BucketScratch* sizer_bkt = nullptr;
  uint64_t memory_waits = 0;          // batches that waited for arena memory
  uint64_t blocked_head = 0;          // id of the request heading a waiting batch (0: none)
  size_t blocked_nq = 0, blocked_need = 0;

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

  ~tq_server() {
    stop();
    slots.clear();
    if (sizer_bkt) vcb::bucket_scratch_delete(sizer_bkt);
  }

  // The search of one batch on stream s with the given scratch (a dry run
  // when vcb::dry_run_flag() is set); returns k_eff.
  size_t run_search(const Target& t, const float* d_q, size_t nq, size_t k, size_t n_probe, float* d_s,
                    uint64_t* d_i, cudaStream_t s, vcb::FlatScratchStore& flat, vcb::BucketScratch& bkt) {
    if (t.flat) {
      const size_t ke = std::min(k, t.flat->n);
      t.flat->search_device(d_q, nq, k, d_s, d_i, ke, s, flat.ref());
      return ke;
    }
    const vcb::LearnedProbe lp{t.mlp, t.coverage, t.min_conf};
    return vcb::bucketed_search_with(t.bkt, d_q, nq, k, n_probe, t.mlp ? &lp : nullptr, d_s, d_i, s, bkt);
  }

  // Exact scratch bytes of a batch: the same host code with no device work,
  // its scratch buffers drawing placeholder pieces from a measuring arena.
  size_t batch_need(const Target& t, size_t nq, size_t k, size_t n_probe) {
    sizer.reset(nullptr, 0, true);
    sizer_flat.bind(&sizer);
    vcb::bucket_scratch_bind(sizer_bkt, &sizer);
    struct DryRun {
      DryRun() { vcb::dry_run_flag() = true; }
      ~DryRun() { vcb::dry_run_flag() = false; }
    } dry;
    run_search(t, nullptr, nq, k, n_probe, nullptr, nullptr, nullptr, sizer_flat, *sizer_bkt);
    return sizer.used;
  }

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
    const size_t ke = run_search(t, sl.d_q.as<float>(), row, r0->k, r0->n_probe, sl.d_s.as<float>(),
                                 sl.d_i.as<uint64_t>(), s, sl.flat, *sl.bkt);
    sl.k_eff = ke;
    vcb::check(cudaMemcpyAsync(sl.h_s, sl.d_s.get(), row * ke * 4, cudaMemcpyDeviceToHost, s), "D2H");
    vcb::check(cudaMemcpyAsync(sl.h_i, sl.d_i.get(), row * ke * 8, cudaMemcpyDeviceToHost, s), "D2H");
    vcb::check(cudaLaunchHostFunc(s, mark_done, &sl), "cudaLaunchHostFunc");
    vcb::check(cudaEventRecord(sl.done, s), "cudaEventRecord");
    sl.busy = true;
    ++batches;
    queries += row;
  }

  void free_region(Slot& sl) {
    if (sl.region_bytes) pool.give(sl.region_off, sl.region_bytes);
    sl.region_bytes = 0;
  }

  void retire(Slot& sl) {
    free_region(sl);
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

  // Oldest waiting request plus later compatible ones, up to max_batch
  // queries (left in the queue until the batch is admitted).
  std::vector<Request*> peek_batch(size_t* total) const {
    std::vector<Request*> b;
    Request* r0 = pending.front();
    b.push_back(r0);
    *total = r0->nq;
    for (auto it = std::next(pending.begin()); it != pending.end(); ++it) {
      Request* r = *it;
      if (r->target == r0->target && r->k == r0->k && r->n_probe == r0->n_probe && *total + r->nq <= max_batch) {
        b.push_back(r);
        *total += r->nq;
      }
    }
    return b;
  }

  void unqueue(const std::vector<Request*>& b) {
    for (Request* r : b) pending.erase(std::find(pending.begin(), pending.end(), r));
  }

  void fail_batch(const std::vector<Request*>& b, int status, const std::string& why) {
    for (Request* r : b) {
      r->status = status;
      r->error = why;
      r->done = true;
    }
    cv_done.notify_all();
  }

  // Admits the batch at the head of the queue into the free slot sl when its
  // scratch fits in the arena. Returns false when it must wait for memory.
  bool admit(Slot& sl) {
    size_t nq = 0;
    std::vector<Request*> b = peek_batch(&nq);
    Request* r0 = b.front();
    const Target& t = targets[r0->target];
    size_t need = 0;
    if (blocked_head == r0->id && blocked_nq == nq) {
      need = blocked_need;  // sized while it waited
    } else {
      try {
        need = batch_need(t, nq, r0->k, r0->n_probe);
      } catch (const std::exception& ex) {
        unqueue(b);
        fail_batch(b, TQ_ERR_CUDA, ex.what());
        return true;
      }
    }
    if (need > arena_bytes && b.size() > 1) {
      // The merged batch is too large for the arena: the oldest request alone.
      b.resize(1);
      nq = r0->nq;
      try {
        need = batch_need(t, nq, r0->k, r0->n_probe);
      } catch (const std::exception& ex) {
        unqueue(b);
        fail_batch(b, TQ_ERR_CUDA, ex.what());
        return true;
      }
    }
    if (need > arena_bytes) {
      unqueue(b);
      fail_batch(b, TQ_ERR_OUT_OF_MEMORY,
                 "batch scratch of " + std::to_string(need) + " bytes exceeds the serving arena (" +
                     std::to_string(arena_bytes) + " bytes)");
      return true;
    }
    size_t off = 0;
    if (!pool.take(need, &off)) {
      if (blocked_head != r0->id) ++memory_waits;
      blocked_head = r0->id;
      blocked_nq = nq;
      blocked_need = need;
      return false;
    }
    blocked_head = 0;
    unqueue(b);
    sl.batch = std::move(b);
    sl.region_off = off;
    sl.region_bytes = need;
    sl.region.reset(static_cast<unsigned char*>(arena.get()) + off, need, false);
    sl.flat.bind(&sl.region);
    vcb::bucket_scratch_bind(sl.bkt, &sl.region);
    arena_peak = std::max(arena_peak, pool.used());
    try {
      launch(sl);
    } catch (const std::exception& ex) {
      // Work queued before the failure may still read the region: free it
      // only after the slot's streams drain.
      cudaStreamSynchronize(sl.stream);
      cudaStreamSynchronize(sl.stream_hi);
      free_region(sl);
      fail_batch(sl.batch, TQ_ERR_CUDA, ex.what());
      sl.batch.clear();
    }
    return true;
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
            free_region(sl);
            fail_batch(sl.batch, TQ_ERR_CUDA, worker_error);
            sl.batch.clear();
            sl.busy = false;
            progress = true;
          }
        }
      }
      if (progress) cv_done.notify_all();
      // Free slots take batches in arrival order while their scratch fits;
      // a batch that must wait for memory holds back the ones behind it.
      bool memory_wait = false;
      for (auto& sp : slots) {
        Slot& sl = *sp;
        if (!sl.busy && !pending.empty() && !memory_wait) {
          if (admit(sl)) {
            progress = true;
          } else {
            memory_wait = true;
          }
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
      // Full-size and two-query searches per index with throwaway scratch:
      // kernels are loaded on their first launch, and that device memory is
      // resident, not part of the scratch arena.
      vcb::DeviceBuffer q, sc_s, sc_i;
      vcb::FlatScratchStore fs;
      fs.range_cap = kServingRangeVectors;
      vcb::BucketScratch* bs = vcb::bucket_scratch_new();
      const size_t m = max_batch;
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
      slots.push_back(std::move(sl));
    }
    slot_bytes = max_batch * (max_dim * 4 + max_k * 12);
    size_t free_b = 0, total_b = 0;
    vcb::check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    resident_bytes = total_b - free_b;  // indexes, kernels, context and the slots' buffers
    // The largest scratch any admissible batch needs: full batches at the
    // largest k and n_probe (and one- and two-query batches, which may take
    // the batch-split scan).
    sizer_flat.range_cap = kServingRangeVectors;
    sizer_bkt = vcb::bucket_scratch_new();
    for (const Target& t : targets) {
      for (size_t m : {max_batch, std::min<size_t>(max_batch, 2), size_t{1}}) {
        max_need = std::max(max_need, batch_need(t, m, t.max_k, t.max_probe));
      }
    }
    if (budget <= resident_bytes || budget - resident_bytes < max_need) {
      vcb::fail(TQ_ERR_OUT_OF_MEMORY, "the HBM budget does not hold the resident indexes plus the scratch of one "
                                      "full batch (" + std::to_string(resident_bytes + max_need) + " bytes needed)");
    }
    arena_bytes = std::min(budget - resident_bytes, max_slots * max_need);
    arena_bytes = arena_bytes / vcb::ScratchArena::kAlign * vcb::ScratchArena::kAlign;
    arena.reserve(arena_bytes);
    pool.reset(arena_bytes);
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

int tq_server_memory(tq_server* h, size_t* arena_bytes, size_t* arena_peak, size_t* max_batch_bytes,
                     uint64_t* memory_waits) {
  return vcb::guarded([&] {
    checked(h);
    require(h->started, TQ_ERR_STATE, "start() the server first");
    std::lock_guard<std::mutex> lk(h->mu);
    if (arena_bytes) *arena_bytes = h->arena_bytes;
    if (arena_peak) *arena_peak = h->arena_peak;
    if (max_batch_bytes) *max_batch_bytes = h->max_need;
    if (memory_waits) *memory_waits = h->memory_waits;
  });
}

int tq_server_batch_bytes(tq_server* h, int target, size_t nq, size_t k, size_t n_probe, size_t* bytes) {
  return vcb::guarded([&] {
    checked(h);
    require(h->started, TQ_ERR_STATE, "start() the server first");
    require(bytes != nullptr, TQ_ERR_INVALID_ARGUMENT, "null argument");
    require(target >= 0 && target < static_cast<int>(h->targets.size()), TQ_ERR_INVALID_ARGUMENT, "no such index");
    const Target& t = h->targets[target];
    require(nq >= 1 && nq <= h->max_batch, TQ_ERR_INVALID_ARGUMENT, "nq must be in [1, max_batch]");
    require(k >= 1 && k <= t.max_k, TQ_ERR_INVALID_ARGUMENT, "k must be in [1, max_k of the index]");
    vcb::DeviceGuard g(h->device);
    std::lock_guard<std::mutex> lk(h->mu);
    *bytes = h->batch_need(t, nq, k, t.flat ? 0 : (n_probe ? n_probe : t.max_probe));
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
