// Internal interfaces the serving loop (tq_server.cu) uses to run searches of
// the bucketed index with caller-owned scratch (defined in tq_bucketed.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/vectorcache_b200.h"

namespace vcb {

struct BucketScratch;
struct LearnedProbe {
  tq_probe_mlp* mlp;
  float coverage;
  float min_confidence;
};

BucketScratch* bucket_scratch_new();
void bucket_scratch_delete(BucketScratch* sc);
// Later reserves of every buffer of sc draw from a (nullptr: cudaMalloc).
struct ScratchArena;
void bucket_scratch_bind(BucketScratch* sc, ScratchArena* a);
size_t bucketed_dim_in(const tq_bucketed* h);
size_t bucketed_size(const tq_bucketed* h);
bool bucketed_prepared(const tq_bucketed* h);
size_t bucketed_search_with(tq_bucketed* h, const float* d_q, size_t nq, size_t k, size_t n_probe,
                            const LearnedProbe* lp, float* d_scores, uint64_t* d_ids, cudaStream_t s,
                            BucketScratch& sc);

}  // namespace vcb
