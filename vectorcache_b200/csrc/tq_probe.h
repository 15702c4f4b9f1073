// Inference entry of the learned n_probe MLP for other translation units
// (the bucketed index's learned search and the serving loop), with caller-owned
// scratch so that batches on different streams can run concurrently.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/vectorcache_b200.h"
#include "tq_index_impl.h"

namespace vcb {

struct ProbeScratch {
  DeviceBuffer x, z, act0, act1;
  void bind(ScratchArena* a) {
    for (DeviceBuffer* b : {&x, &z, &act0, &act1}) b->bind(a);
  }
};

// Grows sc to what probe_predict needs for m queries (no device work).
void probe_reserve(tq_probe_mlp* h, size_t m, ProbeScratch& sc);

// n_probe for m queries from their top routing scores (row stride p; the first
// min(p, 256) columns are used), written to d_out; queued on s. Same decision
// rule as tq_probe_mlp_predict_device.
void probe_predict(tq_probe_mlp* h, const float* d_top, size_t m, int p, float coverage, float min_conf,
                   uint32_t fallback, uint32_t* d_out, cudaStream_t s, ProbeScratch& sc);

// Largest candidate n_probe of the model.
uint32_t probe_max_class(const tq_probe_mlp* h);

}  // namespace vcb
