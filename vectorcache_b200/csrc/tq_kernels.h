// Launch interfaces of the TurboQuant device kernels. Host code (tq_index.cu)
// owns all device memory and passes plain pointers here.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace vcb {

// Scan layout: 512-vector tiles; inside a tile each byte group is one row of
// 128 u32 words, word w holding vectors 4w..4w+3.
constexpr int kTileVectors = 512;
constexpr int kTileWords = kTileVectors / 4;
// Vectors one scan CTA (8 warps x 256 vectors) covers per block iteration.
constexpr int kScanBlockVectors = 2048;
// The reference flushes integer LUT sums into f32 every 256 byte groups
// (constants.hpp kFlushEvery, search_avx2.cpp:98-124).
constexpr int kFlushGroups = 256;

struct EncodeArgs {
  const float* x;            // n rows x dim, 16-byte aligned
  long long n;
  int dim, bits, block;      // block = Walsh-Hadamard block size
  float inv_sqrt_block;
  const uint32_t* perm_sign;  // source index | sign bit 31
  const float* boundaries;    // 15 floats (device), unused tail = 0
  const float* centroids;     // 16 floats (device)
  bool tqplus;
  const float* shift;
  const float* scale;
  const float* inv_scale;
  uint8_t* out_flat;          // n rows x flat_stride bytes (row-major byte groups)
  int flat_stride;
  float* out_alpha;
  unsigned long long* replay_count;  // optional: vectors whose alpha needed the exact replay
  // Code grid of the boundaries (CodeGrid in tq_host_math.h): CodeGrid::kCells
  // entries {base code, inner boundary bits} and its parameters. nullptr: the
  // per-warp row kernel with the binary search encodes.
  const uint2* grid = nullptr;
  float grid_lo = 0.f, grid_hi = 0.f, grid_a = 0.f, grid_k = 0.f;
};

struct RelayoutArgs {
  const uint8_t* flat;   // rows for vectors [src_first, src_first + src_n)
  long long src_first, src_n;
  int flat_stride;
  long long keep_below;  // vectors below this id keep their existing words
  long long n_total;
  long long first_vector;  // set by the launcher
  int nbg, bits;
  uint32_t* codes;       // scan layout
};

struct RotateArgs {
  const float* x;
  long long n;
  int dim, block;
  float inv_sqrt_block;
  const uint32_t* perm_sign;
  float* out_t;  // dim x n (transposed)
};

struct QueryPrepArgs {
  const float* q;  // nq x dim
  long long nq;
  int dim, bits, block, nbg;
  float inv_sqrt_block;
  const uint32_t* perm_sign;
  const float* centroids;  // 16 floats (device)
  bool tqplus;
  const float* shift;
  const float* scale;
  uint8_t* luts;       // nq x nbg x 32
  float* lut_scale;    // nq
  float* lut_bias;     // nq (sum of per-group minima)
  float* bias_corr;    // nq (TQ+ correction, 0 otherwise)
  float* fa_init;      // nq: lut_bias + bias_corr
  float* q_rot;        // optional nq x dim export
  unsigned long long* replay_count;
};

struct ScanArgs {
  const uint32_t* codes;   // scan layout
  const float* alpha;      // padded to the layout capacity
  const uint8_t* luts;     // nq x nbg x 32
  const float* lut_scale;
  const float* fa_init;
  long long n;             // valid vectors
  int nbg;
  long long nq;
  int k;                   // 1 <= k <= kmax of the instantiation
  int q_per_cta;           // queries per CTA (template Q)
  long long range_vectors; // vectors per CTA range (multiple of kScanBlockVectors)
  int n_ranges;
  int lut_chunk_groups;    // groups resident in shared memory at once (multiple of 256 or nbg)
  int bits = 4;            // 3 selects the lookup that skips nibble values >= 8
  float* cand_score;       // nq x n_ranges x k
  uint32_t* cand_id;
  // Optional scratch for the batch-split scan of one or two queries (used
  // when the plan asks for it): integer sums [query][batch][partial_stride]
  // over partial_batches 256-group batches; partial_stride >= the layout
  // capacity. nullptr: the scan never splits.
  uint32_t* partial = nullptr;
  long long partial_stride = 0;
  int partial_batches = 0;
  // With `partial`: one zeroed counter per (query group, block); the CTA that
  // stores a block's last batch sums flushes that block in the same launch.
  // nullptr: a second launch flushes every block.
  unsigned* arrive = nullptr;
};

struct MergeArgs {
  const float* cand_score;
  const uint32_t* cand_id;
  long long nq;
  int n_lists;   // candidate lists per query
  int k;         // entries per list (padded with -inf / 0xffffffff)
  int k_out;     // k_eff = min(k, n)
  float* out_score;     // nq x k_out
  uint64_t* out_id;
  // Id written into result slots no candidate filled (their score is 0).
  uint64_t pad_id = 0;
  // Lists per query in memory (0: n_lists).
  int list_stride = 0;
  // Optional per query: its candidates are the first entry_count[q] entries of
  // its region (list_stride * k entries), unpadded, instead of n_lists lists.
  const uint32_t* entry_count = nullptr;
};

size_t encode_smem_bytes(int dim, bool tqplus);
bool encode_dim_supported(int dim);
cudaError_t launch_encode(const EncodeArgs& a, int sms, cudaStream_t stream);
cudaError_t launch_relayout(const RelayoutArgs& a, cudaStream_t stream);
cudaError_t launch_export_flat(const uint32_t* codes, long long n, int nbg, uint8_t* out,
                               cudaStream_t stream);
cudaError_t launch_rotate_rows_t(const RotateArgs& a, int sms, cudaStream_t stream);
cudaError_t launch_order_stats(const float* yt, long long n, int dim, long long lo_rank,
                               long long hi_rank, float* q_lo, float* q_hi, cudaStream_t stream);

cudaError_t launch_query_prep(const QueryPrepArgs& a, int sms, cudaStream_t stream);

// Rows wider than 2048 coordinates: one CTA per row, row in shared memory
// (tq_bigdim.cu). The launchers above dispatch here by themselves.
constexpr int kRegisterRowMaxDim = 2048;
cudaError_t launch_encode_big(const EncodeArgs& a, int sms, cudaStream_t stream);
cudaError_t launch_query_prep_big(const QueryPrepArgs& a, int sms, cudaStream_t stream);
cudaError_t launch_rotate_rows_t_big(const RotateArgs& a, int sms, cudaStream_t stream);

// Scan plan: queries per CTA, ranges, chunking. Filled by plan_scan().
struct ScanPlan {
  int q_per_cta = 1;
  int kmax = 16;
  long long range_vectors = 0;
  int n_ranges = 1;
  int lut_chunk_groups = 0;
  size_t smem_bytes = 0;
  int lists_per_range = 1;  // candidate lists each (query, range) publishes
  // > 1: batches of the batch-split scan, which pays off for one or two
  // queries over few blocks (whole blocks per CTA would leave the last wave
  // of CTAs part-full); it needs ScanArgs::partial.
  int split_batches = 0;
  // CTAs per SM of the one-query batch-split scan: 4 (8 groups in flight,
  // 64 registers) or 2 (16 groups in flight), whichever wastes less of its
  // last wave.
  int split_ctas_per_sm = 2;
  // CTAs per SM of a one-query whole-row scan on the register ring: 4 (8
  // groups in flight) for 2- and 4-bit codes when four CTAs' LUTs fit, else 2.
  int ring_ctas_per_sm = 2;
  // > 0: the code stream goes through this many shared-memory slots per warp
  // (one or two queries per CTA, register top-k).
  int stages = 0;
};
// max_range_vectors > 0 bounds the vectors one CTA scans (shorter CTAs let
// higher-priority work on other streams start sooner).
// bits: the index's code width (one-query whole-row scans of 2- and 4-bit
// codes take the register ring on four CTAs per SM, 3-bit codes the
// shared-memory slots).
bool plan_scan(long long n, long long nq, int nbg, int k, int sms, ScanPlan* plan, long long max_range_vectors = 0,
               int bits = 4);
cudaError_t launch_scan(const ScanArgs& a, const ScanPlan& plan, cudaStream_t stream);
cudaError_t launch_merge(const MergeArgs& a, cudaStream_t stream);

// Parity/introspection: integer LUT sums and float scores for every
// (query, vector) pair, computed straight from the scan layout.
cudaError_t launch_dense_scores(const uint32_t* codes, const float* alpha, const uint8_t* luts,
                                const float* lut_scale, const float* fa_init, long long n, int nbg,
                                long long nq, uint32_t* out_int, float* out_score,
                                cudaStream_t stream);

constexpr int kMaxK = 256;

// Exact float re-rank of nq rows of k (score, id) in place (tq_rescore.cu).
cudaError_t launch_rescore(const float* queries, long long nq, int dim, const float* corpus, long long n_corpus,
                           int k, float* scores, uint64_t* ids, cudaStream_t stream);

}  // namespace vcb
