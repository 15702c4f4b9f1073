// Launch interfaces of the bucketed (IVF) index kernels (tq_bucket.cu).
//
// Build: spherical k-means (fp32 routing contraction + argmax), deterministic
// fixed-point centroid sums, 2-means fission of oversized buckets, and the
// bucket-ordered slot layout of residual rows. Search: query routing scores,
// top-n_probe selection, (query, bucket) pairs grouped by bucket into work
// items, and the bucket scan: FastScan over each probed bucket's residual codes
// with the per-(query, bucket) offset <q_hat, encode_c> (score_prepared_into,
// search.cpp:1156-1264).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace vcb {

// A bucket starts at a multiple of this many slots: one scan warp covers 256
// vectors (32 lanes x 8), i.e. one half of a 512-vector scan-layout tile.
constexpr int kBucketSlotAlign = 256;
// Queries per bucket-scan work item (two groups of four, one per warp pair).
constexpr int kItemQueries = 8;
// Candidate lists per (query, probe) of the bucket scan: one per tile set
// scanned side by side within an item (one with 2 queries per warp).
constexpr int kBsListsPerProbe = 1;
// Fixed-point scale of the deterministic centroid sums (|x| <= 1 per coordinate).
constexpr double kFixedScale = 4294967296.0;  // 2^32

// Rows scaled to unit L2 norm and zero-padded from dim_in to dim columns (dim >=
// dim_in). Rows with norm below 1e-30 become zero rows.
cudaError_t launch_normalize_rows(const float* x, long long n, int dim_in, int dim, float* out,
                                  cudaStream_t stream);

// C (m x nb, row stride ldc) = A (m x dim) . B (nb x dim)^T of fp32 rows on the
// tensor cores: 3xTF32 products (split hi/lo TF32 operands), fp32
// accumulation, about 2^-21 relative per product.
cudaError_t launch_gemm_nt(const float* A, long long m, const float* B, long long nb, int dim, float* C,
                           long long ldc, cudaStream_t stream);

// Per row of A: the column of the largest A.B^T entry (ties: lower column) and
// its value, in fp32 fused multiply-adds over the coordinates in order.
cudaError_t launch_assign(const float* A, long long m, const float* B, long long nb, int dim,
                          uint32_t* label, float* best, cudaStream_t stream);

// Largest number of buckets one query may probe.
constexpr int kMaxProbe = 2048;
// Probes scanned before the rest to bound the candidates kept from the rest:
// 8, or 32 from 128 probes on (with a floor after 8 of the 32). Measured at
// 1.2M x 100, 4-bit, k = 100 kept candidates, probe 0 scanned alone first: 32
// first probes scan 512 probes 3.3 % and 256 probes 3.8 % faster than 16, 64 is
// no faster than 32; from 128 instead of 256 probes on, a learned per-query
// assignment runs 0.8 % faster and fixed n_probe 128 is unchanged, from 64 on
// fixed n_probe 64 is 5 % slower.
constexpr int kFloorProbes = 8;
constexpr int kFloorProbesWide = 32;
constexpr int kFloorWideFrom = 128;
// Passes of fewer queries skip the floor after 8 probes and keep 8 first
// probes up to 256 probes: there the extra step's launches (pairs, scan,
// merge) cost more than they save (measured at 1.2M x 100: 16 queries at 128
// probes 0.568 -> 0.475 ms, 64 at 512 probes 0.814 -> 0.754 ms without them).
constexpr int kFloorWideFromSmall = 256;
constexpr long long kMidFloorMinQueries = 4096;

// Per row of S (row stride ld, ncols valid columns): the top p entries, score
// descending, equal scores by lower column; p <= kMaxProbe. Rows with fewer
// than p columns are padded with (-inf, 0xffffffff).
cudaError_t launch_select_top(const float* S, long long rows, long long ld, int ncols, int p, float* out_s,
                              uint32_t* out_i, cudaStream_t stream);

// Counting sort of labels: counts[nb] (zeroed inside), starts[nb + 1]
// (exclusive prefix; starts[nb] = total), members[n] (row ids grouped by label,
// in no particular order inside a group). fill[nb] is scratch.
cudaError_t launch_group_by_label(const uint32_t* label, long long n, int nb, uint32_t* counts,
                                  unsigned long long* starts, uint32_t* fill, uint32_t* members,
                                  cudaStream_t stream);

// Sorts every group's members ascending (groups of at most `max_group` rows,
// max_group <= 8192).
cudaError_t launch_sort_groups(const unsigned long long* starts, int nb, int max_group, uint32_t* members,
                               cudaStream_t stream);

// Deterministic centroids: sums in 2^32 fixed point (exact, order-free) of the
// member rows of X; enc[b] = mean (fp32), route[b] = mean / ||mean||. Empty
// groups keep their previous centroids. acc is nb * dim int64 scratch.
cudaError_t launch_centroids(const float* X, int dim, const unsigned long long* starts, const uint32_t* members,
                             int nb, long long* acc, float* enc, float* route, cudaStream_t stream);

// One 2-means split of each listed group: seeds are the member least aligned
// with the group's routing centroid and the member least aligned with that
// seed; members go to the closer seed, the two means are formed, and members go
// to the closer mean. Members on the second side get label new_label[t]. A
// split that leaves one side empty, or any split when force_bits is set,
// divides the members by the lowest id bit that differs among them (an
// arbitrary but balanced-in-expectation halving that always makes progress).
cudaError_t launch_split(const float* X, int dim, const unsigned long long* starts, const uint32_t* members,
                         const uint32_t* groups, const uint32_t* new_label, int n_groups, const float* route,
                         uint32_t* label, bool force_bits, cudaStream_t stream);

// Slot layout: residual rows R[slot] = X[id] - enc[b] for the members of every
// bucket at slot_start[b] + rank (members sorted), zero rows in the padding;
// slot_ids[slot] = id or 0xffffffff.
cudaError_t launch_build_residuals(const float* X, int dim, const unsigned long long* starts,
                                   const uint32_t* members, int nb, const unsigned long long* slot_start,
                                   const float* enc, long long n_slots, float* R, uint32_t* slot_ids,
                                   cudaStream_t stream);

// Residuals of arbitrary rows against the encode centroid of their label.
cudaError_t launch_residual_rows(const float* X, long long n, int dim, const uint32_t* label, const float* enc,
                                 float* R, cudaStream_t stream);

// label[i] = remap[label[i]] for n labels.
cudaError_t launch_relabel(uint32_t* label, long long n, const uint32_t* remap, cudaStream_t stream);
// dst[r] = src[rows[r]] for n_rows rows of dim floats.
cudaError_t launch_gather_rows(const float* src, const uint32_t* rows, long long n_rows, int dim, float* dst,
                               cudaStream_t stream);

// dst (nq x k_out) = the first k_out columns of src (nq x k_src); entries whose
// id is >= n_valid (unfilled slots) become (0, 0).
cudaError_t launch_take_columns(const float* src_s, const uint64_t* src_i, long long nq, int k_src, int k_out,
                                unsigned long long n_valid, float* dst_s, uint64_t* dst_i, cudaStream_t stream);

struct PairArgs {
  const uint32_t* probes;    // nq rows of bucket ids (routing order), row stride probe_stride
  int probe_stride = 0;      // 0: max_probe
  const uint32_t* n_probe;   // per query, or nullptr: every query probes `fixed_probe`
  int fixed_probe;
  int max_probe;
  long long nq;
  int nb;
  // q_hat . enc^T (nq rows, row stride enc_ld: <q_hat, encode centroid> of
  // every bucket), computed before the pairs; offsets are gathered from it.
  const float* enc_scores;
  long long enc_ld;
  // outputs / scratch (device)
  uint32_t* counts;          // nb
  unsigned long long* pair_start;  // nb + 1
  unsigned long long* item_start;  // nb + 1
  uint32_t* fill;            // nb
  uint32_t* pairs;           // nq * max_probe: q * max_probe + j, grouped by bucket
  float* offsets;            // nq * max_probe: <q_hat, enc[probe]>
  uint4* items;              // (bucket, first pair, pair count, 0)
  unsigned long long* n_items;
  // Probe positions [probe_begin, probe_end) of each query get pairs (the
  // search scans its first probes before the rest).
  int probe_begin = 0;
  int probe_end = 1 << 30;
  // 1: also end at the query's own first-probe count, 2: begin there. That
  // count follows the query's n_probe: kFloorProbesWide from wide_from
  // probes, else kFloorProbes (at most its n_probe).
  int first_split = 0;
  int wide_from = kFloorWideFrom;
};
// Groups the (query, probe) pairs by bucket and builds the scan work items.
cudaError_t launch_build_pairs(const PairArgs& a, cudaStream_t stream);
long long max_items(long long nq, int max_probe, int nb);

struct BucketScanArgs {
  const uint32_t* codes;     // scan layout over slots
  const float* alpha;        // per slot
  const uint32_t* slot_ids;  // per slot: original id
  const unsigned long long* slot_start;  // per bucket (multiple of kBucketSlotAlign)
  const uint32_t* bucket_size;
  const uint8_t* luts;       // nq x nbg x 32
  const float* lut_scale;
  const float* fa_init;
  const uint32_t* pairs;
  const float* offsets;
  const uint4* items;
  const unsigned long long* n_items;
  unsigned long long* next_item;  // work counter (zeroed by launch_bucket_scan)
  int nbg, bits, k, max_probe;
  float* cand_score;         // (nq * max_probe * kBsListsPerProbe) lists of k
  uint32_t* cand_id;
  // Optional per query: scores below floor[q] cannot reach the query's top k
  // and are not kept (nullptr: no floor).
  const float* floor = nullptr;
  // Optional per query (zeroed by the caller): the kept candidates of query q
  // are appended, unpadded, to its region of L = max_probe * kBsListsPerProbe
  // lists of k entries at cand_score/cand_id + q * L * k, and append_count[q]
  // counts them. nullptr: one -inf padded list of k per (query, probe, tile set).
  uint32_t* append_count = nullptr;
};
// `grid`: a bound of the item count; the launch runs min(grid, resident CTAs).
cudaError_t launch_bucket_scan(const BucketScanArgs& a, long long grid, cudaStream_t stream);
// floor[q] = the k-th largest score (above -inf) among the first count[q]
// candidates of query q's region (cand + q * stride), -inf when there are
// fewer than k: the k-th score of their merged top k, a lower bound of the
// k-th best over all probes.
cudaError_t launch_kth_floor(const float* cand, long long stride, const uint32_t* count, long long nq, int k,
                             float* floor, cudaStream_t stream);

// ---- multi-index persistent scan (tq_multi.cu) -----------------------------
// One flat index of a multi-index launch: its scan layout, its queries' LUTs
// and constants, and where its candidate lists go: list ((q * n_ranges +
// range) * 2 + tile set), k entries each.
struct MultiIndexDesc {
  const uint32_t* codes;
  const float* alpha;
  long long n;
  long long range_vectors;  // multiple of kBucketSlotAlign
  int n_ranges;
  int nbg, bits, k;
  const uint8_t* luts;
  const float* lut_scale;
  const float* fa_init;
  float* cand_s;
  uint32_t* cand_i;
};
struct MultiItem {
  int index;
  int range;
  int first_query;
  int n_queries;  // <= kItemQueries
};
struct MultiScanArgs {
  const MultiIndexDesc* indexes;
  const MultiItem* items;
  long long n_items;
  unsigned long long* next_item;  // zeroed before the launch
};
// Persistent launch: `ctas` CTAs pull items until none is left. smem_bytes:
// multi_scan_smem_bytes of the largest nbg and k among the indexes.
size_t multi_scan_smem_bytes(int max_nbg, int max_k);
cudaError_t launch_multi_scan(const MultiScanArgs& a, int ctas, size_t smem_bytes, bool any3, bool any24,
                              cudaStream_t stream);
// Resident CTAs per SM of the multi-index scan for a given shared-memory size.
int multi_scan_ctas_per_sm(size_t smem_bytes, bool any3);

}  // namespace vcb
