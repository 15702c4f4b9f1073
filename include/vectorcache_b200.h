/*
 * vectorcache_b200 — C ABI of the B200 (sm_100a) TurboQuant flat index.
 *
 * Drop-in boundary for the flat TurboQuant encode + FastScan search path of
 * nishadtardalkar/vectorcache. The reference exposes this path as C++ only:
 * the free functions fit_calibration / encode / repack / prepare_queries /
 * score_prepared / search_flat and the GPU class gpu::FlatIndex. Each entry
 * point below names the reference interface it replaces (paths inside the
 * reference project).
 *
 * Conventions
 *   - Every function returns 0 on success and a nonzero TQ_ERR_* code on
 *     failure; tq_last_error() returns the calling thread's last message.
 *     Nothing throws across this boundary.
 *   - Host pointers belong to the caller. Device memory belongs to the library,
 *     except for the *_device entry points, whose buffers the caller owns
 *     (16-byte aligned, on the index's device).
 *   - A handle is used by one host thread at a time. Work is queued on the
 *     index's own CUDA stream unless a `stream` (cudaStream_t) is passed.
 *   - Validation follows the reference: dim a positive multiple of 8 and
 *     <= 16384, bits in {2, 3, 4}; search returns k_eff = min(k, n) results
 *     per query, scores descending, equal scores ordered by lower id.
 */
#ifndef VECTORCACHE_B200_H
#define VECTORCACHE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  TQ_OK = 0,
  TQ_ERR_INVALID_ARGUMENT = 1, /* std::invalid_argument in the reference */
  TQ_ERR_STATE = 2,            /* std::runtime_error: wrong call order */
  TQ_ERR_CUDA = 3,             /* CUDA runtime error */
  TQ_ERR_OUT_OF_MEMORY = 4,    /* device allocation failed or over the HBM budget */
  TQ_ERR_UNSUPPORTED = 5       /* valid for the reference, not for this device path */
};

typedef struct tq_index tq_index;

/* Last error message of the calling thread ("" if none). */
const char* tq_last_error(void);

/* Library version string. */
const char* tq_version(void);

/* ---- host-side tables (same values as the reference's setup code) -------- */

/* Lloyd-Max codebook for Beta((dim-1)/2, (dim-1)/2).
 * Replaces vectorcache::codebook (src/quantize/codebook.cpp:203).
 * boundaries: 2^bits - 1 floats, centroids: 2^bits floats. */
int tq_codebook(size_t bits, size_t dim, float* boundaries, float* centroids);

/* Rotation tables: signs[dim] (+-1) and perm[dim].
 * Replaces vectorcache::Rotation::signs/perm (src/transform/rotation.cpp:139-160). */
int tq_rotation_tables(size_t dim, float* signs, uint32_t* perm);

/* ---- index lifecycle ------------------------------------------------------- */

/* Create an empty flat index on CUDA device `device`. flags: reserved, pass 0.
 * Replaces gpu::FlatIndex::FlatIndex(dim, bits)
 * (include/vectorcache/gpu/flat_index.hpp:19, src/gpu/flat_index.cpp:82). */
int tq_index_create(size_t dim, size_t bits, uint32_t flags, int device, tq_index** out);

int tq_index_destroy(tq_index* h);

/* Optional TQ+ calibration from n >= 2 sample rows (host memory). Must precede
 * prepare(). Replaces vectorcache::fit_calibration (src/encode/encode.cpp:327). */
int tq_index_calibrate(tq_index* h, const float* sample, size_t n);
int tq_index_calibrate_device(tq_index* h, const float* d_sample, size_t n, void* stream);

/* Append n rows. Before prepare() rows are staged on the device and encoded by
 * prepare(); after prepare() they are encoded and appended immediately.
 * Replaces gpu::FlatIndex::add (src/gpu/flat_index.cpp:134) and
 * vectorcache::encode (src/encode/encode.cpp:294). */
int tq_index_add(tq_index* h, const float* vectors, size_t n);
int tq_index_add_device(tq_index* h, const float* d_vectors, size_t n, void* stream);

/* Encode staged rows and build the scan layout.
 * Replaces gpu::FlatIndex::prepare (src/gpu/flat_index.cpp:147) and
 * vectorcache::repack (src/pack/pack.cpp:366). */
int tq_index_prepare(tq_index* h);

/* Top-k search. scores/ids hold nq * k entries; rows are written with stride
 * *k_eff = min(k, size). 1 <= k <= 256.
 * Replaces gpu::FlatIndex::search (src/gpu/flat_index.cpp:220) and
 * vectorcache::search_flat (src/search/search.cpp:1293). */
int tq_index_search(tq_index* h, const float* queries, size_t nq, size_t k, float* scores,
                    uint64_t* ids, size_t* k_eff);
/* Same with caller-owned device buffers, queued on `stream` (NULL: the
 * index's stream); returns without synchronizing. */
int tq_index_search_device(tq_index* h, const float* d_queries, size_t nq, size_t k,
                           float* d_scores, uint64_t* d_ids, size_t* k_eff, void* stream);

/* Block until the index's queued work is done. */
int tq_index_synchronize(tq_index* h);

/* ---- persistence and file formats -------------------------------------------
 * Index files: no counterpart in the reference, which keeps no index on disk.
 * The file holds dim, bits, the TQ+ shift/scale, codes_flat, alpha and a
 * checksum; tq_index_load returns a prepared index on `device`. */
int tq_index_save(tq_index* h, const char* path);
int tq_index_load(const char* path, int device, tq_index** out);

/* Append the rows of a float32 C-order (rows, dim) .npy file, streamed in
 * chunks. Replaces NpyReader (include/vectorcache/datasets/npy.hpp:33-61)
 * feeding add(). */
int tq_index_add_npy(tq_index* h, const char* path);

/* .npy float32 matrices: NpyReader / write_npy_f32_matrix
 * (include/vectorcache/datasets/npy.hpp:33-66). */
int tq_npy_f32_info(const char* path, size_t* rows, size_t* cols);
int tq_npy_f32_read(const char* path, size_t row0, size_t nrows, float* out);
int tq_npy_f32_write(const char* path, size_t rows, size_t cols, const float* data);

/* VCEX exact-top-k files (tools/query-bench.cpp:180-340): ground-truth ids
 * nq x k with the index size, seed and three labels. */
int tq_vcex_write(const char* path, const uint64_t* ids, size_t nq, size_t k, uint64_t index_n,
                  uint64_t seed, const char* source_label, const char* split,
                  const char* query_split);
int tq_vcex_read_header(const char* path, size_t* nq, size_t* k, uint64_t* index_n,
                        uint64_t* seed);
int tq_vcex_read_ids(const char* path, uint64_t* ids);

/* ---- exact float re-rank ---------------------------------------------------
 * Re-scores each query's k candidates with the exact float inner product
 * <query, corpus[id]> (the reference's AVX2 summation order) and re-sorts the
 * row: score descending, equal scores by lower id; ids >= n_corpus score -inf.
 * scores/ids are nq x k, rewritten in place. Replaces float_rescore_topk
 * (src/search/float_rescore.cpp:80-164). k <= 4096. */
int tq_rescore(const float* queries, size_t nq, size_t dim, const float* corpus, size_t n_corpus,
               size_t k, float* scores, uint64_t* ids, int device);
/* Device buffers, queued on `stream` (a cudaStream_t; NULL = legacy default). */
int tq_rescore_device(const float* d_queries, size_t nq, size_t dim, const float* d_corpus,
                      size_t n_corpus, size_t k, float* d_scores, uint64_t* d_ids, void* stream);

/* ---- introspection (parity exports) --------------------------------------- */

int tq_index_info(const tq_index* h, size_t* dim, size_t* bits, size_t* n, int* prepared,
                  int* calibrated);

/* Row-major byte-group codes, n * (dim / (8 / bits)) bytes; first code of a
 * byte in the high bits (codes_flat_from_packed, src/pack/pack.cpp:352). */
int tq_index_export_codes_flat(tq_index* h, uint8_t* out);

/* Bit-plane rows exactly as vectorcache::encode writes them:
 * n * bits * dim / 8 bytes (src/encode/encode.cpp:147-153). */
int tq_index_export_packed(tq_index* h, uint8_t* out);

/* Per-vector alpha = ||v|| / <u, x_hat> (encode.cpp:32-37). */
int tq_index_export_alpha(tq_index* h, float* out);

/* TQ+ shift / scale (dim floats each); TQ_ERR_STATE if not calibrated. */
int tq_index_export_calibration(tq_index* h, float* shift, float* scale);

/* Query-side state of prepare_queries (src/search/search.cpp:762):
 * q_rot (nq*dim), bias_corr (nq), LUT bytes (nq * nbg * 32), LUT scale and
 * bias (nq each). Any output pointer may be NULL. */
int tq_index_prepare_queries(tq_index* h, const float* queries, size_t nq, float* q_rot,
                             float* bias_corr, uint8_t* luts, float* lut_scale, float* lut_bias);

/* Dense scores of every (query, vector): integer LUT sums over all groups
 * (nq * n uint32) and the float scores the scan ranks (nq * n floats).
 * Either output may be NULL. */
int tq_index_dense_scores(tq_index* h, const float* queries, size_t nq, uint32_t* int_scores,
                          float* scores);

/* Number of vectors whose alpha (or queries whose TQ+ bias) needed the exact
 * sequential replay since the index was created. */
int tq_index_replay_count(const tq_index* h, uint64_t* count);

/* The scan plan a search of nq queries with this k would use: queries per
 * CTA, vector ranges (one CTA per query group and range), vectors per range
 * (a multiple of the 2048-vector scan block), and the number of 256-group
 * batches a one- or two-query scan splits into (1: no split), and the
 * shared-memory slots per warp its code stream goes through (0: a register
 * prefetch ring). The reference tiles its scan over <= 4 or <= 8 queries and
 * block ranges (src/search/search.cpp:600-758); this reports the device's
 * tiling, for tests that need a given tiling and for measurements. Any out
 * pointer may be null. */
int tq_index_scan_plan(const tq_index* h, size_t nq, size_t k, int* q_per_cta, int* n_ranges,
                       uint64_t* range_vectors, int* split_batches, int* stages);

/* The same plan for an index of n vectors of dim coordinates at bits, on a device
 * of `sms` SMs, computed on the host alone (no index, no device; the plan of a
 * search through the index's own scratch). Outputs as above, plus the CTAs per SM
 * of a one- or two-query batch-split scan (0 when it does not split). No
 * counterpart in the reference: it lets tests check the planning rules and
 * callers size a deployment without a GPU. Any out pointer may be null. */
int tq_scan_plan_shape(uint64_t n, size_t nq, size_t dim, size_t bits, size_t k, int sms, int* q_per_cta,
                       int* n_ranges, uint64_t* range_vectors, int* split_batches, int* stages,
                       int* split_ctas_per_sm);

/* ---- measurement (no counterpart in the reference, which times with
 *      std::chrono around whole calls: tools/gpu-bench.cpp:155-190) ---------- */

/* The index's own CUDA stream (a cudaStream_t), for callers that time or
 * order work around the host-buffer entry points. */
int tq_index_get_stream(tq_index* h, void** stream);

/* Per-kernel device time, recorded with CUDA events around every launch
 * while profiling is enabled. Reading the profile synchronizes the index and
 * resets it. scan_stream_bytes counts the bytes one streaming of the codes +
 * alpha per query group moves: sum over scan launches of
 * query_groups * n * (n_byte_groups + 4). */
typedef struct tq_profile {
  double prep_ms, scan_ms, merge_ms, encode_ms;
  uint64_t prep_launches, scan_launches, merge_launches, encode_launches;
  uint64_t scan_stream_bytes;
  uint64_t scan_queries;
} tq_profile;

int tq_index_set_profiling(tq_index* h, int enabled);
int tq_index_read_profile(tq_index* h, tq_profile* out);
/* The launches timed up to the last tq_index_read_profile, per launch name
 * (e.g. "bucket scan kernel", "pair kernels", "probe network"), in first-seen
 * order: entry i's name (truncated to name_cap - 1 bytes, NUL-terminated),
 * device time and launch count. */
int tq_index_profile_entries(const tq_index* h, size_t* n);
int tq_index_profile_entry(const tq_index* h, size_t i, char* name, size_t name_cap, double* ms,
                           uint64_t* launches);

/* ---- bucketed (IVF) index ---------------------------------------------------
 * BucketedTurboQuantIndex / BucketParams of the reference's README
 * (README.md:56, :91-98, :113-120); the reference ships no implementation of
 * them, only the per-bucket scoring they compose, score_prepared_into
 * (src/search/search.cpp:1156-1264), which the search reproduces bit for bit:
 * score = (fa * alpha) + <q_hat, encode_c> over each probed bucket's residual
 * codes x_hat - encode_c, top-k in (score desc, id asc) order.
 *
 * Rows and queries are L2-normalized (cosine); dim need not be a multiple of 8
 * (rows are zero-padded to the next multiple of 8 internally, dim <= 2048).
 * The partition: ceil(expected_n / energy_soft) seeds, kmeans_iters rounds of
 * spherical k-means, then 2-means fission of every bucket above
 * max_bucket_size; it is deterministic for a given seed. */
typedef struct tq_bucket_params {
  uint32_t n_probe;         /* buckets scanned per query by default (64), <= 2048 */
  uint32_t max_bucket_size; /* hard cap; larger buckets are split (800), <= 8192 */
  uint32_t energy_soft;     /* target mean bucket size of the initial partition (400) */
  uint32_t kmeans_iters;    /* spherical k-means rounds of the initial partition (4) */
  uint32_t rerank_k;        /* 0: off (default). > k: the scan keeps rerank_k candidates,
                               re-scored with the exact float <q_hat, x_hat> (the
                               reference's float_rescore_topk order,
                               src/search/float_rescore.cpp:80-164); top k returned */
  uint32_t reserved;        /* 0 */
  uint64_t expected_n;      /* corpus size the partition is sized for; 0 = rows at prepare() */
  uint64_t seed;            /* seed of the initial centroid choice */
} tq_bucket_params;

typedef struct tq_bucketed tq_bucketed;

/* Default parameters (the values in parentheses above). */
void tq_bucket_params_init(tq_bucket_params* p);

/* params may be NULL (defaults). */
int tq_bucketed_create(size_t dim, size_t bits, const tq_bucket_params* params, int device,
                       tq_bucketed** out);
int tq_bucketed_destroy(tq_bucketed* h);
/* Optional TQ+ calibration sample (host rows); fitted at prepare() on the
 * residuals of these rows against their nearest bucket. */
int tq_bucketed_calibrate(tq_bucketed* h, const float* sample, size_t n);
int tq_bucketed_add(tq_bucketed* h, const float* vectors, size_t n);
int tq_bucketed_add_device(tq_bucketed* h, const float* d_vectors, size_t n, void* stream);
/* Builds the partition and encodes the residuals. Rows added after prepare()
 * are assigned to their nearest routing centroid by the next prepare(), which
 * also splits buckets that grew past max_bucket_size; encode centroids of
 * buckets that were not split stay frozen. */
int tq_bucketed_prepare(tq_bucketed* h);
/* Top-k over the n_probe best-routed buckets (n_probe = 0: the index's
 * default). n_probe_per_query (optional, nq entries, each <= n_probe) scans
 * fewer buckets for some queries — the learned probe predictor's output. */
int tq_bucketed_search(tq_bucketed* h, const float* queries, size_t nq, size_t k, size_t n_probe,
                       const uint32_t* n_probe_per_query, float* scores, uint64_t* ids,
                       size_t* k_eff);
int tq_bucketed_search_device(tq_bucketed* h, const float* d_queries, size_t nq, size_t k,
                              size_t n_probe, const uint32_t* d_n_probe, float* d_scores,
                              uint64_t* d_ids, size_t* k_eff, void* stream);
/* Routing only: the top p (<= 2048) buckets per query and their scores
 * <q_hat, routing centroid>, best first (device buffers nq x p). */
int tq_bucketed_route_device(tq_bucketed* h, const float* d_queries, size_t nq, size_t p,
                             float* d_top_scores, uint32_t* d_top_ids, void* stream);
/* The selection the routing uses, on any device score matrix (rows x ncols,
 * row stride ld floats): per row the top p (<= 2048) columns, score
 * descending, equal scores by lower column; -inf and NaN are never selected
 * and rows with fewer than p selectable columns end in (-inf, 0xffffffff).
 * Outputs rows x p. No counterpart in the reference (its probe order is the
 * heap order of the same key). */
int tq_select_top_device(const float* d_scores, size_t rows, size_t ld, size_t ncols, size_t p,
                         float* d_top_scores, uint32_t* d_top_ids, int device, void* stream);

/* Introspection for parity checks. */
int tq_bucketed_info(const tq_bucketed* h, size_t* dim, size_t* dim_padded, size_t* bits, size_t* n,
                     size_t* n_buckets, size_t* n_slots, int* prepared);
/* Search that also returns the probes (nq x n_probe bucket ids, routing
 * order), the offsets <q_hat, encode_c> of those probes and q_hat
 * (nq x dim_padded). */
int tq_bucketed_search_trace(tq_bucketed* h, const float* queries, size_t nq, size_t k,
                             size_t n_probe, const uint32_t* n_probe_per_query, float* scores,
                             uint64_t* ids, size_t* k_eff, uint32_t* probes, float* offsets,
                             float* q_hat);
/* q_hat (nq x dim_padded) and all routing scores (nq x n_buckets). */
int tq_bucketed_route(tq_bucketed* h, const float* queries, size_t nq, float* q_hat, float* scores);
/* slot_start: n_buckets + 1; bucket_size: n_buckets; slot_ids: n_slots
 * (0xffffffff in padding slots); labels: n (bucket of every row). */
int tq_bucketed_export_layout(tq_bucketed* h, uint64_t* slot_start, uint32_t* bucket_size,
                              uint32_t* slot_ids, uint32_t* labels);
/* routing and encode centroids, n_buckets x dim_padded each. */
int tq_bucketed_export_centroids(tq_bucketed* h, float* route, float* enc);
/* the normalized, padded rows (n x dim_padded). */
int tq_bucketed_export_rows(tq_bucketed* h, float* x_hat);
/* The flat index over the residual slots (owned by h): its codes_flat,
 * alpha, calibration and query LUT exports describe the bucketed layout. */
int tq_bucketed_engine(tq_bucketed* h, tq_index** engine);

/* ---- learned n_probe predictor ----------------------------------------------
 * No counterpart in the reference. A small MLP reads a query's top-256
 * routing scores s_1 >= ... >= s_256 and the gaps s_i - s_{i+1} (512 inputs,
 * standardized by tq_probe_mlp_set_normalization), n_layers hidden layers of
 * `hidden` units (ReLU) and one logit per class; class c stands for the
 * n_probe value classes[c] (increasing, <= 2048). Matrix products use bf16
 * weights and activations with fp32 accumulation; training (Adam) keeps fp32
 * master weights. Everything runs on the GPU. Two training objectives:
 *   TQ_PROBE_OBJECTIVE_CLASSES (default): softmax cross-entropy against one
 *     label class per query (its smallest sufficient n_probe). Prediction:
 *     the smallest class whose cumulative probability reaches `coverage`, or
 *     `fallback` when the largest class probability is below
 *     `min_confidence`.
 *   TQ_PROBE_OBJECTIVE_RECALL: one sigmoid per class, binary cross-entropy
 *     (mean over queries and classes) against the query's measured recall at
 *     each class (targets in [0, 1]); output r_c estimates the recall at
 *     classes[c]. Prediction: the class maximizing
 *     r_c - coverage * classes[c] / classes[last] (the lowest such class on
 *     ties), i.e. `coverage` carries the trade-off: recall given up to save
 *     the largest class's whole probe budget; `fallback` when the largest
 *     r_c is below `min_confidence`. Confidence = the largest r_c.
 * Parameters are flattened as, per layer, W (fan_in x fan_out, row-major)
 * then b (fan_out). */
typedef struct tq_probe_mlp tq_probe_mlp;

enum { TQ_PROBE_OBJECTIVE_CLASSES = 0, TQ_PROBE_OBJECTIVE_RECALL = 1 };

int tq_probe_mlp_create(size_t hidden, size_t n_layers, const uint32_t* classes, size_t n_classes,
                        uint64_t seed, int device, tq_probe_mlp** out);
/* Chooses the training objective and the prediction rule (before training). */
int tq_probe_mlp_set_objective(tq_probe_mlp* h, int objective);
int tq_probe_mlp_destroy(tq_probe_mlp* h);
int tq_probe_mlp_info(const tq_probe_mlp* h, size_t* n_inputs, size_t* n_params, size_t* n_classes);
/* Raw (unstandardized) 512 features of m rows of top routing scores (row
 * stride p <= 256), host buffers. */
int tq_probe_mlp_features(tq_probe_mlp* h, const float* top_scores, size_t m, size_t p, float* raw);
int tq_probe_mlp_set_normalization(tq_probe_mlp* h, const float* mean, const float* stddev);
int tq_probe_mlp_get_params(tq_probe_mlp* h, float* params);
int tq_probe_mlp_set_params(tq_probe_mlp* h, const float* params);
/* Logits (m x n_classes) of host rows. */
int tq_probe_mlp_forward(tq_probe_mlp* h, const float* top_scores, size_t m, size_t p, float* logits);
/* Mean cross-entropy and its gradients (n_params floats) for a host batch,
 * without updating the parameters (classes objective). */
int tq_probe_mlp_gradients(tq_probe_mlp* h, const float* top_scores, const uint32_t* labels, size_t m,
                           size_t p, float* loss, float* grads);
/* The same for the recall objective: recall is m x n_classes, row-major. */
int tq_probe_mlp_recall_gradients(tq_probe_mlp* h, const float* top_scores, const float* recall, size_t m,
                                  size_t p, float* loss, float* grads);
/* One Adam step (lr; beta1 0.9, beta2 0.999, eps 1e-8) on a device batch,
 * queued on `stream` (NULL: the model's own stream); returns when done. */
int tq_probe_mlp_train_step_device(tq_probe_mlp* h, const float* d_top_scores, const uint32_t* d_labels,
                                   size_t m, size_t p, float lr, float* loss, void* stream);
/* The same for the recall objective (d_recall: m x n_classes targets in [0, 1]). */
int tq_probe_mlp_train_step_recall_device(tq_probe_mlp* h, const float* d_top_scores, const float* d_recall,
                                          size_t m, size_t p, float lr, float* loss, void* stream);
/* Per-query n_probe (device, m entries) and optionally the confidence. */
int tq_probe_mlp_predict_device(tq_probe_mlp* h, const float* d_top_scores, size_t m, size_t p,
                                float coverage, float min_confidence, uint32_t fallback,
                                uint32_t* d_n_probe, float* d_confidence, void* stream);
int tq_probe_mlp_synchronize(tq_probe_mlp* h);

/* Bucketed search with the learned n_probe: one routing pass gives both the
 * network's input (top-256 routing scores) and the probes; every query scans
 * its predicted number of buckets (at most fallback_n_probe, which is also the
 * low-confidence fallback; 0 = the index's n_probe). Device buffers, queued
 * on `stream`. */
int tq_bucketed_search_learned_device(tq_bucketed* h, const float* d_queries, size_t nq, size_t k,
                                      tq_probe_mlp* mlp, float coverage, float min_confidence,
                                      size_t fallback_n_probe, float* d_scores, uint64_t* d_ids,
                                      size_t* k_eff, void* stream);

/* ---- serving loop -------------------------------------------------------------
 * No counterpart in the reference (its tools time single synchronous calls).
 * Continuous batching over resident indexes on one GPU: requests wait in a
 * FIFO queue; whenever one of the server's max_slots slots (own CUDA streams,
 * pinned staging, device query / result buffers) is free, the oldest request
 * forms a batch with every later waiting request for the same index, k and
 * n_probe, up to max_batch queries. The batch's search scratch is sized
 * exactly on the host (a dry run of the search code) and taken from one
 * device arena: start() sizes the arena to what hbm_budget_bytes leaves after
 * the resident indexes, kernels and slot buffers (at most max_slots full
 * batches' worth, at least one, else TQ_ERR_OUT_OF_MEMORY). A batch whose
 * scratch does not fit waits, with the requests behind it, until running
 * batches return theirs: requests are admitted as slots and memory free up,
 * and batches in different slots overlap on the device. Serving allocates no
 * device memory. A query's result does not depend on the other queries of its
 * batch. Host buffers of a request must stay valid until tq_server_wait
 * returns for it. */
typedef struct tq_server tq_server;

int tq_server_create(int device, size_t hbm_budget_bytes, size_t max_slots, size_t max_batch,
                     tq_server** out);
int tq_server_destroy(tq_server* h);
/* Register an index (prepared, same device) before start(); *target is its id. */
int tq_server_add_flat(tq_server* h, tq_index* index, size_t max_k, int* target);
/* mlp (optional): the learned n_probe predictor; requests then scan each
 * query's predicted number of buckets, at most their n_probe. */
int tq_server_add_bucketed(tq_server* h, tq_bucketed* index, size_t max_k, size_t max_probe,
                           tq_probe_mlp* mlp, float coverage, float min_confidence, int* target);
int tq_server_start(tq_server* h);
/* slot_bytes: one slot's fixed device buffers; resident_bytes: device memory
 * in use at start() before the scratch arena (indexes, kernels, slots). */
int tq_server_info(tq_server* h, size_t* n_slots, size_t* slot_bytes, size_t* resident_bytes);
/* The scratch arena: its size, the most of it in use at once, the largest
 * scratch of any admissible batch, and how many batches had to wait for
 * arena memory. */
int tq_server_memory(tq_server* h, size_t* arena_bytes, size_t* arena_peak, size_t* max_batch_bytes,
                     uint64_t* memory_waits);
/* Scratch bytes a batch of nq queries of `target` with this k and n_probe
 * takes from the arena (the server's own sizing, on the host). */
int tq_server_batch_bytes(tq_server* h, int target, size_t nq, size_t k, size_t n_probe, size_t* bytes);
/* Queue a request (nq <= max_batch host rows); scores/ids receive nq x k_eff. */
int tq_server_submit(tq_server* h, int target, const float* queries, size_t nq, size_t k,
                     size_t n_probe, float* scores, uint64_t* ids, uint64_t* request);
/* Block until the request is done; latency from submission to the completion
 * of its result copy. */
int tq_server_wait(tq_server* h, uint64_t request, size_t* k_eff, double* latency_us);
int tq_server_stats(tq_server* h, uint64_t* batches, uint64_t* queries, uint64_t* completed,
                    size_t* peak_inflight);

/* Open-loop replay of a request trace: each item is submitted at its arrival
 * time (microseconds after the call starts); latency_us[i] runs from the
 * scheduled arrival to completion. */
typedef struct tq_replay_item {
  double arrival_us;
  int target;
  const float* queries;
  size_t nq, k, n_probe;
  float* scores;
  uint64_t* ids;
} tq_replay_item;
int tq_server_replay(tq_server* h, const tq_replay_item* items, size_t n, double* latency_us,
                     double* wall_s);

/* ---- multi-index launch -----------------------------------------------------
 * No counterpart in the reference. One persistent scan launch serves many
 * prepared flat indexes (same device; any n, dim, bits) with per-index batch
 * sizes and k: work items (index, vector range, up to 8 queries) are pulled
 * from a global counter by a fixed grid of CTAs. tq_multi_plan fixes the batch
 * size nq[i] and k[i] of every index, sizes all scratch, optionally autotunes
 * the item range length and resident CTAs per SM (timed on the planned
 * workload), and captures query-LUT kernels + scan + merges into one CUDA
 * graph; tq_multi_launch replays it. Queries go into the device buffers given
 * by tq_multi_buffers (nq[i] x dim_i floats) before a launch; results come out
 * as nq[i] x k_eff rows, identical to tq_index_search on each index. */
typedef struct tq_multi tq_multi;

int tq_multi_create(tq_index* const* indexes, size_t n_indexes, tq_multi** out);
int tq_multi_destroy(tq_multi* h);
int tq_multi_plan(tq_multi* h, const size_t* nq, const size_t* k, int autotune);
int tq_multi_buffers(tq_multi* h, size_t i, float** d_queries, float** d_scores, uint64_t** d_ids,
                     size_t* k_eff);
/* Graph launch on `stream` (NULL: the multi-index object's stream). */
int tq_multi_launch(tq_multi* h, void* stream);
/* The same sequence issued kernel by kernel (no graph), for comparison. */
int tq_multi_run_uncaptured(tq_multi* h, void* stream);
int tq_multi_synchronize(tq_multi* h);
/* Chosen configuration; tuned_ms receives up to *n_tuned candidate timings
 * (on return *n_tuned = candidates timed). */
int tq_multi_config(tq_multi* h, long long* range_vectors, int* ctas, size_t* n_items, size_t* smem_bytes,
                    double* tuned_ms, size_t* n_tuned);
/* The autotuner's third pass may route the heaviest index batches (by nq x n
 * x byte groups) to the single-index scan kernels, inside the same graph;
 * flags[i] = 1 marks those (n_indexes entries). */
int tq_multi_direct(tq_multi* h, size_t* n_direct, uint8_t* flags);
/* Synchronous copies into / out of the library's device buffers (for callers
 * without their own CUDA runtime). */
int tq_copy_to_device(void* d_dst, const void* src, size_t bytes);
int tq_copy_to_host(void* dst, const void* d_src, size_t bytes);

/* ---- search without device allocation --------------------------------------
 * No counterpart in the reference.
 *
 * Same inputs, outputs and results as tq_index_search_device, but the call
 * allocates no device memory: its temporary buffers (query LUTs, per-query
 * constants, candidate lists) live in one fixed 16 MiB array compiled into the
 * library, which every GPU that loads the library holds until the process
 * exits. It is meant for callers that may not allocate while serving queries —
 * for example a server that hands all free HBM to its own pool up front, or a
 * latency-critical loop that cannot afford cudaMalloc's implicit
 * synchronization. The index itself must already be prepared.
 *
 * Limits: a request must fit in the 16 MiB array — nq * (dim / (8 / bits)) * 32
 * bytes of LUTs plus 16 bytes per query plus the candidate lists (at least
 * nq * 8 * k_eff * 8 bytes). Larger requests fail with TQ_ERR_INVALID_ARGUMENT
 * before any work is queued; split them into smaller batches.
 *
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture. All calls on one device share the array and each
 * call overwrites everything it reads from it (nothing has to start at zero),
 * so calls whose work overlaps on the GPU — on different streams or for
 * different indexes on the same device — race and must be serialized by the
 * caller. Returns without synchronizing `stream` (NULL: the index's stream). */
int tq_index_search_device_noalloc(tq_index* h, const float* d_queries, size_t nq, size_t k,
                                   float* d_scores, uint64_t* d_ids, size_t* k_eff,
                                   void* stream);

#ifdef __cplusplus
}
#endif

#endif /* VECTORCACHE_B200_H */
