/* Test infrastructure only — the CPU oracle for the flat TurboQuant path.
 *
 * A plain-C restatement of the reference's (nishadtardalkar/vectorcache) CPU
 * arithmetic, used by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg as the CHECKER. The product library never links or calls it.
 * Each function names the reference file:line it follows. It is pinned against
 * the reference's own code (oracle/_ref) and against the committed golden
 * vectors in tests/golden/.
 */
#ifndef TQ_ORACLE_H
#define TQ_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ChaCha8 keystream with the rotation seed; signs then Fisher-Yates perm. */
int tqo_rotation(size_t dim, float* signs, uint32_t* perm);

/* Lloyd-Max codebook for Beta((dim-1)/2, (dim-1)/2) on [-1, 1]. */
int tqo_codebook(size_t bits, size_t dim, float* boundaries, float* centroids);

/* Beta(a, a) CDF at t (regularized incomplete beta). */
double tqo_beta_cdf_aa(double a, double t);

/* L2 norm (8 interleaved float chains) + rotation of n rows. */
int tqo_rotate_rows(const float* x, size_t n, size_t dim, float* rot_out, float* norms);

/* TQ+ per-dimension shift / scale from a calibration sample. */
int tqo_fit_calibration(const float* x, size_t n, size_t dim, size_t bits, float* shift,
                        float* scale);

/* Bit-plane encode: packed_out = n * bits * dim/8 bytes, alpha = n floats.
 * shift/scale may be NULL (no TQ+). */
int tqo_encode(const float* x, size_t n, size_t dim, size_t bits, const float* shift,
               const float* scale, uint8_t* packed_out, float* alpha);

/* Bit-plane rows -> row-major codes_flat (n * nbg bytes). */
int tqo_codes_flat(const uint8_t* packed, size_t n, size_t bits, size_t dim, uint8_t* out);

/* Query side: q_rot (nq*dim), bias_corr (nq), luts (nq*nbg*32), lut_scale,
 * lut_bias (nq each). shift/scale may be NULL. */
int tqo_prepare_queries(const float* q, size_t nq, size_t dim, size_t bits, const float* shift,
                        const float* scale, float* q_rot, float* bias_corr, uint8_t* luts,
                        float* lut_scale, float* lut_bias);

/* Integer LUT score sum over all byte groups: out[qi*n + vi]. */
void tqo_int_scores(const uint8_t* luts, size_t nq, const uint8_t* codes_flat, size_t n,
                    size_t nbg, uint32_t* out);

/* Float score exactly as the AVX2 PERM0 scan forms it: out[qi*n + vi]. */
void tqo_float_scores(const uint8_t* luts, const float* lut_scale, const float* lut_bias,
                      const float* bias_corr, size_t nq, const uint8_t* codes_flat,
                      const float* alpha, size_t n, size_t nbg, float* out);

/* Exact top-k per row of a score matrix: score desc, ties by lower id.
 * Rows written with stride k_eff = min(k, n); returns k_eff. */
size_t tqo_topk(const float* scores, size_t nq, size_t n, size_t k, float* out_scores,
                uint64_t* out_ids);

/* End-to-end flat search (prepare + score + top-k) against an encoded index. */
size_t tqo_search_flat(const float* q, size_t nq, size_t dim, size_t bits, const float* shift,
                       const float* scale, const uint8_t* packed, const float* alpha, size_t n,
                       size_t k, float* out_scores, uint64_t* out_ids);

/* Exact float re-rank in place: scores[q][j] = <q, corpus[ids[q][j]]> in the
 * reference's AVX2 summation order, rows re-sorted (score desc, id asc);
 * ids >= n_corpus score -inf. */
void tqo_float_rescore(const float* queries, size_t nq, size_t dim, const float* corpus,
                       size_t n_corpus, size_t k, float* scores, uint64_t* ids);

/* IVF residual search over bucket-ordered slots (score_prepared_into,
 * search.cpp:1156-1264, composed per query over its probed buckets). */
void tqo_ivf_search(const uint8_t* luts, const float* lut_scale, const float* lut_bias,
                    const float* bias_corr, size_t nq, size_t nbg, const uint8_t* codes_flat,
                    const float* alpha, const uint64_t* ids, const uint64_t* bucket_start,
                    const uint64_t* bucket_size, const uint32_t* probes,
                    const uint32_t* n_probe, size_t max_probe, const float* offsets, size_t k,
                    float* out_scores, uint64_t* out_ids);

#ifdef __cplusplus
}
#endif

#endif
