/* Test infrastructure only — the CPU oracle for the flat TurboQuant path.
 *
 * Plain-C restatement of the reference's (nishadtardalkar/vectorcache) CPU
 * arithmetic. tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg
 * use it as the checker; the product library never links or calls it.
 *
 * Parity pins: this file is checked bit-for-bit against the reference's own
 * code compiled in place (oracle/_ref/libtqref.so, see ref_shim.cpp) and
 * against the golden vectors committed in tests/golden/ (generated from that
 * library by tests/golden/make_golden.py).
 *
 * The reference is compiled with -O3 -mavx2 -mfma -ffp-contract=fast
 * (CMakeLists.txt:62-66), so GCC fuses a multiply into the add/sub that
 * consumes it whenever that is the product's only use. This file is compiled
 * with -ffp-contract=off and writes each of those fusions out as fma()/fmaf(),
 * so the arithmetic is stated explicitly rather than left to the compiler.
 */
#include "tq_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ----------------------------------------------------------------------------
 * ChaCha8 keystream (chacha8.cpp:34-85): IETF ChaCha state with a 32-byte key,
 * a 64-bit block counter in words 12-13, zero nonce, 4 double rounds, output
 * words consumed in order; next_u64 = lo | hi << 32.
 * ------------------------------------------------------------------------- */
typedef struct {
  uint32_t key[16];
  uint32_t out[16];
  int pos;
} chacha8_t;

static uint32_t rotl(uint32_t v, int r) { return (v << r) | (v >> (32 - r)); }

#define QR(a, b, c, d)          \
  do {                          \
    a += b; d = rotl(d ^ a, 16); \
    c += d; b = rotl(b ^ c, 12); \
    a += b; d = rotl(d ^ a, 8);  \
    c += d; b = rotl(b ^ c, 7);  \
  } while (0)

static void chacha8_init(chacha8_t* s, const uint8_t seed[32]) {
  static const uint32_t sigma[4] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u};
  for (int i = 0; i < 4; ++i) s->key[i] = sigma[i];
  for (int i = 0; i < 8; ++i) {
    const uint8_t* p = seed + 4 * i;
    s->key[4 + i] = (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) |
                    ((uint32_t)p[3] << 24);
  }
  for (int i = 12; i < 16; ++i) s->key[i] = 0;
  s->pos = 16;
}

static void chacha8_block(chacha8_t* s) {
  uint32_t x[16];
  memcpy(x, s->key, sizeof x);
  for (int r = 0; r < 4; ++r) {
    QR(x[0], x[4], x[8], x[12]);
    QR(x[1], x[5], x[9], x[13]);
    QR(x[2], x[6], x[10], x[14]);
    QR(x[3], x[7], x[11], x[15]);
    QR(x[0], x[5], x[10], x[15]);
    QR(x[1], x[6], x[11], x[12]);
    QR(x[2], x[7], x[8], x[13]);
    QR(x[3], x[4], x[9], x[14]);
  }
  for (int i = 0; i < 16; ++i) s->out[i] = x[i] + s->key[i];
  s->key[12] += 1u;
  if (s->key[12] == 0u) s->key[13] += 1u;
  s->pos = 0;
}

static uint32_t chacha8_u32(chacha8_t* s) {
  if (s->pos >= 16) chacha8_block(s);
  return s->out[s->pos++];
}

static uint64_t chacha8_u64(chacha8_t* s) {
  const uint64_t lo = chacha8_u32(s);
  const uint64_t hi = chacha8_u32(s);
  return lo | (hi << 32);
}

/* Fixed rotation seed (rotation.cpp:18-20). */
static const uint8_t kRotationSeed[32] = {164, 143, 161, 123, 88,  50,  61,  10,
                                          234, 184, 161, 204, 105, 1,   20,  184,
                                          43,  140, 200, 117, 24,  180, 247, 84,
                                          141, 68,  110, 161, 228, 223, 32,  242};

static int dim_ok(size_t dim) { return dim > 0 && dim % 8 == 0 && dim <= 16384; }
static int bits_ok(size_t bits) { return bits >= 2 && bits <= 4; }
static size_t nbg_of(size_t bits, size_t dim) { return dim / (8 / bits); }

/* Rotation tables (rotation.cpp:139-160, fisher_yates :24-35): dim signs from
 * next_u32() & 1 (1 -> -1), then perm = identity shuffled from the top with
 * j = next_u64() % (i + 1). One round (kRotationRounds = 1). */
int tqo_rotation(size_t dim, float* signs, uint32_t* perm) {
  if (!dim_ok(dim)) return 1;
  chacha8_t rng;
  chacha8_init(&rng, kRotationSeed);
  for (size_t i = 0; i < dim; ++i) signs[i] = (chacha8_u32(&rng) & 1u) ? -1.f : 1.f;
  for (size_t i = 0; i < dim; ++i) perm[i] = (uint32_t)i;
  for (size_t i = dim - 1; i >= 1; --i) {
    const size_t j = (size_t)(chacha8_u64(&rng) % ((uint64_t)i + 1));
    const uint32_t t = perm[i];
    perm[i] = perm[j];
    perm[j] = t;
  }
  return 0;
}

/* ----------------------------------------------------------------------------
 * Special functions in double (codebook.cpp:12-110, encode.cpp:42-112).
 * ------------------------------------------------------------------------- */
#define TQ_PI 3.14159265358979323846

/* Lanczos log-gamma, g = 7, nine coefficients (published table). */
static double lgamma_lanczos(double z) {
  static const double c[9] = {0.99999999999980993,  676.5203681218851,     -1259.1392167224028,
                              771.32342877765313,   -176.61502916214059,   12.507343278686905,
                              -0.13857109526572012, 9.984369654078861e-6, 1.5056327351493116e-7};
  if (z < 0.5) {
    return log(TQ_PI) - log(sin(TQ_PI * z)) - lgamma_lanczos(1.0 - z);
  }
  z -= 1.0;
  double s = c[0];
  for (int i = 1; i < 9; ++i) s += c[i] / (z + (double)i);
  const double t = z + 7.5;
  const double half_log_2pi = 0.5 * log(2.0 * TQ_PI);
  /* (z + 0.5) * log(t) fuses into the add of the constant. */
  return fma(z + 0.5, log(t), half_log_2pi) - t + log(s);
}

/* Continued fraction for the incomplete beta (modified Lentz). */
static double beta_cf(double a, double b, double x) {
  const double tiny = 1e-30;
  const double qab = a + b, qap = a + 1.0, qam = a - 1.0;
  double c = 1.0;
  double d = 1.0 - qab * x / qap;
  if (fabs(d) < tiny) d = tiny;
  d = 1.0 / d;
  double h = d;
  for (int m = 1; m <= 200; ++m) {
    const double m2 = 2.0 * m;
    double aa = (double)m * (b - (double)m) * x / ((qam + m2) * (a + m2));
    d = fma(aa, d, 1.0);
    if (fabs(d) < tiny) d = tiny;
    c = 1.0 + aa / c;
    if (fabs(c) < tiny) c = tiny;
    d = 1.0 / d;
    h *= d * c;
    aa = -(a + (double)m) * (qab + (double)m) * x / ((a + m2) * (qap + m2));
    d = fma(aa, d, 1.0);
    if (fabs(d) < tiny) d = tiny;
    c = 1.0 + aa / c;
    if (fabs(c) < tiny) c = tiny;
    d = 1.0 / d;
    const double del = d * c;
    h *= del;
    if (fabs(del - 1.0) < 3e-14) break;
  }
  return h;
}

static double inc_beta(double a, double b, double x) {
  if (x <= 0.0) return 0.0;
  if (x >= 1.0) return 1.0;
  const double lbeta = lgamma_lanczos(a) + lgamma_lanczos(b) - lgamma_lanczos(a + b);
  const double lx = log(x);
  const double l1x = log(1.0 - x);
  const double e = exp(fma(lx, a, l1x * b) - lbeta);
  if (x < (a + 1.0) / (a + b + 2.0)) {
    return e / a * beta_cf(a, b, x);
  }
  return fma(-(e / b), beta_cf(b, a, 1.0 - x), 1.0);
}

double tqo_beta_cdf_aa(double a, double t) { return inc_beta(a, a, t); }

/* Beta(a, a) density on (0, 1). */
static double beta_pdf_aa(double a, double t) {
  if (t <= 0.0 || t >= 1.0) return 0.0;
  const double lbeta = 2.0 * lgamma_lanczos(a) - lgamma_lanczos(2.0 * a);
  const double am1 = a - 1.0;
  return exp(fma(am1, log(t), am1 * log(1.0 - t)) - lbeta);
}

/* Integrand of the conditional mean over a cell: x * p(x) with x in [-1, 1]
 * and p the density of 2*Beta(a,a) - 1. */
static double mean_integrand(double a, double x) {
  const double t = (x + 1.0) / 2.0;
  return x * beta_pdf_aa(a, t) / 2.0;
}

static double simpson_rec(double alpha, double lo, double hi, double flo, double fhi, double fmid,
                          double whole, double tol, int depth) {
  const double mid = (lo + hi) / 2.0;
  const double q1 = (lo + mid) / 2.0;
  const double q3 = (mid + hi) / 2.0;
  const double f1 = mean_integrand(alpha, q1);
  const double f3 = mean_integrand(alpha, q3);
  const double left = (mid - lo) / 6.0 * (flo + 4.0 * f1 + fmid);
  const double right = (hi - mid) / 6.0 * (fmid + 4.0 * f3 + fhi);
  const double both = left + right;
  if (depth == 0 || fabs(both - whole) < 15.0 * tol) {
    return both + (both - whole) / 15.0;
  }
  return simpson_rec(alpha, lo, mid, flo, fmid, f1, left, tol / 2.0, depth - 1) +
         simpson_rec(alpha, mid, hi, fmid, fhi, f3, right, tol / 2.0, depth - 1);
}

static double cell_mean_mass(double alpha, double lo, double hi) {
  const double mid = (lo + hi) / 2.0;
  const double flo = mean_integrand(alpha, lo);
  const double fhi = mean_integrand(alpha, hi);
  const double fmid = mean_integrand(alpha, mid);
  const double whole = (hi - lo) / 6.0 * (flo + 4.0 * fmid + fhi);
  return simpson_rec(alpha, lo, hi, flo, fhi, fmid, whole, 1e-14, 50);
}

/* Lloyd-Max codebook (codebook.cpp:135-195): levels start evenly spaced over
 * +-3 std of the coordinate distribution, then alternate midpoint boundaries
 * and conditional means until no centroid moves by 1e-12 (<= 200 rounds).
 * Centroids are cast to f32; boundaries are f32 midpoints of the f32
 * centroids (codebook.cpp:191-193). */
int tqo_codebook(size_t bits, size_t dim, float* boundaries, float* centroids) {
  if (!bits_ok(bits) || dim < 2) return 1;
  const double a = ((double)dim - 1.0) / 2.0;
  const size_t L = (size_t)1 << bits;
  const double sd = sqrt(2.0 * a / ((2.0 * a + 1.0) * 4.0 * a));
  const double spread = 3.0 * sd;
  double c[16], nc[16], edge[17];
  for (size_t i = 0; i < L; ++i) c[i] = -spread + 2.0 * spread * (double)i / (double)(L - 1);
  for (int it = 0; it < 200; ++it) {
    edge[0] = -1.0;
    for (size_t i = 0; i + 1 < L; ++i) edge[i + 1] = (c[i] + c[i + 1]) / 2.0;
    edge[L] = 1.0;
    for (size_t i = 0; i < L; ++i) {
      const double lo = edge[i], hi = edge[i + 1];
      const double mass = inc_beta(a, a, (hi + 1.0) / 2.0) - inc_beta(a, a, (lo + 1.0) / 2.0);
      nc[i] = (mass < 1e-15) ? c[i] : cell_mean_mass(a, lo, hi) / mass;
    }
    double moved = 0.0;
    for (size_t i = 0; i < L; ++i) {
      const double dlt = fabs(c[i] - nc[i]);
      if (dlt > moved) moved = dlt;
      c[i] = nc[i];
    }
    if (moved < 1e-12) break;
  }
  for (size_t i = 0; i < L; ++i) centroids[i] = (float)c[i];
  for (size_t i = 0; i + 1 < L; ++i) boundaries[i] = (centroids[i] + centroids[i + 1]) * 0.5f;
  return 0;
}

/* ----------------------------------------------------------------------------
 * Row transform.
 * ------------------------------------------------------------------------- */

/* ||row|| with 8 interleaved f32 chains combined as a tree
 * (encode.cpp:16-26, :290); each chain step is a fused multiply-add. */
static float row_norm(const float* row, size_t dim) {
  float ch[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (size_t j = 0; j < dim; ++j) ch[j & 7] = fmaf(row[j], row[j], ch[j & 7]);
  const float s = ((ch[0] + ch[1]) + (ch[2] + ch[3])) + ((ch[4] + ch[5]) + (ch[6] + ch[7]));
  return sqrtf(s);
}

/* y[i] = (x[perm[i]] * inv) * sign[i], then a normalized Walsh-Hadamard
 * transform on each block of B = dim & -dim: stages of butterflies
 * (a + b, a - b) at strides 1, 2, 4, ..., then x 1/sqrt(B)
 * (rotation.cpp:38-121, :185-205). */
static void rotate_row(const float* x, float inv, const float* signs, const uint32_t* perm,
                       size_t dim, float* y) {
  const size_t B = dim & (~dim + 1);
  const float inv_sqrt_b = 1.f / sqrtf((float)B);
  for (size_t i = 0; i < dim; ++i) y[i] = (x[perm[i]] * inv) * signs[i];
  for (size_t off = 0; off < dim; off += B) {
    float* blk = y + off;
    for (size_t len = 1; len < B; len <<= 1) {
      for (size_t i = 0; i < B; i += 2 * len) {
        for (size_t j = i; j < i + len; ++j) {
          const float u = blk[j], v = blk[j + len];
          blk[j] = u + v;
          blk[j + len] = u - v;
        }
      }
    }
    for (size_t i = 0; i < B; ++i) blk[i] *= inv_sqrt_b;
  }
}

int tqo_rotate_rows(const float* x, size_t n, size_t dim, float* rot_out, float* norms) {
  if (!dim_ok(dim)) return 1;
  float* signs = malloc(dim * sizeof(float));
  uint32_t* perm = malloc(dim * sizeof(uint32_t));
  tqo_rotation(dim, signs, perm);
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < (long long)n; ++i) {
    const float* src = x + (size_t)i * dim;
    const float nv = row_norm(src, dim);
    if (norms) norms[i] = nv;
    const float inv = (nv > 1e-10f) ? (1.f / nv) : 0.f;
    rotate_row(src, inv, signs, perm, dim, rot_out + (size_t)i * dim);
  }
  free(signs);
  free(perm);
  return 0;
}

/* ----------------------------------------------------------------------------
 * TQ+ calibration (encode.cpp:233-286, :327-335).
 * ------------------------------------------------------------------------- */
static uint32_t f32_key(float f) {
  uint32_t b;
  memcpy(&b, &f, 4);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

static float f32_unkey(uint32_t k) {
  const uint32_t b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  float f;
  memcpy(&f, &b, 4);
  return f;
}

static int cmp_u32(const void* pa, const void* pb) {
  const uint32_t a = *(const uint32_t*)pa, b = *(const uint32_t*)pb;
  return (a > b) - (a < b);
}

int tqo_fit_calibration(const float* x, size_t n, size_t dim, size_t bits, float* shift,
                        float* scale) {
  if (!dim_ok(dim) || !bits_ok(bits) || n < 2) return 1;
  float bnd[15], cen[16];
  tqo_codebook(bits, dim, bnd, cen);
  const size_t L = (size_t)1 << bits;
  float c_outer = 0.f;
  for (size_t i = 0; i < L; ++i) c_outer = fmaxf(c_outer, fabsf(cen[i]));
  const double a = ((double)dim - 1.0) / 2.0;
  const double p_hi = inc_beta(a, a, ((double)c_outer + 1.0) / 2.0);
  const double p_lo = 1.0 - p_hi;
  const float qc_lo = -c_outer, qc_span = c_outer - (-c_outer);
  size_t lo_idx = (size_t)((double)n * p_lo);
  size_t hi_idx = (size_t)((double)n * p_hi);
  if (hi_idx > n - 1) hi_idx = n - 1;
  if (hi_idx < lo_idx + 1) hi_idx = lo_idx + 1;

  float* rot = malloc(n * dim * sizeof(float));
  tqo_rotate_rows(x, n, dim, rot, NULL);
#pragma omp parallel
  {
    uint32_t* col = malloc(n * sizeof(uint32_t));
#pragma omp for schedule(static)
    for (long long d = 0; d < (long long)dim; ++d) {
      shift[d] = 0.f;
      scale[d] = 1.f;
      for (size_t i = 0; i < n; ++i) col[i] = f32_key(rot[i * dim + (size_t)d]);
      qsort(col, n, sizeof(uint32_t), cmp_u32);
      const float q_lo = f32_unkey(col[lo_idx]);
      const float q_hi = f32_unkey(col[hi_idx]);
      const float span = q_hi - q_lo;
      if (!(span > 1e-12f) || !(qc_span > 0.f)) continue;
      const float s = qc_span / span;
      scale[d] = s;
      shift[d] = qc_lo / s - q_lo;
    }
    free(col);
  }
  free(rot);
  return 0;
}

/* ----------------------------------------------------------------------------
 * Encode (encode.cpp:112-157, :185-231, :294-307).
 * ------------------------------------------------------------------------- */
int tqo_encode(const float* x, size_t n, size_t dim, size_t bits, const float* shift,
               const float* scale, uint8_t* packed_out, float* alpha) {
  if (!dim_ok(dim) || !bits_ok(bits)) return 1;
  float bnd[15], cen[16];
  tqo_codebook(bits, dim, bnd, cen);
  const size_t nb = ((size_t)1 << bits) - 1;
  const size_t bpp = dim / 8;
  float* signs = malloc(dim * sizeof(float));
  uint32_t* perm = malloc(dim * sizeof(uint32_t));
  float* inv_scale = malloc(dim * sizeof(float));
  tqo_rotation(dim, signs, perm);
  /* Without a calibration the plain path runs (encode.cpp:207-214); with one,
   * the calibrated path runs even when it is the identity. */
  const int identity = (shift == NULL);
  if (shift) {
    for (size_t d = 0; d < dim; ++d) inv_scale[d] = 1.f / scale[d];
  }
#pragma omp parallel
  {
    float* y = malloc(dim * sizeof(float));
#pragma omp for schedule(static)
    for (long long ii = 0; ii < (long long)n; ++ii) {
      const size_t i = (size_t)ii;
      const float* src = x + i * dim;
      const float nv = row_norm(src, dim);
      const float inv = (nv > 1e-10f) ? (1.f / nv) : 0.f;
      rotate_row(src, inv, signs, perm, dim, y);
      double ch[4] = {0.0, 0.0, 0.0, 0.0};
      uint8_t* prow = packed_out + i * bits * bpp;
      for (size_t cb = 0; cb < bpp; ++cb) {
        uint8_t code[8];
        for (size_t k = 0; k < 8; ++k) {
          const size_t j = cb * 8 + k;
          const float v = identity ? y[j] : (y[j] + shift[j]) * scale[j];
          unsigned q = 0;
          for (size_t b = 0; b < nb; ++b) q += (v > bnd[b]) ? 1u : 0u;
          code[k] = (uint8_t)q;
          if (identity) {
            ch[j & 3] += (double)y[j] * (double)cen[q];
          } else {
            /* centroid mapped back to the un-calibrated axis, then a fused
             * multiply-add into the chain. */
            const double back = (double)cen[q] * (double)inv_scale[j] - (double)shift[j];
            ch[j & 3] = fma((double)y[j], back, ch[j & 3]);
          }
        }
        for (size_t p = 0; p < bits; ++p) {
          uint8_t byte = 0;
          for (size_t k = 0; k < 8; ++k) byte |= (uint8_t)(((code[k] >> p) & 1u) << (7 - k));
          prow[p * bpp + cb] = byte;
        }
      }
      const double inner = (ch[0] + ch[1]) + (ch[2] + ch[3]);
      alpha[i] = (inner > 1e-12) ? nv / (float)inner : 0.f;
    }
    free(y);
  }
  free(signs);
  free(perm);
  free(inv_scale);
  return 0;
}

/* Bit-plane rows -> row-major codes_flat (pack.cpp:70-131): codes_per_byte =
 * 8 / bits codes share a byte, first code in the high bits, 3-bit codes in a
 * 4-bit field. */
int tqo_codes_flat(const uint8_t* packed, size_t n, size_t bits, size_t dim, uint8_t* out) {
  if (!dim_ok(dim) || !bits_ok(bits)) return 1;
  const size_t bpp = dim / 8;
  const size_t cpb = 8 / bits;
  const size_t field = (bits == 3) ? 4 : bits;
  const size_t nbg = nbg_of(bits, dim);
#pragma omp parallel for schedule(static)
  for (long long vv = 0; vv < (long long)n; ++vv) {
    const size_t v = (size_t)vv;
    const uint8_t* row = packed + v * bits * bpp;
    uint8_t* o = out + v * nbg;
    memset(o, 0, nbg);
    for (size_t j = 0; j < dim; ++j) {
      unsigned code = 0;
      for (size_t p = 0; p < bits; ++p) code |= ((row[p * bpp + j / 8] >> (7 - j % 8)) & 1u) << p;
      const size_t g = j / cpb;
      const size_t sh = (cpb - 1 - j % cpb) * field;
      o[g] |= (uint8_t)(code << sh);
    }
  }
  return 0;
}

/* ----------------------------------------------------------------------------
 * Query side (search.cpp:149-219, :762-860).
 * ------------------------------------------------------------------------- */
static void build_lut(const float* qr, const float* cen, size_t bits, size_t dim, uint8_t* lut,
                      float* out_scale, float* out_bias) {
  const size_t cpb = 8 / bits;
  const size_t cpn = cpb / 2;
  const size_t nbg = dim / cpb;
  const unsigned mask = (1u << bits) - 1u;
  float* vals = malloc(nbg * 32 * sizeof(float));
  float* mins = malloc(nbg * 2 * sizeof(float));
  float span_max = 0.f, bias = 0.f;
  for (size_t g = 0; g < nbg; ++g) {
    const size_t d0 = g * cpb;
    for (int half = 0; half < 2; ++half) {
      float mn = FLT_MAX, mx = -FLT_MAX;
      for (unsigned nv = 0; nv < 16; ++nv) {
        float s = 0.f;
        for (size_t c = 0; c < cpn; ++c) {
          const unsigned code = (nv >> ((cpn - 1 - c) * bits)) & mask;
          s = fmaf(qr[d0 + (size_t)half * cpn + c], cen[code], s);
        }
        vals[g * 32 + (size_t)half * 16 + nv] = s;
        mn = fminf(mn, s);
        mx = fmaxf(mx, s);
      }
      mins[g * 2 + (size_t)half] = mn;
      span_max = fmaxf(span_max, mx - mn);
    }
    bias += mins[g * 2] + mins[g * 2 + 1];
  }
  float scale = (span_max > 0.f) ? span_max / 127.f : 1.f;
  float inv = 1.f;
  if (scale >= FLT_MIN) {
    inv = 1.f / scale;
  } else {
    scale = 1.f;
  }
  for (size_t g = 0; g < nbg; ++g) {
    for (int i = 0; i < 32; ++i) {
      const float mn = mins[g * 2 + (i >= 16 ? 1 : 0)];
      float r = roundf((vals[g * 32 + (size_t)i] - mn) * inv);
      r = r < 0.f ? 0.f : (r > 127.f ? 127.f : r);
      lut[g * 32 + (size_t)i] = (uint8_t)r;
    }
  }
  *out_scale = scale;
  *out_bias = bias;
  free(vals);
  free(mins);
}

int tqo_prepare_queries(const float* q, size_t nq, size_t dim, size_t bits, const float* shift,
                        const float* scale, float* q_rot, float* bias_corr, uint8_t* luts,
                        float* lut_scale, float* lut_bias) {
  if (!dim_ok(dim) || !bits_ok(bits)) return 1;
  float bnd[15], cen[16];
  tqo_codebook(bits, dim, bnd, cen);
  const size_t nbg = nbg_of(bits, dim);
  tqo_rotate_rows(q, nq, dim, q_rot, NULL);
#pragma omp parallel for schedule(static)
  for (long long ii = 0; ii < (long long)nq; ++ii) {
    const size_t i = (size_t)ii;
    float* row = q_rot + i * dim;
    bias_corr[i] = 0.f;
    if (shift) {
      double bc = 0.0;
      for (size_t d = 0; d < dim; ++d) {
        const float r = row[d];
        row[d] = r / scale[d];
        bc -= (double)r * (double)shift[d];
      }
      bias_corr[i] = (float)bc;
    }
    build_lut(row, cen, bits, dim, luts + i * nbg * 32, lut_scale + i, lut_bias + i);
  }
  return 0;
}

/* ----------------------------------------------------------------------------
 * Scan (search_avx2.cpp:24-225).
 * ------------------------------------------------------------------------- */
void tqo_int_scores(const uint8_t* luts, size_t nq, const uint8_t* codes_flat, size_t n,
                    size_t nbg, uint32_t* out) {
#pragma omp parallel for schedule(static) collapse(2)
  for (long long qi = 0; qi < (long long)nq; ++qi) {
    for (long long vi = 0; vi < (long long)n; ++vi) {
      const uint8_t* lut = luts + (size_t)qi * nbg * 32;
      const uint8_t* c = codes_flat + (size_t)vi * nbg;
      uint32_t acc = 0;
      for (size_t g = 0; g < nbg; ++g) acc += lut[g * 32 + (c[g] >> 4)] + lut[g * 32 + 16 + (c[g] & 15)];
      out[(size_t)qi * n + (size_t)vi] = acc;
    }
  }
}

/* fa starts at lut bias + bias_corr; every batch of up to 256 byte groups
 * (kFlushEvery) adds scale * (integer batch sum) with one fused multiply-add;
 * the score is fa * alpha (search_avx2.cpp:24-48, :100-205). */
void tqo_float_scores(const uint8_t* luts, const float* lut_scale, const float* lut_bias,
                      const float* bias_corr, size_t nq, const uint8_t* codes_flat,
                      const float* alpha, size_t n, size_t nbg, float* out) {
#pragma omp parallel for schedule(static) collapse(2)
  for (long long qi = 0; qi < (long long)nq; ++qi) {
    for (long long vi = 0; vi < (long long)n; ++vi) {
      const uint8_t* lut = luts + (size_t)qi * nbg * 32;
      const uint8_t* c = codes_flat + (size_t)vi * nbg;
      float fa = lut_bias[qi] + (bias_corr ? bias_corr[qi] : 0.f);
      for (size_t g0 = 0; g0 < nbg; g0 += 256) {
        const size_t g1 = (g0 + 256 < nbg) ? g0 + 256 : nbg;
        uint32_t acc = 0;
        for (size_t g = g0; g < g1; ++g) acc += lut[g * 32 + (c[g] >> 4)] + lut[g * 32 + 16 + (c[g] & 15)];
        fa = fmaf(lut_scale[qi], (float)acc, fa);
      }
      out[(size_t)qi * n + (size_t)vi] = fa * alpha[vi] + 0.f;
    }
  }
}

/* Top-k with the reference's order: higher score first, equal scores by lower
 * id (topk_heap.hpp:19-22, search.cpp:739-752). Candidates must beat -inf
 * (heap admission is a strict '>' against an initial -inf). */
typedef struct {
  float s;
  uint64_t id;
} cand_t;

static int better(const cand_t* a, const cand_t* b) {
  if (a->s != b->s) return a->s > b->s;
  return a->id < b->id;
}

size_t tqo_topk(const float* scores, size_t nq, size_t n, size_t k, float* out_scores,
                uint64_t* out_ids) {
  const size_t ke = k < n ? k : n;
  if (ke == 0) return 0;
#pragma omp parallel
  {
    cand_t* top = malloc(ke * sizeof(cand_t));
#pragma omp for schedule(static)
    for (long long qi = 0; qi < (long long)nq; ++qi) {
      const float* row = scores + (size_t)qi * n;
      size_t cnt = 0;
      for (size_t v = 0; v < n; ++v) {
        cand_t c = {row[v], v};
        if (!(c.s > -INFINITY)) continue;
        if (cnt == ke && !better(&c, &top[ke - 1])) continue;
        size_t pos = (cnt < ke) ? cnt++ : ke - 1;
        while (pos > 0 && better(&c, &top[pos - 1])) {
          top[pos] = top[pos - 1];
          --pos;
        }
        top[pos] = c;
      }
      for (size_t j = 0; j < ke; ++j) {
        out_scores[(size_t)qi * ke + j] = j < cnt ? top[j].s : 0.f;
        out_ids[(size_t)qi * ke + j] = j < cnt ? top[j].id : 0;
      }
    }
    free(top);
  }
  return ke;
}

size_t tqo_search_flat(const float* q, size_t nq, size_t dim, size_t bits, const float* shift,
                       const float* scale, const uint8_t* packed, const float* alpha, size_t n,
                       size_t k, float* out_scores, uint64_t* out_ids) {
  const size_t nbg = nbg_of(bits, dim);
  float* q_rot = malloc(nq * dim * sizeof(float));
  float* bc = malloc(nq * sizeof(float));
  float* ls = malloc(nq * sizeof(float));
  float* lb = malloc(nq * sizeof(float));
  uint8_t* luts = malloc(nq * nbg * 32);
  uint8_t* flat = malloc(n * nbg + 1);
  float* sc = malloc(nq * n * sizeof(float) + 1);
  tqo_prepare_queries(q, nq, dim, bits, shift, scale, q_rot, bc, luts, ls, lb);
  tqo_codes_flat(packed, n, bits, dim, flat);
  tqo_float_scores(luts, ls, lb, bc, nq, flat, alpha, n, nbg, sc);
  const size_t ke = tqo_topk(sc, nq, n, k, out_scores, out_ids);
  free(q_rot);
  free(bc);
  free(ls);
  free(lb);
  free(luts);
  free(flat);
  free(sc);
  return ke;
}

/* ----------------------------------------------------------------------------
 * Exact float re-rank (float_rescore.cpp:23-58 dot product, :80-164 driver).
 * The dot product: 16 fused multiply-add chains over the first dim - dim % 16
 * elements (element i feeds chain i % 16), chains 8..15 added lane-wise into
 * 0..7, an 8-element tail into chains 0..7 when dim % 16 == 8, then
 * ((c0+c4)+(c1+c5))+((c2+c6)+(c3+c7)).
 * ------------------------------------------------------------------------- */
static float dot_avx2_order(const float* a, const float* b, size_t dim) {
  float c[16] = {0};
  const size_t main_end = dim - dim % 16;
  for (size_t i = 0; i < main_end; ++i) c[i % 16] = fmaf(a[i], b[i], c[i % 16]);
  for (int l = 0; l < 8; ++l) c[l] = c[l] + c[l + 8];
  if (dim % 16 == 8) {
    for (int l = 0; l < 8; ++l) c[l] = fmaf(a[main_end + (size_t)l], b[main_end + (size_t)l], c[l]);
  }
  const float b0 = c[0] + c[4], b1 = c[1] + c[5], b2 = c[2] + c[6], b3 = c[3] + c[7];
  return (b0 + b1) + (b2 + b3);
}

void tqo_float_rescore(const float* queries, size_t nq, size_t dim, const float* corpus,
                       size_t n_corpus, size_t k, float* scores, uint64_t* ids) {
#pragma omp parallel
  {
    cand_t* row = malloc((k ? k : 1) * sizeof(cand_t));
#pragma omp for schedule(static)
    for (long long qq = 0; qq < (long long)nq; ++qq) {
      const size_t qi = (size_t)qq;
      for (size_t j = 0; j < k; ++j) {
        const uint64_t id = ids[qi * k + j];
        row[j].id = id;
        row[j].s = (id < n_corpus) ? dot_avx2_order(queries + qi * dim, corpus + id * dim, dim) : -INFINITY;
      }
      for (size_t j = 1; j < k; ++j) {  /* insertion sort, best first */
        cand_t c = row[j];
        size_t p = j;
        while (p > 0 && better(&c, &row[p - 1])) {
          row[p] = row[p - 1];
          --p;
        }
        row[p] = c;
      }
      for (size_t j = 0; j < k; ++j) {
        scores[qi * k + j] = row[j].s;
        ids[qi * k + j] = row[j].id;
      }
    }
    free(row);
  }
}

/* ----------------------------------------------------------------------------
 * IVF residual search over bucket-ordered slots: the composition of
 * score_prepared_into (search.cpp:1156-1264) the bucketed index performs.
 * Each query visits its probed buckets in probe order; every vector's score is
 * (fa * alpha) + offset with two roundings (search_avx2.cpp:150-161, :217-219:
 * the multiply and the offset add are separate instructions), and enters the
 * query's top-k collector under the reference heap rule (topk_heap.hpp:101-157):
 * admitted only when strictly above the current minimum, replacing the worst
 * entry (lowest score, ties: larger id). The kept entries are finally sorted
 * score descending, equal scores by lower id (heaps_to_search_results,
 * search.cpp:1266-1290); rows with fewer than k entries are padded with
 * (0, 0).
 * ------------------------------------------------------------------------- */
void tqo_ivf_search(const uint8_t* luts, const float* lut_scale, const float* lut_bias,
                    const float* bias_corr, size_t nq, size_t nbg, const uint8_t* codes_flat,
                    const float* alpha, const uint64_t* ids, const uint64_t* bucket_start,
                    const uint64_t* bucket_size, const uint32_t* probes,
                    const uint32_t* n_probe, size_t max_probe, const float* offsets, size_t k,
                    float* out_scores, uint64_t* out_ids) {
#pragma omp parallel
  {
    cand_t* heap = malloc((k ? k : 1) * sizeof(cand_t));
#pragma omp for schedule(dynamic)
    for (long long qi = 0; qi < (long long)nq; ++qi) {
      const uint8_t* lut = luts + (size_t)qi * nbg * 32;
      size_t sz = 0, mi = 0;
      float hmin = -INFINITY;
      for (size_t j = 0; j < n_probe[qi]; ++j) {
        const uint32_t b = probes[(size_t)qi * max_probe + j];
        const float off = offsets[(size_t)qi * max_probe + j];
        for (uint64_t t = 0; t < bucket_size[b]; ++t) {
          const size_t slot = (size_t)(bucket_start[b] + t);
          const uint8_t* c = codes_flat + slot * nbg;
          float fa = lut_bias[qi] + (bias_corr ? bias_corr[qi] : 0.f);
          for (size_t g0 = 0; g0 < nbg; g0 += 256) {
            const size_t g1 = (g0 + 256 < nbg) ? g0 + 256 : nbg;
            uint32_t acc = 0;
            for (size_t g = g0; g < g1; ++g) acc += lut[g * 32 + (c[g] >> 4)] + lut[g * 32 + 16 + (c[g] & 15)];
            fa = fmaf(lut_scale[qi], (float)acc, fa);
          }
          const float prod = fa * alpha[slot];
          const cand_t cd = {prod + off, ids[slot]};
          if (!(cd.s > hmin)) continue;
          if (sz < k) {
            heap[sz++] = cd;
            if (sz < k) continue;
          } else {
            heap[mi] = cd;
          }
          /* rescan for the worst entry */
          mi = 0;
          for (size_t h = 1; h < k; ++h) {
            if (better(&heap[mi], &heap[h])) mi = h;
          }
          hmin = heap[mi].s;
        }
      }
      /* insertion sort, best first */
      for (size_t a = 1; a < sz; ++a) {
        cand_t x = heap[a];
        size_t pos = a;
        while (pos > 0 && better(&x, &heap[pos - 1])) {
          heap[pos] = heap[pos - 1];
          --pos;
        }
        heap[pos] = x;
      }
      for (size_t j = 0; j < k; ++j) {
        out_scores[(size_t)qi * k + j] = j < sz ? heap[j].s : 0.f;
        out_ids[(size_t)qi * k + j] = j < sz ? heap[j].id : 0;
      }
    }
    free(heap);
  }
}
