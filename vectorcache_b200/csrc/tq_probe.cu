// Learned n_probe predictor for the bucketed index: a small MLP trained and run
// on the GPU by this file's own kernels. No counterpart exists in the
// reference.
//
// Input per query: its top-256 routing scores s_1 >= ... >= s_256 and the 255
// gaps s_i - s_{i+1} (a zero pads the gap vector to 256), standardized per
// feature with the mean / std of the training set, rounded to bf16. Network:
// in -> hidden (ReLU) -> hidden (ReLU) -> n_classes logits; one class per
// candidate n_probe value. Weights are bf16 in every matrix product, with fp32
// accumulation; the optimizer (Adam) keeps fp32 master weights and rewrites the
// bf16 copies after each step. Biases, pre-activations and gradients are fp32.
//
// Classes objective (softmax cross-entropy on one label class per query):
// the query gets the smallest n_probe whose cumulative probability reaches
// `coverage`, or the fixed fallback n_probe when the largest class
// probability is below `min_confidence`.
//
// Recall objective (one sigmoid per class, binary cross-entropy against the
// query's measured recall at every class): r_c estimates the recall at
// classes[c], and the query gets the class maximizing
// r_c - lambda * classes[c] / classes[last] with lambda passed as `coverage`.
// One lambda for all queries spends probes where the predicted recall gain
// per probe is largest, instead of asking every query for the same recall.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <vector>

#include "../../include/vectorcache_b200.h"
#include "tq_abi.h"
#include "tq_device.cuh"
#include "tq_index_impl.h"
#include "tq_probe.h"

namespace vcb {
namespace {

constexpr int kRouteFeatures = 256;  // top routing scores per query
constexpr int kInputs = 2 * kRouteFeatures;
constexpr int kMaxClasses = 32;

using bf16 = __nv_bfloat16;

// Raw features -> standardized bf16 inputs. top: m x p (p <= 256) scores
// best first; missing scores (p < 256 or -inf) repeat the last valid one.
__global__ void features_kernel(const float* __restrict__ top, long long m, int p, const float* __restrict__ mu,
                                const float* __restrict__ inv_sd, bf16* __restrict__ x, float* __restrict__ raw) {
  const long long q = blockIdx.x;
  if (q >= m) return;
  __shared__ float s[kRouteFeatures];
  for (int i = threadIdx.x; i < kRouteFeatures; i += blockDim.x) {
    s[i] = i < p ? top[q * p + i] : -INFINITY;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float last = s[0] > -INFINITY ? s[0] : 0.f;
    for (int i = 0; i < kRouteFeatures; ++i) {
      if (s[i] > -INFINITY) {
        last = s[i];
      } else {
        s[i] = last;
      }
    }
  }
  __syncthreads();
  for (int f = threadIdx.x; f < kInputs; f += blockDim.x) {
    float v;
    if (f < kRouteFeatures) {
      v = s[f];
    } else {
      const int i = f - kRouteFeatures;
      v = i + 1 < kRouteFeatures ? __fsub_rn(s[i], s[i + 1]) : 0.f;
    }
    if (raw) raw[q * kInputs + f] = v;
    x[q * kInputs + f] = __float2bfloat16_rn(__fmul_rn(__fsub_rn(v, mu[f]), inv_sd[f]));
  }
}

// C (M x N, fp32, row stride ldc) = A (M x K) . B (K x N) with bf16 operands on
// the tensor cores (mma.sync m16n8k16, fp32 accumulation). Element (i, k) of
// A at A[i * a_r + k * a_c]; (k, j) of B at B[k * b_r + j * b_c]. A T x T tile
// per CTA of 4 warps (T = 64, or 32 when 64-wide tiles would leave most SMs
// idle), each warp a (T/2) x (T/2) piece; 32 coordinates per shared-memory
// stage, staged k-contiguous so every fragment register is one 32-bit load.
template <int T>
__global__ void __launch_bounds__(128) gemm_bf16_tc_kernel(const bf16* __restrict__ A, long long a_r, long long a_c,
                                                           const bf16* __restrict__ B, long long b_r, long long b_c,
                                                           float* __restrict__ C, long long ldc, long long M, int N,
                                                           int K) {
  constexpr int KC = 32, PAD = 8;          // PAD: rows 20 words apart, conflict-free fragment loads
  constexpr int WT = T / 2;                // warp piece
  constexpr int MI = WT / 16, NJ = WT / 8;  // m16 and n8 tiles per warp
  __shared__ __align__(16) bf16 sa[T][KC + PAD];
  __shared__ __align__(16) bf16 sb[T][KC + PAD];
  const long long i0 = static_cast<long long>(blockIdx.y) * T;
  const int j0 = blockIdx.x * T;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = warp & 1, wn = warp >> 1;
  const int g = lane >> 2, q = lane & 3;
  float acc[MI][NJ][4];
#pragma unroll
  for (int i = 0; i < MI; ++i)
#pragma unroll
    for (int j = 0; j < NJ; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;
  const bf16 zero = __float2bfloat16_rn(0.f);
  for (int k0 = 0; k0 < K; k0 += KC) {
    __syncthreads();
    for (int e = threadIdx.x; e < T * KC; e += blockDim.x) {
      const int r = e / KC, c = e % KC;
      const int gk = k0 + c;
      const long long gi = i0 + r;
      sa[r][c] = (gi < M && gk < K) ? A[gi * a_r + gk * a_c] : zero;
      const int gj = j0 + r;
      sb[r][c] = (gj < N && gk < K) ? B[gk * b_r + static_cast<long long>(gj) * b_c] : zero;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < KC; kk += 16) {
      uint32_t af[MI][4], bfr[NJ][2];
#pragma unroll
      for (int i = 0; i < MI; ++i) {
        const int r = wm * WT + i * 16 + g;
        af[i][0] = *reinterpret_cast<const uint32_t*>(&sa[r][kk + 2 * q]);
        af[i][1] = *reinterpret_cast<const uint32_t*>(&sa[r + 8][kk + 2 * q]);
        af[i][2] = *reinterpret_cast<const uint32_t*>(&sa[r][kk + 8 + 2 * q]);
        af[i][3] = *reinterpret_cast<const uint32_t*>(&sa[r + 8][kk + 8 + 2 * q]);
      }
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        const int n = wn * WT + j * 8 + g;
        bfr[j][0] = *reinterpret_cast<const uint32_t*>(&sb[n][kk + 2 * q]);
        bfr[j][1] = *reinterpret_cast<const uint32_t*>(&sb[n][kk + 8 + 2 * q]);
      }
#pragma unroll
      for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
          asm volatile(
              "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
              "{%0,%1,%2,%3};\n"
              : "+f"(acc[i][j][0]), "+f"(acc[i][j][1]), "+f"(acc[i][j][2]), "+f"(acc[i][j][3])
              : "r"(af[i][0]), "r"(af[i][1]), "r"(af[i][2]), "r"(af[i][3]), "r"(bfr[j][0]), "r"(bfr[j][1]));
        }
    }
  }
#pragma unroll
  for (int i = 0; i < MI; ++i)
#pragma unroll
    for (int j = 0; j < NJ; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const long long gi = i0 + wm * WT + i * 16 + g + (e >> 1) * 8;
        const int gj = j0 + wn * WT + j * 8 + 2 * q + (e & 1);
        if (gi < M && gj < N) C[gi * ldc + gj] = acc[i][j][e];
      }
}

// Z += bias; optionally A = bf16(relu(Z)).
__global__ void bias_act_kernel(float* __restrict__ Z, long long M, int N, const float* __restrict__ bias,
                                bf16* __restrict__ act) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= M * N) return;
  const float z = __fadd_rn(Z[i], bias[i % N]);
  Z[i] = z;
  if (act) act[i] = __float2bfloat16_rn(z > 0.f ? z : 0.f);
}

// Row-wise softmax cross-entropy: dZ = (softmax - onehot) / M, loss_rows[q].
__global__ void softmax_xent_kernel(const float* __restrict__ Z, long long M, int N, const uint32_t* __restrict__ label,
                                    float* __restrict__ dZ, float* __restrict__ loss_rows) {
  const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (q >= M) return;
  const float* z = Z + q * N;
  float mx = -INFINITY;
  for (int j = 0; j < N; ++j) mx = fmaxf(mx, z[j]);
  float sum = 0.f;
  for (int j = 0; j < N; ++j) sum = __fadd_rn(sum, expf(__fsub_rn(z[j], mx)));
  const float inv_m = 1.f / static_cast<float>(M);
  const uint32_t y = label[q];
  for (int j = 0; j < N; ++j) {
    const float pj = __fdiv_rn(expf(__fsub_rn(z[j], mx)), sum);
    dZ[q * N + j] = __fmul_rn(__fsub_rn(pj, j == static_cast<int>(y) ? 1.f : 0.f), inv_m);
  }
  loss_rows[q] = __fsub_rn(logf(sum), __fsub_rn(z[y], mx));
}

// Row-wise sigmoid binary cross-entropy against soft targets t in [0, 1]:
// loss_rows[q] = mean_j (max(z, 0) - t z + log(1 + exp(-|z|))),
// dZ = (sigmoid(z) - t) / (M N).
__global__ void sigmoid_bce_kernel(const float* __restrict__ Z, long long M, int N, const float* __restrict__ T,
                                   float* __restrict__ dZ, float* __restrict__ loss_rows) {
  const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (q >= M) return;
  const float inv = 1.f / (static_cast<float>(M) * static_cast<float>(N));
  float row = 0.f;
  for (int j = 0; j < N; ++j) {
    const float z = Z[q * N + j], t = T[q * N + j];
    const float e = expf(-fabsf(z));
    row = __fadd_rn(row, __fadd_rn(__fsub_rn(fmaxf(z, 0.f), __fmul_rn(t, z)), log1pf(e)));
    // sigmoid(z) from e = exp(-|z|) without overflow
    const float sg = z >= 0.f ? __fdiv_rn(1.f, __fadd_rn(1.f, e)) : __fdiv_rn(e, __fadd_rn(1.f, e));
    dZ[q * N + j] = __fmul_rn(__fsub_rn(sg, t), inv);
  }
  loss_rows[q] = __fdiv_rn(row, static_cast<float>(N));
}

// dZ *= (Zprev > 0)
__global__ void relu_grad_kernel(float* __restrict__ dA, const float* __restrict__ Z, long long total) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < total && !(Z[i] > 0.f)) dA[i] = 0.f;
}

// db[j] = sum_i dZ[i, j] (one thread per column, rows in order).
__global__ void colsum_kernel(const float* __restrict__ dZ, long long M, int N, float* __restrict__ db) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  float s = 0.f;
  for (long long i = 0; i < M; ++i) s = __fadd_rn(s, dZ[i * N + j]);
  db[j] = s;
}

__global__ void adam_kernel(float* __restrict__ p, float* __restrict__ m1, float* __restrict__ m2,
                            const float* __restrict__ g, long long n, float lr, float b1, float b2, float eps,
                            float c1, float c2, bf16* __restrict__ shadow, long long shadow_n) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float a = __fmaf_rn(b1, m1[i], __fmul_rn(1.f - b1, gi));
  const float v = __fmaf_rn(b2, m2[i], __fmul_rn(1.f - b2, __fmul_rn(gi, gi)));
  m1[i] = a;
  m2[i] = v;
  const float mh = __fdiv_rn(a, c1), vh = __fdiv_rn(v, c2);
  const float w = __fsub_rn(p[i], __fdiv_rn(__fmul_rn(lr, mh), __fadd_rn(sqrtf(vh), eps)));
  p[i] = w;
  if (i < shadow_n) shadow[i] = __float2bfloat16_rn(w);
}

__global__ void to_bf16_kernel(const float* __restrict__ src, bf16* __restrict__ dst, long long n) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = __float2bfloat16_rn(src[i]);
}

// Logits -> n_probe per query (see the file comment).
// The rule of one query's logits z[0..N): its n_probe, and its confidence
// (largest predicted recall or class probability) in *conf.
__device__ uint32_t predict_row(const float* z, int N, const uint32_t* __restrict__ classes, int objective,
                                float coverage, float min_conf, uint32_t fallback, float* conf) {
  if (objective == TQ_PROBE_OBJECTIVE_RECALL) {
    const float per_probe = coverage / static_cast<float>(classes[N - 1]);
    float best = -INFINITY, top_r = 0.f;
    int pick = N - 1;
    for (int j = 0; j < N; ++j) {
      const float r = 1.f / (1.f + expf(-z[j]));
      const float v = r - per_probe * static_cast<float>(classes[j]);
      if (v > best) {
        best = v;
        pick = j;
      }
      top_r = fmaxf(top_r, r);
    }
    *conf = top_r;
    return top_r < min_conf ? fallback : classes[pick];
  }
  float mx = -INFINITY;
  for (int j = 0; j < N; ++j) mx = fmaxf(mx, z[j]);
  float sum = 0.f;
  for (int j = 0; j < N; ++j) sum += expf(z[j] - mx);
  float cum = 0.f, best = 0.f;
  int pick = N - 1;
  bool picked = false;
  for (int j = 0; j < N; ++j) {
    const float pj = expf(z[j] - mx) / sum;
    best = fmaxf(best, pj);
    cum += pj;
    if (!picked && cum >= coverage) {
      pick = j;
      picked = true;
    }
  }
  *conf = best;
  return best < min_conf ? fallback : classes[pick];
}

__global__ void predict_kernel(const float* __restrict__ Z, long long M, int N, const uint32_t* __restrict__ classes,
                               int objective, float coverage, float min_conf, uint32_t fallback,
                               uint32_t* __restrict__ out, float* __restrict__ conf_out) {
  const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (q >= M) return;
  float conf;
  out[q] = predict_row(Z + q * N, N, classes, objective, coverage, min_conf, fallback, &conf);
  if (conf_out) conf_out[q] = conf;
}

// ---------------------------------------------------------------------------
// Fused prediction for the default shape (512 inputs, two hidden layers of
// 128, at most 32 classes): the features, the three products with their bias
// (and ReLU) epilogues, and the rule, for 64 queries per CTA of 4 warps (16
// rows each), in one launch instead of eight. Every output is accumulated by
// the same m16n8k16 sequence (k ascending in steps of 16, from zero) as in
// gemm_bf16_tc_kernel, and the epilogues round as bias_act_kernel does, so the
// logits and the picks are those of the unfused kernels.
// ---------------------------------------------------------------------------
constexpr int kFuseRows = 64, kFuseHidden = 128, kFuseKC = 32, kFusePad = 8;
struct FusedSmem {
  bf16 x[kFuseRows][kInputs + kFusePad];      // standardized inputs (rows 1,040 B apart)
  bf16 h[kFuseRows][kFuseHidden + kFusePad];  // hidden activations
  bf16 w[kFuseHidden][kFuseKC + kFusePad];    // one 32-deep chunk of a layer's weights, n-major
  float z[kFuseRows][kMaxClasses + 1];        // logits
};

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// acc (this warp's 16 rows x NJ*8 columns) = A (rows of lda bf16) . W, W the
// layer's K x N bf16 weights (row-major, global); columns >= N get zeros.
template <int NJ>
__device__ __forceinline__ void fused_product(const bf16* A, int lda, int K, const bf16* __restrict__ W, int N,
                                              FusedSmem& sm, float (&acc)[NJ][4]) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  const bf16 zero = __float2bfloat16_rn(0.f);
#pragma unroll
  for (int j = 0; j < NJ; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[j][e] = 0.f;
  for (int k0 = 0; k0 < K; k0 += kFuseKC) {
    __syncthreads();  // the previous chunk is consumed (and A's rows are written)
    for (int e = threadIdx.x; e < NJ * 8 * kFuseKC; e += blockDim.x) {
      const int c = e / (NJ * 8), n = e % (NJ * 8);  // coalesced along n
      sm.w[n][c] = n < N ? W[static_cast<long long>(k0 + c) * N + n] : zero;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kFuseKC; kk += 16) {
      const int r = warp * 16 + g, k = k0 + kk + 2 * q;
      uint32_t af[4];
      af[0] = *reinterpret_cast<const uint32_t*>(A + r * lda + k);
      af[1] = *reinterpret_cast<const uint32_t*>(A + (r + 8) * lda + k);
      af[2] = *reinterpret_cast<const uint32_t*>(A + r * lda + k + 8);
      af[3] = *reinterpret_cast<const uint32_t*>(A + (r + 8) * lda + k + 8);
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        const uint32_t b0 = *reinterpret_cast<const uint32_t*>(&sm.w[j * 8 + g][kk + 2 * q]);
        const uint32_t b1 = *reinterpret_cast<const uint32_t*>(&sm.w[j * 8 + g][kk + 8 + 2 * q]);
        mma_bf16(acc[j], af, b0, b1);
      }
    }
  }
}

// bias, ReLU, bf16 into this warp's rows of sm.h
__device__ __forceinline__ void fused_hidden_epilogue(const float (&acc)[kFuseHidden / 8][4],
                                                      const float* __restrict__ bias, FusedSmem& sm) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  __syncwarp();  // every lane of the warp is done reading its rows of sm.h
#pragma unroll
  for (int j = 0; j < kFuseHidden / 8; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int r = warp * 16 + g + (e >> 1) * 8, c = j * 8 + 2 * q + (e & 1);
      const float zv = __fadd_rn(acc[j][e], bias[c]);
      sm.h[r][c] = __float2bfloat16_rn(zv > 0.f ? zv : 0.f);
    }
}

__global__ void __launch_bounds__(128) predict_fused_kernel(const float* __restrict__ top, long long m, int p,
                                                            const float* __restrict__ mu,
                                                            const float* __restrict__ inv_sd,
                                                            const bf16* __restrict__ w0, const float* __restrict__ b0,
                                                            const bf16* __restrict__ w1, const float* __restrict__ b1,
                                                            const bf16* __restrict__ w2, const float* __restrict__ b2,
                                                            int n_classes, const uint32_t* __restrict__ classes,
                                                            int objective, float coverage, float min_conf,
                                                            uint32_t fallback, uint32_t* __restrict__ out,
                                                            float* __restrict__ conf_out) {
  extern __shared__ __align__(16) unsigned char fused_smem[];
  FusedSmem& sm = *reinterpret_cast<FusedSmem*>(fused_smem);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long q0 = static_cast<long long>(blockIdx.x) * kFuseRows;
  // Features of this warp's 16 queries; lane l holds scores 8l .. 8l+7.
  for (int rr = 0; rr < 16; ++rr) {
    const int r = warp * 16 + rr;
    const long long qi = q0 + r;
    float s[8];
    int any = 0;
    float last = 0.f;  // this lane's last valid score
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int i = lane * 8 + j;
      s[j] = (qi < m && i < p) ? top[qi * p + i] : -INFINITY;
      if (s[j] > -INFINITY) {
        any = 1;
        last = s[j];
      }
    }
    // Missing scores repeat the last valid one before them (0 when there is
    // none): an inclusive scan over lanes of "the last valid score so far",
    // then this lane's carry-in from the lane before.
#pragma unroll
    for (int o = 1; o < kWarp; o <<= 1) {
      const float lv = __shfl_up_sync(full_mask(), last, o);
      const int la = __shfl_up_sync(full_mask(), any, o);
      if (lane >= o && la && !any) {
        last = lv;
        any = 1;
      }
    }
    const float carry = __shfl_up_sync(full_mask(), last, 1);
    const int have = __shfl_up_sync(full_mask(), any, 1);
    float cur = (lane >= 1 && have) ? carry : 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if (s[j] > -INFINITY) {
        cur = s[j];
      } else {
        s[j] = cur;
      }
    }
    const float next = __shfl_down_sync(full_mask(), s[0], 1);  // score 8l + 8
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int i = lane * 8 + j;
      const float gap = i + 1 < kRouteFeatures ? __fsub_rn(s[j], j < 7 ? s[j + 1] : next) : 0.f;
      sm.x[r][i] = __float2bfloat16_rn(__fmul_rn(__fsub_rn(s[j], mu[i]), inv_sd[i]));
      sm.x[r][kRouteFeatures + i] =
          __float2bfloat16_rn(__fmul_rn(__fsub_rn(gap, mu[kRouteFeatures + i]), inv_sd[kRouteFeatures + i]));
    }
  }
  float acc[kFuseHidden / 8][4];
  fused_product<kFuseHidden / 8>(&sm.x[0][0], kInputs + kFusePad, kInputs, w0, kFuseHidden, sm, acc);
  fused_hidden_epilogue(acc, b0, sm);
  fused_product<kFuseHidden / 8>(&sm.h[0][0], kFuseHidden + kFusePad, kFuseHidden, w1, kFuseHidden, sm, acc);
  fused_hidden_epilogue(acc, b1, sm);
  float lz[kMaxClasses / 8][4];
  fused_product<kMaxClasses / 8>(&sm.h[0][0], kFuseHidden + kFusePad, kFuseHidden, w2, n_classes, sm, lz);
  {
    const int g = lane >> 2, q = lane & 3;
#pragma unroll
    for (int j = 0; j < kMaxClasses / 8; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int r = warp * 16 + g + (e >> 1) * 8, c = j * 8 + 2 * q + (e & 1);
        if (c < n_classes) sm.z[r][c] = __fadd_rn(lz[j][e], b2[c]);
      }
  }
  __syncthreads();
  if (threadIdx.x < kFuseRows && q0 + threadIdx.x < m) {
    const long long qi = q0 + threadIdx.x;
    float conf;
    out[qi] = predict_row(sm.z[threadIdx.x], n_classes, classes, objective, coverage, min_conf, fallback, &conf);
    if (conf_out) conf_out[qi] = conf;
  }
}

// Every MLP product (forward, dW = X^T.dZ, dX = dZ.W^T) has bf16 operands and
// runs on the tensor cores; 32 x 32 tiles when 64 x 64 tiles would fill fewer
// than two CTAs per SM (e.g. 1,310 x 128 outputs: 42 tiles of 64, 164 of 32).
cudaError_t gemm(const bf16* A, long long a_r, long long a_c, const bf16* B, long long b_r, long long b_c,
                 float* C, long long ldc, long long M, int N, int K, cudaStream_t s) {
  if (M == 0 || N == 0) return cudaSuccess;
  const long long tiles64 = ((N + 63) / 64) * ((M + 63) / 64);
  if (tiles64 < 2 * 148) {
    dim3 grid(static_cast<unsigned>((N + 31) / 32), static_cast<unsigned>((M + 31) / 32));
    if (grid.y > 65535) return cudaErrorInvalidValue;
    gemm_bf16_tc_kernel<32><<<grid, 128, 0, s>>>(A, a_r, a_c, B, b_r, b_c, C, ldc, M, N, K);
    return cudaGetLastError();
  }
  dim3 grid(static_cast<unsigned>((N + 63) / 64), static_cast<unsigned>((M + 63) / 64));
  if (grid.y > 65535) return cudaErrorInvalidValue;
  gemm_bf16_tc_kernel<64><<<grid, 128, 0, s>>>(A, a_r, a_c, B, b_r, b_c, C, ldc, M, N, K);
  return cudaGetLastError();
}

inline unsigned blocks(long long n, int t = 256) { return static_cast<unsigned>((n + t - 1) / t); }

}  // namespace
}  // namespace vcb

struct tq_probe_mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  int hidden = 128, n_layers = 2, n_classes = 0;
  int objective = TQ_PROBE_OBJECTIVE_CLASSES;
  std::vector<uint32_t> classes;
  std::vector<int> fan_in, fan_out;  // per linear layer
  std::vector<size_t> w_off, b_off;  // offsets into the flat fp32 parameter vector
  size_t n_params = 0;
  vcb::DeviceBuffer d_params, d_m1, d_m2, d_grad, d_wbf, d_mu, d_isd, d_classes;
  std::vector<size_t> wbf_off;
  size_t n_wbf = 0;
  int64_t step = 0;
  // scratch
  vcb::DeviceBuffer d_x, d_raw, d_top, d_labels, d_targets, d_loss, d_out;
  vcb::DeviceBuffer z[5], a[5], dz[5];  // per linear layer (n_layers <= 4)
  vcb::DeviceBuffer dzb;                 // bf16 copy of one layer's dZ (the products' operand)

  ~tq_probe_mlp() {
    if (stream) {
      cudaStreamSynchronize(stream);
      cudaStreamDestroy(stream);
    }
  }

  void sync() { vcb::check(cudaStreamSynchronize(stream), "cudaStreamSynchronize"); }
  int n_lin() const { return n_layers + 1; }

  void reserve_batch(size_t m) {
    d_x.reserve(m * vcb::kInputs * 2);
    for (int l = 0; l < n_lin(); ++l) {
      z[l].reserve(m * fan_out[l] * 4);
      a[l].reserve(m * fan_out[l] * 2);
      dz[l].reserve(m * fan_out[l] * 4);
      dzb.reserve(m * fan_out[l] * 2);
    }
    d_loss.reserve(m * 4);
  }

  const vcb::bf16* wbf(int l) const { return d_wbf.as<vcb::bf16>() + wbf_off[l]; }
  const float* bias(int l) const { return d_params.as<float>() + b_off[l]; }

  // features(top) -> d_x; then the forward pass; logits in z[last].
  void forward(const float* d_top, size_t m, int p, cudaStream_t s) {
    reserve_batch(m);
    vcb::features_kernel<<<static_cast<unsigned>(m), 256, 0, s>>>(d_top, static_cast<long long>(m), p,
                                                                  d_mu.as<float>(), d_isd.as<float>(),
                                                                  d_x.as<vcb::bf16>(), nullptr);
    vcb::check(cudaGetLastError(), "features kernel");
    const vcb::bf16* in = d_x.as<vcb::bf16>();
    for (int l = 0; l < n_lin(); ++l) {
      const int K = fan_in[l], N = fan_out[l];
      vcb::check(vcb::gemm(in, K, 1, wbf(l), N, 1, z[l].as<float>(), N, static_cast<long long>(m), N, K, s),
                 "mlp gemm");
      const bool last = l + 1 == n_lin();
      vcb::bias_act_kernel<<<vcb::blocks(static_cast<long long>(m) * N), 256, 0, s>>>(
          z[l].as<float>(), static_cast<long long>(m), N, bias(l), last ? nullptr : a[l].as<vcb::bf16>());
      vcb::check(cudaGetLastError(), "bias kernel");
      in = a[l].as<vcb::bf16>();
    }
  }

  // Gradients of the mean loss into d_grad; returns the loss. Labels (classes
  // objective) or recall targets (recall objective), by the model's objective.
  float backward(const uint32_t* d_lab, const float* d_tgt, size_t m, cudaStream_t s) {
    const long long M = static_cast<long long>(m);
    const int L = n_lin();
    if (objective == TQ_PROBE_OBJECTIVE_RECALL) {
      vcb::sigmoid_bce_kernel<<<vcb::blocks(M), 256, 0, s>>>(z[L - 1].as<float>(), M, n_classes, d_tgt,
                                                              dz[L - 1].as<float>(), d_loss.as<float>());
    } else {
      vcb::softmax_xent_kernel<<<vcb::blocks(M), 256, 0, s>>>(z[L - 1].as<float>(), M, n_classes, d_lab,
                                                               dz[L - 1].as<float>(), d_loss.as<float>());
    }
    vcb::check(cudaGetLastError(), "loss kernel");
    float* g = d_grad.as<float>();
    for (int l = L - 1; l >= 0; --l) {
      const int K = fan_in[l], N = fan_out[l];
      const vcb::bf16* in = l == 0 ? d_x.as<vcb::bf16>() : a[l - 1].as<vcb::bf16>();
      // The products take dZ in bf16 (fp32 accumulation); the bias gradient
      // sums the fp32 dZ.
      vcb::to_bf16_kernel<<<vcb::blocks(M * N), 256, 0, s>>>(dz[l].as<float>(), dzb.as<vcb::bf16>(), M * N);
      vcb::check(cudaGetLastError(), "bf16 kernel");
      // dW = in^T . dZ  (K x N)
      vcb::check(vcb::gemm(in, 1, K, dzb.as<vcb::bf16>(), N, 1, g + w_off[l], N, K, N, static_cast<int>(M), s),
                 "mlp gemm");
      vcb::colsum_kernel<<<vcb::blocks(N), 256, 0, s>>>(dz[l].as<float>(), M, N, g + b_off[l]);
      vcb::check(cudaGetLastError(), "colsum kernel");
      if (l > 0) {
        // dA_{l-1} = dZ . W^T (M x K), then the ReLU mask of layer l-1.
        vcb::check(vcb::gemm(dzb.as<vcb::bf16>(), N, 1, wbf(l), 1, N, dz[l - 1].as<float>(), K, M, K, N, s),
                   "mlp gemm");
        vcb::relu_grad_kernel<<<vcb::blocks(M * K), 256, 0, s>>>(dz[l - 1].as<float>(), z[l - 1].as<float>(),
                                                                 M * K);
        vcb::check(cudaGetLastError(), "relu grad kernel");
      }
    }
    std::vector<float> lr(m);
    vcb::check(cudaMemcpyAsync(lr.data(), d_loss.get(), m * 4, cudaMemcpyDeviceToHost, s), "D2H");
    vcb::check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    double tot = 0.0;
    for (float v : lr) tot += v;
    return static_cast<float>(tot / static_cast<double>(m));
  }

  void adam(float lr, cudaStream_t s) {
    ++step;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, static_cast<float>(step));
    const float c2 = 1.f - std::pow(b2, static_cast<float>(step));
    // Each weight matrix: its fp32 master and its bf16 copy.
    for (int l = 0; l < n_lin(); ++l) {
      const long long nw = static_cast<long long>(fan_in[l]) * fan_out[l];
      vcb::adam_kernel<<<vcb::blocks(nw), 256, 0, s>>>(d_params.as<float>() + w_off[l], d_m1.as<float>() + w_off[l],
                                                       d_m2.as<float>() + w_off[l], d_grad.as<float>() + w_off[l], nw,
                                                       lr, b1, b2, 1e-8f, c1, c2, d_wbf.as<vcb::bf16>() + wbf_off[l],
                                                       nw);
      vcb::check(cudaGetLastError(), "adam kernel");
      const long long nbias = fan_out[l];
      vcb::adam_kernel<<<vcb::blocks(nbias), 256, 0, s>>>(d_params.as<float>() + b_off[l],
                                                          d_m1.as<float>() + b_off[l], d_m2.as<float>() + b_off[l],
                                                          d_grad.as<float>() + b_off[l], nbias, lr, b1, b2, 1e-8f, c1,
                                                          c2, nullptr, 0);
      vcb::check(cudaGetLastError(), "adam kernel");
    }
  }

  void refresh_bf16(cudaStream_t s) {
    for (int l = 0; l < n_lin(); ++l) {
      const long long nw = static_cast<long long>(fan_in[l]) * fan_out[l];
      vcb::to_bf16_kernel<<<vcb::blocks(nw), 256, 0, s>>>(d_params.as<float>() + w_off[l],
                                                          d_wbf.as<vcb::bf16>() + wbf_off[l], nw);
      vcb::check(cudaGetLastError(), "bf16 kernel");
    }
  }
};

namespace vcb {

void probe_reserve(tq_probe_mlp* h, size_t m, ProbeScratch& sc) {
  int widest = 1;
  for (int l = 0; l < h->n_lin(); ++l) widest = std::max(widest, h->fan_out[l]);
  sc.x.reserve(m * kInputs * 2);
  sc.z.reserve(m * widest * 4);
  sc.act0.reserve(m * widest * 2);
  sc.act1.reserve(m * widest * 2);
}

// The default shape (512 inputs, two hidden layers of 128) predicts in one
// fused launch; false for other shapes.
bool predict_fused(tq_probe_mlp* h, const float* d_top, long long M, int p, float coverage, float min_conf,
                   uint32_t fallback, uint32_t* d_out, float* d_conf, cudaStream_t s) {
  if (!(h->n_layers == 2 && h->fan_in[0] == kInputs && h->fan_out[0] == kFuseHidden &&
        h->fan_out[1] == kFuseHidden && h->n_classes <= kMaxClasses)) {
    return false;
  }
  constexpr size_t smem = sizeof(FusedSmem);
  check(cudaFuncSetAttribute(predict_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem)),
        "fused predict attribute");
  predict_fused_kernel<<<static_cast<unsigned>((M + kFuseRows - 1) / kFuseRows), 128, smem, s>>>(
      d_top, M, p, h->d_mu.as<float>(), h->d_isd.as<float>(), h->wbf(0), h->bias(0), h->wbf(1), h->bias(1),
      h->wbf(2), h->bias(2), h->n_classes, h->d_classes.as<uint32_t>(), h->objective, coverage, min_conf, fallback,
      d_out, d_conf);
  check(cudaGetLastError(), "fused predict kernel");
  return true;
}

void probe_predict(tq_probe_mlp* h, const float* d_top, size_t m, int p, float coverage, float min_conf,
                   uint32_t fallback, uint32_t* d_out, cudaStream_t s, ProbeScratch& sc) {
  if (m == 0) return;
  const long long M = static_cast<long long>(m);
  if (predict_fused(h, d_top, M, p, coverage, min_conf, fallback, d_out, nullptr, s)) return;
  probe_reserve(h, m, sc);
  features_kernel<<<static_cast<unsigned>(m), 256, 0, s>>>(d_top, M, p, h->d_mu.as<float>(), h->d_isd.as<float>(),
                                                           sc.x.as<bf16>(), nullptr);
  check(cudaGetLastError(), "features kernel");
  const bf16* in = sc.x.as<bf16>();
  for (int l = 0; l < h->n_lin(); ++l) {
    const int K = h->fan_in[l], N = h->fan_out[l];
    check(gemm(in, K, 1, h->wbf(l), N, 1, sc.z.as<float>(), N, M, N, K, s), "mlp gemm");
    const bool last = l + 1 == h->n_lin();
    bf16* out = (l & 1) ? sc.act1.as<bf16>() : sc.act0.as<bf16>();
    bias_act_kernel<<<blocks(M * N), 256, 0, s>>>(sc.z.as<float>(), M, N, h->bias(l), last ? nullptr : out);
    check(cudaGetLastError(), "bias kernel");
    in = out;
  }
  predict_kernel<<<blocks(M), 256, 0, s>>>(sc.z.as<float>(), M, h->n_classes, h->d_classes.as<uint32_t>(),
                                           h->objective, coverage, min_conf, fallback, d_out, nullptr);
  check(cudaGetLastError(), "predict kernel");
}

uint32_t probe_max_class(const tq_probe_mlp* h) { return h->classes.back(); }

}  // namespace vcb

namespace {

using vcb::require;

tq_probe_mlp* checked(tq_probe_mlp* h) {
  require(h != nullptr, TQ_ERR_INVALID_ARGUMENT, "null model");
  return h;
}

}  // namespace

extern "C" {

int tq_probe_mlp_create(size_t hidden, size_t n_layers, const uint32_t* classes, size_t n_classes, uint64_t seed,
                        int device, tq_probe_mlp** out) {
  return vcb::guarded([&] {
    require(out != nullptr, TQ_ERR_INVALID_ARGUMENT, "out must not be NULL");
    *out = nullptr;
    require(hidden >= 1 && hidden <= 1024, TQ_ERR_INVALID_ARGUMENT, "hidden must be in [1, 1024]");
    require(n_layers >= 1 && n_layers <= 4, TQ_ERR_INVALID_ARGUMENT, "n_layers must be in [1, 4]");
    require(classes != nullptr && n_classes >= 2 && n_classes <= static_cast<size_t>(vcb::kMaxClasses),
            TQ_ERR_INVALID_ARGUMENT, "need 2..32 classes");
    for (size_t i = 0; i < n_classes; ++i) {
      require(classes[i] >= 1 && classes[i] <= 2048 && (i == 0 || classes[i] > classes[i - 1]),
              TQ_ERR_INVALID_ARGUMENT, "classes must be increasing n_probe values in [1, 2048]");
    }
    int count = 0;
    vcb::check(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
    require(device >= 0 && device < count, TQ_ERR_INVALID_ARGUMENT, "no such CUDA device");
    vcb::DeviceGuard g(device);
    auto h = std::make_unique<tq_probe_mlp>();
    h->device = device;
    vcb::check(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    h->hidden = static_cast<int>(hidden);
    h->n_layers = static_cast<int>(n_layers);
    h->n_classes = static_cast<int>(n_classes);
    h->classes.assign(classes, classes + n_classes);
    int in = vcb::kInputs;
    for (int l = 0; l <= h->n_layers; ++l) {
      const int o = l == h->n_layers ? h->n_classes : h->hidden;
      h->fan_in.push_back(in);
      h->fan_out.push_back(o);
      h->w_off.push_back(h->n_params);
      h->n_params += static_cast<size_t>(in) * o;
      h->b_off.push_back(h->n_params);
      h->n_params += o;
      h->wbf_off.push_back(h->n_wbf);
      h->n_wbf += static_cast<size_t>(in) * o;
      in = o;
    }
    // He-uniform initial weights, zero biases (mt19937_64(seed)).
    std::vector<float> init(h->n_params, 0.f);
    std::mt19937_64 rng(seed);
    for (int l = 0; l <= h->n_layers; ++l) {
      const float lim = std::sqrt(6.f / static_cast<float>(h->fan_in[l]));
      std::uniform_real_distribution<float> U(-lim, lim);
      for (size_t i = 0; i < static_cast<size_t>(h->fan_in[l]) * h->fan_out[l]; ++i) init[h->w_off[l] + i] = U(rng);
    }
    h->d_params.reserve(h->n_params * 4);
    h->d_m1.reserve(h->n_params * 4);
    h->d_m2.reserve(h->n_params * 4);
    h->d_grad.reserve(h->n_params * 4);
    h->d_wbf.reserve(h->n_wbf * 2);
    h->d_mu.reserve(vcb::kInputs * 4);
    h->d_isd.reserve(vcb::kInputs * 4);
    h->d_classes.reserve(n_classes * 4);
    std::vector<float> mu(vcb::kInputs, 0.f), isd(vcb::kInputs, 1.f);
    vcb::check(cudaMemcpyAsync(h->d_params.get(), init.data(), h->n_params * 4, cudaMemcpyHostToDevice, h->stream),
               "H2D");
    vcb::check(cudaMemsetAsync(h->d_m1.get(), 0, h->n_params * 4, h->stream), "memset");
    vcb::check(cudaMemsetAsync(h->d_m2.get(), 0, h->n_params * 4, h->stream), "memset");
    vcb::check(cudaMemcpyAsync(h->d_mu.get(), mu.data(), mu.size() * 4, cudaMemcpyHostToDevice, h->stream), "H2D");
    vcb::check(cudaMemcpyAsync(h->d_isd.get(), isd.data(), isd.size() * 4, cudaMemcpyHostToDevice, h->stream), "H2D");
    vcb::check(cudaMemcpyAsync(h->d_classes.get(), classes, n_classes * 4, cudaMemcpyHostToDevice, h->stream), "H2D");
    h->refresh_bf16(h->stream);
    h->sync();
    *out = h.release();
  });
}

int tq_probe_mlp_set_objective(tq_probe_mlp* h, int objective) {
  return vcb::guarded([&] {
    checked(h);
    require(objective == TQ_PROBE_OBJECTIVE_CLASSES || objective == TQ_PROBE_OBJECTIVE_RECALL,
            TQ_ERR_INVALID_ARGUMENT, "unknown objective");
    h->objective = objective;
  });
}

int tq_probe_mlp_destroy(tq_probe_mlp* h) {
  return vcb::guarded([&] {
    if (!h) return;
    vcb::DeviceGuard g(h->device);
    delete h;
  });
}

int tq_probe_mlp_info(const tq_probe_mlp* h, size_t* n_inputs, size_t* n_params, size_t* n_classes) {
  return vcb::guarded([&] {
    require(h != nullptr, TQ_ERR_INVALID_ARGUMENT, "null model");
    if (n_inputs) *n_inputs = vcb::kInputs;
    if (n_params) *n_params = h->n_params;
    if (n_classes) *n_classes = static_cast<size_t>(h->n_classes);
  });
}

int tq_probe_mlp_features(tq_probe_mlp* h, const float* top_scores, size_t m, size_t p, float* raw) {
  return vcb::guarded([&] {
    checked(h);
    require(top_scores && raw, TQ_ERR_INVALID_ARGUMENT, "null buffer");
    require(p >= 1 && p <= 256, TQ_ERR_INVALID_ARGUMENT, "p must be in [1, 256]");
    if (m == 0) return;
    vcb::DeviceGuard g(h->device);
    vcb::DeviceBuffer top, r, x;
    top.reserve(m * p * 4);
    r.reserve(m * vcb::kInputs * 4);
    x.reserve(m * vcb::kInputs * 2);
    vcb::check(cudaMemcpyAsync(top.get(), top_scores, m * p * 4, cudaMemcpyHostToDevice, h->stream), "H2D");
    vcb::features_kernel<<<static_cast<unsigned>(m), 256, 0, h->stream>>>(
        top.as<float>(), static_cast<long long>(m), static_cast<int>(p), h->d_mu.as<float>(), h->d_isd.as<float>(),
        x.as<vcb::bf16>(), r.as<float>());
    vcb::check(cudaGetLastError(), "features kernel");
    vcb::check(cudaMemcpyAsync(raw, r.get(), m * vcb::kInputs * 4, cudaMemcpyDeviceToHost, h->stream), "D2H");
    h->sync();
  });
}

int tq_probe_mlp_set_normalization(tq_probe_mlp* h, const float* mean, const float* stddev) {
  return vcb::guarded([&] {
    checked(h);
    require(mean && stddev, TQ_ERR_INVALID_ARGUMENT, "null buffer");
    vcb::DeviceGuard g(h->device);
    std::vector<float> isd(vcb::kInputs);
    for (int i = 0; i < vcb::kInputs; ++i) isd[i] = stddev[i] > 1e-12f ? 1.f / stddev[i] : 0.f;
    vcb::check(cudaMemcpyAsync(h->d_mu.get(), mean, vcb::kInputs * 4, cudaMemcpyHostToDevice, h->stream), "H2D");
    vcb::check(cudaMemcpyAsync(h->d_isd.get(), isd.data(), vcb::kInputs * 4, cudaMemcpyHostToDevice, h->stream),
               "H2D");
    h->sync();
  });
}

int tq_probe_mlp_get_params(tq_probe_mlp* h, float* params) {
  return vcb::guarded([&] {
    checked(h);
    require(params != nullptr, TQ_ERR_INVALID_ARGUMENT, "null buffer");
    vcb::DeviceGuard g(h->device);
    vcb::check(cudaMemcpyAsync(params, h->d_params.get(), h->n_params * 4, cudaMemcpyDeviceToHost, h->stream), "D2H");
    h->sync();
  });
}

int tq_probe_mlp_set_params(tq_probe_mlp* h, const float* params) {
  return vcb::guarded([&] {
    checked(h);
    require(params != nullptr, TQ_ERR_INVALID_ARGUMENT, "null buffer");
    vcb::DeviceGuard g(h->device);
    vcb::check(cudaMemcpyAsync(h->d_params.get(), params, h->n_params * 4, cudaMemcpyHostToDevice, h->stream), "H2D");
    h->refresh_bf16(h->stream);
    h->sync();
  });
}

int tq_probe_mlp_forward(tq_probe_mlp* h, const float* top_scores, size_t m, size_t p, float* logits) {
  return vcb::guarded([&] {
    checked(h);
    require(top_scores && logits, TQ_ERR_INVALID_ARGUMENT, "null buffer");
    require(p >= 1 && p <= 256, TQ_ERR_INVALID_ARGUMENT, "p must be in [1, 256]");
    if (m == 0) return;
    vcb::DeviceGuard g(h->device);
    h->d_top.reserve(m * p * 4);
    vcb::check(cudaMemcpyAsync(h->d_top.get(), top_scores, m * p * 4, cudaMemcpyHostToDevice, h->stream), "H2D");
    h->forward(h->d_top.as<float>(), m, static_cast<int>(p), h->stream);
    vcb::check(cudaMemcpyAsync(logits, h->z[h->n_lin() - 1].get(), m * h->n_classes * 4, cudaMemcpyDeviceToHost,
                               h->stream),
               "D2H");
    h->sync();
  });
}

int tq_probe_mlp_gradients(tq_probe_mlp* h, const float* top_scores, const uint32_t* labels, size_t m, size_t p,
                           float* loss, float* grads) {
  return vcb::guarded([&] {
    checked(h);
    require(top_scores && labels && grads, TQ_ERR_INVALID_ARGUMENT, "null buffer");
    require(p >= 1 && p <= 256, TQ_ERR_INVALID_ARGUMENT, "p must be in [1, 256]");
    require(m >= 1, TQ_ERR_INVALID_ARGUMENT, "empty batch");
    require(h->objective == TQ_PROBE_OBJECTIVE_CLASSES, TQ_ERR_STATE, "model has the recall objective");
    for (size_t i = 0; i < m; ++i) {
      require(labels[i] < static_cast<uint32_t>(h->n_classes), TQ_ERR_INVALID_ARGUMENT, "label out of range");
    }
    vcb::DeviceGuard g(h->device);
    h->d_top.reserve(m * p * 4);
    h->d_labels.reserve(m * 4);
    vcb::check(cudaMemcpyAsync(h->d_top.get(), top_scores, m * p * 4, cudaMemcpyHostToDevice, h->stream), "H2D");
    vcb::check(cudaMemcpyAsync(h->d_labels.get(), labels, m * 4, cudaMemcpyHostToDevice, h->stream), "H2D");
    h->forward(h->d_top.as<float>(), m, static_cast<int>(p), h->stream);
    const float l = h->backward(h->d_labels.as<uint32_t>(), nullptr, m, h->stream);
    if (loss) *loss = l;
    vcb::check(cudaMemcpyAsync(grads, h->d_grad.get(), h->n_params * 4, cudaMemcpyDeviceToHost, h->stream), "D2H");
    h->sync();
  });
}

int tq_probe_mlp_recall_gradients(tq_probe_mlp* h, const float* top_scores, const float* recall, size_t m, size_t p,
                                  float* loss, float* grads) {
  return vcb::guarded([&] {
    checked(h);
    require(top_scores && recall && grads, TQ_ERR_INVALID_ARGUMENT, "null buffer");
    require(p >= 1 && p <= 256, TQ_ERR_INVALID_ARGUMENT, "p must be in [1, 256]");
    require(m >= 1, TQ_ERR_INVALID_ARGUMENT, "empty batch");
    require(h->objective == TQ_PROBE_OBJECTIVE_RECALL, TQ_ERR_STATE, "model has the classes objective");
    const size_t nt = m * static_cast<size_t>(h->n_classes);
    for (size_t i = 0; i < nt; ++i) {
      require(recall[i] >= 0.f && recall[i] <= 1.f, TQ_ERR_INVALID_ARGUMENT, "recall targets must be in [0, 1]");
    }
    vcb::DeviceGuard g(h->device);
    h->d_top.reserve(m * p * 4);
    h->d_targets.reserve(nt * 4);
    vcb::check(cudaMemcpyAsync(h->d_top.get(), top_scores, m * p * 4, cudaMemcpyHostToDevice, h->stream), "H2D");
    vcb::check(cudaMemcpyAsync(h->d_targets.get(), recall, nt * 4, cudaMemcpyHostToDevice, h->stream), "H2D");
    h->forward(h->d_top.as<float>(), m, static_cast<int>(p), h->stream);
    const float l = h->backward(nullptr, h->d_targets.as<float>(), m, h->stream);
    if (loss) *loss = l;
    vcb::check(cudaMemcpyAsync(grads, h->d_grad.get(), h->n_params * 4, cudaMemcpyDeviceToHost, h->stream), "D2H");
    h->sync();
  });
}

namespace {

// One Adam step on a device batch: labels or recall targets, by objective.
void train_step(tq_probe_mlp* h, const float* d_top_scores, const uint32_t* d_labels, const float* d_recall, size_t m,
                size_t p, float lr, float* loss, void* stream) {
  require(d_top_scores && (d_labels || d_recall), TQ_ERR_INVALID_ARGUMENT, "null buffer");
  require(p >= 1 && p <= 256, TQ_ERR_INVALID_ARGUMENT, "p must be in [1, 256]");
  require(m >= 1, TQ_ERR_INVALID_ARGUMENT, "empty batch");
  vcb::DeviceGuard g(h->device);
  // On the caller's stream (where the batch was produced); the step ends
  // with the loss read back, so it returns with its work complete.
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->stream;
  if (s != h->stream) h->sync();
  h->forward(d_top_scores, m, static_cast<int>(p), s);
  const float l = h->backward(d_labels, d_recall, m, s);
  h->adam(lr, s);
  vcb::check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  if (loss) *loss = l;
}

}  // namespace

int tq_probe_mlp_train_step_device(tq_probe_mlp* h, const float* d_top_scores, const uint32_t* d_labels, size_t m,
                                   size_t p, float lr, float* loss, void* stream) {
  return vcb::guarded([&] {
    checked(h);
    require(h->objective == TQ_PROBE_OBJECTIVE_CLASSES, TQ_ERR_STATE, "model has the recall objective");
    require(d_labels != nullptr, TQ_ERR_INVALID_ARGUMENT, "null buffer");
    train_step(h, d_top_scores, d_labels, nullptr, m, p, lr, loss, stream);
  });
}

int tq_probe_mlp_train_step_recall_device(tq_probe_mlp* h, const float* d_top_scores, const float* d_recall, size_t m,
                                          size_t p, float lr, float* loss, void* stream) {
  return vcb::guarded([&] {
    checked(h);
    require(h->objective == TQ_PROBE_OBJECTIVE_RECALL, TQ_ERR_STATE, "model has the classes objective");
    require(d_recall != nullptr, TQ_ERR_INVALID_ARGUMENT, "null buffer");
    train_step(h, d_top_scores, nullptr, d_recall, m, p, lr, loss, stream);
  });
}

int tq_probe_mlp_predict_device(tq_probe_mlp* h, const float* d_top_scores, size_t m, size_t p, float coverage,
                                float min_confidence, uint32_t fallback, uint32_t* d_n_probe, float* d_confidence,
                                void* stream) {
  return vcb::guarded([&] {
    checked(h);
    require(d_top_scores && d_n_probe, TQ_ERR_INVALID_ARGUMENT, "null buffer");
    require(p >= 1 && p <= 256, TQ_ERR_INVALID_ARGUMENT, "p must be in [1, 256]");
    require(fallback >= 1 && fallback <= 2048, TQ_ERR_INVALID_ARGUMENT, "fallback must be in [1, 2048]");
    if (m == 0) return;
    vcb::DeviceGuard g(h->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->stream;
    if (s != h->stream) h->sync();
    if (vcb::predict_fused(h, d_top_scores, static_cast<long long>(m), static_cast<int>(p), coverage,
                           min_confidence, fallback, d_n_probe, d_confidence, s)) {
      return;
    }
    h->forward(d_top_scores, m, static_cast<int>(p), s);
    vcb::predict_kernel<<<vcb::blocks(static_cast<long long>(m)), 256, 0, s>>>(
        h->z[h->n_lin() - 1].as<float>(), static_cast<long long>(m), h->n_classes, h->d_classes.as<uint32_t>(),
        h->objective, coverage, min_confidence, fallback, d_n_probe, d_confidence);
    vcb::check(cudaGetLastError(), "predict kernel");
  });
}

int tq_probe_mlp_synchronize(tq_probe_mlp* h) {
  return vcb::guarded([&] {
    checked(h);
    vcb::DeviceGuard g(h->device);
    h->sync();
  });
}

}  // extern "C"
