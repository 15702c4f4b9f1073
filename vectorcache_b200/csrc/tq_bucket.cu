// Bucketed (IVF) index kernels on sm_100a: build (spherical k-means, 2-means
// fission, residual slot layout) and search (routing, probe pairs, bucket
// scan). Interfaces and layout in tq_bucket.h.
//
// The bucket scan applies the reference's IVF residual scoring
// (score_prepared_into, search.cpp:1156-1264; search_avx2.cpp:150-161):
// FastScan integer LUT sums flushed into f32 every 256 byte groups, then
// score = (fa * alpha) + <q_hat, encode_c>, two separately rounded operations,
// and top-k in (score desc, id asc) order over the original ids.
#include <algorithm>
#include <cfloat>
#include <climits>

#include "tq_bucket.h"
#include "tq_device.cuh"
#include "tq_kernels.h"

namespace vcb {
namespace {

constexpr int kTile = 128;  // rows of A per GEMM CTA
constexpr int kTileB = 64;  // rows of B per GEMM CTA step
constexpr int kKc = 16;     // coordinates per shared-memory stage

// ---------------------------------------------------------------------------
// Row normalization
// ---------------------------------------------------------------------------
__global__ void normalize_rows_kernel(const float* __restrict__ x, long long n, int dim_in, int dim,
                                      float* __restrict__ out) {
  const long long row = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) / kWarp;
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  const float* xr = x + row * dim_in;
  float s = 0.f;
  for (int i = lane; i < dim_in; i += kWarp) s = __fmaf_rn(xr[i], xr[i], s);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s = __fadd_rn(s, __shfl_xor_sync(full_mask(), s, o));
  const float nrm = __fsqrt_rn(s);
  const float inv = nrm > 1e-30f ? __frcp_rn(nrm) : 0.f;
  float* orow = out + row * dim;
  for (int i = lane; i < dim; i += kWarp) orow[i] = i < dim_in ? __fmul_rn(xr[i], inv) : 0.f;
}

// ---------------------------------------------------------------------------
// fp32 A . B^T tiles: 256 threads, 128 x 64 outputs per step, 8 x 4 per thread,
// coordinates staged through shared memory 16 at a time.
// ---------------------------------------------------------------------------
struct GemmTile {
  float a[kKc][kTile + 4];
  float b[kKc][kTileB + 4];
};

__device__ __forceinline__ void stage_a(GemmTile& t, const float* __restrict__ A, long long m, int dim,
                                        long long r0, int k0) {
  for (int e = threadIdx.x; e < kTile * kKc; e += blockDim.x) {
    const int r = e / kKc, c = e % kKc;
    const long long row = r0 + r;
    const int col = k0 + c;
    t.a[c][r] = (row < m && col < dim) ? A[row * dim + col] : 0.f;
  }
}

__device__ __forceinline__ void stage_b(GemmTile& t, const float* __restrict__ B, long long nb, int dim,
                                        long long c0, int k0) {
  for (int e = threadIdx.x; e < kTileB * kKc; e += blockDim.x) {
    const int r = e / kKc, c = e % kKc;
    const long long row = c0 + r;
    const int col = k0 + c;
    t.b[c][r] = (row < nb && col < dim) ? B[row * dim + col] : 0.f;
  }
}

// acc[i][j] = sum over coordinates of A[r0 + ty*8 + i] * B[c0 + tx*4 + j].
__device__ __forceinline__ void tile_product(GemmTile& t, const float* __restrict__ A, long long m,
                                             const float* __restrict__ B, long long nb, int dim, long long r0,
                                             long long c0, float (&acc)[8][4]) {
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
  for (int k0 = 0; k0 < dim; k0 += kKc) {
    __syncthreads();
    stage_a(t, A, m, dim, r0, k0);
    stage_b(t, B, nb, dim, c0, k0);
    __syncthreads();
#pragma unroll
    for (int c = 0; c < kKc; ++c) {
      const float4 a0 = *reinterpret_cast<const float4*>(&t.a[c][ty * 8]);
      const float4 a1 = *reinterpret_cast<const float4*>(&t.a[c][ty * 8 + 4]);
      const float4 bv = *reinterpret_cast<const float4*>(&t.b[c][tx * 4]);
      const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      const float bw[4] = {bv.x, bv.y, bv.z, bv.w};
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = __fmaf_rn(av[i], bw[j], acc[i][j]);
    }
  }
}

// ---------------------------------------------------------------------------
// Routing and offset products on the tensor cores (mma.sync m16n8k8 TF32,
// fp32 accumulation) in 3xTF32 form (Markidis et al., "NVIDIA Tensor Core
// Programmability, Performance & Precision", IPDPSW 2018): each fp32 operand
// splits as x = hi + lo with hi = tf32(x) and lo = tf32(x - hi), and a product
// is accumulated as lo_a*hi_b + hi_a*lo_b + hi_a*hi_b, about 2^-21 relative
// per product, well inside the 1e-5 the routing scores are checked to against
// fp64. A CTA of 8 warps (4 along A's rows x 2 along B's rows) computes a
// 128 x 64 tile of C; every warp a 32 x 32 piece: 2 x 4 m16n8 tiles.
// ---------------------------------------------------------------------------
constexpr int kTcM = 128, kTcN = 64, kTcK = 32, kTcPad = 4;

struct TcTile {
  float a[kTcM][kTcK + kTcPad];  // rows of A, coordinates k0 .. k0+31
  float b[kTcN][kTcK + kTcPad];  // rows of B
};

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
  hi = to_tf32(x);
  lo = to_tf32(__fsub_rn(x, __uint_as_float(hi)));
}

__device__ __forceinline__ void mma_tf32(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__global__ void __launch_bounds__(256) gemm_nt_tc_kernel(const float* __restrict__ A, long long m,
                                                         const float* __restrict__ B, long long nb, int dim,
                                                         float* __restrict__ C, long long ldc) {
  __shared__ __align__(16) TcTile t;
  const long long r0 = static_cast<long long>(blockIdx.y) * kTcM;
  const long long c0 = static_cast<long long>(blockIdx.x) * kTcN;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = warp & 3, wn = warp >> 2;  // warp's 32 x 32 piece
  const int g = lane >> 2, q = lane & 3;    // mma group and thread in group
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;

  const bool vec = (dim % 4) == 0;
  for (int k0 = 0; k0 < dim; k0 += kTcK) {
    __syncthreads();
    // Stage A (128 x 32) and B (64 x 32), zero outside the matrices.
    for (int e = threadIdx.x; e < (kTcM + kTcN) * (kTcK / 4); e += blockDim.x) {
      const int row = e / (kTcK / 4), c4 = (e % (kTcK / 4)) * 4;
      const bool is_a = row < kTcM;
      const long long src_row = is_a ? r0 + row : c0 + (row - kTcM);
      const long long rows = is_a ? m : nb;
      const float* src = is_a ? A : B;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      const int col = k0 + c4;
      if (src_row < rows) {
        const float* p = src + src_row * dim + col;
        if (vec && col + 4 <= dim) {
          v = *reinterpret_cast<const float4*>(p);
        } else {
          v.x = col < dim ? p[0] : 0.f;
          v.y = col + 1 < dim ? p[1] : 0.f;
          v.z = col + 2 < dim ? p[2] : 0.f;
          v.w = col + 3 < dim ? p[3] : 0.f;
        }
      }
      float* dst = is_a ? &t.a[row][c4] : &t.b[row - kTcM][c4];
      *reinterpret_cast<float4*>(dst) = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kTcK; kk += 8) {
      uint32_t ah[2][4], al[2][4], bh[4][2], bl[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r = wm * 32 + i * 16 + g;
        split_tf32(t.a[r][kk + q], ah[i][0], al[i][0]);
        split_tf32(t.a[r + 8][kk + q], ah[i][1], al[i][1]);
        split_tf32(t.a[r][kk + q + 4], ah[i][2], al[i][2]);
        split_tf32(t.a[r + 8][kk + q + 4], ah[i][3], al[i][3]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int n = wn * 32 + j * 8 + g;
        split_tf32(t.b[n][kk + q], bh[j][0], bl[j][0]);
        split_tf32(t.b[n][kk + q + 4], bh[j][1], bl[j][1]);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          mma_tf32(acc[i][j], al[i], bh[j]);
          mma_tf32(acc[i][j], ah[i], bl[j]);
          mma_tf32(acc[i][j], ah[i], bh[j]);
        }
    }
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const long long row = r0 + wm * 32 + i * 16 + g + (e >> 1) * 8;
        const long long col = c0 + wn * 32 + j * 8 + 2 * q + (e & 1);
        if (row < m && col < nb) C[row * ldc + col] = acc[i][j][e];
      }
}

__global__ void __launch_bounds__(256) assign_kernel(const float* __restrict__ A, long long m,
                                                     const float* __restrict__ B, long long nb, int dim,
                                                     uint32_t* __restrict__ label, float* __restrict__ best) {
  __shared__ __align__(16) GemmTile t;
  const long long r0 = static_cast<long long>(blockIdx.x) * kTile;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  float bs[8];
  uint32_t bc[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    bs[i] = -INFINITY;
    bc[i] = 0xffffffffu;
  }
  for (long long c0 = 0; c0 < nb; c0 += kTileB) {
    float acc[8][4];
    tile_product(t, A, m, B, nb, dim, r0, c0, acc);
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const long long col = c0 + tx * 4 + j;
        if (col < nb && better(acc[i][j], static_cast<uint32_t>(col), bs[i], bc[i])) {
          bs[i] = acc[i][j];
          bc[i] = static_cast<uint32_t>(col);
        }
      }
  }
  // The 16 threads of a row group are one half of a warp.
#pragma unroll
  for (int i = 0; i < 8; ++i) {
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) {
      const float os = __shfl_xor_sync(full_mask(), bs[i], o);
      const uint32_t oc = __shfl_xor_sync(full_mask(), bc[i], o);
      if (better(os, oc, bs[i], bc[i])) {
        bs[i] = os;
        bc[i] = oc;
      }
    }
    const long long row = r0 + ty * 8 + i;
    if (tx == 0 && row < m) {
      label[row] = bc[i];
      if (best) best[row] = bs[i];
    }
  }
}

// ---------------------------------------------------------------------------
// Top-p per row (score desc, column asc): candidates stream through a buffer
// that is sorted together with the best p kept so far.
// ---------------------------------------------------------------------------
constexpr int kSelThreads = 256;
constexpr int kSelChunk = 1024;

// Sort buffer capacity for top-p: a power of two >= kSelChunk + p.
__host__ __device__ inline int sel_cap(int p) {
  int c = 2;
  while (c < kSelChunk + p) c <<= 1;
  return c;
}

__device__ void cta_sort(float* s, uint32_t* id, int p) {
  for (int size = 2; size <= p; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int t = threadIdx.x; t < (p >> 1); t += blockDim.x) {
        const int i = (t / stride) * 2 * stride + (t % stride);
        const int j = i + stride;
        const bool up = (i & size) == 0;
        const float si = s[i], sj = s[j];
        const uint32_t ii = id[i], ij = id[j];
        if (better(sj, ij, si, ii) == up) {
          s[i] = sj;
          s[j] = si;
          id[i] = ij;
          id[j] = ii;
        }
      }
      __syncthreads();
    }
  }
}

// Top-p by radix selection, for rows that fit in shared memory: the row's
// scores become order-preserving 32-bit keys, four 8-bit histogram passes find
// the p-th largest key T, every key above T and the lowest columns holding T
// are gathered, and only those p entries are sorted. Same output as
// select_top_kernel (a score order with ties by column; -inf and NaN never
// selected).
constexpr int kRadixThreads = 256;
constexpr int kRadixMaxCols = 32768;

// Scores that can be selected map to keys > 0 ordered like the scores (-0 as +0).
__device__ __forceinline__ uint32_t select_key(float v) {
  if (!(v > -INFINITY)) return 0u;
  uint32_t u = __float_as_uint(v);
  if (u == 0x80000000u) u = 0u;
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Bitonic sort of 256 * E 64-bit keys, largest first; thread t holds elements
// t*E .. t*E+E-1. Strides below E exchange registers, strides below 32E (the
// warp's elements) shuffle, only the longer ones go through `tmp` (256 * E
// keys of shared memory) with two barriers each: 6 of the 55 stages at 1,024
// keys instead of every stage.
template <int E, int SIZE, int STRIDE>
__device__ __forceinline__ void bitonic_stage(uint64_t (&k)[E], uint64_t* tmp) {
  const int t = threadIdx.x;
  if constexpr (STRIDE >= 32 * E) {
#pragma unroll
    for (int r = 0; r < E; ++r) tmp[t * E + r] = k[r];
    __syncthreads();
#pragma unroll
    for (int r = 0; r < E; ++r) {
      const int e = t * E + r;
      const uint64_t o = tmp[e ^ STRIDE];
      const bool keep_max = ((e & STRIDE) == 0) == ((e & SIZE) == 0);
      k[r] = keep_max ? (k[r] > o ? k[r] : o) : (k[r] < o ? k[r] : o);
    }
    __syncthreads();
  } else if constexpr (STRIDE >= E) {
#pragma unroll
    for (int r = 0; r < E; ++r) {
      const int e = t * E + r;
      const uint64_t o = __shfl_xor_sync(full_mask(), k[r], STRIDE / E);
      const bool keep_max = ((e & STRIDE) == 0) == ((e & SIZE) == 0);
      k[r] = keep_max ? (k[r] > o ? k[r] : o) : (k[r] < o ? k[r] : o);
    }
  } else {
#pragma unroll
    for (int r = 0; r < E; ++r) {
      if ((r & STRIDE) == 0) {
        const bool up = ((t * E + r) & SIZE) == 0;
        const uint64_t a = k[r], b = k[r + STRIDE];
        if (up ? a < b : a > b) {
          k[r] = b;
          k[r + STRIDE] = a;
        }
      }
    }
  }
}

// The stages of merge size SIZE from STRIDE down, then the larger sizes.
template <int E, int SIZE, int STRIDE>
__device__ __forceinline__ void bitonic_from(uint64_t (&k)[E], uint64_t* tmp) {
  if constexpr (SIZE <= kRadixThreads * E) {
    if constexpr (STRIDE == 0) {
      bitonic_from<E, SIZE * 2, SIZE>(k, tmp);
    } else {
      bitonic_stage<E, SIZE, STRIDE>(k, tmp);
      bitonic_from<E, SIZE, STRIDE / 2>(k, tmp);
    }
  }
}

// Bitonic sort of 256 * E 64-bit keys, largest first; thread t holds elements
// t*E .. t*E+E-1. Strides below E exchange registers, strides below 32E (the
// warp's elements) shuffle, only the longer ones go through `tmp` (256 * E
// keys of shared memory) with two barriers each: 6 of the 55 stages at 1,024
// keys instead of every stage.
template <int E>
__device__ __forceinline__ void cta_sort_keys(uint64_t (&k)[E], uint64_t* tmp) {
  bitonic_from<E, 2, 1>(k, tmp);
}

// E = max(256, next power of two >= p) / 256 keys per thread in the final sort.
template <int E>
__global__ void __launch_bounds__(kRadixThreads) select_radix_kernel(const float* __restrict__ S, long long ld,
                                                                     int ncols, int p, float* __restrict__ out_s,
                                                                     uint32_t* __restrict__ out_i) {
  extern __shared__ __align__(16) unsigned char rad_smem[];
  constexpr int N = kRadixThreads * E;
  // selected (key << 32 | ~column): larger is better, ties to the lower column
  uint64_t* ks = reinterpret_cast<uint64_t*>(rad_smem);
  uint32_t* keys = reinterpret_cast<uint32_t*>(ks + N);  // ncols
  __shared__ unsigned hist[256];
  __shared__ unsigned s_valid, s_eq, s_n, s_bin, s_above, s_warp[kRadixThreads / kWarp];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long row = blockIdx.x;
  const float* sr = S + row * ld;
  if (threadIdx.x == 0) {
    s_valid = 0u;
    s_eq = 0u;
    s_n = 0u;
  }
  __syncthreads();
  unsigned mine = 0;
  for (int c = threadIdx.x; c < ncols; c += blockDim.x) {
    const uint32_t k = select_key(sr[c]);
    keys[c] = k;
    mine += k != 0u;
  }
  atomicAdd(&s_valid, mine);
  __syncthreads();
  const unsigned n_valid = s_valid;
  // T: the p-th largest key (0 when every valid key is taken); rank: how many
  // keys equal to T belong to the top p.
  uint32_t T = 0u, mask = 0u;
  unsigned rank = 0u;
  if (n_valid > static_cast<unsigned>(p)) {
    rank = static_cast<unsigned>(p);
    for (int shift = 24; shift >= 0; shift -= 8) {
      hist[threadIdx.x] = 0u;  // blockDim.x == 256
      __syncthreads();
      for (int c = threadIdx.x; c < ncols; c += blockDim.x) {
        const uint32_t k = keys[c];
        if (k != 0u && (k & mask) == T) atomicAdd(&hist[(k >> shift) & 255u], 1u);
      }
      __syncthreads();
      if (warp == 0) {
        // lane l holds bins 255 - 8l .. 248 - 8l (highest first)
        unsigned c8[8], sum = 0u;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          c8[j] = hist[255 - (lane * 8 + j)];
          sum += c8[j];
        }
        unsigned incl = sum;
#pragma unroll
        for (int o = 1; o < kWarp; o <<= 1) {
          const unsigned t = __shfl_up_sync(full_mask(), incl, o);
          if (lane >= o) incl += t;
        }
        const unsigned excl = incl - sum;
        if (excl < rank && rank <= incl) {
          unsigned acc = excl;
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            if (acc + c8[j] >= rank) {
              s_bin = 255u - static_cast<unsigned>(lane * 8 + j);
              s_above = acc;
              break;
            }
            acc += c8[j];
          }
        }
      }
      __syncthreads();
      T |= s_bin << shift;
      mask |= 0xffu << shift;
      rank -= s_above;
      __syncthreads();  // s_bin / s_above are rewritten by the next pass
    }
    for (int c = threadIdx.x; c < ncols; c += blockDim.x) {
      if (keys[c] == T) atomicAdd(&s_eq, 1u);
    }
    __syncthreads();
  }
  const unsigned n_eq = s_eq;
  // Every key above T (all valid keys when T = 0), and the keys equal to T
  // when all of them belong to the top p.
  const bool all_eq = n_eq <= rank;
  for (int c = threadIdx.x; c < ncols; c += blockDim.x) {
    const uint32_t k = keys[c];
    if (k > T || (k == T && k != 0u && all_eq)) {
      const unsigned pos = atomicAdd(&s_n, 1u);
      ks[pos] = (static_cast<uint64_t>(k) << 32) | static_cast<uint32_t>(~c);
    }
  }
  if (!all_eq) {
    // More keys equal T than fit: the lowest `rank` columns, in column order.
    unsigned base = 0u;
    for (int c0 = 0; c0 < ncols; c0 += blockDim.x) {
      const int c = c0 + threadIdx.x;
      const bool eq = c < ncols && keys[c] == T;
      const unsigned bal = __ballot_sync(full_mask(), eq);
      __syncthreads();
      if (lane == 0) s_warp[warp] = __popc(bal);
      __syncthreads();
      unsigned before = base;
      for (int w = 0; w < warp; ++w) before += s_warp[w];
      before += __popc(bal & ((1u << lane) - 1u));
      if (eq && before < rank) {
        const unsigned pos = atomicAdd(&s_n, 1u);
        ks[pos] = (static_cast<uint64_t>(T) << 32) | static_cast<uint32_t>(~c);
      }
      for (int w = 0; w < kRadixThreads / kWarp; ++w) base += s_warp[w];
    }
  }
  __syncthreads();
  const int n = static_cast<int>(s_n);
  for (int t = n + threadIdx.x; t < N; t += blockDim.x) ks[t] = 0ull;  // below every selected key
  __syncthreads();
  uint64_t k8[E];
#pragma unroll
  for (int r = 0; r < E; ++r) k8[r] = ks[threadIdx.x * E + r];
  cta_sort_keys<E>(k8, ks);
#pragma unroll
  for (int r = 0; r < E; ++r) {
    const int t = threadIdx.x * E + r;
    if (t >= p) break;
    const bool have = k8[r] != 0ull;
    const uint32_t c = ~static_cast<uint32_t>(k8[r]);
    out_s[row * p + t] = have ? sr[c] : -INFINITY;
    out_i[row * p + t] = have ? c : 0xffffffffu;
  }
}

__global__ void __launch_bounds__(kSelThreads) select_top_kernel(const float* __restrict__ S, long long ld,
                                                                 int ncols, int p, float* __restrict__ out_s,
                                                                 uint32_t* __restrict__ out_i) {
  extern __shared__ __align__(16) unsigned char sel_smem[];
  const int cap = sel_cap(p);
  float* buf_s = reinterpret_cast<float*>(sel_smem);
  uint32_t* buf_i = reinterpret_cast<uint32_t*>(buf_s + cap);
  float* keep_s = reinterpret_cast<float*>(buf_i + cap);
  uint32_t* keep_i = reinterpret_cast<uint32_t*>(keep_s + p);
  __shared__ int n_new;
  const long long row = blockIdx.x;
  const float* sr = S + row * ld;
  int nkeep = 0;
  float thr_s = -FLT_MAX;
  uint32_t thr_i = 0xffffffffu;
  for (int base = 0; base < ncols; base += kSelChunk) {
    if (threadIdx.x == 0) n_new = 0;
    __syncthreads();
    for (int t = threadIdx.x; t < kSelChunk; t += blockDim.x) {
      const int c = base + t;
      if (c < ncols) {
        const float v = sr[c];
        if (v > -INFINITY && (nkeep < p || better(v, static_cast<uint32_t>(c), thr_s, thr_i))) {
          const int pos = atomicAdd(&n_new, 1);
          buf_s[pos] = v;
          buf_i[pos] = static_cast<uint32_t>(c);
        }
      }
    }
    __syncthreads();
    const int fresh = n_new;
    __syncthreads();
    if (fresh == 0) continue;
    for (int t = threadIdx.x; t < nkeep; t += blockDim.x) {
      buf_s[fresh + t] = keep_s[t];
      buf_i[fresh + t] = keep_i[t];
    }
    const int tot = fresh + nkeep;
    int q = 2;
    while (q < tot) q <<= 1;
    for (int t = tot + threadIdx.x; t < q; t += blockDim.x) {
      buf_s[t] = -INFINITY;
      buf_i[t] = 0xffffffffu;
    }
    __syncthreads();
    cta_sort(buf_s, buf_i, q);
    nkeep = min(p, tot);
    for (int t = threadIdx.x; t < nkeep; t += blockDim.x) {
      keep_s[t] = buf_s[t];
      keep_i[t] = buf_i[t];
    }
    if (nkeep == p) {
      thr_s = buf_s[p - 1];
      thr_i = buf_i[p - 1];
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < p; t += blockDim.x) {
    const bool have = t < nkeep;
    out_s[row * p + t] = have ? keep_s[t] : -INFINITY;
    out_i[row * p + t] = have ? keep_i[t] : 0xffffffffu;
  }
}

// ---------------------------------------------------------------------------
// Counting sort by label and prefix sums
// ---------------------------------------------------------------------------
__global__ void label_hist_kernel(const uint32_t* __restrict__ label, long long n, uint32_t* __restrict__ counts) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) atomicAdd(&counts[label[i]], 1u);
}

// Exclusive prefix sums of counts (and of ceil(counts / div) when div > 0) in
// one CTA; out[nb] = total.
__global__ void __launch_bounds__(1024) prefix_kernel(const uint32_t* __restrict__ counts, int nb,
                                                      unsigned long long* __restrict__ out, int div,
                                                      unsigned long long* __restrict__ out_div,
                                                      unsigned long long* __restrict__ total_div) {
  __shared__ unsigned long long part[1024];
  __shared__ unsigned long long part_d[1024];
  __shared__ unsigned long long carry, carry_d;
  if (threadIdx.x == 0) {
    carry = 0;
    carry_d = 0;
  }
  __syncthreads();
  for (int base = 0; base < nb; base += 1024) {
    const int i = base + threadIdx.x;
    const unsigned long long c = i < nb ? counts[i] : 0ull;
    const unsigned long long cd = (i < nb && div > 0) ? (c + div - 1) / div : 0ull;
    part[threadIdx.x] = c;
    part_d[threadIdx.x] = cd;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
      const unsigned long long v = threadIdx.x >= o ? part[threadIdx.x - o] : 0ull;
      const unsigned long long vd = threadIdx.x >= o ? part_d[threadIdx.x - o] : 0ull;
      __syncthreads();
      part[threadIdx.x] += v;
      part_d[threadIdx.x] += vd;
      __syncthreads();
    }
    if (i < nb) {
      out[i] = carry + part[threadIdx.x] - c;
      if (div > 0) out_div[i] = carry_d + part_d[threadIdx.x] - cd;
    }
    __syncthreads();
    if (threadIdx.x == 1023) {
      carry += part[1023];
      carry_d += part_d[1023];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[nb] = carry;
    if (div > 0) {
      out_div[nb] = carry_d;
      if (total_div) *total_div = carry_d;
    }
  }
}

__global__ void label_scatter_kernel(const uint32_t* __restrict__ label, long long n,
                                     const unsigned long long* __restrict__ starts, uint32_t* __restrict__ fill,
                                     uint32_t* __restrict__ members) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t b = label[i];
  const unsigned long long pos = starts[b] + atomicAdd(&fill[b], 1u);
  members[pos] = static_cast<uint32_t>(i);
}

__global__ void __launch_bounds__(512) sort_groups_kernel(const unsigned long long* __restrict__ starts,
                                                          uint32_t* __restrict__ members) {
  extern __shared__ uint32_t sm[];
  const int b = blockIdx.x;
  const unsigned long long s0 = starts[b], s1 = starts[b + 1];
  const int n = static_cast<int>(s1 - s0);
  if (n < 2) return;
  int p = 2;
  while (p < n) p <<= 1;
  for (int t = threadIdx.x; t < p; t += blockDim.x) sm[t] = t < n ? members[s0 + t] : 0xffffffffu;
  __syncthreads();
  for (int size = 2; size <= p; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int t = threadIdx.x; t < (p >> 1); t += blockDim.x) {
        const int i = (t / stride) * 2 * stride + (t % stride);
        const int j = i + stride;
        const bool up = (i & size) == 0;
        const uint32_t a = sm[i], c = sm[j];
        if ((c < a) == up) {
          sm[i] = c;
          sm[j] = a;
        }
      }
      __syncthreads();
    }
  }
  for (int t = threadIdx.x; t < n; t += blockDim.x) members[s0 + t] = sm[t];
}

// ---------------------------------------------------------------------------
// Deterministic centroids
// ---------------------------------------------------------------------------
constexpr int kCentSplit = 8;
constexpr int kCentThreads = 256;
constexpr int kCentMaxDim = 4096;

__device__ __forceinline__ long long to_fixed(float v) {
  return __double2ll_rn(static_cast<double>(v) * kFixedScale);
}

__global__ void __launch_bounds__(kCentThreads) centroid_sum_kernel(const float* __restrict__ X, int dim,
                                                                    const unsigned long long* __restrict__ starts,
                                                                    const uint32_t* __restrict__ members,
                                                                    long long* __restrict__ acc) {
  const int b = blockIdx.x, part = blockIdx.y;
  const unsigned long long s0 = starts[b], s1 = starts[b + 1];
  const unsigned long long n = s1 - s0;
  if (n == 0) return;
  const unsigned long long per = (n + kCentSplit - 1) / kCentSplit;
  const unsigned long long m0 = s0 + part * per;
  const unsigned long long m1 = min(s1, m0 + per);
  if (m0 >= m1) return;
  constexpr int kR = kCentMaxDim / kCentThreads;
  long long sum[kR];
#pragma unroll
  for (int r = 0; r < kR; ++r) sum[r] = 0;
  for (unsigned long long m = m0; m < m1; ++m) {
    const float* row = X + static_cast<long long>(members[m]) * dim;
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      const int d = threadIdx.x + r * kCentThreads;
      if (d < dim) sum[r] += to_fixed(row[d]);
    }
  }
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    const int d = threadIdx.x + r * kCentThreads;
    if (d < dim) {
      atomicAdd(reinterpret_cast<unsigned long long*>(acc + static_cast<long long>(b) * dim + d),
                static_cast<unsigned long long>(sum[r]));
    }
  }
}

// One warp per group: enc = fixed-point sum / (count * 2^32); route = enc / ||enc||.
__global__ void centroid_finish_kernel(const long long* __restrict__ acc, int dim, int nb,
                                       const unsigned long long* __restrict__ starts, float* __restrict__ enc,
                                       float* __restrict__ route) {
  const int b = (blockIdx.x * blockDim.x + threadIdx.x) / kWarp;
  const int lane = threadIdx.x & 31;
  if (b >= nb) return;
  const unsigned long long n = starts[b + 1] - starts[b];
  if (n == 0) return;
  const double inv = 1.0 / (static_cast<double>(n) * kFixedScale);
  double ss = 0.0;
  for (int d = lane; d < dim; d += kWarp) {
    const float v = static_cast<float>(static_cast<double>(acc[static_cast<long long>(b) * dim + d]) * inv);
    enc[static_cast<long long>(b) * dim + d] = v;
    ss += static_cast<double>(v) * v;
  }
  ss = warp_sum_d(ss);
  const double rn = ss > 0.0 ? 1.0 / sqrt(ss) : 0.0;
  for (int d = lane; d < dim; d += kWarp) {
    route[static_cast<long long>(b) * dim + d] =
        static_cast<float>(static_cast<double>(enc[static_cast<long long>(b) * dim + d]) * rn);
  }
}

// ---------------------------------------------------------------------------
// 2-means fission
// ---------------------------------------------------------------------------
constexpr int kSplitThreads = 256;

__device__ __forceinline__ float warp_dot(const float* __restrict__ a, const float* __restrict__ b, int dim,
                                          int lane) {
  float s = 0.f;
  for (int d = lane; d < dim; d += kWarp) s = __fmaf_rn(a[d], b[d], s);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s = __fadd_rn(s, __shfl_xor_sync(full_mask(), s, o));
  return s;
}

// Lowest (value, id) over the CTA; every thread gets the winner's id.
__device__ uint32_t cta_argmin(float v, uint32_t id, float* red_v, uint32_t* red_i) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float ov = __shfl_xor_sync(full_mask(), v, o);
    const uint32_t oi = __shfl_xor_sync(full_mask(), id, o);
    if (ov < v || (ov == v && oi < id)) {
      v = ov;
      id = oi;
    }
  }
  __syncthreads();
  if (lane == 0) {
    red_v[warp] = v;
    red_i[warp] = id;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kSplitThreads / kWarp; ++w) {
      if (red_v[w] < red_v[0] || (red_v[w] == red_v[0] && red_i[w] < red_i[0])) {
        red_v[0] = red_v[w];
        red_i[0] = red_i[w];
      }
    }
  }
  __syncthreads();
  return red_i[0];
}

__global__ void __launch_bounds__(kSplitThreads) split_kernel(const float* __restrict__ X, int dim,
                                                              const unsigned long long* __restrict__ starts,
                                                              const uint32_t* __restrict__ members,
                                                              const uint32_t* __restrict__ groups,
                                                              const uint32_t* __restrict__ new_label,
                                                              const float* __restrict__ route,
                                                              uint32_t* __restrict__ label, int force_bits) {
  extern __shared__ __align__(16) unsigned char smem[];
  float* cA = reinterpret_cast<float*>(smem);             // dim
  float* cB = cA + dim;                                   // dim
  unsigned long long* sum0 = reinterpret_cast<unsigned long long*>(cB + dim);  // dim
  unsigned long long* sum1 = sum0 + dim;                  // dim
  __shared__ float red_v[kSplitThreads / kWarp];
  __shared__ uint32_t red_i[kSplitThreads / kWarp];
  __shared__ unsigned int n_side[2];
  __shared__ unsigned int id_or, id_and;
  const int g = groups[blockIdx.x];
  const uint32_t lab1 = new_label[blockIdx.x];
  const unsigned long long s0 = starts[g], s1 = starts[g + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int kWarps = kSplitThreads / kWarp;
  const float* c = route + static_cast<long long>(g) * dim;

  // Seed A: the member least aligned with the routing centroid.
  float bv = INFINITY;
  uint32_t bi = 0xffffffffu;
  for (unsigned long long m = s0 + warp; m < s1; m += kWarps) {
    const uint32_t id = members[m];
    const float d = warp_dot(X + static_cast<long long>(id) * dim, c, dim, lane);
    if (d < bv || (d == bv && id < bi)) {
      bv = d;
      bi = id;
    }
  }
  const uint32_t seed_a = cta_argmin(bv, bi, red_v, red_i);
  for (int d = threadIdx.x; d < dim; d += blockDim.x) cA[d] = X[static_cast<long long>(seed_a) * dim + d];
  __syncthreads();
  // Seed B: the member least aligned with seed A.
  bv = INFINITY;
  bi = 0xffffffffu;
  for (unsigned long long m = s0 + warp; m < s1; m += kWarps) {
    const uint32_t id = members[m];
    const float d = warp_dot(X + static_cast<long long>(id) * dim, cA, dim, lane);
    if (d < bv || (d == bv && id < bi)) {
      bv = d;
      bi = id;
    }
  }
  const uint32_t seed_b = cta_argmin(bv, bi, red_v, red_i);
  for (int d = threadIdx.x; d < dim; d += blockDim.x) cB[d] = X[static_cast<long long>(seed_b) * dim + d];
  for (int d = threadIdx.x; d < dim; d += blockDim.x) {
    sum0[d] = 0ull;
    sum1[d] = 0ull;
  }
  if (threadIdx.x < 2) n_side[threadIdx.x] = 0u;
  __syncthreads();
  // Members to the closer seed; fixed-point sums of the two sides.
  for (unsigned long long m = s0 + warp; m < s1; m += kWarps) {
    const uint32_t id = members[m];
    const float* row = X + static_cast<long long>(id) * dim;
    const float da = warp_dot(row, cA, dim, lane), db = warp_dot(row, cB, dim, lane);
    unsigned long long* sum = (db > da) ? sum1 : sum0;
    for (int d = lane; d < dim; d += kWarp) atomicAdd(&sum[d], static_cast<unsigned long long>(to_fixed(row[d])));
  }
  __syncthreads();
  // The two means (sums; their scale does not matter for the cosine comparison).
  for (int d = threadIdx.x; d < dim; d += blockDim.x) {
    const float a = static_cast<float>(static_cast<double>(static_cast<long long>(sum0[d])) / kFixedScale);
    const float b = static_cast<float>(static_cast<double>(static_cast<long long>(sum1[d])) / kFixedScale);
    cA[d] = a;
    cB[d] = b;
  }
  __syncthreads();
  // Members to the closer mean (cosine): compare <x, a>/|a| with <x, b>/|b|.
  __shared__ float norm_ab[2];
  if (warp == 0) {
    const float na = warp_dot(cA, cA, dim, lane), nb = warp_dot(cB, cB, dim, lane);
    if (lane == 0) {
      norm_ab[0] = __fsqrt_rn(na);
      norm_ab[1] = __fsqrt_rn(nb);
    }
  }
  if (threadIdx.x == 0) {
    id_or = 0u;
    id_and = 0xffffffffu;
  }
  __syncthreads();
  const float na = norm_ab[0], nb = norm_ab[1];
  for (unsigned long long m = s0 + warp; m < s1; m += kWarps) {
    const uint32_t id = members[m];
    const float* row = X + static_cast<long long>(id) * dim;
    const float da = warp_dot(row, cA, dim, lane), db = warp_dot(row, cB, dim, lane);
    // db / nb > da / na, cross-multiplied (norms are >= 0)
    const bool side = __fmul_rn(db, na) > __fmul_rn(da, nb);
    if (lane == 0) {
      atomicAdd(&n_side[side ? 1 : 0], 1u);
      atomicOr(&id_or, id);
      atomicAnd(&id_and, id);
    }
  }
  __syncthreads();
  const bool degenerate = force_bits || n_side[0] == 0u || n_side[1] == 0u;
  // Degenerate split (e.g. identical rows): divide by the lowest id bit that
  // differs among the members (ids are distinct, so one does).
  const unsigned diff = id_or ^ id_and;
  const int bit = diff ? __ffs(static_cast<int>(diff)) - 1 : 0;
  for (unsigned long long m = s0 + warp; m < s1; m += kWarps) {
    const uint32_t id = members[m];
    bool side;
    if (degenerate) {
      side = (id >> bit) & 1u;
    } else {
      const float* row = X + static_cast<long long>(id) * dim;
      const float da = warp_dot(row, cA, dim, lane), db = warp_dot(row, cB, dim, lane);
      side = __fmul_rn(db, na) > __fmul_rn(da, nb);
    }
    if (lane == 0 && side) label[id] = lab1;
  }
}

// ---------------------------------------------------------------------------
// Residual slot layout
// ---------------------------------------------------------------------------
__global__ void build_residuals_kernel(const float* __restrict__ X, int dim,
                                       const unsigned long long* __restrict__ starts,
                                       const uint32_t* __restrict__ members,
                                       const unsigned long long* __restrict__ slot_start,
                                       const float* __restrict__ enc, float* __restrict__ R,
                                       uint32_t* __restrict__ slot_ids) {
  const int b = blockIdx.x;
  const unsigned long long s0 = starts[b], n = starts[b + 1] - s0;
  const unsigned long long t0 = slot_start[b], t1 = slot_start[b + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x / kWarp;
  const float* c = enc + static_cast<long long>(b) * dim;
  for (unsigned long long t = t0 + warp; t < t1; t += warps) {
    const unsigned long long r = t - t0;
    float* out = R + static_cast<long long>(t) * dim;
    if (r < n) {
      const uint32_t id = members[s0 + r];
      const float* row = X + static_cast<long long>(id) * dim;
      for (int d = lane; d < dim; d += kWarp) out[d] = __fsub_rn(row[d], c[d]);
      if (lane == 0) slot_ids[t] = id;
    } else {
      for (int d = lane; d < dim; d += kWarp) out[d] = 0.f;
      if (lane == 0) slot_ids[t] = 0xffffffffu;
    }
  }
}

__global__ void residual_rows_kernel(const float* __restrict__ X, long long n, int dim,
                                     const uint32_t* __restrict__ label, const float* __restrict__ enc,
                                     float* __restrict__ R) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n * dim) return;
  const long long row = i / dim;
  const int d = static_cast<int>(i % dim);
  R[i] = __fsub_rn(X[i], enc[static_cast<long long>(label[row]) * dim + d]);
}

// ---------------------------------------------------------------------------
// Probe pairs and work items
// ---------------------------------------------------------------------------
__device__ __forceinline__ int probes_of(const PairArgs& a, long long q) {
  const int np = a.n_probe ? static_cast<int>(a.n_probe[q]) : a.fixed_probe;
  return np < a.max_probe ? np : a.max_probe;
}

// Probe position j of query q gets a pair in this build.
__device__ __forceinline__ bool pair_in_range(const PairArgs& a, long long q, int j) {
  const int np = probes_of(a, q);
  int lo = a.probe_begin, hi = a.probe_end;
  if (a.first_split) {
    int f = np >= a.wide_from ? kFloorProbesWide : kFloorProbes;
    f = f < np ? f : np;
    if (a.first_split == 1) {
      hi = hi < f ? hi : f;
    } else {
      lo = lo > f ? lo : f;
    }
  }
  return j >= lo && j < hi && j < np;
}

__global__ void pair_count_kernel(PairArgs a) {
  const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= a.nq * a.max_probe) return;
  const long long q = t / a.max_probe;
  const int j = static_cast<int>(t % a.max_probe);
  if (!pair_in_range(a, q, j)) return;
  const uint32_t b = a.probes[q * (a.probe_stride ? a.probe_stride : a.max_probe) + j];
  if (b < static_cast<uint32_t>(a.nb)) atomicAdd(&a.counts[b], 1u);
}

__global__ void pair_scatter_kernel(PairArgs a) {
  const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= a.nq * a.max_probe) return;
  const long long q = t / a.max_probe;
  const int j = static_cast<int>(t % a.max_probe);
  if (!pair_in_range(a, q, j)) return;
  const uint32_t b = a.probes[q * (a.probe_stride ? a.probe_stride : a.max_probe) + j];
  if (b >= static_cast<uint32_t>(a.nb)) return;
  const unsigned long long pos = a.pair_start[b] + atomicAdd(&a.fill[b], 1u);
  a.pairs[pos] = static_cast<uint32_t>(t);
}

// One thread per (query, probe): the offset <q_hat, enc[b]> read from the
// q_hat . enc^T product computed before the pairs.
__global__ void pair_offset_gather_kernel(PairArgs a) {
  const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= a.nq * a.max_probe) return;
  const long long q = t / a.max_probe;
  const int j = static_cast<int>(t % a.max_probe);
  if (!pair_in_range(a, q, j)) return;
  const uint32_t b = a.probes[q * (a.probe_stride ? a.probe_stride : a.max_probe) + j];
  if (b >= static_cast<uint32_t>(a.nb)) return;
  a.offsets[t] = a.enc_scores[q * a.enc_ld + b];
}

__global__ void item_build_kernel(PairArgs a) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= a.nb) return;
  const unsigned long long c = a.pair_start[b + 1] - a.pair_start[b];
  const unsigned long long i0 = a.item_start[b];
  for (unsigned long long t = 0; t * kItemQueries < c; ++t) {
    const unsigned long long first = a.pair_start[b] + t * kItemQueries;
    const unsigned long long cnt = min(static_cast<unsigned long long>(kItemQueries), c - t * kItemQueries);
    a.items[i0 + t] = make_uint4(static_cast<unsigned>(b), static_cast<unsigned>(first),
                                 static_cast<unsigned>(cnt), 0u);
  }
}

// ---------------------------------------------------------------------------
// Bucket scan
// ---------------------------------------------------------------------------
constexpr int kBsWarps = 4;
constexpr int kBsQueriesPerWarp = 2;  // bucket scan; the multi-index scan keeps 4
static_assert(kBsWarps / (kItemQueries / kBsQueriesPerWarp) == kBsListsPerProbe,
              "bucket-scan tile sets per item must match the candidate lists per probe");
constexpr int kBsPrefetch = 4;
constexpr int kBsBuf = 512;  // per-warp sort buffer: up to 256 new + 256 kept

// Per-warp top-k list capacity for k (k <= 256).
__host__ __device__ inline int kmax_of(int k) { return k <= 32 ? 32 : (k <= 64 ? 64 : (k <= 128 ? 128 : 256)); }

// j-th largest (1-based, j <= 8) of the lane's valid scores, -inf if fewer.
__device__ __forceinline__ float lane_jth_largest(const float (&sc)[8], unsigned ok, int j) {
  float v[8];
#pragma unroll
  for (int t = 0; t < 8; ++t) v[t] = (ok >> t & 1u) ? sc[t] : -INFINITY;
  // partial selection: j passes of max extraction
  float out = -INFINITY;
  for (int r = 0; r < j; ++r) {
    int bi = 0;
    float bv = v[0];
#pragma unroll
    for (int t = 1; t < 8; ++t) {
      if (v[t] > bv) {
        bv = v[t];
        bi = t;
      }
    }
    out = bv;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      if (t == bi) v[t] = -INFINITY;
    }
  }
  return out;
}

// One scan work item: up to kItemQueries queries against one range of slots
// of a scan layout (a probed bucket, or a vector range of a flat index).
struct ItemView {
  const uint32_t* codes;
  const float* alpha;
  const uint32_t* slot_ids;  // original id per slot; nullptr: the id is the slot
  long long slot0;           // multiple of kBucketSlotAlign
  int size;                  // slots of the range
  int nbg;
  const uint8_t* luts;       // LUT rows (nbg x 32 bytes each)
  int k;
  int pc;                    // queries of the item
  float* cand_s;
  uint32_t* cand_i;
  // nullptr: each (query, tile set) writes its own list of k entries at
  // ItemQueries::list, -inf padded. Otherwise ItemQueries::list is the start
  // (in lists of k) of the query's candidate region and the kept candidates
  // are appended there at append_count[query] (atomically), unpadded.
  uint32_t* append_count = nullptr;
};

// The item's queries, in shared memory (filled by the calling kernel).
struct ItemQueries {
  int q[kItemQueries];           // LUT row (-1: no query)
  long long list[kItemQueries];  // candidate list written by tile set 0 (tile set 1: list + 1)
  float scale[kItemQueries], init[kItemQueries], off[kItemQueries];
  float floor[kItemQueries];     // scores below it are not kept (-inf: keep all)
};

// Scans one item with the CTA's 4 warps and writes one candidate list of k per
// (query, tile set). QW = 4: 2 groups of 4 queries x 2 tile sets (a warp scans
// every other 256-slot tile set); QW = 2: 4 groups of 2 queries x 1 tile set
// (a warp scans every tile set: half the registers for accumulators, so more
// CTAs fit on an SM; the bucket scan takes this form).
// WHOLE: every 256-group batch of the item's index is a whole number of
// kBsPrefetch-group rings (nbg a multiple of kBsPrefetch); the ring loop then
// runs without bounds checks.
template <bool NIBBLE8, int QW = 4, bool WHOLE = false>
__device__ __forceinline__ void scan_item(const ItemView& v, const ItemQueries& iq, unsigned char* smem) {
  constexpr int kGroups = kItemQueries / QW;  // query groups per item
  constexpr int kTsets = kBsWarps / kGroups;  // tile sets scanned side by side
  const int nbg = v.nbg, k = v.k, pc = v.pc;
  const int chunk = nbg < kFlushGroups ? nbg : kFlushGroups;
  const bool resident = chunk >= nbg;

  LutHalf* s_lut = reinterpret_cast<LutHalf*>(smem);  // [kItemQueries][chunk][2]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int kmax = kmax_of(k);
  // Per-warp top-k lists and sort buffer after the LUT area.
  unsigned char* warp_area = smem + static_cast<size_t>(kItemQueries) * chunk * 32 +
                             warp * (static_cast<size_t>(QW) * kmax * 8 + kBsBuf * 8);
  float* list_s = reinterpret_cast<float*>(warp_area);
  uint32_t* list_i = reinterpret_cast<uint32_t*>(list_s + QW * kmax);
  float* buf_s = reinterpret_cast<float*>(list_i + QW * kmax);
  uint32_t* buf_i = reinterpret_cast<uint32_t*>(buf_s + kBsBuf);

  auto load_lut_chunk = [&](int g_first, int g_count) {
    const int halves = g_count * 2;
    for (int t = threadIdx.x; t < kItemQueries * halves; t += blockDim.x) {
      const int q = t / halves, r = t % halves;
      LutHalf h = {{0u, 0u, 0u, 0u}};
      if (iq.q[q] >= 0) {
        h = *reinterpret_cast<const LutHalf*>(v.luts + (static_cast<long long>(iq.q[q]) * nbg + g_first) * 32LL +
                                              r * 16LL);
      }
      s_lut[q * chunk * 2 + r] = h;
    }
  };
  if (resident) {
    load_lut_chunk(0, nbg);
    __syncthreads();
  }

  const int quad = warp % kGroups, tset = warp / kGroups;
  const bool quad_ok = quad * QW < pc;
  const unsigned long long slot0 = static_cast<unsigned long long>(v.slot0);
  const int size = v.size;
  const int n_sub = (size + kBucketSlotAlign - 1) / kBucketSlotAlign;
  // per-query constants stay in shared memory (iq): fewer live registers
  float thr_s[QW];
  uint32_t thr_i[QW];
  int cnt[QW];
#pragma unroll
  for (int q = 0; q < QW; ++q) {
    thr_s[q] = -FLT_MAX;
    thr_i[q] = 0xffffffffu;
    cnt[q] = 0;
  }
  const int j_rank = (k + 31) / 32;           // per-lane rank used by the prefilter
  const int k_rank = (k + j_rank - 1) / j_rank;  // rank among the 32 lane values
  constexpr long long kGroupStride = kTileWords / 2;  // uint2 per group row

  const int rounds = (n_sub + kTsets - 1) / kTsets;
  for (int r = 0; r < rounds; ++r) {
    const int st = tset + kTsets * r;
    const bool active = quad_ok && st < n_sub;
    const long long sub = static_cast<long long>(slot0 / kBucketSlotAlign) + st;
    const long long tile = sub >> 1;
    const int half = static_cast<int>(sub & 1);
    const uint2* wp = reinterpret_cast<const uint2*>(v.codes + tile * nbg * kTileWords + half * 64) + lane;
    const long long vbase = sub * kBucketSlotAlign + 8 * lane;
    float fa[QW][8];
    uint32_t acc[QW][8];
#pragma unroll
    for (int q = 0; q < QW; ++q)
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        fa[q][j] = iq.init[quad * QW + q];
        acc[q][j] = 0u;
      }
    for (int gb = 0; gb < nbg; gb += kFlushGroups) {
      const int g_stop = min(gb + kFlushGroups, nbg);
      if (!resident) {
        __syncthreads();
        load_lut_chunk(gb, g_stop - gb);
        __syncthreads();
      }
      if (!active) continue;
      const int chunk_base = resident ? 0 : gb;
      const LutHalf* lq = s_lut + (quad * QW) * chunk * 2;  // this warp's queries
      uint2 ring[kBsPrefetch];
      if constexpr (WHOLE) {
        // Every batch is a whole number of rings: no bounds checks, loads at
        // immediate offsets of a running pointer.
        const uint2* src = wp + static_cast<long long>(gb) * kGroupStride;
#pragma unroll
        for (int u = 0; u < kBsPrefetch; ++u) ring[u] = src[u * kGroupStride];
        src += kBsPrefetch * kGroupStride;
        int g = gb;
        for (; g + kBsPrefetch < g_stop; g += kBsPrefetch) {
          uint2 cur[kBsPrefetch];
#pragma unroll
          for (int u = 0; u < kBsPrefetch; ++u) {
            cur[u] = ring[u];
            ring[u] = src[u * kGroupStride];
          }
          src += kBsPrefetch * kGroupStride;
#pragma unroll
          for (int u = 0; u < kBsPrefetch; u += 2) {
            lookup_group_pair<QW, NIBBLE8>(cur[u], cur[u + 1], lq + (g + u - chunk_base) * 2, chunk * 2, acc);
          }
        }
#pragma unroll
        for (int u = 0; u < kBsPrefetch; u += 2) {
          lookup_group_pair<QW, NIBBLE8>(ring[u], ring[u + 1], lq + (g + u - chunk_base) * 2, chunk * 2, acc);
        }
      } else {
#pragma unroll
        for (int u = 0; u < kBsPrefetch; ++u) {
          ring[u] = (gb + u < g_stop) ? wp[(gb + u) * kGroupStride] : make_uint2(0u, 0u);
        }
        for (int g = gb; g < g_stop; g += kBsPrefetch) {
          uint2 cur[kBsPrefetch];
#pragma unroll
          for (int u = 0; u < kBsPrefetch; ++u) {
            cur[u] = ring[u];
            const int gn = g + kBsPrefetch + u;
            ring[u] = (gn < g_stop) ? wp[gn * kGroupStride] : make_uint2(0u, 0u);
          }
          // Groups in pairs (nbg and the 256-group batches are even).
#pragma unroll
          for (int u = 0; u < kBsPrefetch; u += 2) {
            if (g + u >= g_stop) break;
            lookup_group_pair<QW, NIBBLE8>(cur[u], cur[u + 1], lq + (g + u - chunk_base) * 2, chunk * 2, acc);
          }
        }
      }
      // f32 flush of this batch (search_avx2.cpp:24-48).
#pragma unroll
      for (int q = 0; q < QW; ++q)
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          fa[q][j] = __fmaf_rn(iq.scale[quad * QW + q], __uint2float_rn(acc[q][j]), fa[q][j]);
          acc[q][j] = 0u;
        }
    }
    if (!active) continue;  // warp-uniform; no CTA barrier follows in this round

    float al[8];
    uint32_t ids[8];
    {
      const float4 x0 = *reinterpret_cast<const float4*>(v.alpha + vbase);
      const float4 x1 = *reinterpret_cast<const float4*>(v.alpha + vbase + 4);
      al[0] = x0.x; al[1] = x0.y; al[2] = x0.z; al[3] = x0.w;
      al[4] = x1.x; al[5] = x1.y; al[6] = x1.z; al[7] = x1.w;
      if (v.slot_ids) {
        const uint4 i0 = *reinterpret_cast<const uint4*>(v.slot_ids + vbase);
        const uint4 i1 = *reinterpret_cast<const uint4*>(v.slot_ids + vbase + 4);
        ids[0] = i0.x; ids[1] = i0.y; ids[2] = i0.z; ids[3] = i0.w;
        ids[4] = i1.x; ids[5] = i1.y; ids[6] = i1.z; ids[7] = i1.w;
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) ids[j] = static_cast<uint32_t>(vbase + j);
      }
    }
    unsigned valid = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if (vbase + j - static_cast<long long>(slot0) < size) valid |= 1u << j;
    }
#pragma unroll
    for (int q = 0; q < QW; ++q) {
      if (quad * QW + q >= pc) break;  // warp-uniform
      float sc[8];
      unsigned ok = 0;
      const float fl = iq.floor[quad * QW + q];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        sc[j] = __fadd_rn(__fmul_rn(fa[q][j], al[j]), iq.off[quad * QW + q]);
        if ((valid >> j & 1u) && sc[j] > -INFINITY && !(sc[j] < fl)) ok |= 1u << j;
      }
      if (!__any_sync(full_mask(), ok != 0u)) continue;  // nothing at or above the floor
      if (r == rounds - 1) {
        // Last block and every admissible score fits in the list: append them
        // all, unsorted (published lists need not be ordered; the merge
        // selects and sorts), without the prefilter.
        const int n_ok = __popc(ok);
        int incl_ok = n_ok;
#pragma unroll
        for (int o = 1; o < kWarp; o <<= 1) {
          const int t = __shfl_up_sync(full_mask(), incl_ok, o);
          if (lane >= o) incl_ok += t;
        }
        const int total_ok = __shfl_sync(full_mask(), incl_ok, kWarp - 1);
        if (cnt[q] + total_ok <= k) {
          float* ls = list_s + q * kmax;
          uint32_t* li = list_i + q * kmax;
          int at = cnt[q] + incl_ok - n_ok;
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            if (ok >> j & 1u) {
              ls[at] = sc[j];
              li[at] = ids[j];
              ++at;
            }
          }
          cnt[q] += total_ok;
          __syncwarp();
          continue;
        }
      }
      unsigned pass = 0;
      if (cnt[q] == k) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          if ((ok >> j & 1u) && better(sc[j], ids[j], thr_s[q], thr_i[q])) pass |= 1u << j;
        }
      } else {
        // At least k_rank lanes hold j_rank scores >= bound, i.e. >= k scores of
        // this block are >= bound, so a score below it cannot be in the top-k.
        const float mine = lane_jth_largest(sc, ok, j_rank);
        const float bound = warp_kth_largest(mine, k_rank, lane);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          if ((ok >> j & 1u) && !(sc[j] < bound)) pass |= 1u << j;
        }
      }
      const int n_mine = __popc(pass);
      int incl = n_mine;
#pragma unroll
      for (int o = 1; o < kWarp; o <<= 1) {
        const int t = __shfl_up_sync(full_mask(), incl, o);
        if (lane >= o) incl += t;
      }
      const int total = __shfl_sync(full_mask(), incl, kWarp - 1);
      if (total == 0) continue;
      float* ls = list_s + q * kmax;
      uint32_t* li = list_i + q * kmax;
      if (r == rounds - 1 && cnt[q] + total <= k) {
        // Last block and the prefiltered scores fit: append without sorting.
        int at = cnt[q] + incl - n_mine;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          if (pass >> j & 1u) {
            ls[at] = sc[j];
            li[at] = ids[j];
            ++at;
          }
        }
        cnt[q] += total;
        __syncwarp();
        continue;
      }
      int pos = incl - n_mine;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if (pass >> j & 1u) {
          buf_s[pos] = sc[j];
          buf_i[pos] = ids[j];
          ++pos;
        }
      }
      for (int t = lane; t < cnt[q]; t += kWarp) {
        buf_s[total + t] = ls[t];
        buf_i[total + t] = li[t];
      }
      const int tot = total + cnt[q];
      int p = 32;
      while (p < tot) p <<= 1;
      for (int t = tot + lane; t < p; t += kWarp) {
        buf_s[t] = -INFINITY;
        buf_i[t] = 0xffffffffu;
      }
      __syncwarp();
      warp_sort_best_first(buf_s, buf_i, p, lane);
      const int keep = min(k, tot);
      for (int t = lane; t < keep; t += kWarp) {
        ls[t] = buf_s[t];
        li[t] = buf_i[t];
      }
      cnt[q] = keep;
      if (keep == k) {
        thr_s[q] = buf_s[k - 1];
        thr_i[q] = buf_i[k - 1];
      }
      __syncwarp();
    }
  }
  // Publish the list (tile set 0's list + tile set) of every valid query of this warp.
  if (!quad_ok) return;
  if (v.append_count) {
#pragma unroll
    for (int q = 0; q < QW; ++q) {
      if (quad * QW + q >= pc) break;
      const int c = cnt[q];
      if (c == 0) continue;  // warp-uniform
      unsigned at = 0;
      if (lane == 0) at = atomicAdd(v.append_count + iq.q[quad * QW + q], static_cast<unsigned>(c));
      at = __shfl_sync(full_mask(), at, 0);
      const long long base = iq.list[quad * QW + q] * k + at;
      for (int t = lane; t < c; t += kWarp) {
        v.cand_s[base + t] = list_s[q * kmax + t];
        v.cand_i[base + t] = list_i[q * kmax + t];
      }
    }
    return;
  }
#pragma unroll
  for (int q = 0; q < QW; ++q) {
    if (quad * QW + q >= pc) break;
    const long long list = iq.list[quad * QW + q] + tset;
    float* os = v.cand_s + list * k;
    uint32_t* oi = v.cand_i + list * k;
    for (int t = lane; t < k; t += kWarp) {
      const bool have = t < cnt[q];
      os[t] = have ? list_s[q * kmax + t] : -INFINITY;
      oi[t] = have ? list_i[q * kmax + t] : 0xffffffffu;
    }
  }
}

// One work item (a bucket and up to kItemQueries of its probing queries).
template <bool NIBBLE8, bool WHOLE>
__device__ __forceinline__ void bucket_scan_item(const BucketScanArgs& a, const uint4 it, ItemQueries& iq,
                                                 unsigned char* smem) {
  const int b = static_cast<int>(it.x);
  const int pc = static_cast<int>(it.z);
  if (threadIdx.x < kItemQueries) {
    const int t = threadIdx.x;
    if (t < pc) {
      const uint32_t pr = a.pairs[it.y + t];
      const int q = static_cast<int>(pr / static_cast<uint32_t>(a.max_probe));
      iq.q[t] = q;
      // (query, probe) lists, or the query's region when appending
      iq.list[t] = (a.append_count ? static_cast<long long>(q) * a.max_probe : static_cast<long long>(pr)) *
                   kBsListsPerProbe;
      iq.scale[t] = a.lut_scale[q];
      iq.init[t] = a.fa_init[q];
      iq.off[t] = a.offsets[pr];
      iq.floor[t] = a.floor ? a.floor[q] : -INFINITY;
    } else {
      iq.q[t] = -1;
      iq.list[t] = 0;
      iq.scale[t] = 0.f;
      iq.init[t] = 0.f;
      iq.off[t] = 0.f;
      iq.floor[t] = -INFINITY;
    }
  }
  __syncthreads();
  const ItemView v{a.codes, a.alpha, a.slot_ids, static_cast<long long>(a.slot_start[b]),
                   static_cast<int>(a.bucket_size[b]), a.nbg, a.luts, a.k, pc, a.cand_score, a.cand_id,
                   a.append_count};
  scan_item<NIBBLE8, kBsQueriesPerWarp, WHOLE>(v, iq, smem);
}

// kBsQueriesPerWarp = 2: 96 registers, 5 CTAs per SM (20 warps; 4 queries per
// warp held 4 CTAs); measured 8 % faster at 1.2M x 100, n_probe 512. The grid
// is the resident CTA count; each CTA pulls the next item from a device
// counter until none is left, so a host bound far above the real item count
// (per-query probe counts up to a large maximum) costs no empty CTAs. (A fixed
// stride over the items instead measured 9 % slower than one item per CTA:
// items are uneven; pulling balances them as the block scheduler does.)
template <bool NIBBLE8, bool WHOLE>
__global__ void __launch_bounds__(kBsWarps * 32, 5) bucket_scan_kernel(BucketScanArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ ItemQueries iq;
  __shared__ unsigned long long s_item;
  const unsigned long long n_items = *a.n_items;
  while (true) {
    __syncthreads();  // the previous item is done with iq and the LUT area
    if (threadIdx.x == 0) s_item = atomicAdd(a.next_item, 1ull);
    __syncthreads();
    const unsigned long long item = s_item;
    if (item >= n_items) return;
    bucket_scan_item<NIBBLE8, WHOLE>(a, a.items[item], iq, smem);
  }
}

// ---------------------------------------------------------------------------
// Multi-index persistent scan: a fixed grid of CTAs pulls work items — (flat
// index, vector range, up to 8 of its queries) — from a global counter until
// none is left, so one launch serves indexes of any n, dim and bits.
// ---------------------------------------------------------------------------
template <bool ANY3, bool ANY24>
__global__ void __launch_bounds__(kBsWarps * 32, 4) multi_scan_kernel(MultiScanArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ ItemQueries iq;
  __shared__ long long s_item;
  while (true) {
    __syncthreads();  // the previous item is done with iq and the LUT area
    if (threadIdx.x == 0) s_item = static_cast<long long>(atomicAdd(a.next_item, 1ull));
    __syncthreads();
    const long long item = s_item;
    if (item >= a.n_items) return;
    const MultiItem it = a.items[item];
    const MultiIndexDesc d = a.indexes[it.index];
    if (threadIdx.x < kItemQueries) {
      const int t = threadIdx.x;
      if (t < it.n_queries) {
        const int q = it.first_query + t;
        iq.q[t] = q;
        iq.list[t] = (static_cast<long long>(q) * d.n_ranges + it.range) * 2;
        iq.scale[t] = d.lut_scale[q];
        iq.init[t] = d.fa_init[q];
        iq.off[t] = 0.f;
      } else {
        iq.q[t] = -1;
        iq.list[t] = 0;
        iq.scale[t] = 0.f;
        iq.init[t] = 0.f;
        iq.off[t] = 0.f;
      }
      iq.floor[t] = -INFINITY;
    }
    __syncthreads();
    const long long slot0 = static_cast<long long>(it.range) * d.range_vectors;
    const long long left = d.n - slot0;
    const int size = static_cast<int>(left < d.range_vectors ? left : d.range_vectors);
    const ItemView v{d.codes, d.alpha, nullptr, slot0, size, d.nbg, d.luts, d.k, it.n_queries, d.cand_s, d.cand_i};
    if (ANY3 && d.bits == 3) {
      scan_item<true>(v, iq, smem);
    } else if (ANY24) {
      scan_item<false>(v, iq, smem);
    }
  }
}

__global__ void relabel_kernel(uint32_t* __restrict__ label, long long n, const uint32_t* __restrict__ remap) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) label[i] = remap[label[i]];
}

__global__ void gather_rows_kernel(const float* __restrict__ src, const uint32_t* __restrict__ rows, long long n,
                                   int dim, float* __restrict__ dst) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n * dim) return;
  const long long r = i / dim;
  dst[i] = src[static_cast<long long>(rows[r]) * dim + (i % dim)];
}

__global__ void take_columns_kernel(const float* __restrict__ src_s, const uint64_t* __restrict__ src_i,
                                    long long nq, int k_src, int k_out, unsigned long long n_valid,
                                    float* __restrict__ dst_s, uint64_t* __restrict__ dst_i) {
  const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= nq * k_out) return;
  const long long q = t / k_out;
  const int j = static_cast<int>(t % k_out);
  const uint64_t id = src_i[q * k_src + j];
  const bool ok = id < n_valid;
  dst_s[t] = ok ? src_s[q * k_src + j] : 0.f;
  dst_i[t] = ok ? id : 0ull;
}

}  // namespace

// ---------------------------------------------------------------------------
// Launchers
cudaError_t launch_take_columns(const float* src_s, const uint64_t* src_i, long long nq, int k_src, int k_out,
                                unsigned long long n_valid, float* dst_s, uint64_t* dst_i, cudaStream_t stream) {
  const long long total = nq * k_out;
  if (total == 0) return cudaSuccess;
  take_columns_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, stream>>>(src_s, src_i, nq, k_src, k_out,
                                                                                       n_valid, dst_s, dst_i);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
cudaError_t launch_normalize_rows(const float* x, long long n, int dim_in, int dim, float* out,
                                  cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  const long long threads = n * kWarp;
  normalize_rows_kernel<<<static_cast<unsigned>((threads + 255) / 256), 256, 0, stream>>>(x, n, dim_in, dim, out);
  return cudaGetLastError();
}

cudaError_t launch_gemm_nt(const float* A, long long m, const float* B, long long nb, int dim, float* C,
                           long long ldc, cudaStream_t stream) {
  if (m == 0 || nb == 0) return cudaSuccess;
  dim3 grid(static_cast<unsigned>((nb + kTcN - 1) / kTcN), static_cast<unsigned>((m + kTcM - 1) / kTcM));
  if (grid.y > 65535) return cudaErrorInvalidValue;
  gemm_nt_tc_kernel<<<grid, 256, 0, stream>>>(A, m, B, nb, dim, C, ldc);
  return cudaGetLastError();
}

cudaError_t launch_assign(const float* A, long long m, const float* B, long long nb, int dim, uint32_t* label,
                          float* best, cudaStream_t stream) {
  if (m == 0) return cudaSuccess;
  assign_kernel<<<static_cast<unsigned>((m + kTile - 1) / kTile), 256, 0, stream>>>(A, m, B, nb, dim, label, best);
  return cudaGetLastError();
}

cudaError_t launch_select_top(const float* S, long long rows, long long ld, int ncols, int p, float* out_s,
                              uint32_t* out_i, cudaStream_t stream) {
  if (rows == 0) return cudaSuccess;
  if (p < 1 || p > kMaxProbe) return cudaErrorInvalidValue;
  if (ncols <= kRadixMaxCols) {
    int n2 = kRadixThreads;
    while (n2 < p) n2 <<= 1;
    const size_t rsmem = static_cast<size_t>(n2) * 8 + static_cast<size_t>(ncols) * 4;
    auto kern = n2 == kRadixThreads       ? select_radix_kernel<1>
                : n2 == 2 * kRadixThreads ? select_radix_kernel<2>
                : n2 == 4 * kRadixThreads ? select_radix_kernel<4>
                                          : select_radix_kernel<8>;
    static_assert(kMaxProbe <= 8 * kRadixThreads, "p fits the largest sort");
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(rsmem));
    if (e != cudaSuccess) return e;
    kern<<<static_cast<unsigned>(rows), kRadixThreads, rsmem, stream>>>(S, ld, ncols, p, out_s, out_i);
    return cudaGetLastError();
  }
  const size_t smem = static_cast<size_t>(sel_cap(p)) * 8 + static_cast<size_t>(p) * 8;
  cudaError_t e = cudaFuncSetAttribute(select_top_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  select_top_kernel<<<static_cast<unsigned>(rows), kSelThreads, smem, stream>>>(S, ld, ncols, p, out_s, out_i);
  return cudaGetLastError();
}

cudaError_t launch_group_by_label(const uint32_t* label, long long n, int nb, uint32_t* counts,
                                  unsigned long long* starts, uint32_t* fill, uint32_t* members,
                                  cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(counts, 0, static_cast<size_t>(nb) * 4, stream);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(fill, 0, static_cast<size_t>(nb) * 4, stream);
  if (e != cudaSuccess) return e;
  if (n > 0) {
    label_hist_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, stream>>>(label, n, counts);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  prefix_kernel<<<1, 1024, 0, stream>>>(counts, nb, starts, 0, nullptr, nullptr);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (n > 0) {
    label_scatter_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, stream>>>(label, n, starts, fill,
                                                                                      members);
  }
  return cudaGetLastError();
}

cudaError_t launch_sort_groups(const unsigned long long* starts, int nb, int max_group, uint32_t* members,
                               cudaStream_t stream) {
  if (nb == 0) return cudaSuccess;
  if (max_group > 8192) return cudaErrorInvalidValue;
  int p = 2;
  while (p < max_group) p <<= 1;
  const size_t smem = static_cast<size_t>(p) * 4;
  cudaError_t e = cudaFuncSetAttribute(sort_groups_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  sort_groups_kernel<<<nb, 512, smem, stream>>>(starts, members);
  return cudaGetLastError();
}

cudaError_t launch_centroids(const float* X, int dim, const unsigned long long* starts, const uint32_t* members,
                             int nb, long long* acc, float* enc, float* route, cudaStream_t stream) {
  if (nb == 0) return cudaSuccess;
  if (dim > kCentMaxDim) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(acc, 0, static_cast<size_t>(nb) * dim * 8, stream);
  if (e != cudaSuccess) return e;
  centroid_sum_kernel<<<dim3(nb, kCentSplit), kCentThreads, 0, stream>>>(X, dim, starts, members, acc);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const long long threads = static_cast<long long>(nb) * kWarp;
  centroid_finish_kernel<<<static_cast<unsigned>((threads + 255) / 256), 256, 0, stream>>>(acc, dim, nb, starts,
                                                                                            enc, route);
  return cudaGetLastError();
}

cudaError_t launch_split(const float* X, int dim, const unsigned long long* starts, const uint32_t* members,
                         const uint32_t* groups, const uint32_t* new_label, int n_groups, const float* route,
                         uint32_t* label, bool force_bits, cudaStream_t stream) {
  if (n_groups == 0) return cudaSuccess;
  const size_t smem = static_cast<size_t>(dim) * (4 + 4 + 8 + 8);
  cudaError_t e = cudaFuncSetAttribute(split_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  split_kernel<<<n_groups, kSplitThreads, smem, stream>>>(X, dim, starts, members, groups, new_label, route, label,
                                                          force_bits ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_build_residuals(const float* X, int dim, const unsigned long long* starts,
                                   const uint32_t* members, int nb, const unsigned long long* slot_start,
                                   const float* enc, long long n_slots, float* R, uint32_t* slot_ids,
                                   cudaStream_t stream) {
  (void)n_slots;
  if (nb == 0) return cudaSuccess;
  build_residuals_kernel<<<nb, 256, 0, stream>>>(X, dim, starts, members, slot_start, enc, R, slot_ids);
  return cudaGetLastError();
}

cudaError_t launch_residual_rows(const float* X, long long n, int dim, const uint32_t* label, const float* enc,
                                 float* R, cudaStream_t stream) {
  const long long total = n * dim;
  if (total == 0) return cudaSuccess;
  residual_rows_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, stream>>>(X, n, dim, label, enc, R);
  return cudaGetLastError();
}

cudaError_t launch_relabel(uint32_t* label, long long n, const uint32_t* remap, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  relabel_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, stream>>>(label, n, remap);
  return cudaGetLastError();
}

cudaError_t launch_gather_rows(const float* src, const uint32_t* rows, long long n_rows, int dim, float* dst,
                               cudaStream_t stream) {
  const long long total = n_rows * dim;
  if (total == 0) return cudaSuccess;
  gather_rows_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, stream>>>(src, rows, n_rows, dim, dst);
  return cudaGetLastError();
}

long long max_items(long long nq, int max_probe, int nb) {
  return (nq * max_probe + kItemQueries - 1) / kItemQueries + nb;
}

cudaError_t launch_build_pairs(const PairArgs& a, cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(a.counts, 0, static_cast<size_t>(a.nb) * 4, stream);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(a.fill, 0, static_cast<size_t>(a.nb) * 4, stream);
  if (e != cudaSuccess) return e;
  const long long total = a.nq * a.max_probe;
  if (total > 0) {
    pair_count_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, stream>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  prefix_kernel<<<1, 1024, 0, stream>>>(a.counts, a.nb, a.pair_start, kItemQueries, a.item_start, a.n_items);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (total > 0) {
    pair_scatter_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, stream>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    pair_offset_gather_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, stream>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  item_build_kernel<<<static_cast<unsigned>((a.nb + 255) / 256), 256, 0, stream>>>(a);
  return cudaGetLastError();
}

// floor[q] = the k-th largest admitted score (above -inf, not NaN) among the
// first count[q] entries of query q's candidate region, -inf when it has fewer
// than k: the k-th score of the merged top k of those candidates (ties do not
// change that value), found without sorting by a radix select over
// order-preserving 32-bit keys, 8 bits per pass, one CTA of 256 threads per
// query. The region is L2-resident (just written by the scan); each pass
// re-reads it.
__global__ void __launch_bounds__(256) kth_floor_kernel(const float* __restrict__ cand, long long stride,
                                                        const uint32_t* __restrict__ count, int k,
                                                        float* __restrict__ floor) {
  __shared__ uint32_t hist[256];
  __shared__ uint32_t s_digit, s_need, s_total;
  const long long q = blockIdx.x;
  const long long n = count[q];
  const float* cs = cand + q * stride;
  uint32_t prefix = 0, mask = 0, need = static_cast<uint32_t>(k);
  for (int shift = 24; shift >= 0; shift -= 8) {
    hist[threadIdx.x] = 0u;
    __syncthreads();
    for (long long i = threadIdx.x; i < n; i += 256) {
      const float v = cs[i];
      if (v > -INFINITY) {
        const uint32_t u = __float_as_uint(v);
        const uint32_t key = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
        if ((key & mask) == prefix) atomicAdd(&hist[(key >> shift) & 255u], 1u);
      }
    }
    __syncthreads();
    if (threadIdx.x < kWarp) {
      // lane l holds digits 255 - 8l down to 248 - 8l; counts from the top
      const int lane = threadIdx.x;
      uint32_t c[8], sum = 0;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        c[j] = hist[255 - 8 * lane - j];
        sum += c[j];
      }
      uint32_t incl = sum;
#pragma unroll
      for (int o = 1; o < kWarp; o <<= 1) {
        const uint32_t t = __shfl_up_sync(full_mask(), incl, o);
        if (lane >= o) incl += t;
      }
      const uint32_t excl = incl - sum;
      if (shift == 24 && lane == kWarp - 1) s_total = incl;
      if (excl < need && need <= incl) {
        uint32_t above = excl;
        int d = 255 - 8 * lane;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          if (above + c[j] >= need) {
            d = 255 - 8 * lane - j;
            break;
          }
          above += c[j];
        }
        s_digit = static_cast<uint32_t>(d);
        s_need = need - above;
      }
    }
    __syncthreads();
    if (s_total < static_cast<uint32_t>(k)) {  // fewer than k admitted candidates
      if (threadIdx.x == 0) floor[q] = -INFINITY;
      return;
    }
    prefix |= s_digit << shift;
    mask |= 255u << shift;
    need = s_need;
    __syncthreads();  // everyone has read s_digit / s_need before the next pass
  }
  if (threadIdx.x == 0) floor[q] = __uint_as_float((prefix & 0x80000000u) ? (prefix & 0x7fffffffu) : ~prefix);
}

cudaError_t launch_kth_floor(const float* cand, long long stride, const uint32_t* count, long long nq, int k,
                             float* floor, cudaStream_t stream) {
  if (nq <= 0) return cudaSuccess;
  if (k < 1) return cudaErrorInvalidValue;
  kth_floor_kernel<<<static_cast<unsigned>(nq), 256, 0, stream>>>(cand, stride, count, k, floor);
  return cudaGetLastError();
}

size_t multi_scan_smem_bytes(int max_nbg, int max_k) {
  const int chunk = max_nbg < kFlushGroups ? max_nbg : kFlushGroups;
  const int kmax = kmax_of(max_k);
  return static_cast<size_t>(kItemQueries) * chunk * 32 +
         static_cast<size_t>(kBsWarps) * (static_cast<size_t>(4) * kmax * 8 + kBsBuf * 8);
}

int multi_scan_ctas_per_sm(size_t smem_bytes, bool any3) {
  int blocks = 0;
  auto kern = any3 ? multi_scan_kernel<true, true> : multi_scan_kernel<false, true>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem_bytes)) !=
      cudaSuccess) {
    return 0;
  }
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, kBsWarps * 32, smem_bytes) != cudaSuccess) {
    return 0;
  }
  return blocks;
}

cudaError_t launch_multi_scan(const MultiScanArgs& a, int ctas, size_t smem_bytes, bool any3, bool any24,
                              cudaStream_t stream) {
  if (a.n_items <= 0 || ctas <= 0) return cudaSuccess;
  auto kern = any3 ? (any24 ? multi_scan_kernel<true, true> : multi_scan_kernel<true, false>)
                   : multi_scan_kernel<false, true>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem_bytes));
  if (e != cudaSuccess) return e;
  kern<<<ctas, kBsWarps * 32, smem_bytes, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_bucket_scan(const BucketScanArgs& a, long long grid, cudaStream_t stream) {
  if (grid <= 0) return cudaSuccess;
  if (a.k < 1 || a.k > kMaxK || a.next_item == nullptr) return cudaErrorInvalidValue;
  const int chunk = a.nbg < kFlushGroups ? a.nbg : kFlushGroups;
  const int kmax = kmax_of(a.k);
  const size_t smem =
      static_cast<size_t>(kItemQueries) * chunk * 32 +
      static_cast<size_t>(kBsWarps) * (static_cast<size_t>(kBsQueriesPerWarp) * kmax * 8 + kBsBuf * 8);
  // Whole rings when nbg is a multiple of the ring (no bounds checks).
  const bool whole = a.nbg % kBsPrefetch == 0;
  auto kern = a.bits == 3 ? (whole ? bucket_scan_kernel<true, true> : bucket_scan_kernel<true, false>)
                          : (whole ? bucket_scan_kernel<false, true> : bucket_scan_kernel<false, false>);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  // Resident CTAs of this shape, cached per thread (device, variant, size).
  struct Resident {
    int device = -1;
    size_t smem = 0;
    const void* kern = nullptr;
    int ctas = 0;
  };
  static thread_local Resident cache[4];
  int device = 0;
  if ((e = cudaGetDevice(&device)) != cudaSuccess) return e;
  Resident* hit = nullptr;
  for (Resident& r : cache) {
    if (r.device == device && r.smem == smem && r.kern == reinterpret_cast<const void*>(kern)) hit = &r;
  }
  if (hit == nullptr) {
    int sms = 0, per_sm = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBsWarps * 32, smem)) != cudaSuccess) {
      return e;
    }
    for (int i = 3; i > 0; --i) cache[i] = cache[i - 1];
    cache[0] = Resident{device, smem, reinterpret_cast<const void*>(kern), std::max(1, per_sm) * sms};
    hit = &cache[0];
  }
  if ((e = cudaMemsetAsync(a.next_item, 0, sizeof(unsigned long long), stream)) != cudaSuccess) return e;
  const long long ctas = std::min<long long>(grid, hit->ctas);
  kern<<<static_cast<unsigned>(ctas), kBsWarps * 32, smem, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace vcb
