// Device-side building blocks shared by the TurboQuant kernels (sm_100a).
//
// Arithmetic contract: every floating-point step that decides a code, an
// alpha, a LUT byte or a score is written with an explicitly rounded intrinsic
// (__fadd_rn, __fmul_rn, __fmaf_rn, __fdiv_rn, __dadd_rn, ...). The library is
// also compiled with -fmad=false, so nothing is contracted behind our back.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace vcb {

constexpr int kWarp = 32;
constexpr float kMinInputNorm = 1e-10f;   // constants.hpp kMinInputNorm
constexpr double kDegenerateInner = 1e-12;  // constants.hpp kDegenerateInnerEps

__device__ __forceinline__ unsigned full_mask() { return 0xffffffffu; }

// Asynchronous 16-byte global -> shared copies (cp.async, L1 bypassed): the
// bytes in flight occupy shared memory, not registers. A thread's copies are
// complete after cp_async_wait<N> (at most N of its commit groups pending);
// other threads see them after a barrier (__syncwarp / __syncthreads).
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { cp_async_wait<0>(); }

// Sum of squares with 8 interleaved chains (chain j % 8, in index order, one
// fused multiply-add per step) combined as ((c0+c1)+(c2+c3))+((c4+c5)+(c6+c7))
// (encode.cpp:16-26). Lane l of the warp owns chain l % 8 of row l / 8, so one
// warp handles four rows; every lane returns the norm of its own row.
__device__ __forceinline__ float warp_norm4(const float* __restrict__ row, int dim, bool valid,
                                            int lane) {
  const int c = lane & 7;
  float s = 0.f;
  if (valid) {
    const int steps = dim >> 3;
    int t = 0;
    for (; t + 8 <= steps; t += 8) {
      float v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = __ldg(row + 8 * (t + u) + c);
#pragma unroll
      for (int u = 0; u < 8; ++u) s = __fmaf_rn(v[u], v[u], s);
    }
    for (; t < steps; ++t) {
      const float v = __ldg(row + 8 * t + c);
      s = __fmaf_rn(v, v, s);
    }
  }
  s = __fadd_rn(s, __shfl_xor_sync(full_mask(), s, 1));
  s = __fadd_rn(s, __shfl_xor_sync(full_mask(), s, 2));
  s = __fadd_rn(s, __shfl_xor_sync(full_mask(), s, 4));
  return __fsqrt_rn(s);
}

// Rotation of one row held by a warp: element i lives in lane i % 32,
// register i / 32. y[i] = (x[perm[i]] * inv) * sign[i], then a Walsh-Hadamard
// butterfly network on each block of B coordinates with strides 1, 2, 4, ...
// (a + b, a - b per pair, same order of stages as rotation.cpp:38-85), then
// y *= 1/sqrt(B). perm_sign packs the source index in bits 0..30 and the sign
// in bit 31. Strides below 32 exchange lanes with shuffles; larger strides pair
// registers of the same lane.
template <int R>
__device__ __forceinline__ void warp_rotate(const float* __restrict__ xs,
                                            const uint32_t* __restrict__ perm_sign, int dim,
                                            int block, float inv, float inv_sqrt_block,
                                            float (&y)[R], int lane) {
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int i = lane + kWarp * r;
    float v = 0.f;
    if (i < dim) {
      const uint32_t e = perm_sign[i];
      v = __fmul_rn(xs[e & 0x7fffffffu], inv);
      if (e >> 31) v = -v;
    }
    y[r] = v;
  }
#pragma unroll
  for (int len = 1; len < kWarp; len <<= 1) {
    if (len < block) {
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const float o = __shfl_xor_sync(full_mask(), y[r], len);
        y[r] = (lane & len) ? __fsub_rn(o, y[r]) : __fadd_rn(y[r], o);
      }
    }
  }
#pragma unroll
  for (int s = 1; s < R; s <<= 1) {
    if (kWarp * s < block) {
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if ((r & s) == 0 && (r | s) < R) {
          const float a = y[r], b = y[r | s];
          y[r] = __fadd_rn(a, b);
          y[r | s] = __fsub_rn(a, b);
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r) y[r] = __fmul_rn(y[r], inv_sqrt_block);
}

// Count of boundaries strictly below v (encode.cpp:126-140). The boundaries
// are strictly increasing, so a branch-free binary search gives the same count.
__device__ __forceinline__ unsigned quantize_code(float v, const float* __restrict__ bnd, int bits) {
  unsigned idx = 0;
  for (int step = 1 << (bits - 1); step > 0; step >>= 1) {
    if (v > bnd[idx + step - 1]) idx += step;
  }
  return idx;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = __dadd_rn(v, __shfl_xor_sync(full_mask(), v, o));
  return v;
}

__device__ __forceinline__ float warp_max_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(full_mask(), v, o));
  return v;
}

// Decides float(S) for a double S that the reference accumulates sequentially
// (recursive summation, one rounding per term) from an estimate E of the same
// exact sum computed in a different order. |S - exact| <= gamma_m * A and
// |E - exact| <= gamma_m' * A, where A bounds the sum of |terms|; `steps` is an
// upper bound on m + m'. If every double in [E - bound, E + bound] rounds to the
// same float, that float is float(S). Returns false when the interval straddles
// a float rounding boundary (or the threshold `gate`), in which case the caller
// replays the sequential sum exactly.
__device__ __forceinline__ bool decide_float_of_sum(double E, double A, int steps, double gate,
                                                    bool* above_gate, float* out) {
  const double bound = __dmul_ru(__dmul_ru(static_cast<double>(steps + 8), 0x1p-52), A);
  const double lo = __dadd_rd(E, -bound);
  const double hi = __dadd_ru(E, bound);
  if (lo > gate) {
    *above_gate = true;
  } else if (hi <= gate) {
    *above_gate = false;
  } else {
    return false;
  }
  const float flo = __double2float_rn(lo);
  const float fhi = __double2float_rn(hi);
  if (__float_as_uint(flo) != __float_as_uint(fhi)) return false;
  *out = flo;
  return true;
}

// prmt.b32 in its default mode: each selector nibble picks one of eight source
// bytes (bits 0..2); when bit 3 is set the byte's sign bit is replicated
// instead. LUT bytes are <= 127, so a selector nibble >= 8 yields 0x00.
__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
  uint32_t d;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(sel));
  return d;
}

// Total order of the reference's top-k (topk_heap.hpp:19-22): higher score
// first; equal scores by lower id.
__device__ __forceinline__ bool better(float sa, uint32_t ia, float sb, uint32_t ib) {
  return (sa > sb) || (sa == sb && ia < ib);
}


// 16 bytes of a query LUT (one nibble's 16 entries of one byte group).
struct __align__(16) LutHalf {
  uint32_t w[4];
};

// Warp-cooperative bitonic sort of p (a power of two) entries in
// shared memory, best first under `better`.
__device__ __forceinline__ void warp_sort_best_first(float* s, uint32_t* id, int p, int lane) {
  for (int size = 2; size <= p; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int t = lane; t < (p >> 1); t += kWarp) {
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
      __syncwarp();
    }
  }
}

// k-th largest of the 32 lane values (k <= 32), by a shuffle bitonic sort.
__device__ __forceinline__ float warp_kth_largest(float v, int k, int lane) {
#pragma unroll
  for (int size = 2; size <= kWarp; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      const float o = __shfl_xor_sync(full_mask(), v, stride);
      const bool lower = (lane & stride) == 0;
      const bool desc = (lane & size) == 0;  // final pass: descending everywhere
      // keep the larger value in the lower lane of a descending block
      const bool take_max = (lower == desc);
      v = take_max ? fmaxf(v, o) : fminf(v, o);
    }
  }
  return __shfl_sync(full_mask(), v, k - 1);
}

}  // namespace vcb
