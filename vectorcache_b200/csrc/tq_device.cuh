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

// The lookups of one pair of byte groups (codes ca = group g, cb = group g + 1,
// 8 vectors of a lane) for Q queries, added into acc. The LUT halves of query
// q start at lg + q * q_stride: [F(g), S(g), F(g+1), S(g+1)], F the 16 entries
// of the high nibble (first half of the group's codes), S of the low nibble.
// The second-half lookups of both groups add into one byte per vector
// (<= 2 * 127), the first-half lookups into another; one prmt interleaves the
// two bytes of each vector so a single dp4a adds both. Measured and rejected
// (bit-exact, slower or equal): the selector shifts on the FMA pipe as mul.hi
// (1M x 1536 one query 0.187 -> 0.191 ms), every byte-sum addition as a
// multiply-add (-> 0.195 ms), the last addition of each four-lookup sum as a
// multiply-add with four queries per CTA (10k queries 870.0 -> 876.0 ms with
// the unchecked 4-group ring, 853.6 vs 853.3 ms with the 8-group ring).
// DIRECT: vectors 0..3 add their two bytes with two dp4a instead of the
// interleave prmt (see below).
template <int Q, bool NIBBLE8, bool DIRECT = (Q >= 4 && !NIBBLE8)>
__device__ __forceinline__ void lookup_group_pair(uint2 ca, uint2 cb, const LutHalf* lg, int q_stride,
                                                  uint32_t (&acc)[Q][8]) {
  auto hi16 = [](uint32_t x) -> uint32_t { return x >> 16; };
  auto add2 = [](uint32_t x, uint32_t y) -> uint32_t { return x + y; };
  auto add4 = [](uint32_t x, uint32_t y, uint32_t z, uint32_t w) -> uint32_t { return x + y + z + w; };
  const uint32_t a0 = ca.x, a1 = ca.y, b0 = cb.x, b1 = cb.y;
  const uint32_t a0h = hi16(a0), a1h = hi16(a1), b0h = hi16(b0), b1h = hi16(b1);
  [[maybe_unused]] uint32_t ta0 = 0, ta1 = 0, tb0 = 0, tb1 = 0, ta0h = 0, ta1h = 0, tb0h = 0, tb1h = 0;
  if constexpr (!NIBBLE8) {
    ta0 = a0 ^ 0x88888888u;
    ta1 = a1 ^ 0x88888888u;
    tb0 = b0 ^ 0x88888888u;
    tb1 = b1 ^ 0x88888888u;
    ta0h = hi16(ta0);
    ta1h = hi16(ta1);
    tb0h = hi16(tb0);
    tb1h = hi16(tb1);
  }
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const LutHalf Fa = lg[q * q_stride];      // group g: entries 0..15 (high nibble)
    const LutHalf Sa = lg[q * q_stride + 1];  //          entries 16..31 (low nibble)
    const LutHalf Fb = lg[q * q_stride + 2];  // group g + 1
    const LutHalf Sb = lg[q * q_stride + 3];
    uint32_t lo0, hi0, lo1, hi1;
    if constexpr (NIBBLE8) {
      // 3-bit codes: every nibble is < 8, entries 8..15 are never used.
      lo0 = add2(prmt(Sa.w[0], Sa.w[1], a0), prmt(Sb.w[0], Sb.w[1], b0));
      hi0 = add2(prmt(Fa.w[0], Fa.w[1], a0h), prmt(Fb.w[0], Fb.w[1], b0h));
      lo1 = add2(prmt(Sa.w[0], Sa.w[1], a1), prmt(Sb.w[0], Sb.w[1], b1));
      hi1 = add2(prmt(Fa.w[0], Fa.w[1], a1h), prmt(Fb.w[0], Fb.w[1], b1h));
    } else {
      lo0 = add4(prmt(Sa.w[0], Sa.w[1], a0), prmt(Sa.w[2], Sa.w[3], ta0), prmt(Sb.w[0], Sb.w[1], b0),
                 prmt(Sb.w[2], Sb.w[3], tb0));
      hi0 = add4(prmt(Fa.w[0], Fa.w[1], a0h), prmt(Fa.w[2], Fa.w[3], ta0h), prmt(Fb.w[0], Fb.w[1], b0h),
                 prmt(Fb.w[2], Fb.w[3], tb0h));
      lo1 = add4(prmt(Sa.w[0], Sa.w[1], a1), prmt(Sa.w[2], Sa.w[3], ta1), prmt(Sb.w[0], Sb.w[1], b1),
                 prmt(Sb.w[2], Sb.w[3], tb1));
      hi1 = add4(prmt(Fa.w[0], Fa.w[1], a1h), prmt(Fa.w[2], Fa.w[3], ta1h), prmt(Fb.w[0], Fb.w[1], b1h),
                 prmt(Fb.w[2], Fb.w[3], tb1h));
    }
    // [lo.b0, hi.b0, lo.b1, hi.b1] and [lo.b2, hi.b2, lo.b3, hi.b3]. With four
    // or more queries over 2- or 4-bit codes the prmt lookups keep the ALU pipe
    // busier than the FMA pipe (82 % against 40 %), so vectors 0..3 skip the
    // interleave and add their lo and hi bytes with two dp4a each (10k queries
    // x 1M x 1536: 853.3 -> 840.2 ms; all eight vectors this way: 878.3 ms).
    // The 3-bit lookups (one prmt per nibble) leave the ALU pipe room, and
    // there the extra dp4a only cost (the multi-index workload, whose largest
    // index is 3-bit: 103.6 -> 111.0 ms), as they did with k = 64 (one CTA of
    // shared-memory lists per SM: 1M x 1536 4-bit 10,678 -> 10,561 QPS).
    if constexpr (DIRECT) {
      acc[q][0] = __dp4a(hi0, 0x00000001u, __dp4a(lo0, 0x00000001u, acc[q][0]));
      acc[q][1] = __dp4a(hi0, 0x00000100u, __dp4a(lo0, 0x00000100u, acc[q][1]));
      acc[q][2] = __dp4a(hi0, 0x00010000u, __dp4a(lo0, 0x00010000u, acc[q][2]));
      acc[q][3] = __dp4a(hi0, 0x01000000u, __dp4a(lo0, 0x01000000u, acc[q][3]));
    } else {
      const uint32_t m00 = prmt(lo0, hi0, 0x5140u), m01 = prmt(lo0, hi0, 0x7362u);
      acc[q][0] = __dp4a(m00, 0x00000101u, acc[q][0]);
      acc[q][1] = __dp4a(m00, 0x01010000u, acc[q][1]);
      acc[q][2] = __dp4a(m01, 0x00000101u, acc[q][2]);
      acc[q][3] = __dp4a(m01, 0x01010000u, acc[q][3]);
    }
    const uint32_t m10 = prmt(lo1, hi1, 0x5140u), m11 = prmt(lo1, hi1, 0x7362u);
    acc[q][4] = __dp4a(m10, 0x00000101u, acc[q][4]);
    acc[q][5] = __dp4a(m10, 0x01010000u, acc[q][5]);
    acc[q][6] = __dp4a(m11, 0x00000101u, acc[q][6]);
    acc[q][7] = __dp4a(m11, 0x01010000u, acc[q][7]);
  }
}

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
