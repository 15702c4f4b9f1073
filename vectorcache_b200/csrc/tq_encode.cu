// Encode path on sm_100a: norm -> rotation -> (TQ+) -> Lloyd-Max code ->
// alpha -> row-major codes, then the relayout into the scan layout.
//
// Follows the reference's encode (src/encode/encode.cpp:112-231, :294-307) and
// pack (src/pack/pack.cpp:70-131) arithmetic bit for bit; see tq_device.cuh for
// the rounding contract.
#include <type_traits>

#include "tq_host_math.h"
#include "tq_kernels.h"
#include "tq_device.cuh"

namespace vcb {
namespace {

// Encodes four rows per warp iteration (the norm phase uses all 32 lanes as
// 4 rows x 8 chains); the rotation/quantize phase then walks the four rows
// with the whole warp. Shared memory: perm|sign table, TQ+ tables, one staged
// input row per warp.
template <int R>
__global__ void __launch_bounds__(256) encode_rows_kernel(EncodeArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int dim = a.dim;
  uint32_t* s_perm = reinterpret_cast<uint32_t*>(smem);
  float* s_shift = reinterpret_cast<float*>(s_perm + dim);
  float* s_scale = s_shift + (a.tqplus ? dim : 0);
  float* s_inv_scale = s_scale + (a.tqplus ? dim : 0);
  float* s_bnd = s_inv_scale + (a.tqplus ? dim : 0);
  float* s_cen = s_bnd + 16;
  float* s_rows = s_cen + 16;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* xrow = s_rows + static_cast<size_t>(warp) * dim;

  for (int i = threadIdx.x; i < dim; i += blockDim.x) {
    s_perm[i] = a.perm_sign[i];
    if (a.tqplus) {
      s_shift[i] = a.shift[i];
      s_scale[i] = a.scale[i];
      s_inv_scale[i] = a.inv_scale[i];
    }
  }
  if (threadIdx.x < 16) {
    s_bnd[threadIdx.x] = threadIdx.x < 15 ? a.boundaries[threadIdx.x] : 0.f;
    s_cen[threadIdx.x] = a.centroids[threadIdx.x];
  }
  __syncthreads();

  const int cpb = 8 / a.bits;                 // codes per byte group
  const int field = (a.bits == 3) ? 4 : a.bits;  // bits per code inside the byte
  const int lanes_per_word = 4 * cpb;         // lanes whose codes fill one u32 of codes_flat
  const int nc = (dim + 3) / 4;               // terms per inner-product chain

  const long long warps_total = static_cast<long long>(gridDim.x) * (blockDim.x >> 5);
  for (long long quad = static_cast<long long>(blockIdx.x) * (blockDim.x >> 5) + warp;
       quad * 4 < a.n; quad += warps_total) {
    const long long v_lane = quad * 4 + (lane >> 3);
    const bool lane_valid = v_lane < a.n;
    const float nrm_lane =
        warp_norm4(a.x + (lane_valid ? v_lane : 0) * static_cast<long long>(dim), dim, lane_valid, lane);

    for (int j = 0; j < 4; ++j) {
      const long long v = quad * 4 + j;
      const float nrm = __shfl_sync(full_mask(), nrm_lane, 8 * j);
      if (v >= a.n) break;
      const float* src = a.x + v * static_cast<long long>(dim);
      __syncwarp();
      for (int i = lane * 4; i < dim; i += kWarp * 4) {
        *reinterpret_cast<float4*>(xrow + i) = __ldg(reinterpret_cast<const float4*>(src + i));
      }
      __syncwarp();
      const float inv = (nrm > kMinInputNorm) ? __fdiv_rn(1.f, nrm) : 0.f;
      float y[R];
      warp_rotate<R>(xrow, s_perm, dim, a.block, inv, a.inv_sqrt_block, y, lane);

      // Quantize, inner-product estimate, codes_flat words.
      double est = 0.0, mag = 0.0;
      uint8_t* flat_row = a.out_flat + v * static_cast<long long>(a.flat_stride);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = lane + kWarp * r;
        unsigned code = 0;
        if (i < dim) {
          double term;
          if (a.tqplus) {
            const float c = __fmul_rn(__fadd_rn(y[r], s_shift[i]), s_scale[i]);
            code = quantize_code(c, s_bnd, a.bits);
            const double back = __dsub_rn(
                __dmul_rn(static_cast<double>(s_cen[code]), static_cast<double>(s_inv_scale[i])),
                static_cast<double>(s_shift[i]));
            term = __dmul_rn(static_cast<double>(y[r]), back);
          } else {
            code = quantize_code(y[r], s_bnd, a.bits);
            term = __dmul_rn(static_cast<double>(y[r]), static_cast<double>(s_cen[code]));
          }
          est = __dadd_rn(est, term);
          mag = __dadd_rn(mag, fabs(term));
        }
        // Row-major byte groups: codes_per_byte codes per byte, first code in
        // the high bits (pack.cpp:70-131). OR-reduce over the lanes of a word.
        const int e = lane % lanes_per_word;
        uint32_t word = code << (8 * (e / cpb) + field * (cpb - 1 - e % cpb));
        for (int o = 1; o < lanes_per_word; o <<= 1) word |= __shfl_xor_sync(full_mask(), word, o);
        const int byte_off = (kWarp * r) / cpb + 4 * (lane / lanes_per_word);
        if (e == 0 && kWarp * r + lane < dim) {
          *reinterpret_cast<uint32_t*>(flat_row + byte_off) = word;
        }
      }
      est = warp_sum_d(est);
      mag = warp_sum_d(mag);

      float alpha = 0.f;
      bool above = false;
      float inner_f = 0.f;
      if (decide_float_of_sum(est, mag, nc + 2 + R + 6, kDegenerateInner, &above, &inner_f)) {
        alpha = above ? __fdiv_rn(nrm, inner_f) : 0.f;
      } else {
        // Exact replay of the reference's four sequential double chains
        // (chain i % 4, one fused multiply-add per term; encode.cpp:117-156).
        // The staged input row is no longer needed: park y there.
        __syncwarp();
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int i = lane + kWarp * r;
          if (i < dim) xrow[i] = y[r];
        }
        __syncwarp();
        double ch = 0.0;
        if (lane < 4) {
#pragma unroll 1
          for (int i = lane; i < dim; i += 4) {
            const float yv = xrow[i];
            if (a.tqplus) {
              const float c = __fmul_rn(__fadd_rn(yv, s_shift[i]), s_scale[i]);
              const unsigned code = quantize_code(c, s_bnd, a.bits);
              const double back = __dsub_rn(__dmul_rn(static_cast<double>(s_cen[code]),
                                                      static_cast<double>(s_inv_scale[i])),
                                            static_cast<double>(s_shift[i]));
              ch = __fma_rn(static_cast<double>(yv), back, ch);
            } else {
              const unsigned code = quantize_code(yv, s_bnd, a.bits);
              ch = __fma_rn(static_cast<double>(yv), static_cast<double>(s_cen[code]), ch);
            }
          }
        }
        const double c0 = __shfl_sync(full_mask(), ch, 0), c1 = __shfl_sync(full_mask(), ch, 1);
        const double c2 = __shfl_sync(full_mask(), ch, 2), c3 = __shfl_sync(full_mask(), ch, 3);
        const double inner = __dadd_rn(__dadd_rn(c0, c1), __dadd_rn(c2, c3));
        alpha = inner > kDegenerateInner ? __fdiv_rn(nrm, __double2float_rn(inner)) : 0.f;
        if (lane == 0 && a.replay_count) atomicAdd(a.replay_count, 1ull);
      }
      if (lane == 0) a.out_alpha[v] = alpha;
    }
  }
}

// codes_flat rows (stride flat_stride) -> scan layout words. One CTA converts
// 128 consecutive vectors x 32 byte groups through shared memory so both the
// reads and the word writes are coalesced. Vectors below `keep_below` belong to
// an earlier add() and keep their existing nibbles.
__global__ void __launch_bounds__(256) relayout_kernel(RelayoutArgs a) {
  __shared__ uint32_t tile[128][9];  // 128 vectors x 32 bytes (+1 word pad)
  const long long v0 = a.first_vector + static_cast<long long>(blockIdx.x) * 128;
  const int g0 = blockIdx.y * 32;
  for (int t = threadIdx.x; t < 128 * 8; t += blockDim.x) {
    const int vr = t >> 3, wcol = t & 7;
    const long long v = v0 + vr;
    uint32_t w = 0;
    if (v >= a.src_first && v < a.src_first + a.src_n) {
      w = *reinterpret_cast<const uint32_t*>(a.flat + (v - a.src_first) * a.flat_stride + g0 + 4 * wcol);
    }
    tile[vr][wcol] = w;
  }
  __syncthreads();
  const int q = threadIdx.x & 31;  // quad inside the 128-vector strip
  const int cpb = 8 / a.bits;
  for (int gi = threadIdx.x >> 5; gi < 32; gi += blockDim.x >> 5) {
    const int g = g0 + gi;
    if (g >= a.nbg) break;
    uint32_t word = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const uint32_t byte = (tile[4 * q + j][gi >> 2] >> (8 * (gi & 3))) & 0xffu;
      word |= (byte & 0xfu) << (4 * j);          // second half of the group's codes
      word |= (byte >> 4) << (16 + 4 * j);       // first half
    }
    const long long vq = v0 + 4 * q;  // first vector of this quad
    if (vq >= a.n_total) continue;
    const long long tile_idx = vq / kTileVectors;
    const int wq = static_cast<int>((vq % kTileVectors) / 4);
    uint32_t* dst = a.codes + (tile_idx * a.nbg + g) * kTileWords + wq;
    if (vq < a.keep_below) {
      // Merge with the nibbles of vectors that were encoded by an earlier add().
      uint32_t keep = 0;
      for (int j = 0; j < 4; ++j) {
        if (vq + j < a.keep_below) keep |= (0xfu << (4 * j)) | (0xfu << (16 + 4 * j));
      }
      word = (*dst & keep) | (word & ~keep);
    }
    *dst = word;
    (void)cpb;
  }
}

// Scan layout -> codes_flat rows (introspection and parity export).
__global__ void export_flat_kernel(const uint32_t* __restrict__ codes, long long n, int nbg,
                                   uint8_t* __restrict__ out) {
  const long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= n * nbg) return;
  const long long v = idx / nbg;
  const int g = static_cast<int>(idx % nbg);
  const long long tile = v / kTileVectors;
  const int wq = static_cast<int>((v % kTileVectors) / 4), j = static_cast<int>(v & 3);
  const uint32_t w = codes[(tile * nbg + g) * kTileWords + wq];
  const uint32_t lo = (w >> (4 * j)) & 0xfu, hi = (w >> (16 + 4 * j)) & 0xfu;
  out[idx] = static_cast<uint8_t>((hi << 4) | lo);
}

// Rotated (and normalized) rows, transposed to dim x n, for the TQ+ fit.
template <int R>
__global__ void __launch_bounds__(256) rotate_rows_t_kernel(RotateArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int dim = a.dim;
  uint32_t* s_perm = reinterpret_cast<uint32_t*>(smem);
  float* s_rows = reinterpret_cast<float*>(s_perm + dim);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* xrow = s_rows + static_cast<size_t>(warp) * dim;
  for (int i = threadIdx.x; i < dim; i += blockDim.x) s_perm[i] = a.perm_sign[i];
  __syncthreads();
  const long long warps_total = static_cast<long long>(gridDim.x) * (blockDim.x >> 5);
  for (long long quad = static_cast<long long>(blockIdx.x) * (blockDim.x >> 5) + warp;
       quad * 4 < a.n; quad += warps_total) {
    const long long v_lane = quad * 4 + (lane >> 3);
    const bool lane_valid = v_lane < a.n;
    const float nrm_lane =
        warp_norm4(a.x + (lane_valid ? v_lane : 0) * static_cast<long long>(dim), dim, lane_valid, lane);
    for (int j = 0; j < 4; ++j) {
      const long long v = quad * 4 + j;
      const float nrm = __shfl_sync(full_mask(), nrm_lane, 8 * j);
      if (v >= a.n) break;
      const float* src = a.x + v * static_cast<long long>(dim);
      __syncwarp();
      for (int i = lane * 4; i < dim; i += kWarp * 4) {
        *reinterpret_cast<float4*>(xrow + i) = __ldg(reinterpret_cast<const float4*>(src + i));
      }
      __syncwarp();
      const float inv = (nrm > kMinInputNorm) ? __fdiv_rn(1.f, nrm) : 0.f;
      float y[R];
      warp_rotate<R>(xrow, s_perm, dim, a.block, inv, a.inv_sqrt_block, y, lane);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = lane + kWarp * r;
        if (i < dim) a.out_t[static_cast<long long>(i) * a.n + v] = y[r];
      }
    }
  }
}

// Per-dimension order statistics of the rotated sample (radix select on the
// f32 total-order key, encode.cpp:60-69, :262-276). One CTA per dimension
// selects the lo-th and hi-th smallest keys.
__device__ __forceinline__ uint32_t f32_order_key(float f) {
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__device__ __forceinline__ float f32_from_order_key(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

__global__ void __launch_bounds__(256) order_stats_kernel(const float* __restrict__ yt, long long n,
                                                          long long lo_rank, long long hi_rank,
                                                          float* __restrict__ q_lo,
                                                          float* __restrict__ q_hi) {
  __shared__ unsigned int hist[2][256];
  __shared__ uint32_t prefix[2];
  __shared__ long long rank[2];
  const float* col = yt + static_cast<long long>(blockIdx.x) * n;
  if (threadIdx.x < 2) {
    prefix[threadIdx.x] = 0;
    rank[threadIdx.x] = threadIdx.x == 0 ? lo_rank : hi_rank;
  }
  for (int shift = 24; shift >= 0; shift -= 8) {
    for (int b = threadIdx.x; b < 512; b += blockDim.x) hist[b >> 8][b & 255] = 0;
    __syncthreads();
    const uint32_t hmask = (shift == 24) ? 0u : (0xffffffffu << (shift + 8));
    const uint32_t p0 = prefix[0], p1 = prefix[1];
    for (long long i = threadIdx.x; i < n; i += blockDim.x) {
      const uint32_t k = f32_order_key(col[i]);
      const uint32_t d = (k >> shift) & 255u;
      if ((k & hmask) == (p0 & hmask)) atomicAdd(&hist[0][d], 1u);
      if ((k & hmask) == (p1 & hmask)) atomicAdd(&hist[1][d], 1u);
    }
    __syncthreads();
    if (threadIdx.x < 2) {
      const int s = threadIdx.x;
      long long r = rank[s];
      uint32_t d = 0;
      for (; d < 256; ++d) {
        if (r < static_cast<long long>(hist[s][d])) break;
        r -= hist[s][d];
      }
      rank[s] = r;
      prefix[s] |= d << shift;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    q_lo[blockIdx.x] = f32_from_order_key(prefix[0]);
    q_hi[blockIdx.x] = f32_from_order_key(prefix[1]);
  }
}

// ---------------------------------------------------------------------------
// Pipelined encode (dims whose register layout below applies; others use
// encode_rows_kernel). Persistent CTAs, one per SM; each warp encodes ROWS
// rows per iteration:
//   * the rows arrive in shared memory by cp.async (16-byte copies), issued for
//     the warp's next rows as soon as each row's gather has read its slot, so
//     the loads of the next rows overlap the arithmetic of the current ones;
//   * the norm: lane 8j + c runs chain c of row j (the reference's 8-chain
//     order) out of shared memory;
//   * the rotation: element i of the row lives in lane l, register r with
//     i = (r / E) * 32E + l * E + r % E, so butterfly strides below E pair
//     registers of one lane, strides E .. 16E pair lanes (one shuffle and one
//     fused multiply-add by +-1 per element, which rounds exactly like the
//     reference's a + b / a - b), larger strides pair register segments;
//   * a lane's E consecutive codes pack into whole codes_flat bytes in its own
//     registers (no cross-lane packing) and leave as one 2-8 byte store.
// The per-element tables (source offset and sign of the permutation, TQ+
// shift/scale and the inv_scale of the inner-product estimate) are
// stored in the same (register, lane) order, so every table read is one
// conflict-free shared-memory access.

// Index of the row element held by (lane, register r).
template <int E>
__device__ __forceinline__ int pipe_elem(int r, int lane) {
  return (r / E) * (32 * E) + lane * E + (r % E);
}

struct PipeLayout {
  int stride;         // floats per row slot (>= dim + 1, == 8 mod 32)
  size_t off_bk, off_ss, off_cen, off_grid, off_src, off_bnd, off_rows, total;
};

__host__ __device__ inline PipeLayout pipe_layout(int dim, int r_regs, bool tqplus, int warps, int rows) {
  PipeLayout L;
  int pad = (8 - dim % 32 + 32) % 32;
  if (pad == 0) pad = 32;
  L.stride = dim + pad;
  const size_t slots = static_cast<size_t>(r_regs) * 32;
  size_t o = 0;
  L.off_bk = o;
  o += tqplus ? slots * 4 : 0;
  L.off_ss = o;
  o += tqplus ? slots * 8 : 0;
  L.off_cen = o;
  o += 16 * 8;  // 16 float centroids, padded to keep the grid 8-byte aligned
  L.off_grid = o;
  o += static_cast<size_t>(CodeGrid::kCells) * 8;
  L.off_src = o;
  o += slots * 4;
  L.off_bnd = o;
  o += 16 * 4;
  o = (o + 15) / 16 * 16;
  L.off_rows = o;
  o += static_cast<size_t>(warps) * rows * L.stride * 4;
  L.total = o;
  return L;
}

// Count of boundaries strictly below v, boundaries in shared memory, BITS levels.
template <int BITS>
__device__ __forceinline__ unsigned pipe_code(float v, const float* __restrict__ bnd) {
  unsigned idx = 0;
#pragma unroll
  for (int step = 1 << (BITS - 1); step > 0; step >>= 1) {
    if (v > bnd[idx + step - 1]) idx += step;
  }
  return idx;
}

// The code of v from the host-built grid (CodeGrid in tq_host_math.h): one
// fused multiply-add picks a cell holding at most one boundary, so the count
// of boundaries strictly below v is the cell's base plus one compare.
__device__ __forceinline__ unsigned grid_code(float v, const uint2* __restrict__ grid, float lo, float hi, float ga,
                                              float gk) {
  const float c = fminf(fmaxf(v, lo), hi);  // NaN -> lo: code 0, as v > b is false for every b
  const int cell = __float_as_int(__fmaf_rn(c, ga, gk)) - 0x4B400000;
  const uint2 e = grid[cell];
  return e.x + (c > __uint_as_float(e.y) ? 1u : 0u);
}

template <int R, int E, int BITS, int ROWS, int MAXW, bool TQ>
__global__ void __launch_bounds__(MAXW * 32, 1) encode_pipe_kernel(EncodeArgs a) {
  static_assert(R % E == 0, "segments of E registers");
  constexpr int SEG = R / E;
  constexpr int CPB = 8 / BITS;                 // codes per codes_flat byte
  constexpr int FIELD = BITS == 3 ? 4 : BITS;   // bits per code inside the byte
  constexpr int RUN_BYTES = E / CPB;            // bytes of one lane's E codes
  static_assert(RUN_BYTES == 1 || RUN_BYTES == 2 || RUN_BYTES == 4 || RUN_BYTES == 8, "run size");
  using Run = typename std::conditional<RUN_BYTES == 8, unsigned long long,
              typename std::conditional<RUN_BYTES == 4, uint32_t,
              typename std::conditional<RUN_BYTES == 2, uint16_t, uint8_t>::type>::type>::type;

  extern __shared__ __align__(16) unsigned char smem[];
  const int dim = a.dim;
  const int warps = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const PipeLayout L = pipe_layout(dim, R, a.tqplus, warps, ROWS);
  // TQ+: inv_scale as float (widened to double where the estimate needs it,
  // exactly; a 16-byte double table cost 3 more shared-memory wavefronts per
  // element), and {shift, scale}.
  float* s_bk = reinterpret_cast<float*>(smem + L.off_bk);
  float2* s_ss = reinterpret_cast<float2*>(smem + L.off_ss);     // {shift, scale} (TQ+)
  // Float centroids, widened to double where used (exact): a 16-float table is
  // one conflict-free wavefront per lookup, a 16-double table two.
  float* s_cen = reinterpret_cast<float*>(smem + L.off_cen);
  uint2* s_grid = reinterpret_cast<uint2*>(smem + L.off_grid);     // {base code, inner boundary bits}
  uint32_t* s_src = reinterpret_cast<uint32_t*>(smem + L.off_src);
  float* s_bnd = reinterpret_cast<float*>(smem + L.off_bnd);
  float* rows = reinterpret_cast<float*>(smem + L.off_rows) + static_cast<size_t>(warp) * ROWS * L.stride;

  // Tables in (register, lane) order. Elements past dim read the zero word at
  // column dim of every row slot and have zero TQ+ tables, so they add nothing.
  for (int t = threadIdx.x; t < R * 32; t += blockDim.x) {
    const int r = t / 32, l = t % 32;
    const int i = pipe_elem<E>(r, l);
    uint32_t src = static_cast<uint32_t>(dim) * 4u;
    float bk = 0.f;
    float2 ss = make_float2(0.f, 0.f);
    if (i < dim) {
      const uint32_t e = a.perm_sign[i];
      src = ((e & 0x7fffffffu) * 4u) | (e & 0x80000000u);
      if (a.tqplus) {
        bk = a.inv_scale[i];
        ss = make_float2(a.shift[i], a.scale[i]);
      }
    }
    s_src[t] = src;
    if (a.tqplus) {
      s_bk[t] = bk;
      s_ss[t] = ss;
    }
  }
  if (threadIdx.x < 16) {
    s_cen[threadIdx.x] = a.centroids[threadIdx.x];
    s_bnd[threadIdx.x] = threadIdx.x < 15 ? a.boundaries[threadIdx.x] : 0.f;
  }
  for (int j = threadIdx.x; j < CodeGrid::kCells; j += blockDim.x) s_grid[j] = a.grid[j];
  const float g_lo = a.grid_lo, g_hi = a.grid_hi, g_a = a.grid_a, g_k = a.grid_k;
  for (int j = lane; j < ROWS; j += 32) rows[j * L.stride + dim] = 0.f;

  const long long n_groups = (a.n + ROWS - 1) / ROWS;
  const long long g_step = static_cast<long long>(gridDim.x) * warps;
  const int chunks = dim / 4;  // 16-byte pieces of a row
  auto prefetch = [&](long long v, int j) {
    const float* src = a.x + v * static_cast<long long>(dim);
    float* dst = rows + j * L.stride;
    for (int c = lane; c < chunks; c += 32) cp_async16(dst + 4 * c, src + 4 * c);
  };
  long long grp = static_cast<long long>(blockIdx.x) * warps + warp;
  if (grp < n_groups) {
#pragma unroll
    for (int j = 0; j < ROWS; ++j) {
      if (grp * ROWS + j < a.n) prefetch(grp * ROWS + j, j);
    }
  }
  cp_async_commit();
  __syncthreads();

  constexpr bool tq = TQ;
  for (; grp < n_groups; grp += g_step) {
    cp_async_wait_all();
    __syncwarp();

    // Norms: lane 8j + c runs chain c of row j (encode.cpp:16-26).
    float nrm_lane;
    {
      const int j = min(lane >> 3, ROWS - 1), c = lane & 7;
      const float* xr = rows + j * L.stride + c;
      float s = 0.f;
      const int steps = dim >> 3;
      int t = 0;
      for (; t + 4 <= steps; t += 4) {
        const float v0 = xr[8 * t], v1 = xr[8 * t + 8], v2 = xr[8 * t + 16], v3 = xr[8 * t + 24];
        s = __fmaf_rn(v0, v0, s);
        s = __fmaf_rn(v1, v1, s);
        s = __fmaf_rn(v2, v2, s);
        s = __fmaf_rn(v3, v3, s);
      }
      for (; t < steps; ++t) {
        const float v = xr[8 * t];
        s = __fmaf_rn(v, v, s);
      }
      s = __fadd_rn(s, __shfl_xor_sync(full_mask(), s, 1));
      s = __fadd_rn(s, __shfl_xor_sync(full_mask(), s, 2));
      s = __fadd_rn(s, __shfl_xor_sync(full_mask(), s, 4));
      nrm_lane = __fsqrt_rn(s);
    }

    const long long next = grp + g_step;
#pragma unroll 1
    for (int j = 0; j < ROWS; ++j) {
      const long long v = grp * ROWS + j;
      const float nrm = __shfl_sync(full_mask(), nrm_lane, 8 * j);
      if (v >= a.n) break;
      const float inv = (nrm > kMinInputNorm) ? __fdiv_rn(1.f, nrm) : 0.f;
      const uint32_t inv_bits = __float_as_uint(inv);

      // Gather y = (x[perm[i]] * inv) * sign[i] (rotation.cpp:185-205).
      float y[R];
      {
        const unsigned char* xb = reinterpret_cast<const unsigned char*>(rows + j * L.stride);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const uint32_t e = s_src[r * 32 + lane];
          const float xv = *reinterpret_cast<const float*>(xb + (e & 0x7fffffffu));
          y[r] = __uint_as_float(__float_as_uint(__fmul_rn(xv, __uint_as_float(inv_bits))) ^ (e & 0x80000000u));
        }
      }
      __syncwarp();
      // The slot is free: bring in this warp's row j of its next group.
      if (next < n_groups && next * ROWS + j < a.n) prefetch(next * ROWS + j, j);
      cp_async_commit();

      // Walsh-Hadamard butterflies, strides 1, 2, 4, ... < block (rotation.cpp:38-85).
      const int block = a.block;
#pragma unroll
      for (int s = 1; s < E; s <<= 1) {
        if (s < block) {
#pragma unroll
          for (int r = 0; r < R; ++r) {
            if ((r & s) == 0) {
              const float p = y[r], q = y[r | s];
              y[r] = __fadd_rn(p, q);
              y[r | s] = __fsub_rn(p, q);
            }
          }
        }
      }
#pragma unroll
      for (int m = 1; m < 32; m <<= 1) {
        if (m * E < block) {
          const float sgn = (lane & m) ? -1.f : 1.f;
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const float o = __shfl_xor_sync(full_mask(), y[r], m);
            y[r] = __fmaf_rn(sgn, y[r], o);  // lower lane: y + o; upper lane: o - y
          }
        }
      }
#pragma unroll
      for (int sg = 1; sg < SEG; sg <<= 1) {
        if (32 * E * sg < block) {
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int seg = r / E;
            if ((seg & sg) == 0 && (seg | sg) < SEG) {
              const float p = y[r], q = y[r + sg * E];
              y[r] = __fadd_rn(p, q);
              y[r + sg * E] = __fsub_rn(p, q);
            }
          }
        }
      }
#pragma unroll
      for (int r = 0; r < R; ++r) y[r] = __fmul_rn(y[r], a.inv_sqrt_block);

      // Codes, packed runs, inner-product estimate (encode.cpp:112-157).
      double est = 0.0, mag = 0.0;
      uint8_t* flat_row = a.out_flat + v * static_cast<long long>(a.flat_stride);
#pragma unroll
      for (int sgi = 0; sgi < SEG; ++sgi) {
        Run run = 0;
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int r = sgi * E + e;
          unsigned code;
          double term;
          if constexpr (tq) {
            const float2 ss = s_ss[r * 32 + lane];
            const float c = __fmul_rn(__fadd_rn(y[r], ss.x), ss.y);
            code = grid_code(c, s_grid, g_lo, g_hi, g_a, g_k);
            const double back = __dsub_rn(__dmul_rn(static_cast<double>(s_cen[code]),
                                                    static_cast<double>(s_bk[r * 32 + lane])),
                                          static_cast<double>(ss.x));
            term = __dmul_rn(static_cast<double>(y[r]), back);
          } else {
            code = grid_code(y[r], s_grid, g_lo, g_hi, g_a, g_k);
            term = __dmul_rn(static_cast<double>(y[r]), static_cast<double>(s_cen[code]));
          }
          est = __dadd_rn(est, term);
          mag = __dadd_rn(mag, fabs(term));
          // codes_flat: CPB codes per byte, first code in the high bits (pack.cpp:70-131)
          const int byte = e / CPB, slot = e % CPB;
          run |= static_cast<Run>(code) << (8 * byte + FIELD * (CPB - 1 - slot));
        }
        const int i0 = sgi * 32 * E + lane * E;
        if (i0 < dim) *reinterpret_cast<Run*>(flat_row + i0 / CPB) = run;
      }
      est = warp_sum_d(est);
      mag = warp_sum_d(mag);

      float alpha = 0.f;
      bool above = false;
      float inner_f = 0.f;
      const int nc = (dim + 3) / 4;
      if (decide_float_of_sum(est, mag, nc + 2 + R + 6, kDegenerateInner, &above, &inner_f)) {
        alpha = above ? __fdiv_rn(nrm, inner_f) : 0.f;
      } else {
        // Exact replay of the reference's four sequential double chains
        // (chain i % 4, one fused multiply-add per term, encode.cpp:117-156).
        // Chain c visits its elements in index order; a lane holds E
        // consecutive elements of a segment, so each chain's running value
        // passes from lane to lane (a shuffle per lane), segment after segment.
        double ch[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int sgi = 0; sgi < SEG; ++sgi) {
#pragma unroll 1
          for (int l = 0; l < 32; ++l) {
            if (lane == l) {
#pragma unroll
              for (int e = 0; e < E; ++e) {
                const int r = sgi * E + e;
                if (pipe_elem<E>(r, lane) < dim) {
                  double back;
                  if constexpr (tq) {
                    const float2 ss = s_ss[r * 32 + lane];
                    const float c = __fmul_rn(__fadd_rn(y[r], ss.x), ss.y);
                    const unsigned code = pipe_code<BITS>(c, s_bnd);
                    back = __dsub_rn(__dmul_rn(static_cast<double>(s_cen[code]),
                                               static_cast<double>(s_bk[r * 32 + lane])),
                                     static_cast<double>(ss.x));
                  } else {
                    back = static_cast<double>(s_cen[pipe_code<BITS>(y[r], s_bnd)]);
                  }
                  ch[e & 3] = __fma_rn(static_cast<double>(y[r]), back, ch[e & 3]);
                }
              }
            }
#pragma unroll
            for (int c = 0; c < 4; ++c) ch[c] = __shfl_sync(full_mask(), ch[c], l);
          }
        }
        const double inner = __dadd_rn(__dadd_rn(ch[0], ch[1]), __dadd_rn(ch[2], ch[3]));
        alpha = inner > kDegenerateInner ? __fdiv_rn(nrm, __double2float_rn(inner)) : 0.f;
        if (lane == 0 && a.replay_count) atomicAdd(a.replay_count, 1ull);
      }
      if (lane == 0) a.out_alpha[v] = alpha;
    }
  }
  cp_async_wait_all();
}

// (R, E) of the pipelined kernel for a dim, or false when no instantiated
// layout fits (those dims use encode_rows_kernel).
bool pipe_shape(int dim, int* r_out, int* e_out) {
  static const int shapes[][2] = {{4, 4}, {8, 8}, {12, 4}, {16, 16}, {24, 8}, {32, 16}, {48, 16}, {64, 16}};
  for (const auto& sh : shapes) {
    const int r = sh[0], e = sh[1];
    // every element has a slot, and no lane's run of E codes crosses dim
    if (32 * r < dim || dim % e != 0) continue;
    *r_out = r;
    *e_out = e;
    return true;
  }
  return false;
}

template <int R, int E, int BITS, int ROWS, int MAXW, bool TQ>
cudaError_t launch_pipe_t(const EncodeArgs& a, int sms, int max_smem, cudaStream_t stream) {
  int warps = MAXW;
  while (warps > 1 && pipe_layout(a.dim, R, a.tqplus, warps, ROWS).total > static_cast<size_t>(max_smem)) --warps;
  const size_t smem = pipe_layout(a.dim, R, a.tqplus, warps, ROWS).total;
  if (smem > static_cast<size_t>(max_smem)) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(encode_pipe_kernel<R, E, BITS, ROWS, MAXW, TQ>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  const long long groups = (a.n + ROWS - 1) / ROWS;
  long long ctas = (groups + warps - 1) / warps;
  if (ctas > sms) ctas = sms;
  encode_pipe_kernel<R, E, BITS, ROWS, MAXW, TQ><<<static_cast<unsigned>(ctas), warps * 32, smem, stream>>>(a);
  return cudaGetLastError();
}

template <int R, int E, int ROWS, int MAXW>
cudaError_t launch_pipe_bits(const EncodeArgs& a, int sms, int max_smem, cudaStream_t stream) {
  switch (a.bits) {
    case 2:
      return a.tqplus ? launch_pipe_t<R, E, 2, ROWS, MAXW, true>(a, sms, max_smem, stream)
                      : launch_pipe_t<R, E, 2, ROWS, MAXW, false>(a, sms, max_smem, stream);
    case 3:
      return a.tqplus ? launch_pipe_t<R, E, 3, ROWS, MAXW, true>(a, sms, max_smem, stream)
                      : launch_pipe_t<R, E, 3, ROWS, MAXW, false>(a, sms, max_smem, stream);
    case 4:
      return a.tqplus ? launch_pipe_t<R, E, 4, ROWS, MAXW, true>(a, sms, max_smem, stream)
                      : launch_pipe_t<R, E, 4, ROWS, MAXW, false>(a, sms, max_smem, stream);
    default: return cudaErrorInvalidValue;
  }
}

int rows_template(int dim) {
  const int need = (dim + kWarp - 1) / kWarp;
  const int options[] = {1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64};
  for (int r : options) {
    if (r >= need) return r;
  }
  return -1;
}

int grid_for_quads(long long n, int sms) {
  const long long quads = (n + 3) / 4;
  long long ctas = (quads + 7) / 8;
  const long long cap = static_cast<long long>(sms) * 8;
  if (ctas > cap) ctas = cap;
  return static_cast<int>(ctas < 1 ? 1 : ctas);
}

}  // namespace

size_t encode_smem_bytes(int dim, bool tqplus) {
  return static_cast<size_t>(dim) * 4 * (tqplus ? 4 : 1) + 32 * 4 + static_cast<size_t>(8) * dim * 4;
}

bool encode_dim_supported(int dim) { return dim > 0 && dim <= 16384; }

#define VCB_ROWS_CASES(X) X(1) X(2) X(3) X(4) X(6) X(8) X(12) X(16) X(24) X(32) X(48) X(64)

cudaError_t launch_encode(const EncodeArgs& a, int sms, cudaStream_t stream) {
  if (a.n == 0) return cudaSuccess;
  if (a.dim > kRegisterRowMaxDim) return launch_encode_big(a, sms, stream);
  int pr = 0, pe = 0;
  if (a.grid && pipe_shape(a.dim, &pr, &pe)) {
    int device = 0, max_smem = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e != cudaSuccess) return e;
    // Warps per CTA as shared memory allows (1536-d: 16 warps of two 6 KB row
    // slots beside 24 KB of tables; 5.26 -> 5.16 ms per 1M rows against 14).
#define VCB_PIPE(RR, EE)                                                                            \
    if (pr == RR && pe == EE) {                                                                     \
      return launch_pipe_bits<RR, EE, (RR <= 32 ? 4 : 2), (RR <= 24 ? 16 : (RR == 32 ? 12 : (RR == 48 ? 16 : 10)))>( \
          a, sms, max_smem, stream);                                                                \
    }
    VCB_PIPE(4, 4) VCB_PIPE(8, 8) VCB_PIPE(12, 4) VCB_PIPE(16, 16) VCB_PIPE(24, 8) VCB_PIPE(32, 16)
    VCB_PIPE(48, 16) VCB_PIPE(64, 16)
#undef VCB_PIPE
  }
  const int r = rows_template(a.dim);
  const size_t smem = encode_smem_bytes(a.dim, a.tqplus);
  const int grid = grid_for_quads(a.n, sms);
  switch (r) {
#define VCB_CASE(RR)                                                                          \
  case RR: {                                                                                  \
    cudaError_t e = cudaFuncSetAttribute(encode_rows_kernel<RR>,                              \
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,         \
                                         static_cast<int>(smem));                             \
    if (e != cudaSuccess) return e;                                                           \
    encode_rows_kernel<RR><<<grid, 256, smem, stream>>>(a);                                   \
    return cudaGetLastError();                                                                \
  }
    VCB_ROWS_CASES(VCB_CASE)
#undef VCB_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

cudaError_t launch_relayout(const RelayoutArgs& a, cudaStream_t stream) {
  const long long first = (a.keep_below / 128) * 128;
  const long long strips = (a.n_total - first + 127) / 128;
  if (strips <= 0) return cudaSuccess;
  RelayoutArgs b = a;
  b.first_vector = first;
  dim3 grid(static_cast<unsigned>(strips), static_cast<unsigned>((a.nbg + 31) / 32));
  relayout_kernel<<<grid, 256, 0, stream>>>(b);
  return cudaGetLastError();
}

cudaError_t launch_export_flat(const uint32_t* codes, long long n, int nbg, uint8_t* out,
                               cudaStream_t stream) {
  const long long total = n * nbg;
  if (total == 0) return cudaSuccess;
  export_flat_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, stream>>>(codes, n, nbg, out);
  return cudaGetLastError();
}

cudaError_t launch_rotate_rows_t(const RotateArgs& a, int sms, cudaStream_t stream) {
  if (a.n == 0) return cudaSuccess;
  if (a.dim > kRegisterRowMaxDim) return launch_rotate_rows_t_big(a, sms, stream);
  const int r = rows_template(a.dim);
  const size_t smem = static_cast<size_t>(a.dim) * 4 + static_cast<size_t>(8) * a.dim * 4;
  const int grid = grid_for_quads(a.n, sms);
  switch (r) {
#define VCB_CASE(RR)                                                                          \
  case RR: {                                                                                  \
    cudaError_t e = cudaFuncSetAttribute(rotate_rows_t_kernel<RR>,                            \
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,         \
                                         static_cast<int>(smem));                             \
    if (e != cudaSuccess) return e;                                                           \
    rotate_rows_t_kernel<RR><<<grid, 256, smem, stream>>>(a);                                 \
    return cudaGetLastError();                                                                \
  }
    VCB_ROWS_CASES(VCB_CASE)
#undef VCB_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

cudaError_t launch_order_stats(const float* yt, long long n, int dim, long long lo_rank,
                               long long hi_rank, float* q_lo, float* q_hi, cudaStream_t stream) {
  order_stats_kernel<<<dim, 256, 0, stream>>>(yt, n, lo_rank, hi_rank, q_lo, q_hi);
  return cudaGetLastError();
}

}  // namespace vcb
