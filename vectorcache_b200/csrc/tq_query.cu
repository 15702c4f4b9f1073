// Query preparation on sm_100a: norm -> rotation -> TQ+ divide and bias
// correction -> per-query uint8 nibble LUTs with their scale and bias.
//
// Follows the reference's prepare_queries / build_query_lut
// (src/search/search.cpp:149-219, :762-860) bit for bit.
//
// One CTA of 8 warps prepares 4 queries: the rows are staged in shared memory,
// warp 0 runs the 8 sequential norm chains of all 4 rows, warp w < 4 rotates
// query w in registers, and then all 256 threads divide by the TQ+ scale and
// build the 4 queries' LUTs together (so a single query still gets the whole
// CTA for its divides and byte groups).
#include <cfloat>

#include "tq_kernels.h"
#include "tq_device.cuh"

namespace vcb {
namespace {

constexpr int kPrepQueries = 4;  // queries per CTA; warp w < 4 rotates query w
constexpr int kPrepThreads = 256;  // all 8 warps share the TQ+ divides and the LUT passes

// The 16 entries of one LUT half: entry nv = sum over the cpn codes packed in
// nibble value nv (first code in the high bits) of q[c] * centroid[code], each
// step one fused multiply-add from 0 (search.cpp:159-173). Fully unrolled so
// the entries stay in registers.
template <int BITS>
__device__ __forceinline__ void lut_half(const float* __restrict__ qd, const float* __restrict__ cen,
                                         float (&v)[16]) {
  if constexpr (BITS == 2) {
    const float q0 = qd[0], q1 = qd[1];
#pragma unroll
    for (int nv = 0; nv < 16; ++nv) {
      v[nv] = __fmaf_rn(q1, cen[nv & 3], __fmaf_rn(q0, cen[(nv >> 2) & 3], 0.f));
    }
  } else {
    const float q0 = qd[0];
#pragma unroll
    for (int nv = 0; nv < 16; ++nv) v[nv] = __fmaf_rn(q0, cen[nv & ((1 << BITS) - 1)], 0.f);
  }
}

template <int BITS>
__device__ __forceinline__ void half_min_max(const float (&v)[16], float* mn, float* mx) {
  float lo = FLT_MAX, hi = -FLT_MAX;
#pragma unroll
  for (int nv = 0; nv < 16; ++nv) {
    lo = (v[nv] < lo) ? v[nv] : lo;  // std::min / std::max semantics
    hi = (hi < v[nv]) ? v[nv] : hi;
  }
  *mn = lo;
  *mx = hi;
}

template <int R, int BITS>
__global__ void __launch_bounds__(kPrepThreads, 2) query_prep_kernel(QueryPrepArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int dim = a.dim, nbg = a.nbg;
  constexpr int kCpb = 8 / BITS;      // codes per byte group
  constexpr int kCpn = kCpb / 2;      // codes per nibble
  uint32_t* s_perm = reinterpret_cast<uint32_t*>(smem);
  float* s_shift = reinterpret_cast<float*>(s_perm + dim);
  float* s_scale = s_shift + (a.tqplus ? dim : 0);
  float* s_rows = s_scale + (a.tqplus ? dim : 0);   // 4 x dim
  float* s_gmin = s_rows + kPrepQueries * dim;         // 4 x nbg
  __shared__ float s_cen[16];
  __shared__ float s_norm[kPrepQueries];
  __shared__ float s_bias_corr[kPrepQueries];
  __shared__ unsigned s_span_bits[kPrepQueries];
  __shared__ float s_inv[kPrepQueries];
  __shared__ float s_lut_scale[kPrepQueries];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  // Tables in 16-byte pieces (dim is a multiple of 8), four pieces per thread
  // loaded before any is stored so their latencies overlap.
  const int n4 = dim >> 2;
  for (int i0 = threadIdx.x; i0 < n4; i0 += 4 * kPrepThreads) {
    uint4 p[4];
    float4 sh[4], sc[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * kPrepThreads;
      if (i < n4) {
        p[u] = __ldg(reinterpret_cast<const uint4*>(a.perm_sign) + i);
        if (a.tqplus) {
          sh[u] = __ldg(reinterpret_cast<const float4*>(a.shift) + i);
          sc[u] = __ldg(reinterpret_cast<const float4*>(a.scale) + i);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * kPrepThreads;
      if (i < n4) {
        reinterpret_cast<uint4*>(s_perm)[i] = p[u];
        if (a.tqplus) {
          reinterpret_cast<float4*>(s_shift)[i] = sh[u];
          reinterpret_cast<float4*>(s_scale)[i] = sc[u];
        }
      }
    }
  }
  if (threadIdx.x < 16) s_cen[threadIdx.x] = a.centroids[threadIdx.x];

  for (long long q0 = static_cast<long long>(blockIdx.x) * kPrepQueries; q0 < a.nq;
       q0 += static_cast<long long>(gridDim.x) * kPrepQueries) {
    const int nloc = static_cast<int>(min(static_cast<long long>(kPrepQueries), a.nq - q0));
    __syncthreads();
    // Stage the rows (coalesced 16-byte loads).
    const int vec_per_row = dim / 4;
    for (int t0 = threadIdx.x; t0 < nloc * vec_per_row; t0 += 4 * kPrepThreads) {
      float4 v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int t = t0 + u * kPrepThreads;
        if (t < nloc * vec_per_row) {
          const int r = t / vec_per_row, c = t % vec_per_row;
          v[u] = __ldg(reinterpret_cast<const float4*>(a.q + (q0 + r) * static_cast<long long>(dim)) + c);
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int t = t0 + u * kPrepThreads;
        if (t < nloc * vec_per_row) reinterpret_cast<float4*>(s_rows)[t] = v[u];
      }
    }
    if (threadIdx.x < kPrepQueries) s_span_bits[threadIdx.x] = 0u;
    __syncthreads();

    // Norms: lane 8v + c of warp 0 runs chain c of row v (encode.cpp:16-26).
    if (warp == 0) {
      const int v = lane >> 3, c = lane & 7;
      float s = 0.f;
      if (v < nloc) {
        const float* row = s_rows + v * dim;
        int j = c;
        for (; j + 56 < dim; j += 64) {  // 8 loads ahead of the chain's FMAs, same order
          float x[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) x[u] = row[j + 8 * u];
#pragma unroll
          for (int u = 0; u < 8; ++u) s = __fmaf_rn(x[u], x[u], s);
        }
        for (; j < dim; j += 8) s = __fmaf_rn(row[j], row[j], s);
      }
      s = __fadd_rn(s, __shfl_xor_sync(full_mask(), s, 1));
      s = __fadd_rn(s, __shfl_xor_sync(full_mask(), s, 2));
      s = __fadd_rn(s, __shfl_xor_sync(full_mask(), s, 4));
      if (c == 0 && v < nloc) s_norm[v] = __fsqrt_rn(s);
    }
    __syncthreads();

    // Rotation (and TQ+) of query `warp`, written back over its staged row.
    if (warp < nloc) {
      const long long qi = q0 + warp;
      float* row = s_rows + warp * dim;
      const float nrm = s_norm[warp];
      const float inv = (nrm > kMinInputNorm) ? __fdiv_rn(1.f, nrm) : 0.f;
      float y[R];
      warp_rotate<R>(row, s_perm, dim, a.block, inv, a.inv_sqrt_block, y, lane);
      float bias_corr = 0.f;
      if (a.tqplus) {
        // bias_corr = -sum_d y_d * shift_d, sequential in double in the
        // reference (search.cpp:792-799); the products are exact in double.
        double est = 0.0, mag = 0.0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int i = lane + kWarp * r;
          if (i < dim) {
            const double p = __dmul_rn(static_cast<double>(y[r]), static_cast<double>(s_shift[i]));
            est = __dsub_rn(est, p);
            mag = __dadd_rn(mag, fabs(p));
          }
        }
        est = warp_sum_d(est);
        mag = warp_sum_d(mag);
        bool above;
        if (!decide_float_of_sum(est, mag, dim + R + 8, -DBL_MAX, &above, &bias_corr)) {
          __syncwarp();
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int i = lane + kWarp * r;
            if (i < dim) row[i] = y[r];
          }
          __syncwarp();
          double bc = 0.0;
          if (lane == 0) {
#pragma unroll 1
            for (int i = 0; i < dim; ++i) {
              bc = __dsub_rn(bc, __dmul_rn(static_cast<double>(row[i]), static_cast<double>(s_shift[i])));
            }
          }
          bias_corr = __double2float_rn(__shfl_sync(full_mask(), bc, 0));
          if (lane == 0 && a.replay_count) atomicAdd(a.replay_count, 1ull);
        }
      }
      __syncwarp();
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = lane + kWarp * r;
        if (i < dim) {
          row[i] = y[r];
          if (a.q_rot && !a.tqplus) a.q_rot[qi * dim + i] = y[r];
        }
      }
      if (lane == 0) s_bias_corr[warp] = bias_corr;
    }
    __syncthreads();
    if (a.tqplus) {
      // q_rot_d = y_d / scale_d (search.cpp:792-797), spread over the whole CTA.
      const int total = nloc * dim;
      for (int t0 = threadIdx.x; t0 < total; t0 += 4 * kPrepThreads) {
        float v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int t = t0 + u * kPrepThreads;
          v[u] = (t < total) ? __fdiv_rn(s_rows[t], s_scale[t % dim]) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int t = t0 + u * kPrepThreads;
          if (t < total) {
            s_rows[t] = v[u];
            if (a.q_rot) a.q_rot[q0 * dim + t] = v[u];
          }
        }
      }
      __syncthreads();
    }

    // LUT pass 1: per-group minima and per-query largest span (search.cpp:163-199).
    float span[kPrepQueries] = {0.f, 0.f, 0.f, 0.f};
    for (int t = threadIdx.x; t < nloc * nbg; t += blockDim.x) {
      const int r = t / nbg, g = t % nbg;
      const float* qd = s_rows + r * dim + g * kCpb;
      float v[16], mn0, mx0, mn1, mx1;
      lut_half<BITS>(qd, s_cen, v);
      half_min_max<BITS>(v, &mn0, &mx0);
      lut_half<BITS>(qd + kCpn, s_cen, v);
      half_min_max<BITS>(v, &mn1, &mx1);
      const float d0 = __fsub_rn(mx0, mn0), d1 = __fsub_rn(mx1, mn1);
      float sp = (0.f < d0) ? d0 : 0.f;
      sp = (sp < d1) ? d1 : sp;
#pragma unroll
      for (int rr = 0; rr < kPrepQueries; ++rr) {
        if (rr == r) span[rr] = (span[rr] < sp) ? sp : span[rr];
      }
      s_gmin[r * nbg + g] = __fadd_rn(mn0, mn1);
    }
#pragma unroll
    for (int rr = 0; rr < kPrepQueries; ++rr) {
      const float m = warp_max_f(span[rr]);
      // Spans are >= 0, so their IEEE bit patterns order like the values.
      if (lane == 0 && rr < nloc) atomicMax(&s_span_bits[rr], __float_as_uint(m));
    }
    __syncthreads();
    if (threadIdx.x < nloc) {
      const float sp = __uint_as_float(s_span_bits[threadIdx.x]);
      float scale = (sp > 0.f) ? __fdiv_rn(sp, 127.f) : 1.f;
      float inv = 1.f;
      if (scale >= FLT_MIN) {
        inv = __fdiv_rn(1.f, scale);
      } else {
        scale = 1.f;
      }
      s_lut_scale[threadIdx.x] = scale;
      s_inv[threadIdx.x] = inv;
    }
    __syncthreads();

    // LUT pass 2: quantized bytes, 32 per group (first half indexed by the
    // high nibble, second half by the low nibble).
    for (int t = threadIdx.x; t < nloc * nbg; t += blockDim.x) {
      const int r = t / nbg, g = t % nbg;
      const float* qd = s_rows + r * dim + g * kCpb;
      const float inv = s_inv[r];
      uint32_t words[8];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        float v[16], mn, mx;
        lut_half<BITS>(qd + h * kCpn, s_cen, v);
        half_min_max<BITS>(v, &mn, &mx);
#pragma unroll
        for (int w = 0; w < 4; ++w) {
          uint32_t word = 0;
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            float x = roundf(__fmul_rn(__fsub_rn(v[4 * w + b], mn), inv));
            x = (x < 0.f) ? 0.f : ((127.f < x) ? 127.f : x);  // std::clamp
            word |= static_cast<uint32_t>(x) << (8 * b);
          }
          words[4 * h + w] = word;
        }
      }
      uint4* dst = reinterpret_cast<uint4*>(a.luts + ((q0 + r) * nbg + g) * 32LL);
      dst[0] = make_uint4(words[0], words[1], words[2], words[3]);
      dst[1] = make_uint4(words[4], words[5], words[6], words[7]);
    }
    __syncthreads();

    // The LUT bias is a sequential f32 sum over groups (search.cpp:196).
    if (threadIdx.x < nloc) {
      const int r = threadIdx.x;
      float bias = 0.f;
      const float* gm = s_gmin + r * nbg;
      int g = 0;
      for (; g + 8 <= nbg; g += 8) {  // loads ahead of the in-order adds
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = gm[g + u];
#pragma unroll
        for (int u = 0; u < 8; ++u) bias = __fadd_rn(bias, v[u]);
      }
      for (; g < nbg; ++g) bias = __fadd_rn(bias, gm[g]);
      const long long qi = q0 + r;
      a.lut_scale[qi] = s_lut_scale[r];
      a.lut_bias[qi] = bias;
      a.bias_corr[qi] = s_bias_corr[r];
      a.fa_init[qi] = __fadd_rn(bias, s_bias_corr[r]);
    }
  }
}

int rows_template_q(int dim) {
  const int need = (dim + kWarp - 1) / kWarp;
  const int options[] = {1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64};
  for (int r : options) {
    if (r >= need) return r;
  }
  return -1;
}

template <int R, int BITS>
cudaError_t launch_prep_t(const QueryPrepArgs& a, size_t smem, unsigned grid, cudaStream_t stream) {
  cudaError_t e = cudaFuncSetAttribute(query_prep_kernel<R, BITS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  query_prep_kernel<R, BITS><<<grid, kPrepThreads, smem, stream>>>(a);
  return cudaGetLastError();
}

template <int R>
cudaError_t launch_prep_bits(const QueryPrepArgs& a, size_t smem, unsigned grid, cudaStream_t stream) {
  switch (a.bits) {
    case 2:
      return launch_prep_t<R, 2>(a, smem, grid, stream);
    case 3:
      return launch_prep_t<R, 3>(a, smem, grid, stream);
    case 4:
      return launch_prep_t<R, 4>(a, smem, grid, stream);
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace

cudaError_t launch_query_prep(const QueryPrepArgs& a, int sms, cudaStream_t stream) {
  if (a.nq == 0) return cudaSuccess;
  if (a.dim > kRegisterRowMaxDim) return launch_query_prep_big(a, sms, stream);
  const int r = rows_template_q(a.dim);
  const size_t smem = static_cast<size_t>(a.dim) * 4 * (a.tqplus ? 3 : 1) +
                      static_cast<size_t>(kPrepQueries) * (a.dim + a.nbg) * 4;
  long long grid = (a.nq + kPrepQueries - 1) / kPrepQueries;
  if (grid > static_cast<long long>(sms) * 16) grid = static_cast<long long>(sms) * 16;
  const unsigned g = static_cast<unsigned>(grid);
  switch (r) {
#define VCB_CASE(RR) \
  case RR:           \
    return launch_prep_bits<RR>(a, smem, g, stream);
    VCB_CASE(1) VCB_CASE(2) VCB_CASE(3) VCB_CASE(4) VCB_CASE(6) VCB_CASE(8) VCB_CASE(12)
    VCB_CASE(16) VCB_CASE(24) VCB_CASE(32) VCB_CASE(48) VCB_CASE(64)
#undef VCB_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace vcb
