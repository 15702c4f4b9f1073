// Query preparation on sm_100a: norm -> rotation -> TQ+ divide and bias
// correction -> per-query uint8 nibble LUTs with their scale and bias.
//
// Follows the reference's prepare_queries / build_query_lut
// (src/search/search.cpp:149-219, :762-860) bit for bit.
#include <cfloat>

#include "tq_kernels.h"
#include "tq_device.cuh"

namespace vcb {
namespace {

constexpr int kPrepWarps = 4;

template <int R>
__global__ void __launch_bounds__(kPrepWarps * 32) query_prep_kernel(QueryPrepArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int dim = a.dim, nbg = a.nbg;
  uint32_t* s_perm = reinterpret_cast<uint32_t*>(smem);
  float* s_shift = reinterpret_cast<float*>(s_perm + dim);
  float* s_scale = s_shift + (a.tqplus ? dim : 0);
  float* s_cen = s_scale + (a.tqplus ? dim : 0);
  float* s_rows = s_cen + 16;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* qrow = s_rows + static_cast<size_t>(warp) * (dim + 4 * nbg);
  float* gmin = qrow + dim;  // 4 queries x nbg per-group (min_first + min_second)

  for (int i = threadIdx.x; i < dim; i += blockDim.x) {
    s_perm[i] = a.perm_sign[i];
    if (a.tqplus) {
      s_shift[i] = a.shift[i];
      s_scale[i] = a.scale[i];
    }
  }
  if (threadIdx.x < 16) s_cen[threadIdx.x] = a.centroids[threadIdx.x];
  __syncthreads();

  const int cpb = 8 / a.bits;
  const int cpn = cpb / 2;  // codes per nibble
  const unsigned code_mask = (1u << a.bits) - 1u;

  const long long warps_total = static_cast<long long>(gridDim.x) * kPrepWarps;
  for (long long quad = static_cast<long long>(blockIdx.x) * kPrepWarps + warp; quad * 4 < a.nq;
       quad += warps_total) {
    const long long q_lane = quad * 4 + (lane >> 3);
    const bool lane_valid = q_lane < a.nq;
    const float nrm_lane =
        warp_norm4(a.q + (lane_valid ? q_lane : 0) * static_cast<long long>(dim), dim, lane_valid, lane);
    float my_bias_corr = 0.f;   // lane j (< 4) keeps query j's values for the final step
    float my_span = 0.f;

    for (int j = 0; j < 4; ++j) {
      const long long qi = quad * 4 + j;
      const float nrm = __shfl_sync(full_mask(), nrm_lane, 8 * j);
      if (qi >= a.nq) break;
      const float* src = a.q + qi * static_cast<long long>(dim);
      __syncwarp();
      for (int i = lane * 4; i < dim; i += kWarp * 4) {
        *reinterpret_cast<float4*>(qrow + i) = __ldg(reinterpret_cast<const float4*>(src + i));
      }
      __syncwarp();
      const float inv = (nrm > kMinInputNorm) ? __fdiv_rn(1.f, nrm) : 0.f;
      float y[R];
      warp_rotate<R>(qrow, s_perm, dim, a.block, inv, a.inv_sqrt_block, y, lane);

      float bias_corr = 0.f;
      if (a.tqplus) {
        // bias_corr = -sum_d y_d * shift_d, accumulated sequentially in double by
        // the reference (search.cpp:792-799); the products are exact in double.
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
            if (i < dim) qrow[i] = y[r];
          }
          __syncwarp();
          double bc = 0.0;
          if (lane == 0) {
#pragma unroll 1
            for (int i = 0; i < dim; ++i) {
              bc = __dsub_rn(bc, __dmul_rn(static_cast<double>(qrow[i]), static_cast<double>(s_shift[i])));
            }
          }
          bias_corr = __double2float_rn(__shfl_sync(full_mask(), bc, 0));
          if (lane == 0 && a.replay_count) atomicAdd(a.replay_count, 1ull);
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int i = lane + kWarp * r;
          if (i < dim) y[r] = __fdiv_rn(y[r], s_scale[i]);
        }
      }
      __syncwarp();
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = lane + kWarp * r;
        if (i < dim) {
          qrow[i] = y[r];
          if (a.q_rot) a.q_rot[qi * dim + i] = y[r];
        }
      }
      __syncwarp();

      // Pass 1: per-group minima and the largest span (search.cpp:163-199).
      float span = 0.f;
      for (int g = lane; g < nbg; g += kWarp) {
        const float* qd = qrow + g * cpb;
        float mins[2];
        for (int h = 0; h < 2; ++h) {
          float mn = FLT_MAX, mx = -FLT_MAX;
          for (unsigned nv = 0; nv < 16; ++nv) {
            float s = 0.f;
            for (int c = 0; c < cpn; ++c) {
              const unsigned code = (nv >> ((cpn - 1 - c) * a.bits)) & code_mask;
              s = __fmaf_rn(qd[h * cpn + c], s_cen[code], s);
            }
            mn = (s < mn) ? s : mn;  // std::min / std::max semantics
            mx = (mx < s) ? s : mx;
          }
          mins[h] = mn;
          const float d = __fsub_rn(mx, mn);
          span = (span < d) ? d : span;
        }
        gmin[j * nbg + g] = __fadd_rn(mins[0], mins[1]);
      }
      span = warp_max_f(span);
      float lut_scale = (span > 0.f) ? __fdiv_rn(span, 127.f) : 1.f;
      float lut_inv = 1.f;
      if (lut_scale >= FLT_MIN) {
        lut_inv = __fdiv_rn(1.f, lut_scale);
      } else {
        lut_scale = 1.f;
      }

      // Pass 2: quantized LUT bytes, 32 per group: first half indexed by the
      // high nibble, second half by the low nibble.
      uint8_t* out = a.luts + qi * static_cast<long long>(nbg) * 32;
      for (int g = lane; g < nbg; g += kWarp) {
        const float* qd = qrow + g * cpb;
        uint32_t words[8];
        for (int h = 0; h < 2; ++h) {
          float vals[16];
          float mn = FLT_MAX;
          for (unsigned nv = 0; nv < 16; ++nv) {
            float s = 0.f;
            for (int c = 0; c < cpn; ++c) {
              const unsigned code = (nv >> ((cpn - 1 - c) * a.bits)) & code_mask;
              s = __fmaf_rn(qd[h * cpn + c], s_cen[code], s);
            }
            vals[nv] = s;
            mn = (s < mn) ? s : mn;
          }
          for (int w = 0; w < 4; ++w) {
            uint32_t word = 0;
            for (int b = 0; b < 4; ++b) {
              float r = roundf(__fmul_rn(__fsub_rn(vals[4 * w + b], mn), lut_inv));
              r = (r < 0.f) ? 0.f : ((127.f < r) ? 127.f : r);  // std::clamp
              word |= static_cast<uint32_t>(r) << (8 * b);
            }
            words[4 * h + w] = word;
          }
        }
        uint4* dst = reinterpret_cast<uint4*>(out + static_cast<long long>(g) * 32);
        dst[0] = make_uint4(words[0], words[1], words[2], words[3]);
        dst[1] = make_uint4(words[4], words[5], words[6], words[7]);
      }
      if (lane == j) {
        my_bias_corr = bias_corr;
        my_span = lut_scale;
      }
    }
    __syncwarp();
    // The LUT bias is a sequential f32 sum over groups (search.cpp:196); lane j
    // replays it for query j of this quad.
    const long long qi = quad * 4 + lane;
    if (lane < 4 && qi < a.nq) {
      float bias = 0.f;
      for (int g = 0; g < nbg; ++g) bias = __fadd_rn(bias, gmin[lane * nbg + g]);
      a.lut_scale[qi] = my_span;
      a.lut_bias[qi] = bias;
      a.bias_corr[qi] = my_bias_corr;
      a.fa_init[qi] = __fadd_rn(bias, my_bias_corr);
    }
    __syncwarp();
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

}  // namespace

cudaError_t launch_query_prep(const QueryPrepArgs& a, int sms, cudaStream_t stream) {
  if (a.nq == 0) return cudaSuccess;
  if (a.dim > kRegisterRowMaxDim) return launch_query_prep_big(a, sms, stream);
  const int r = rows_template_q(a.dim);
  const size_t smem = static_cast<size_t>(a.dim) * 4 * (a.tqplus ? 3 : 1) + 16 * 4 +
                      static_cast<size_t>(kPrepWarps) * (a.dim + 4 * a.nbg) * 4;
  const long long quads = (a.nq + 3) / 4;
  long long grid = (quads + kPrepWarps - 1) / kPrepWarps;
  if (grid > static_cast<long long>(sms) * 16) grid = static_cast<long long>(sms) * 16;
  switch (r) {
#define VCB_CASE(RR)                                                                          \
  case RR: {                                                                                  \
    cudaError_t e = cudaFuncSetAttribute(query_prep_kernel<RR>,                               \
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,         \
                                         static_cast<int>(smem));                             \
    if (e != cudaSuccess) return e;                                                           \
    query_prep_kernel<RR><<<static_cast<unsigned>(grid), kPrepWarps * 32, smem, stream>>>(a); \
    return cudaGetLastError();                                                                \
  }
    VCB_CASE(1) VCB_CASE(2) VCB_CASE(3) VCB_CASE(4) VCB_CASE(6) VCB_CASE(8) VCB_CASE(12)
    VCB_CASE(16) VCB_CASE(24) VCB_CASE(32) VCB_CASE(48) VCB_CASE(64)
#undef VCB_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace vcb
