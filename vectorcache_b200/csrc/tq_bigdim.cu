// Rows wider than 2048 coordinates (up to the reference's 16384): one CTA per
// row with the row in shared memory. Same arithmetic as the register kernels
// in tq_encode.cu / tq_query.cu (rotation.cpp:38-121, encode.cpp:112-231,
// search.cpp:149-219, :762-860); slower, but these widths are rare.
#include <cfloat>

#include "tq_kernels.h"
#include "tq_device.cuh"

namespace vcb {
namespace {

constexpr int kBigThreads = 256;

__device__ __forceinline__ double block_sum_d(double v, double* red) {
  v = warp_sum_d(v);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = (lane < (blockDim.x >> 5)) ? red[lane] : 0.0;
  if (warp == 0) t = warp_sum_d(t);
  if (threadIdx.x == 0) red[0] = t;
  __syncthreads();
  const double r = red[0];
  __syncthreads();
  return r;
}

__device__ __forceinline__ float block_max_f(float v, float* red) {
  v = warp_max_f(v);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  float t = (lane < (blockDim.x >> 5)) ? red[lane] : 0.f;
  if (warp == 0) t = warp_max_f(t);
  if (threadIdx.x == 0) red[0] = t;
  __syncthreads();
  const float r = red[0];
  __syncthreads();
  return r;
}

// ||x|| with the reference's 8 sequential chains (threads 0..7), then the tree.
__device__ float block_norm(const float* __restrict__ row, int dim, float* red) {
  if (threadIdx.x < 8) {
    float s = 0.f;
    for (int j = threadIdx.x; j < dim; j += 8) s = __fmaf_rn(row[j], row[j], s);
    red[threadIdx.x] = s;
  }
  __syncthreads();
  const float n = __fsqrt_rn(__fadd_rn(__fadd_rn(__fadd_rn(red[0], red[1]), __fadd_rn(red[2], red[3])),
                                       __fadd_rn(__fadd_rn(red[4], red[5]), __fadd_rn(red[6], red[7]))));
  __syncthreads();
  return n;
}

// y = WHT_blocks(P S x * inv) * 1/sqrt(B), in shared memory.
__device__ void block_rotate(const float* __restrict__ x, const uint32_t* __restrict__ perm_sign, int dim,
                             int block, float inv, float inv_sqrt_block, float* y) {
  for (int i = threadIdx.x; i < dim; i += blockDim.x) {
    const uint32_t e = perm_sign[i];
    float v = __fmul_rn(x[e & 0x7fffffffu], inv);
    if (e >> 31) v = -v;
    y[i] = v;
  }
  __syncthreads();
  for (int len = 1; len < block; len <<= 1) {
    for (int t = threadIdx.x; t < dim / 2; t += blockDim.x) {
      const int i = (t / len) * 2 * len + (t % len);  // lower element of the pair
      const float a = y[i], b = y[i + len];
      y[i] = __fadd_rn(a, b);
      y[i + len] = __fsub_rn(a, b);
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < dim; i += blockDim.x) y[i] = __fmul_rn(y[i], inv_sqrt_block);
  __syncthreads();
}

// One CTA per row: encode (codes_flat bytes + alpha).
__global__ void __launch_bounds__(kBigThreads) encode_big_kernel(EncodeArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int dim = a.dim;
  float* x = reinterpret_cast<float*>(smem);
  float* y = x + dim;
  __shared__ double red_d[32];
  __shared__ float red_f[32];
  __shared__ float s_bnd[16], s_cen[16];
  if (threadIdx.x < 16) {
    s_bnd[threadIdx.x] = threadIdx.x < 15 ? a.boundaries[threadIdx.x] : 0.f;
    s_cen[threadIdx.x] = a.centroids[threadIdx.x];
  }
  const int cpb = 8 / a.bits, field = (a.bits == 3) ? 4 : a.bits;
  const int nbg = dim / cpb;
  for (long long v = blockIdx.x; v < a.n; v += gridDim.x) {
    const float* src = a.x + v * static_cast<long long>(dim);
    __syncthreads();
    for (int i = threadIdx.x * 4; i < dim; i += blockDim.x * 4) {
      *reinterpret_cast<float4*>(x + i) = __ldg(reinterpret_cast<const float4*>(src + i));
    }
    __syncthreads();
    const float nrm = block_norm(x, dim, red_f);
    const float inv = (nrm > kMinInputNorm) ? __fdiv_rn(1.f, nrm) : 0.f;
    block_rotate(x, a.perm_sign, dim, a.block, inv, a.inv_sqrt_block, y);
    // Codes go to x (reused as bytes); the inner-product estimate is reduced.
    uint8_t* code = reinterpret_cast<uint8_t*>(x);
    double est = 0.0, mag = 0.0;
    for (int i = threadIdx.x; i < dim; i += blockDim.x) {
      double term;
      unsigned c;
      if (a.tqplus) {
        c = quantize_code(__fmul_rn(__fadd_rn(y[i], a.shift[i]), a.scale[i]), s_bnd, a.bits);
        const double back = __dsub_rn(__dmul_rn(static_cast<double>(s_cen[c]), static_cast<double>(a.inv_scale[i])),
                                      static_cast<double>(a.shift[i]));
        term = __dmul_rn(static_cast<double>(y[i]), back);
      } else {
        c = quantize_code(y[i], s_bnd, a.bits);
        term = __dmul_rn(static_cast<double>(y[i]), static_cast<double>(s_cen[c]));
      }
      code[i] = static_cast<uint8_t>(c);
      est = __dadd_rn(est, term);
      mag = __dadd_rn(mag, fabs(term));
    }
    est = block_sum_d(est, red_d);
    mag = block_sum_d(mag, red_d);
    uint8_t* flat_row = a.out_flat + v * static_cast<long long>(a.flat_stride);
    for (int g = threadIdx.x; g < nbg; g += blockDim.x) {
      unsigned byte = 0;
      for (int c = 0; c < cpb; ++c) byte |= static_cast<unsigned>(code[g * cpb + c]) << (field * (cpb - 1 - c));
      flat_row[g] = static_cast<uint8_t>(byte);
    }
    const int steps = (dim + 3) / 4 + 2 + dim / kBigThreads + 12;
    float inner_f = 0.f;
    bool above = false;
    float alpha;
    if (decide_float_of_sum(est, mag, steps, kDegenerateInner, &above, &inner_f)) {
      alpha = above ? __fdiv_rn(nrm, inner_f) : 0.f;
    } else {
      // Exact replay of the four sequential double chains.
      if (threadIdx.x < 4) {
        double ch = 0.0;
        for (int i = threadIdx.x; i < dim; i += 4) {
          const unsigned c = code[i];
          if (a.tqplus) {
            const double back = __dsub_rn(__dmul_rn(static_cast<double>(s_cen[c]), static_cast<double>(a.inv_scale[i])),
                                          static_cast<double>(a.shift[i]));
            ch = __fma_rn(static_cast<double>(y[i]), back, ch);
          } else {
            ch = __fma_rn(static_cast<double>(y[i]), static_cast<double>(s_cen[c]), ch);
          }
        }
        red_d[threadIdx.x] = ch;
      }
      __syncthreads();
      const double inner = __dadd_rn(__dadd_rn(red_d[0], red_d[1]), __dadd_rn(red_d[2], red_d[3]));
      alpha = inner > kDegenerateInner ? __fdiv_rn(nrm, __double2float_rn(inner)) : 0.f;
      if (threadIdx.x == 0 && a.replay_count) atomicAdd(a.replay_count, 1ull);
      __syncthreads();
    }
    if (threadIdx.x == 0) a.out_alpha[v] = alpha;
  }
}

// One CTA per query: rotation, TQ+ divide and bias correction, LUT bytes.
__global__ void __launch_bounds__(kBigThreads) query_prep_big_kernel(QueryPrepArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int dim = a.dim, nbg = a.nbg;
  float* x = reinterpret_cast<float*>(smem);
  float* y = x + dim;
  float* gmin = y + dim;  // nbg
  __shared__ double red_d[32];
  __shared__ float red_f[32];
  __shared__ float s_cen[16];
  __shared__ float s_bc;
  if (threadIdx.x < 16) s_cen[threadIdx.x] = a.centroids[threadIdx.x];
  const int cpb = 8 / a.bits, cpn = cpb / 2;
  const unsigned code_mask = (1u << a.bits) - 1u;
  for (long long qi = blockIdx.x; qi < a.nq; qi += gridDim.x) {
    const float* src = a.q + qi * static_cast<long long>(dim);
    __syncthreads();
    for (int i = threadIdx.x * 4; i < dim; i += blockDim.x * 4) {
      *reinterpret_cast<float4*>(x + i) = __ldg(reinterpret_cast<const float4*>(src + i));
    }
    __syncthreads();
    const float nrm = block_norm(x, dim, red_f);
    const float inv = (nrm > kMinInputNorm) ? __fdiv_rn(1.f, nrm) : 0.f;
    block_rotate(x, a.perm_sign, dim, a.block, inv, a.inv_sqrt_block, y);
    float bias_corr = 0.f;
    if (a.tqplus) {
      double est = 0.0, mag = 0.0;
      for (int i = threadIdx.x; i < dim; i += blockDim.x) {
        const double p = __dmul_rn(static_cast<double>(y[i]), static_cast<double>(a.shift[i]));
        est = __dsub_rn(est, p);
        mag = __dadd_rn(mag, fabs(p));
      }
      est = block_sum_d(est, red_d);
      mag = block_sum_d(mag, red_d);
      bool above;
      if (!decide_float_of_sum(est, mag, dim + dim / kBigThreads + 12, -DBL_MAX, &above, &bias_corr)) {
        if (threadIdx.x == 0) {
          double bc = 0.0;
          for (int i = 0; i < dim; ++i) {
            bc = __dsub_rn(bc, __dmul_rn(static_cast<double>(y[i]), static_cast<double>(a.shift[i])));
          }
          s_bc = __double2float_rn(bc);
          if (a.replay_count) atomicAdd(a.replay_count, 1ull);
        }
        __syncthreads();
        bias_corr = s_bc;
        __syncthreads();
      }
      for (int i = threadIdx.x; i < dim; i += blockDim.x) y[i] = __fdiv_rn(y[i], a.scale[i]);
      __syncthreads();
    }
    if (a.q_rot) {
      for (int i = threadIdx.x; i < dim; i += blockDim.x) a.q_rot[qi * dim + i] = y[i];
    }
    float span = 0.f;
    for (int g = threadIdx.x; g < nbg; g += blockDim.x) {
      const float* qd = y + g * cpb;
      float mins[2];
      for (int h = 0; h < 2; ++h) {
        float mn = FLT_MAX, mx = -FLT_MAX;
        for (unsigned nv = 0; nv < 16; ++nv) {
          float s = 0.f;
          for (int c = 0; c < cpn; ++c) {
            s = __fmaf_rn(qd[h * cpn + c], s_cen[(nv >> ((cpn - 1 - c) * a.bits)) & code_mask], s);
          }
          mn = (s < mn) ? s : mn;
          mx = (mx < s) ? s : mx;
        }
        mins[h] = mn;
        const float d = __fsub_rn(mx, mn);
        span = (span < d) ? d : span;
      }
      gmin[g] = __fadd_rn(mins[0], mins[1]);
    }
    span = block_max_f(span, red_f);
    float lut_scale = (span > 0.f) ? __fdiv_rn(span, 127.f) : 1.f;
    float lut_inv = 1.f;
    if (lut_scale >= FLT_MIN) {
      lut_inv = __fdiv_rn(1.f, lut_scale);
    } else {
      lut_scale = 1.f;
    }
    uint8_t* out = a.luts + qi * static_cast<long long>(nbg) * 32;
    for (int g = threadIdx.x; g < nbg; g += blockDim.x) {
      const float* qd = y + g * cpb;
      uint32_t words[8];
      for (int h = 0; h < 2; ++h) {
        float vals[16];
        float mn = FLT_MAX;
        for (unsigned nv = 0; nv < 16; ++nv) {
          float s = 0.f;
          for (int c = 0; c < cpn; ++c) {
            s = __fmaf_rn(qd[h * cpn + c], s_cen[(nv >> ((cpn - 1 - c) * a.bits)) & code_mask], s);
          }
          vals[nv] = s;
          mn = (s < mn) ? s : mn;
        }
        for (int w = 0; w < 4; ++w) {
          uint32_t word = 0;
          for (int b = 0; b < 4; ++b) {
            float r = roundf(__fmul_rn(__fsub_rn(vals[4 * w + b], mn), lut_inv));
            r = (r < 0.f) ? 0.f : ((127.f < r) ? 127.f : r);
            word |= static_cast<uint32_t>(r) << (8 * b);
          }
          words[4 * h + w] = word;
        }
      }
      uint4* dst = reinterpret_cast<uint4*>(out + static_cast<long long>(g) * 32);
      dst[0] = make_uint4(words[0], words[1], words[2], words[3]);
      dst[1] = make_uint4(words[4], words[5], words[6], words[7]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      float bias = 0.f;
      for (int g = 0; g < nbg; ++g) bias = __fadd_rn(bias, gmin[g]);
      a.lut_scale[qi] = lut_scale;
      a.lut_bias[qi] = bias;
      a.bias_corr[qi] = bias_corr;
      a.fa_init[qi] = __fadd_rn(bias, bias_corr);
    }
  }
}

// One CTA per row: rotated, normalized row written transposed (TQ+ fit).
__global__ void __launch_bounds__(kBigThreads) rotate_rows_t_big_kernel(RotateArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int dim = a.dim;
  float* x = reinterpret_cast<float*>(smem);
  float* y = x + dim;
  __shared__ float red_f[32];
  for (long long v = blockIdx.x; v < a.n; v += gridDim.x) {
    const float* src = a.x + v * static_cast<long long>(dim);
    __syncthreads();
    for (int i = threadIdx.x * 4; i < dim; i += blockDim.x * 4) {
      *reinterpret_cast<float4*>(x + i) = __ldg(reinterpret_cast<const float4*>(src + i));
    }
    __syncthreads();
    const float nrm = block_norm(x, dim, red_f);
    const float inv = (nrm > kMinInputNorm) ? __fdiv_rn(1.f, nrm) : 0.f;
    block_rotate(x, a.perm_sign, dim, a.block, inv, a.inv_sqrt_block, y);
    for (int i = threadIdx.x; i < dim; i += blockDim.x) a.out_t[static_cast<long long>(i) * a.n + v] = y[i];
  }
}

int big_grid(long long rows, int sms) {
  long long g = rows;
  const long long cap = static_cast<long long>(sms) * 4;
  if (g > cap) g = cap;
  return static_cast<int>(g < 1 ? 1 : g);
}

template <typename K>
cudaError_t set_smem(K kernel, size_t bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
}

}  // namespace

cudaError_t launch_encode_big(const EncodeArgs& a, int sms, cudaStream_t stream) {
  if (a.n == 0) return cudaSuccess;
  const size_t smem = static_cast<size_t>(a.dim) * 8;
  cudaError_t e = set_smem(encode_big_kernel, smem);
  if (e != cudaSuccess) return e;
  encode_big_kernel<<<big_grid(a.n, sms), kBigThreads, smem, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_query_prep_big(const QueryPrepArgs& a, int sms, cudaStream_t stream) {
  if (a.nq == 0) return cudaSuccess;
  const size_t smem = static_cast<size_t>(a.dim) * 8 + static_cast<size_t>(a.nbg) * 4;
  cudaError_t e = set_smem(query_prep_big_kernel, smem);
  if (e != cudaSuccess) return e;
  query_prep_big_kernel<<<big_grid(a.nq, sms), kBigThreads, smem, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_rotate_rows_t_big(const RotateArgs& a, int sms, cudaStream_t stream) {
  if (a.n == 0) return cudaSuccess;
  const size_t smem = static_cast<size_t>(a.dim) * 8;
  cudaError_t e = set_smem(rotate_rows_t_big_kernel, smem);
  if (e != cudaSuccess) return e;
  rotate_rows_t_big_kernel<<<big_grid(a.n, sms), kBigThreads, smem, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace vcb
