// Exact float inner-product re-rank of a top-k result, in place
// (the reference's float_rescore_topk, src/search/float_rescore.cpp:80-164).
//
// Each score is the reference's AVX2 dot product (float_rescore.cpp:34-58):
// 16 sequential fused multiply-add chains (element i feeds chain i % 16 while
// i < dim - dim % 16), chains 8..15 added into 0..7, an 8-wide tail when dim %
// 16 == 8, then the horizontal sum ((c0+c4)+(c1+c5))+((c2+c6)+(c3+c7)).
// Candidates are then re-sorted: higher score first, equal scores by lower id;
// an id outside the corpus scores -inf (float_rescore.cpp:118-124, :140-150).
#include <cfloat>

#include "tq_kernels.h"
#include "tq_device.cuh"

namespace vcb {
namespace {

constexpr int kRescoreThreads = 256;

// Half-warp h (lanes 16h..16h+15) scores one candidate; lane l of the half owns
// chain l. Returns the dot product on lane 16h.
__device__ __forceinline__ float dot_reference_order(const float* __restrict__ q, const float* __restrict__ c,
                                                     int dim, int lane) {
  const int l = lane & 15;
  const int main_end = dim - (dim % 16);
  float acc = 0.f;
  for (int i = l; i < main_end; i += 16) acc = __fmaf_rn(__ldg(q + i), __ldg(c + i), acc);
  // chains 8..15 into 0..7
  const float hi = __shfl_down_sync(full_mask(), acc, 8, 16);
  if (l < 8) acc = __fadd_rn(acc, hi);
  if (dim % 16 == 8 && l < 8) acc = __fmaf_rn(__ldg(q + main_end + l), __ldg(c + main_end + l), acc);
  // ((a0+a4)+(a1+a5)) + ((a2+a6)+(a3+a7))
  const float b = __fadd_rn(acc, __shfl_down_sync(full_mask(), acc, 4, 16));   // l<4: a_l + a_{l+4}
  const float c2 = __fadd_rn(b, __shfl_down_sync(full_mask(), b, 1, 16));      // l=0: b0+b1, l=2: b2+b3
  return __fadd_rn(c2, __shfl_down_sync(full_mask(), c2, 2, 16));              // l=0: (b0+b1)+(b2+b3)
}

__global__ void __launch_bounds__(kRescoreThreads) rescore_kernel(const float* __restrict__ queries, long long nq,
                                                                  int dim, const float* __restrict__ corpus,
                                                                  long long n_corpus, int k, float* scores,
                                                                  uint64_t* ids) {
  extern __shared__ __align__(16) unsigned char smem[];
  const long long qi = blockIdx.x;
  if (qi >= nq) return;
  int p = 2;
  while (p < k) p <<= 1;
  float* s = reinterpret_cast<float*>(smem);
  uint64_t* id = reinterpret_cast<uint64_t*>(smem + ((static_cast<size_t>(p) * 4 + 15) / 16) * 16);
  const float* q = queries + qi * static_cast<long long>(dim);
  float* row_s = scores + qi * k;
  uint64_t* row_i = ids + qi * k;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int halves = (blockDim.x >> 5) * 2;
  for (int j0 = warp * 2; j0 < k; j0 += halves) {
    const int j = j0 + (lane >> 4);
    const bool have = j < k;
    const uint64_t cid = have ? row_i[j] : 0;
    const bool in = have && cid < static_cast<uint64_t>(n_corpus);
    const float* c = in ? corpus + static_cast<long long>(cid) * dim : q;  // q: any readable row
    const float d = dot_reference_order(q, c, dim, lane);
    if (have && (lane & 15) == 0) {
      s[j] = in ? d : -INFINITY;
      id[j] = cid;
    }
  }
  for (int t = k + threadIdx.x; t < p; t += blockDim.x) {
    s[t] = -INFINITY;
    id[t] = ~0ull;
  }
  __syncthreads();
  // Bitonic sort, best first: score descending, then id ascending.
  for (int size = 2; size <= p; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int t = threadIdx.x; t < (p >> 1); t += blockDim.x) {
        const int i = (t / stride) * 2 * stride + (t % stride);
        const int jj = i + stride;
        const bool up = (i & size) == 0;
        const float si = s[i], sj = s[jj];
        const uint64_t ii = id[i], ij = id[jj];
        const bool j_better = (sj > si) || (sj == si && ij < ii);
        if (j_better == up) {
          s[i] = sj;
          s[jj] = si;
          id[i] = ij;
          id[jj] = ii;
        }
      }
      __syncthreads();
    }
  }
  for (int t = threadIdx.x; t < k; t += blockDim.x) {
    row_s[t] = s[t];
    row_i[t] = id[t];
  }
}

}  // namespace

size_t rescore_smem_bytes(int k) {
  int p = 2;
  while (p < k) p <<= 1;
  return ((static_cast<size_t>(p) * 4 + 15) / 16) * 16 + static_cast<size_t>(p) * 8;
}

cudaError_t launch_rescore(const float* queries, long long nq, int dim, const float* corpus, long long n_corpus,
                           int k, float* scores, uint64_t* ids, cudaStream_t stream) {
  if (nq == 0 || k == 0) return cudaSuccess;
  const size_t smem = rescore_smem_bytes(k);
  cudaError_t e = cudaFuncSetAttribute(rescore_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  rescore_kernel<<<static_cast<unsigned>(nq), kRescoreThreads, smem, stream>>>(queries, nq, dim, corpus, n_corpus,
                                                                               k, scores, ids);
  return cudaGetLastError();
}

}  // namespace vcb
