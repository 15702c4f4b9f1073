// FastScan search on sm_100a: nibble-LUT lookups with integer accumulation,
// f32 flush every 256 byte groups, alpha scaling and an exact top-k with the
// reference's (score desc, id asc) order.
//
// Reference arithmetic: search_avx2.cpp:24-225 (score of one vector),
// topk_heap.hpp:19-157 and search.cpp:600-758 (top-k and merge order).
//
// Scan layout (built by relayout_kernel): 512-vector tiles; for every byte
// group a tile holds 128 u32 words, word w covering vectors 4w..4w+3 with the
// low nibbles (second half of the group's codes) in bits 4j..4j+3 and the high
// nibbles (first half) in bits 16+4j..16+4j+3 for vector j of the word.
//
// Per thread and group, one 8-byte load brings the codes of 8 vectors. Each
// nibble is looked up with prmt.b32 against the 16-byte half of the group's
// LUT held in registers: entries 0..7 come from a prmt on (w), entries 8..15
// from a prmt on (w ^ 0x8888) — a selector nibble >= 8 returns the replicated
// sign of a LUT byte, which is 0 because LUT bytes are <= 127. Four prmt give
// the four per-vector byte sums (<= 254), and dp4a adds each byte into its
// vector's 32-bit accumulator.
#include <cfloat>
#include <climits>

#include "tq_kernels.h"
#include "tq_device.cuh"

namespace vcb {
namespace {

constexpr int kScanWarps = 8;
constexpr int kMergeBuf = 512;  // per-warp sort buffer: 256 new + up to 256 kept

struct __align__(16) LutHalf {
  uint32_t w[4];
};

// Warp-cooperative bitonic sort of p (power of two, <= kMergeBuf) entries in
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

template <int Q, int KMAX>
__global__ void __launch_bounds__(kScanWarps * 32) scan_kernel(ScanArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int nbg = a.nbg;
  const int chunk = a.lut_chunk_groups;
  LutHalf* s_lut = reinterpret_cast<LutHalf*>(smem);  // [Q][chunk][2]
  unsigned char* warp_area = smem + static_cast<size_t>(Q) * chunk * 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t warp_bytes = static_cast<size_t>(Q) * KMAX * 8 + kMergeBuf * 8;
  float* list_s = reinterpret_cast<float*>(warp_area + warp * warp_bytes);
  uint32_t* list_i = reinterpret_cast<uint32_t*>(list_s + Q * KMAX);
  float* buf_s = reinterpret_cast<float*>(list_i + Q * KMAX);
  uint32_t* buf_i = reinterpret_cast<uint32_t*>(buf_s + kMergeBuf);

  const long long q0 = static_cast<long long>(blockIdx.x) * Q;
  const int range = blockIdx.y;
  const long long v_begin = static_cast<long long>(range) * a.range_vectors;
  long long v_end = v_begin + a.range_vectors;
  if (v_end > a.n) v_end = a.n;
  const int k = a.k;

  float scale[Q], init[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const bool ok = q0 + q < a.nq;
    scale[q] = ok ? a.lut_scale[q0 + q] : 0.f;
    init[q] = ok ? a.fa_init[q0 + q] : 0.f;
  }
  float thr_s[Q];
  uint32_t thr_i[Q];
  int cnt[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    thr_s[q] = -FLT_MAX;
    thr_i[q] = 0xffffffffu;
    cnt[q] = 0;
  }

  auto load_lut_chunk = [&](int g_first, int g_count) {
    const int words_per_q = g_count * 2;  // 16-byte halves
    for (int t = threadIdx.x; t < Q * words_per_q; t += blockDim.x) {
      const int q = t / words_per_q, r = t % words_per_q;
      LutHalf h = {{0u, 0u, 0u, 0u}};
      if (q0 + q < a.nq) {
        h = *reinterpret_cast<const LutHalf*>(a.luts + ((q0 + q) * nbg + g_first) * 32LL + r * 16LL);
      }
      s_lut[q * chunk * 2 + r] = h;
    }
  };

  const bool resident = chunk >= nbg;
  if (resident) {
    load_lut_chunk(0, nbg);
    __syncthreads();
  }

  const int half = warp & 1;
  for (long long blk = v_begin; blk < v_end; blk += kScanBlockVectors) {
    const long long tile = blk / kTileVectors + (warp >> 1);
    const uint2* wp = reinterpret_cast<const uint2*>(a.codes + tile * nbg * kTileWords + half * 64) + lane;
    const long long vbase = tile * kTileVectors + half * 256 + 8 * lane;

    float fa[Q][8];
    uint32_t acc[Q][8];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        fa[q][j] = init[q];
        acc[q][j] = 0u;
      }
    }

    for (int gb = 0; gb < nbg; gb += kFlushGroups) {
      const int g_stop = min(gb + kFlushGroups, nbg);
      if (!resident && gb % chunk == 0) {
        __syncthreads();
        load_lut_chunk(gb, min(chunk, nbg - gb));
        __syncthreads();
      }
      const int chunk_base = resident ? 0 : (gb / chunk) * chunk;
      uint2 nxt = wp[static_cast<long long>(gb) * (kTileWords / 2)];
      for (int g = gb; g < g_stop; ++g) {
        const uint2 w = nxt;
        if (g + 1 < g_stop) nxt = wp[static_cast<long long>(g + 1) * (kTileWords / 2)];
        const uint32_t x0 = w.x, x1 = w.y;
        const uint32_t t0 = x0 ^ 0x88888888u, t1 = x1 ^ 0x88888888u;
        const uint32_t x0h = x0 >> 16, x1h = x1 >> 16, t0h = t0 >> 16, t1h = t1 >> 16;
        const LutHalf* lg = s_lut + (g - chunk_base) * 2;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          const LutHalf F = lg[q * chunk * 2];      // entries 0..15: high nibble
          const LutHalf S = lg[q * chunk * 2 + 1];  // entries 16..31: low nibble
          const uint32_t s0 = prmt(S.w[0], S.w[1], x0) + prmt(S.w[2], S.w[3], t0) +
                              prmt(F.w[0], F.w[1], x0h) + prmt(F.w[2], F.w[3], t0h);
          const uint32_t s1 = prmt(S.w[0], S.w[1], x1) + prmt(S.w[2], S.w[3], t1) +
                              prmt(F.w[0], F.w[1], x1h) + prmt(F.w[2], F.w[3], t1h);
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            acc[q][j] = __dp4a(s0, 1u << (8 * j), acc[q][j]);
            acc[q][4 + j] = __dp4a(s1, 1u << (8 * j), acc[q][4 + j]);
          }
        }
      }
      // f32 flush of this batch (search_avx2.cpp:24-48).
#pragma unroll
      for (int q = 0; q < Q; ++q) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          fa[q][j] = __fmaf_rn(scale[q], __uint2float_rn(acc[q][j]), fa[q][j]);
          acc[q][j] = 0u;
        }
      }
    }

    // Scores (fa * alpha) and the warp's running top-k per query.
    float al[8];
    {
      const float4 a0 = *reinterpret_cast<const float4*>(a.alpha + vbase);
      const float4 a1 = *reinterpret_cast<const float4*>(a.alpha + vbase + 4);
      al[0] = a0.x; al[1] = a0.y; al[2] = a0.z; al[3] = a0.w;
      al[4] = a1.x; al[5] = a1.y; al[6] = a1.z; al[7] = a1.w;
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      if (q0 + q >= a.nq) break;  // warp-uniform
      float sc[8];
      unsigned pass = 0;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        sc[j] = __fadd_rn(__fmul_rn(fa[q][j], al[j]), 0.f);
        const long long v = vbase + j;
        const bool ok = v < v_end && v >= v_begin && sc[j] > -INFINITY &&
                        (cnt[q] < k ? true : better(sc[j], static_cast<uint32_t>(v), thr_s[q], thr_i[q]));
        pass |= static_cast<unsigned>(ok) << j;
      }
      const int mine = __popc(pass);
      int incl = mine;
#pragma unroll
      for (int o = 1; o < kWarp; o <<= 1) {
        const int t = __shfl_up_sync(full_mask(), incl, o);
        if (lane >= o) incl += t;
      }
      const int total = __shfl_sync(full_mask(), incl, kWarp - 1);
      if (total == 0) continue;
      int pos = incl - mine;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if (pass >> j & 1u) {
          buf_s[pos] = sc[j];
          buf_i[pos] = static_cast<uint32_t>(vbase + j);
          ++pos;
        }
      }
      float* ls = list_s + q * KMAX;
      uint32_t* li = list_i + q * KMAX;
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

  // Each warp publishes its sorted list per query; the merge kernel combines
  // the n_ranges * 8 lists of a query.
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    if (q0 + q >= a.nq) break;
    const long long list = ((q0 + q) * a.n_ranges + range) * kScanWarps + warp;
    float* os = a.cand_score + list * k;
    uint32_t* oi = a.cand_id + list * k;
    for (int t = lane; t < k; t += kWarp) {
      const bool have = t < cnt[q];
      os[t] = have ? list_s[q * KMAX + t] : -INFINITY;
      oi[t] = have ? list_i[q * KMAX + t] : 0xffffffffu;
    }
  }
}

// One CTA per query: streams the candidate lists in chunks, keeps the best
// k_out (score desc, id asc) in shared memory.
constexpr int kMergeThreads = 256;
constexpr int kMergeChunk = 1024;
constexpr int kMergeCap = 2048;  // >= kMergeChunk + kMaxK, power of two

__device__ void cta_sort_best_first(float* s, uint32_t* id, int p) {
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

__global__ void __launch_bounds__(kMergeThreads) merge_kernel(MergeArgs a) {
  __shared__ float buf_s[kMergeCap];
  __shared__ uint32_t buf_i[kMergeCap];
  __shared__ float best_s[kMaxK];
  __shared__ uint32_t best_i[kMaxK];
  __shared__ int n_new;
  const long long qi = blockIdx.x;
  const long long total = static_cast<long long>(a.n_lists) * a.k;
  const float* cs = a.cand_score + qi * total;
  const uint32_t* ci = a.cand_id + qi * total;
  const int kout = a.k_out;
  int nbest = 0;
  float thr_s = -FLT_MAX;
  uint32_t thr_i = 0xffffffffu;
  for (long long base = 0; base < total; base += kMergeChunk) {
    if (threadIdx.x == 0) n_new = 0;
    __syncthreads();
    for (int t = threadIdx.x; t < kMergeChunk; t += blockDim.x) {
      const long long idx = base + t;
      if (idx < total) {
        const float s = cs[idx];
        const uint32_t id = ci[idx];
        if (s > -INFINITY && (nbest < kout || better(s, id, thr_s, thr_i))) {
          const int pos = atomicAdd(&n_new, 1);
          buf_s[pos] = s;
          buf_i[pos] = id;
        }
      }
    }
    __syncthreads();
    const int fresh = n_new;
    __syncthreads();  // everyone has read n_new before thread 0 resets it
    if (fresh == 0) continue;
    for (int t = threadIdx.x; t < nbest; t += blockDim.x) {
      buf_s[fresh + t] = best_s[t];
      buf_i[fresh + t] = best_i[t];
    }
    const int tot = fresh + nbest;
    int p = 2;
    while (p < tot) p <<= 1;
    for (int t = tot + threadIdx.x; t < p; t += blockDim.x) {
      buf_s[t] = -INFINITY;
      buf_i[t] = 0xffffffffu;
    }
    __syncthreads();
    cta_sort_best_first(buf_s, buf_i, p);
    nbest = min(kout, tot);
    for (int t = threadIdx.x; t < nbest; t += blockDim.x) {
      best_s[t] = buf_s[t];
      best_i[t] = buf_i[t];
    }
    if (nbest == kout) {
      thr_s = buf_s[kout - 1];
      thr_i = buf_i[kout - 1];
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < kout; t += blockDim.x) {
    const bool have = t < nbest;
    a.out_score[qi * kout + t] = have ? best_s[t] : 0.f;
    a.out_id[qi * kout + t] = have ? static_cast<uint64_t>(best_i[t]) : 0ull;
  }
}

// Dense integer / float scores for parity checks: one thread per (query, vector).
__global__ void dense_scores_kernel(const uint32_t* __restrict__ codes, const float* __restrict__ alpha,
                                    const uint8_t* __restrict__ luts, const float* __restrict__ lut_scale,
                                    const float* __restrict__ fa_init, long long n, int nbg, long long nq,
                                    uint32_t* __restrict__ out_int, float* __restrict__ out_score) {
  const long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= n * nq) return;
  const long long qi = idx / n, v = idx % n;
  const long long tile = v / kTileVectors;
  const int wq = static_cast<int>((v % kTileVectors) / 4), j = static_cast<int>(v & 3);
  const uint8_t* lut = luts + qi * nbg * 32LL;
  uint32_t total = 0, batch = 0;
  float fa = fa_init[qi];
  for (int g = 0; g < nbg; ++g) {
    const uint32_t w = codes[(tile * nbg + g) * kTileWords + wq];
    const uint32_t lo = (w >> (4 * j)) & 0xfu, hi = (w >> (16 + 4 * j)) & 0xfu;
    const uint32_t s = lut[g * 32 + hi] + lut[g * 32 + 16 + lo];
    total += s;
    batch += s;
    if ((g + 1) % kFlushGroups == 0 || g + 1 == nbg) {
      fa = __fmaf_rn(lut_scale[qi], __uint2float_rn(batch), fa);
      batch = 0;
    }
  }
  if (out_int) out_int[idx] = total;
  if (out_score) out_score[idx] = __fadd_rn(__fmul_rn(fa, alpha[v]), 0.f);
}

template <int Q, int KMAX>
cudaError_t launch_scan_t(const ScanArgs& a, const ScanPlan& plan, cudaStream_t stream) {
  cudaError_t e = cudaFuncSetAttribute(scan_kernel<Q, KMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(plan.smem_bytes));
  if (e != cudaSuccess) return e;
  dim3 grid(static_cast<unsigned>((a.nq + Q - 1) / Q), static_cast<unsigned>(plan.n_ranges));
  scan_kernel<Q, KMAX><<<grid, kScanWarps * 32, plan.smem_bytes, stream>>>(a);
  return cudaGetLastError();
}

size_t scan_warp_bytes(int q, int kmax) {
  return static_cast<size_t>(q) * kmax * 8 + kMergeBuf * 8;
}

}  // namespace

bool plan_scan(long long n, long long nq, int nbg, int k, int sms, ScanPlan* plan) {
  if (k < 1 || k > kMaxK || n <= 0 || nq <= 0) return false;
  const int kmax = k <= 16 ? 16 : (k <= 64 ? 64 : 256);
  int q = 4;
  if (kmax == 256) q = 2;
  while (q > 1 && nq <= q / 2) q >>= 1;
  const size_t budget = 220 * 1024;
  size_t warp_total = kScanWarps * scan_warp_bytes(q, kmax);
  int chunk = nbg;
  while (static_cast<size_t>(q) * chunk * 32 + warp_total > budget) {
    if (chunk > kFlushGroups) {
      chunk = ((chunk - 1) / kFlushGroups) * kFlushGroups;
      if (chunk < kFlushGroups) chunk = kFlushGroups;
    } else if (q > 1) {
      q >>= 1;
      warp_total = kScanWarps * scan_warp_bytes(q, kmax);
      chunk = nbg;
    } else {
      return false;
    }
  }
  const long long blocks = (n + kScanBlockVectors - 1) / kScanBlockVectors;
  const long long qgroups = (nq + q - 1) / q;
  const long long target = static_cast<long long>(sms) * 4;
  long long ranges = (target + qgroups - 1) / qgroups;
  if (ranges < 1) ranges = 1;
  if (ranges > blocks) ranges = blocks;
  if (ranges > 65535) ranges = 65535;
  const long long blocks_per_range = (blocks + ranges - 1) / ranges;
  ranges = (blocks + blocks_per_range - 1) / blocks_per_range;
  plan->q_per_cta = q;
  plan->kmax = kmax;
  plan->range_vectors = blocks_per_range * kScanBlockVectors;
  plan->n_ranges = static_cast<int>(ranges);
  plan->lut_chunk_groups = chunk;
  plan->smem_bytes = static_cast<size_t>(q) * chunk * 32 + warp_total;
  return true;
}

cudaError_t launch_scan(const ScanArgs& a, const ScanPlan& plan, cudaStream_t stream) {
  const int q = plan.q_per_cta, km = plan.kmax;
#define VCB_SCAN(QQ, KK) \
  if (q == QQ && km == KK) return launch_scan_t<QQ, KK>(a, plan, stream);
  VCB_SCAN(1, 16) VCB_SCAN(2, 16) VCB_SCAN(4, 16)
  VCB_SCAN(1, 64) VCB_SCAN(2, 64) VCB_SCAN(4, 64)
  VCB_SCAN(1, 256) VCB_SCAN(2, 256)
#undef VCB_SCAN
  return cudaErrorInvalidValue;
}

cudaError_t launch_merge(const MergeArgs& a, cudaStream_t stream) {
  if (a.nq == 0 || a.k_out == 0) return cudaSuccess;
  merge_kernel<<<static_cast<unsigned>(a.nq), kMergeThreads, 0, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_dense_scores(const uint32_t* codes, const float* alpha, const uint8_t* luts,
                                const float* lut_scale, const float* fa_init, long long n, int nbg,
                                long long nq, uint32_t* out_int, float* out_score,
                                cudaStream_t stream) {
  const long long total = n * nq;
  if (total == 0) return cudaSuccess;
  dense_scores_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, stream>>>(
      codes, alpha, luts, lut_scale, fa_init, n, nbg, nq, out_int, out_score);
  return cudaGetLastError();
}

}  // namespace vcb
