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
#include <algorithm>
#include <cfloat>
#include <climits>
#include <type_traits>

#include "tq_kernels.h"
#include "tq_device.cuh"

namespace vcb {
namespace {

constexpr int kScanWarps = 8;
constexpr int kMergeBuf = 512;  // per-warp sort buffer: 256 new + up to 256 kept
constexpr int kRegTopK = 32;    // k up to this is kept in registers, one entry per lane

// Running top-k of one warp for one query, one entry per lane (k <= 32),
// sorted best first; empty slots hold (-inf, 0xffffffff).
struct RegTopK {
  float s = -INFINITY;
  uint32_t i = 0xffffffffu;
  float thr_s = -INFINITY;  // entry k-1
  uint32_t thr_i = 0xffffffffu;

  __device__ __forceinline__ void insert(float cs, uint32_t ci, int k, int lane) {
    const unsigned ahead = __ballot_sync(full_mask(), lane < k && better(s, i, cs, ci));
    const int pos = __popc(ahead);
    const float up_s = __shfl_up_sync(full_mask(), s, 1);
    const uint32_t up_i = __shfl_up_sync(full_mask(), i, 1);
    if (lane > pos) {
      s = up_s;
      i = up_i;
    } else if (lane == pos) {
      s = cs;
      i = ci;
    }
    thr_s = __shfl_sync(full_mask(), s, k - 1);
    thr_i = __shfl_sync(full_mask(), i, k - 1);
  }

  // Offer the 8 scores of every lane (vectors vbase..vbase+7 of that lane).
  __device__ __forceinline__ void offer(const float (&sc)[8], unsigned valid, uint32_t vbase, int k,
                                        int lane) {
    unsigned pass = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if ((valid >> j & 1u) && better(sc[j], vbase + j, thr_s, thr_i)) pass |= 1u << j;
    }
    if (!(thr_s > -INFINITY)) {
      // List not full yet (first block): a lane maximum ranked k-th among the
      // 32 lane maxima is a lower bound of the k-th best score, so anything
      // strictly below it cannot enter the final top-k.
      float mx = -INFINITY;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if (pass >> j & 1u) mx = fmaxf(mx, sc[j]);
      }
      const float bound = warp_kth_largest(mx, k, lane);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if ((pass >> j & 1u) && sc[j] < bound) pass &= ~(1u << j);
      }
    }
    unsigned any = __ballot_sync(full_mask(), pass != 0);
    while (any) {
      const int src = __ffs(any) - 1;
      const int my_j = __ffs(pass) - 1;
      float my_s = sc[0];
#pragma unroll
      for (int j = 1; j < 8; ++j) {
        if (j == my_j) my_s = sc[j];
      }
      const int j = __shfl_sync(full_mask(), my_j, src);
      const float cs = __shfl_sync(full_mask(), my_s, src);
      const uint32_t ci = __shfl_sync(full_mask(), vbase, src) + static_cast<uint32_t>(j);
      if (lane == src) pass &= pass - 1;
      any = __ballot_sync(full_mask(), pass != 0);
      if (better(cs, ci, thr_s, thr_i)) insert(cs, ci, k, lane);
    }
  }

  // offer() for candidates with arbitrary ids (merging candidate lists).
  __device__ __forceinline__ void offer_ids(const float (&sc)[8], const uint32_t (&id)[8], unsigned valid, int k,
                                            int lane) {
    unsigned pass = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if ((valid >> j & 1u) && better(sc[j], id[j], thr_s, thr_i)) pass |= 1u << j;
    }
    if (!(thr_s > -INFINITY)) {
      float mx = -INFINITY;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if (pass >> j & 1u) mx = fmaxf(mx, sc[j]);
      }
      const float bound = warp_kth_largest(mx, k, lane);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if ((pass >> j & 1u) && sc[j] < bound) pass &= ~(1u << j);
      }
    }
    unsigned any = __ballot_sync(full_mask(), pass != 0);
    while (any) {
      const int src = __ffs(any) - 1;
      const int my_j = __ffs(pass) - 1;
      float my_s = sc[0];
      uint32_t my_i = id[0];
#pragma unroll
      for (int j = 1; j < 8; ++j) {
        if (j == my_j) {
          my_s = sc[j];
          my_i = id[j];
        }
      }
      const float cs = __shfl_sync(full_mask(), my_s, src);
      const uint32_t ci = __shfl_sync(full_mask(), my_i, src);
      if (lane == src) pass &= pass - 1;
      any = __ballot_sync(full_mask(), pass != 0);
      if (better(cs, ci, thr_s, thr_i)) insert(cs, ci, k, lane);
    }
  }
};

// Staged code stream: group rows per slot, and slots per warp by queries per
// CTA (shared memory: 8 warps x slots x 8 rows x 256 bytes = 96 KB at one
// query, 80 KB at two, beside the LUTs, two CTAs per SM).
constexpr int kStageGroups = 8;
constexpr int stages_for(int q) { return q == 1 ? 6 : 5; }
// Byte offset of the slots: after the LUT area, which the register top-k's
// end-of-range merge also uses (Q x 8 warps x 32 lanes x 8 bytes).
__host__ __device__ constexpr size_t scan_stage_offset(int q, int chunk) {
  return static_cast<size_t>(q) * chunk * 32 > static_cast<size_t>(q) * kScanWarps * 32 * 8
             ? static_cast<size_t>(q) * chunk * 32
             : static_cast<size_t>(q) * kScanWarps * 32 * 8;
}
constexpr size_t scan_stage_bytes(int q) {
  return static_cast<size_t>(kScanWarps) * stages_for(q) * kStageGroups * 256;
}

// PF: byte groups of codes in flight per thread. Few queries per CTA leave
// the kernel memory-bound, where a deeper ring keeps more bytes in flight.
// MODE 0 scans every byte group and keeps the top k. For one or two queries
// over an index of few blocks, the work splits by 256-group batch instead:
// MODE 1 scans only batch blockIdx.z of one block and stores the integer sums
// in a.partial; MODE 2 then flushes those sums in batch order (the same f32
// arithmetic as MODE 0) and keeps the top k, without lookups. MODE 3 is MODE 1
// followed, in the CTA that stores a block's last batch (a counter per block,
// threadfence-reduction style, no waiting), by MODE 2 for that block.
//
// STAGES > 0 (whole-row scans of one or two queries, k <= 32, nbg a multiple
// of PF): the code stream reaches the lookups through shared memory instead of
// a register ring. Each warp owns STAGES slots of PF group rows (its 256-byte half of a
// tile row each), filled by 16-byte cp.async copies STAGES - 1 slots ahead of
// the lookups; the bytes in flight no longer cost registers, so a memory-bound
// scan keeps more of them in flight (a wait_group and a __syncwarp per slot,
// no spin loop).
template <int Q, int KMAX, int MIN_BLOCKS, bool NIBBLE8, int PF, int MODE = 0, int STAGES = 0, bool WHOLE = false>
__global__ void __launch_bounds__(kScanWarps * 32, MIN_BLOCKS) scan_kernel(ScanArgs a) {
  static_assert(PF % 2 == 0, "byte groups are consumed in pairs");
  static_assert(STAGES == 0 || (STAGES >= 2 && KMAX <= kRegTopK && MODE == 0),
                "staged code stream: register top-k, whole-row scans");
  constexpr bool kReg = KMAX <= kRegTopK;
  extern __shared__ __align__(16) unsigned char smem[];
  const int nbg = a.nbg;
  const int chunk = a.lut_chunk_groups;
  LutHalf* s_lut = reinterpret_cast<LutHalf*>(smem);  // [Q][chunk][2]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  [[maybe_unused]] uint2* s_stage = nullptr;  // this warp's STAGES x PF rows of 32 uint2
  if constexpr (STAGES > 0) {
    s_stage = reinterpret_cast<uint2*>(smem + scan_stage_offset(Q, chunk)) + warp * (STAGES * PF * 32);
  }

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

  // Top-k state: registers for k <= 32, shared memory lists otherwise.
  RegTopK top[kReg ? Q : 1];
  float thr_s[Q];
  uint32_t thr_i[Q];
  int cnt[Q];
  float* list_s = nullptr;
  uint32_t* list_i = nullptr;
  float* buf_s = nullptr;
  uint32_t* buf_i = nullptr;
  if constexpr (!kReg) {
    unsigned char* warp_area = smem + static_cast<size_t>(Q) * chunk * 32;
    const size_t warp_bytes = static_cast<size_t>(Q) * KMAX * 8 + kMergeBuf * 8;
    list_s = reinterpret_cast<float*>(warp_area + warp * warp_bytes);
    list_i = reinterpret_cast<uint32_t*>(list_s + Q * KMAX);
    buf_s = reinterpret_cast<float*>(list_i + Q * KMAX);
    buf_i = reinterpret_cast<uint32_t*>(buf_s + kMergeBuf);
  }
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

  // Byte groups this CTA scans: all (MODE 0), one batch (MODE 1), none (MODE 2).
  constexpr bool kBatch = MODE == 1 || MODE == 3;  // scans one 256-group batch
  const int g_first = kBatch ? static_cast<int>(blockIdx.z) * kFlushGroups : 0;
  const int g_last = kBatch ? min(g_first + kFlushGroups, nbg) : (MODE == 2 ? 0 : nbg);
  const bool resident = MODE != 0 || chunk >= nbg;
  constexpr long long kGroupStride = kTileWords / 2;  // uint2 per group row
  if constexpr (kBatch) {
    load_lut_chunk(g_first, g_last - g_first);
    __syncthreads();
  } else if constexpr (MODE == 0) {
    if (resident) {
      load_lut_chunk(0, nbg);
      __syncthreads();
    }
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

    // Staged stream: slot st holds group rows g_first + st * PF .. + PF - 1.
    [[maybe_unused]] int st = 0;
    [[maybe_unused]] const int n_st = (g_last - g_first) / PF;
    [[maybe_unused]] auto issue = [&](int s_idx) {
      if constexpr (STAGES > 0) {
        if (s_idx < n_st) {
          const uint2* src = (wp - lane) + static_cast<long long>(g_first + s_idx * PF) * kGroupStride;
          uint2* dst = s_stage + (s_idx % STAGES) * (PF * 32);
#pragma unroll
          for (int i = 0; i < PF / 2; ++i) {
            const int c = lane + 32 * i;  // 16-byte chunk c: row c / 16, bytes 16 * (c % 16)
            cp_async16(dst + (c >> 4) * 32 + (c & 15) * 2, src + (c >> 4) * kGroupStride + (c & 15) * 2);
          }
        }
        cp_async_commit();  // empty groups past the end keep the wait counts uniform
      }
    };
    if constexpr (STAGES > 0) {
      __syncwarp();  // every lane is done reading the previous block's slots
#pragma unroll
      for (int s0 = 0; s0 < STAGES - 1; ++s0) issue(s0);
    }

    for (int gb = g_first; gb < g_last; gb += kFlushGroups) {
      const int g_stop = min(gb + kFlushGroups, nbg);
      if (!resident && gb % chunk == 0) {
        __syncthreads();
        load_lut_chunk(gb, min(chunk, nbg - gb));
        __syncthreads();
      }
      const int chunk_base = kBatch ? g_first : (resident ? 0 : (gb / chunk) * chunk);
      // The lookups of PF code groups held in `cur`, starting at group g
      // (CHECKED: only those below g_stop), in pairs of byte groups (nbg and
      // every 256-group batch are even).
      auto process = [&](const uint2 (&cur)[PF], int g, auto checked) {
#pragma unroll
        for (int u = 0; u < PF; u += 2) {
          if constexpr (decltype(checked)::value) {
            if (g + u >= g_stop) break;
          }
          lookup_group_pair<Q, NIBBLE8, (Q >= 4 && !NIBBLE8 && kReg)>(cur[u], cur[u + 1],
                                                                     s_lut + (g + u - chunk_base) * 2, chunk * 2,
                                                                     acc);
        }
      };
      if constexpr (STAGES > 0) {
        for (int g = gb; g < g_stop; g += PF, ++st) {
          cp_async_wait<STAGES - 2>();  // slot st has landed (this lane's copies)
          __syncwarp();                 // ... and every lane's; slot st - 1 is free
          issue(st + STAGES - 1);
          const uint2* slot = s_stage + (st % STAGES) * (PF * 32) + lane;
          uint2 cur[PF];
#pragma unroll
          for (int u = 0; u < PF; ++u) cur[u] = slot[u * 32];
          process(cur, g, std::false_type{});
        }
      } else {
        uint2 ring[PF];
        // Whole rings (every batch a multiple of PF groups) run without bounds
        // checks, loading at immediate offsets of a running pointer: one or two
        // queries decide per batch; four queries take the WHOLE instance
        // (launched when nbg is a multiple of PF), which holds no checked copy
        // of the lookup body — both copies do not fit their 128 registers.
        // At 10k queries x 1M x 1536 the unchecked ring scans in 870.0 ms,
        // the checked one in 992.7 ms (same 4-group ring).
        if (WHOLE || (Q <= 2 && (g_stop - gb) % PF == 0)) {
          const uint2* src = wp + static_cast<long long>(gb) * kGroupStride;
#pragma unroll
          for (int u = 0; u < PF; ++u) ring[u] = src[u * kGroupStride];
          src += PF * kGroupStride;
          int g = gb;
          for (; g + PF < g_stop; g += PF) {
            uint2 cur[PF];
#pragma unroll
            for (int u = 0; u < PF; ++u) {
              cur[u] = ring[u];
              ring[u] = src[u * kGroupStride];
            }
            src += PF * kGroupStride;
            process(cur, g, std::false_type{});
          }
          process(ring, g, std::false_type{});
        } else {
#pragma unroll
          for (int u = 0; u < PF; ++u) {
            ring[u] = (gb + u < g_stop) ? wp[(gb + u) * kGroupStride] : make_uint2(0u, 0u);
          }
          for (int g = gb; g < g_stop; g += PF) {
            uint2 cur[PF];
#pragma unroll
            for (int u = 0; u < PF; ++u) {
              cur[u] = ring[u];
              const int gn = g + PF + u;
              ring[u] = (gn < g_stop) ? wp[gn * kGroupStride] : make_uint2(0u, 0u);
            }
            process(cur, g, std::true_type{});
          }
        }
      }
      // f32 flush of this batch (search_avx2.cpp:24-48).
      if constexpr (MODE == 0) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            fa[q][j] = __fmaf_rn(scale[q], __uint2float_rn(acc[q][j]), fa[q][j]);
            acc[q][j] = 0u;
          }
        }
      }
    }
    if constexpr (kBatch) {
      // The batch's integer sums of this lane's 8 vectors, for the flush.
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        if (q0 + q >= a.nq) break;
        uint4* dst = reinterpret_cast<uint4*>(
            a.partial + ((q0 + q) * a.partial_batches + blockIdx.z) * a.partial_stride + vbase);
        dst[0] = make_uint4(acc[q][0], acc[q][1], acc[q][2], acc[q][3]);
        dst[1] = make_uint4(acc[q][4], acc[q][5], acc[q][6], acc[q][7]);
      }
      if constexpr (MODE == 1) continue;
      if constexpr (MODE == 3) {
        // Publish the sums, then count this batch in; only the CTA that
        // completes the block goes on (no CTA ever waits for another).
        __shared__ unsigned s_last;
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
          unsigned* c = a.arrive + static_cast<long long>(blockIdx.x) * gridDim.y + blockIdx.y;
          s_last = atomicAdd(c, 1u) == static_cast<unsigned>(a.partial_batches - 1) ? 1u : 0u;
        }
        __syncthreads();
        if (!s_last) return;
        __threadfence();
      }
    }
    if constexpr (MODE == 2 || MODE == 3) {
      // The same flushes as MODE 0, batch by batch in order, from the stored
      // sums (read past L1: other CTAs wrote them).
      for (int b = 0; b < a.partial_batches; ++b) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          uint4 s0 = make_uint4(0u, 0u, 0u, 0u), s1 = s0;
          if (q0 + q < a.nq) {
            const uint4* src = reinterpret_cast<const uint4*>(
                a.partial + ((q0 + q) * a.partial_batches + b) * a.partial_stride + vbase);
            s0 = __ldcg(src);
            s1 = __ldcg(src + 1);
          }
          const uint32_t sv[8] = {s0.x, s0.y, s0.z, s0.w, s1.x, s1.y, s1.z, s1.w};
#pragma unroll
          for (int j = 0; j < 8; ++j) fa[q][j] = __fmaf_rn(scale[q], __uint2float_rn(sv[j]), fa[q][j]);
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
    unsigned valid = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const long long v = vbase + j;
      if (v < v_end) valid |= 1u << j;
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      if (q0 + q >= a.nq) break;  // warp-uniform
      float sc[8];
      unsigned ok_mask = 0;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        sc[j] = __fadd_rn(__fmul_rn(fa[q][j], al[j]), 0.f);
        if ((valid >> j & 1u) && sc[j] > -INFINITY) ok_mask |= 1u << j;
      }
      if constexpr (kReg) {
        top[q].offer(sc, ok_mask, static_cast<uint32_t>(vbase), k, lane);
      } else {
        unsigned pass = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const bool ok = (ok_mask >> j & 1u) &&
                          (cnt[q] < k ? true : better(sc[j], static_cast<uint32_t>(vbase + j), thr_s[q], thr_i[q]));
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
  }

  if constexpr (MODE == 1) return;  // sums only; MODE 2 keeps the top k
  if constexpr (kReg) {
    // The CTA merges its 8 warp lists of each query in shared memory (the LUT
    // area is free now) and publishes one list per (query, range).
    __syncthreads();
    float* m_s = reinterpret_cast<float*>(smem);  // [Q][8 warps x 32]
    uint32_t* m_i = reinterpret_cast<uint32_t*>(m_s + Q * kScanWarps * kWarp);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int slot = (q * kScanWarps + warp) * kWarp + lane;
      m_s[slot] = lane < k ? top[q].s : -INFINITY;
      m_i[slot] = lane < k ? top[q].i : 0xffffffffu;
    }
    __syncthreads();
    for (int q = warp; q < Q; q += kScanWarps) {
      if (q0 + q >= a.nq) break;
      float* qs = m_s + q * kScanWarps * kWarp;
      uint32_t* qi = m_i + q * kScanWarps * kWarp;
      warp_sort_best_first(qs, qi, kScanWarps * kWarp, lane);
      const long long list = (q0 + q) * a.n_ranges + range;
      if (lane < k) {
        a.cand_score[list * k + lane] = qs[lane];
        a.cand_id[list * k + lane] = qi[lane];
      }
    }
  } else {
    // Shared-memory lists (k > 32): each warp publishes its own sorted list;
    // the merge kernel combines the n_ranges * 8 lists of a query.
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
  const long long stride = static_cast<long long>(a.list_stride ? a.list_stride : a.n_lists) * a.k;
  const long long total = a.entry_count ? static_cast<long long>(a.entry_count[qi])
                                        : static_cast<long long>(a.n_lists) * a.k;
  const float* cs = a.cand_score + qi * stride;
  const uint32_t* ci = a.cand_id + qi * stride;
  const int kout = a.k_out;
  int nbest = 0;
  float thr_s = -FLT_MAX;
  uint32_t thr_i = 0xffffffffu;
  constexpr int kPer = kMergeChunk / kMergeThreads;
  for (long long base = 0; base < total; base += kMergeChunk) {
    // Scores first: a chunk with nothing at or above the current k-th best
    // (padding, or candidates of far probes) costs one barrier.
    float s[kPer];
    bool any = false;
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const long long v = base + threadIdx.x + u * kMergeThreads;
      s[u] = v < total ? cs[v] : -INFINITY;
      any |= s[u] > -INFINITY && (nbest < kout || !(s[u] < thr_s));
    }
    if (!__syncthreads_or(any)) continue;
    if (threadIdx.x == 0) n_new = 0;
    __syncthreads();
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      if (s[u] > -INFINITY && (nbest < kout || !(s[u] < thr_s))) {
        const uint32_t id = ci[base + threadIdx.x + u * kMergeThreads];
        if (nbest < kout || better(s[u], id, thr_s, thr_i)) {
          const int pos = atomicAdd(&n_new, 1);
          buf_s[pos] = s[u];
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
    a.out_id[qi * kout + t] = have ? static_cast<uint64_t>(best_i[t]) : a.pad_id;
  }
}

// k_out <= 32: one CTA per query, every warp keeps a register top-k over a
// strided share of the candidates (8 consecutive entries per lane, the
// first-block prefilter bounds the work), then one warp merges the 8 lists.
// Same result as merge_kernel: best k_out by (score desc, id asc), -inf and
// NaN never admitted, unfilled slots (0, pad_id).
__global__ void __launch_bounds__(kMergeThreads) merge_reg_kernel(MergeArgs a) {
  constexpr int kWarps = kMergeThreads / kWarp;
  __shared__ float m_s[kMergeThreads];
  __shared__ uint32_t m_i[kMergeThreads];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long qi = blockIdx.x;
  const long long stride = static_cast<long long>(a.list_stride ? a.list_stride : a.n_lists) * a.k;
  const long long total = a.entry_count ? static_cast<long long>(a.entry_count[qi])
                                        : static_cast<long long>(a.n_lists) * a.k;
  const float* cs = a.cand_score + qi * stride;
  const uint32_t* ci = a.cand_id + qi * stride;
  const int kout = a.k_out;
  // Warps that receive candidates (one warp covers 256 per round); the same
  // value in every thread of the CTA.
  const int active = static_cast<int>(min(static_cast<long long>(kWarps), (total + kWarp * 8 - 1) / (kWarp * 8)));
  RegTopK top;
  for (long long base = static_cast<long long>(warp) * kWarp * 8; warp < active && base < total;
       base += static_cast<long long>(kWarps) * kWarp * 8) {
    float sc[8];
    uint32_t id[8];
    unsigned ok = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const long long idx = base + lane * 8 + j;
      sc[j] = -INFINITY;
      id[j] = 0xffffffffu;
      if (idx < total) {
        sc[j] = cs[idx];
        id[j] = ci[idx];
        if (sc[j] > -INFINITY) ok |= 1u << j;
      }
    }
    top.offer_ids(sc, id, ok, kout, lane);
  }
  if (active <= 1) {
    // Warp 0's list (sorted best first) is the answer.
    if (warp == 0 && lane < kout) {
      const bool have = top.s > -INFINITY;
      a.out_score[qi * kout + lane] = have ? top.s : 0.f;
      a.out_id[qi * kout + lane] = have ? static_cast<uint64_t>(top.i) : a.pad_id;
    }
    return;  // taken by the whole CTA (active is CTA-uniform)
  }
  m_s[threadIdx.x] = lane < kout ? top.s : -INFINITY;
  m_i[threadIdx.x] = lane < kout ? top.i : 0xffffffffu;
  __syncthreads();
  if (warp == 0) {
    int p = kWarp * 2;
    while (p < kWarp * active) p <<= 1;  // lists of warps >= active are all empty
    warp_sort_best_first(m_s, m_i, p, lane);
    if (lane < kout) {
      const bool have = m_s[lane] > -INFINITY;
      a.out_score[qi * kout + lane] = have ? m_s[lane] : 0.f;
      a.out_id[qi * kout + lane] = have ? static_cast<uint64_t>(m_i[lane]) : a.pad_id;
    }
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

template <int Q, int KMAX, int MINB, bool N8, int PF, int STAGES = 0, bool WHOLE = false>
cudaError_t launch_scan_t(const ScanArgs& a, const ScanPlan& plan, cudaStream_t stream) {
  auto kern = scan_kernel<Q, KMAX, MINB, N8, PF, 0, STAGES, WHOLE>;
  cudaError_t e =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(plan.smem_bytes));
  if (e != cudaSuccess) return e;
  dim3 grid(static_cast<unsigned>((a.nq + Q - 1) / Q), static_cast<unsigned>(plan.n_ranges));
  kern<<<grid, kScanWarps * 32, plan.smem_bytes, stream>>>(a);
  return cudaGetLastError();
}

// Prefetch depth per queries-per-CTA: the one-query kernel is memory-bound and
// keeps 16 byte groups in flight per thread; the 4-query kernel is issue-bound
// and keeps 8 (10k queries x 1M x 1536 with the unchecked ring: 4 groups
// 870.0 ms, 8 groups 853.3 ms, 16 groups 935.4 ms, register spills).
constexpr int prefetch_for(int q) { return q == 1 ? 16 : (q == 2 ? 8 : 8); }

// Batch-split scan: (block, batch) CTAs store integer sums, then one CTA per
// (query group, range) flushes them in batch order and keeps the top k.
template <int Q, bool N8, int PF, int MINB>
cudaError_t launch_split_mode(const ScanArgs& a, const ScanPlan& plan, cudaStream_t stream, long long blocks) {
  const unsigned qgroups = static_cast<unsigned>((a.nq + Q - 1) / Q);
  ScanArgs s = a;
  s.range_vectors = kScanBlockVectors;
  s.n_ranges = static_cast<int>(blocks);
  s.lut_chunk_groups = kFlushGroups;
  s.partial_batches = plan.split_batches;
  const size_t smem1 = static_cast<size_t>(Q) * kFlushGroups * 32;
  if (a.arrive && plan.n_ranges == blocks) {
    // One launch: the CTA completing a block flushes it (its lists are the
    // plan's ranges, one block each). The LUT area also holds the merge.
    const size_t smem3 = std::max(smem1, static_cast<size_t>(Q) * kScanWarps * kWarp * 8);
    cudaError_t e3 = cudaFuncSetAttribute(scan_kernel<Q, kRegTopK, MINB, N8, PF, 3>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem3));
    if (e3 != cudaSuccess) return e3;
    scan_kernel<Q, kRegTopK, MINB, N8, PF, 3><<<dim3(qgroups, static_cast<unsigned>(blocks),
                                                   static_cast<unsigned>(plan.split_batches)),
                                              kScanWarps * 32, smem3, stream>>>(s);
    return cudaGetLastError();
  }
  cudaError_t e = cudaFuncSetAttribute(scan_kernel<Q, kRegTopK, MINB, N8, PF, 1>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem1));
  if (e != cudaSuccess) return e;
  scan_kernel<Q, kRegTopK, MINB, N8, PF, 1><<<dim3(qgroups, static_cast<unsigned>(blocks),
                                                 static_cast<unsigned>(plan.split_batches)),
                                            kScanWarps * 32, smem1, stream>>>(s);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  ScanArgs c = a;
  c.partial_batches = plan.split_batches;
  const size_t smem2 = static_cast<size_t>(Q) * kScanWarps * kWarp * 8;  // the top-k merge area
  e = cudaFuncSetAttribute(scan_kernel<Q, kRegTopK, MINB, N8, PF, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(smem2));
  if (e != cudaSuccess) return e;
  scan_kernel<Q, kRegTopK, MINB, N8, PF, 2><<<dim3(qgroups, static_cast<unsigned>(plan.n_ranges)), kScanWarps * 32,
                                            smem2, stream>>>(c);
  return cudaGetLastError();
}

template <int Q, bool N8>
cudaError_t launch_split_t(const ScanArgs& a, const ScanPlan& plan, cudaStream_t stream) {
  constexpr int kPf = prefetch_for(Q);
  const long long blocks = (a.n + kScanBlockVectors - 1) / kScanBlockVectors;
  if (Q == 1 && plan.split_ctas_per_sm == 4) {
    // One query, four CTAs per SM: 8 groups in flight within 64 registers.
    return launch_split_mode<1, N8, 8, 4>(a, plan, stream, blocks);
  }
  return launch_split_mode<Q, N8, kPf, 2>(a, plan, stream, blocks);
}

size_t scan_warp_bytes(int q, int kmax) {
  if (kmax <= kRegTopK) return 0;
  return static_cast<size_t>(q) * kmax * 8 + kMergeBuf * 8;
}

}  // namespace

bool plan_scan(long long n, long long nq, int nbg, int k, int sms, ScanPlan* plan, long long max_range_vectors,
               int bits) {
  if (k < 1 || k > kMaxK || n <= 0 || nq <= 0) return false;
  const int kmax = k <= kRegTopK ? kRegTopK : (k <= 64 ? 64 : 256);
  const bool reg = kmax <= kRegTopK;
  // Register top-k leaves shared memory to the LUTs: two CTAs per SM.
  const size_t budget = reg ? 110 * 1024 : 220 * 1024;
  int q = (kmax == 256) ? 2 : 4;
  while (q > 1 && nq <= q / 2) q >>= 1;
  // Prefer fewer queries per CTA over streaming the LUT in chunks.
  while (q > 1 && static_cast<size_t>(q) * nbg * 32 + kScanWarps * scan_warp_bytes(q, kmax) > budget &&
         static_cast<size_t>(q / 2) * nbg * 32 + kScanWarps * scan_warp_bytes(q / 2, kmax) <= budget) {
    q >>= 1;
  }
  const size_t warp_total = kScanWarps * scan_warp_bytes(q, kmax);
  // One or two queries with the register top-k stream the codes through
  // shared-memory slots (nbg a multiple of the slot rows); the slots share
  // the CTA's budget with the LUTs. One query over 2- or 4-bit codes instead
  // keeps an 8-group register ring on four CTAs per SM (one query, 4M x 1536
  // 4-bit: 0.612 ms staged, 0.562 ms ring); the lighter 3-bit lookups gain
  // more from the slots' bytes in flight (10M x 768: 0.568 ms staged, 0.583
  // ms ring). The ring needs four CTAs' resident LUTs on an SM (at most 48 KB
  // each: nbg <= 1536, 3072 dims at 4 bits); wider rows keep the slots.
  const bool ring4 = reg && q == 1 && bits != 3 && static_cast<size_t>(nbg) * 32 <= 48 * 1024;
  const bool staged = reg && q <= 2 && nbg % kStageGroups == 0 && !ring4;
  const size_t stage_total = staged ? scan_stage_bytes(q) : 0;
  auto lut_area = [&](int c) {
    return staged ? scan_stage_offset(q, c) : static_cast<size_t>(q) * c * 32 + warp_total;
  };
  int chunk = nbg;
  while (lut_area(chunk) + stage_total > budget) {
    if (chunk > kFlushGroups) {
      chunk = ((chunk - 1) / kFlushGroups) * kFlushGroups;
      if (chunk < kFlushGroups) chunk = kFlushGroups;
    } else {
      return false;
    }
  }
  const long long blocks = (n + kScanBlockVectors - 1) / kScanBlockVectors;
  const long long qgroups = (nq + q - 1) / q;
  const long long resident = static_cast<long long>(sms) * (reg ? 2 : 1);  // CTAs per wave
  const long long target = static_cast<long long>(sms) * (reg ? 8 : 4);
  long long base = (target + qgroups - 1) / qgroups;
  if (base < 1) base = 1;
  // Among up to 4x the minimum range count, take the one whose last wave of
  // CTAs is fullest (fewer idle SMs at the tail); ties keep fewer ranges.
  long long ranges = base, best_waste = -1;
  for (long long r = base; r <= base * 4; ++r) {
    long long rr = r > blocks ? blocks : r;
    const long long per = (blocks + rr - 1) / rr;
    rr = (blocks + per - 1) / per;
    const long long ctas = qgroups * rr;
    const long long waste = ((ctas + resident - 1) / resident) * resident - ctas;
    // compare waste relative to the work: waste / ctas, as a cross-multiplied ratio
    if (best_waste < 0 || waste * ranges < best_waste * rr) {
      best_waste = waste;
      ranges = rr;
    }
    if (rr == blocks) break;
  }
  if (max_range_vectors > 0) {
    const long long cap_blocks = std::max(1LL, max_range_vectors / kScanBlockVectors);
    ranges = std::max(ranges, (blocks + cap_blocks - 1) / cap_blocks);
  }
  if (ranges > 65535) ranges = 65535;
  const long long blocks_per_range = (blocks + ranges - 1) / ranges;
  ranges = (blocks + blocks_per_range - 1) / blocks_per_range;
  plan->q_per_cta = q;
  plan->kmax = kmax;
  plan->range_vectors = blocks_per_range * kScanBlockVectors;
  plan->n_ranges = static_cast<int>(ranges);
  plan->lut_chunk_groups = chunk;
  plan->smem_bytes = static_cast<size_t>(q) * chunk * 32 + warp_total;
  if (reg) {
    // the end-of-range merge of the 8 warp lists reuses the LUT area
    plan->smem_bytes = std::max(plan->smem_bytes, static_cast<size_t>(q) * kScanWarps * kWarp * 8);
  }
  plan->stages = staged ? stages_for(q) : 0;
  plan->ring_ctas_per_sm = ring4 ? 4 : 2;
  if (staged) plan->smem_bytes = scan_stage_offset(q, chunk) + stage_total;
  plan->lists_per_range = reg ? 1 : kScanWarps;
  // One or two queries over at most two waves of blocks: whole blocks per CTA
  // leave the last wave part-full (1M vectors = 489 blocks over 296 resident
  // CTAs), so the work splits by 256-group batch as well. Measured at 1536-d
  // 4-bit: 1M vectors scan 10 % faster split (one query 0.210 -> 0.191 ms);
  // at 2M (977 blocks) the split no longer pays for its extra CTA start-ups.
  const int n_batches = (nbg + kFlushGroups - 1) / kFlushGroups;
  if (reg && q <= 2 && n_batches > 1 && blocks <= 2 * resident) {
    plan->split_batches = n_batches;
    // A split CTA streams a single 256-group batch, too short to amortize
    // filling the shared-memory slots: the split scans keep the register
    // ring (1M x 1536 4-bit, one query: 0.173 ms with the ring, 0.185 staged;
    // whole rows staged: 4M x 1536 0.659 -> 0.612 ms, 10M x 768 3-bit
    // 0.633 -> 0.571 ms).
    plan->stages = 0;
    // One query: 4 CTAs per SM (8 groups in flight, 64 registers) stream
    // about 1.3x faster per resident wave than 2 (16 groups in flight, 111
    // registers), but hold twice the CTAs per wave; take the shape with the
    // smaller (waves x CTAs per SM / relative rate). Measured, one query:
    // 1M x 1536 4-bit 0.174 -> 0.160 ms and 1M x 768 3-bit 0.105 -> 0.089 ms
    // with 4; 500k x 1536 0.093 ms with 2 against 0.102 with 4.
    if (q == 1) {
      const long long ctas = qgroups * blocks * n_batches;
      auto waves = [&](long long per_sm) { return (ctas + per_sm * sms - 1) / (per_sm * sms); };
      const double cost2 = static_cast<double>(waves(2)) * 2.0;
      const double cost4 = static_cast<double>(waves(4)) * 4.0 / 1.3;
      plan->split_ctas_per_sm = cost4 < cost2 ? 4 : 2;
    }
  }
  return true;
}

cudaError_t launch_scan(const ScanArgs& a, const ScanPlan& plan, cudaStream_t stream) {
  const int q = plan.q_per_cta, km = plan.kmax;
  const bool n8 = a.bits == 3;  // 3-bit codes never set a nibble's top bit
  if (a.partial && plan.split_batches > 1 && km == kRegTopK && q <= 2) {
    const long long span = (a.n + kScanBlockVectors - 1) / kScanBlockVectors * kScanBlockVectors;
    if (a.partial_stride < span || a.partial_batches != plan.split_batches) return cudaErrorInvalidValue;
    if (q == 1) return n8 ? launch_split_t<1, true>(a, plan, stream) : launch_split_t<1, false>(a, plan, stream);
    return n8 ? launch_split_t<2, true>(a, plan, stream) : launch_split_t<2, false>(a, plan, stream);
  }
  if (plan.stages > 0 && km == kRegTopK && q <= 2) {
    if (q == 1) {
      return n8 ? launch_scan_t<1, kRegTopK, 2, true, kStageGroups, stages_for(1)>(a, plan, stream)
                : launch_scan_t<1, kRegTopK, 2, false, kStageGroups, stages_for(1)>(a, plan, stream);
    }
    return n8 ? launch_scan_t<2, kRegTopK, 2, true, kStageGroups, stages_for(2)>(a, plan, stream)
              : launch_scan_t<2, kRegTopK, 2, false, kStageGroups, stages_for(2)>(a, plan, stream);
  }
#define VCB_SCAN(QQ, KK, MB)                                                             \
  if (q == QQ && km == KK) {                                                             \
    return n8 ? launch_scan_t<QQ, KK, MB, true, prefetch_for(QQ)>(a, plan, stream)       \
              : launch_scan_t<QQ, KK, MB, false, prefetch_for(QQ)>(a, plan, stream);     \
  }
  // Four queries over batches that are whole rings: the unchecked instance.
  if (q == 4 && km == 32 && a.nbg % prefetch_for(4) == 0) {
    return n8 ? launch_scan_t<4, 32, 2, true, prefetch_for(4), 0, true>(a, plan, stream)
              : launch_scan_t<4, 32, 2, false, prefetch_for(4), 0, true>(a, plan, stream);
  }
  if (q == 4 && km == 64 && a.nbg % prefetch_for(4) == 0) {
    return n8 ? launch_scan_t<4, 64, 1, true, prefetch_for(4), 0, true>(a, plan, stream)
              : launch_scan_t<4, 64, 1, false, prefetch_for(4), 0, true>(a, plan, stream);
  }
  // One query over 2- or 4-bit codes: the 8-group ring on four CTAs per SM.
  if (q == 1 && km == 32 && !n8 && plan.ring_ctas_per_sm == 4) {
    return launch_scan_t<1, 32, 4, false, 8>(a, plan, stream);
  }
  VCB_SCAN(1, 32, 2) VCB_SCAN(2, 32, 2) VCB_SCAN(4, 32, 2)
  VCB_SCAN(1, 64, 1) VCB_SCAN(2, 64, 1) VCB_SCAN(4, 64, 1)
  VCB_SCAN(1, 256, 1) VCB_SCAN(2, 256, 1)
#undef VCB_SCAN
  return cudaErrorInvalidValue;
}

cudaError_t launch_merge(const MergeArgs& a, cudaStream_t stream) {
  if (a.nq == 0 || a.k_out == 0) return cudaSuccess;
  if (a.k_out <= kRegTopK) {
    merge_reg_kernel<<<static_cast<unsigned>(a.nq), kMergeThreads, 0, stream>>>(a);
    return cudaGetLastError();
  }
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
