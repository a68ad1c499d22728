// Learned candidate pruner: features of the K1 index hits, the BF16 MLP on tensor cores, and the selection of the
// hits to rescore.
//
// The pruner sees the hits the plain path shortlists: the top-K of each spectrum before pair closure (vk_select_topk
// with pair_closure = 0), so the pruned candidates are always a subset of the plain path's.  Features per hit
// (label-free): K1 count, summed matched intensity (fraction of the TIC, from K1's fixed-point sums), precursor mass
// error in ppm (hypothesis mass vs the row's Sage f32 mass), precursor charge, peptide length, missed cleavages,
// standardised with the model's (mu, sd) and stored as 16 BF16 values (6 used).
//
// MLP: x(16) -> 256 (ReLU) -> 256 (ReLU) -> 1 logit; BF16 weights, FP32 accumulation.  Inference uses mma.sync
// m16n8k16 (BF16 in, FP32 accumulate): a warp scores 16 hits; the layer-1 accumulators are repacked in registers as
// the layer-2 A fragments (BF16), layer 2 runs in chunks of 64 output columns whose ReLU output is dotted with the
// layer-3 weights at once, so no activation leaves the registers.  The weights live in shared memory with padded
// rows (no bank conflicts on the B fragments).
//
// Selection per spectrum (one warp): hits with logit >= tau plus the min_keep best (logit desc, count desc, hit
// order desc), at most max_keep of them by the same order; then pair closure, sort by (row, hypothesis) and merge of
// duplicate rows exactly as the top-K selection (topk.cu) -- only the ranking key differs.
#include <cuda_bf16.h>

#include "common.cuh"

namespace {

constexpr int MLP_IN = 16;
constexpr int MLP_H = 256;
constexpr int W1_STRIDE = MLP_IN + 8;   // bf16 elements per W1 row in shared memory
constexpr int W2_STRIDE = MLP_H + 8;    // bf16 elements per W2 row in shared memory
constexpr int INF_WARPS = 8;

// ------------------------------------------------------------------------------------------------ features
// The 16 standardised BF16 features of one hit (hypothesis h, row r, K1 count, fixed-point intensity sum) into
// feat_row (32 bytes, 16-byte aligned): the six used ones first, the rest zero.
__device__ __forceinline__ void hit_features(int64_t h, int64_t r, int64_t cnt, uint32_t isum_fx, const float* h_M,
                                             const int8_t* h_z, const float* mass32, const uint8_t* len,
                                             const uint8_t* missed, const float* mu, const float* sd,
                                             __nv_bfloat16* feat_row) {
  const float mr = mass32[r];
  float raw[6];
  raw[0] = (float)cnt;
  raw[1] = (float)isum_fx * (1.0f / 16777216.0f);
  raw[2] = (h_M[h] - mr) / mr * 1.0e6f;
  raw[3] = (float)h_z[h];
  raw[4] = (float)len[r];
  raw[5] = (float)missed[r];
  __nv_bfloat162 v0 = __floats2bfloat162_rn((raw[0] - mu[0]) / sd[0], (raw[1] - mu[1]) / sd[1]);
  __nv_bfloat162 v1 = __floats2bfloat162_rn((raw[2] - mu[2]) / sd[2], (raw[3] - mu[3]) / sd[3]);
  __nv_bfloat162 v2 = __floats2bfloat162_rn((raw[4] - mu[4]) / sd[4], (raw[5] - mu[5]) / sd[5]);
  uint4 a;
  a.x = *reinterpret_cast<uint32_t*>(&v0);
  a.y = *reinterpret_cast<uint32_t*>(&v1);
  a.z = *reinterpret_cast<uint32_t*>(&v2);
  a.w = 0u;
  uint4* f = reinterpret_cast<uint4*>(feat_row);
  f[0] = a;
  f[1] = make_uint4(0u, 0u, 0u, 0u);
}

// One thread per candidate hit (hypothesis, row, count): its window position is win_off[h] + row - lo[h].
__global__ void cand_features_k(int64_t n, const int64_t* n_dev, const int64_t* c_hyp, const int64_t* c_row,
                                const int64_t* c_cnt, const int64_t* win_off, const int64_t* h_lo, const uint32_t* isum,
                                const float* h_M, const int8_t* h_z, const float* mass32, const uint8_t* len,
                                const uint8_t* missed, const float* mu, const float* sd, __nv_bfloat16* feat) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n_dev) n = min(n, *n_dev);
  if (i >= n) return;
  const int64_t h = c_hyp[i], r = c_row[i];
  // the intensity sum from the dense K1 sums, or (win_off NULL) one per candidate, from the hit-list shortlist
  const uint32_t is = win_off ? isum[win_off[h] + (r - h_lo[h])] : isum[i];
  hit_features(h, r, c_cnt[i], is, h_M, h_z, mass32, len, missed, mu, sd, feat + i * MLP_IN);
}

// The hit-list shortlist's per-spectrum slots compacted (as vk_compact_hits does) and every hit's features written
// on the way: the features kernel's second read of the compacted hits is saved.  A group of 2^g_log lanes per
// spectrum (the smallest power of two >= cap, at most 32): with the short lists the pruner sees (cap = the shortlist
// cap, e.g. 8) a warp per spectrum would leave most lanes idle on this latency-bound gather.
constexpr int CF_THREADS = 256;

__global__ void __launch_bounds__(CF_THREADS)
compact_features_k(int n_spec, int cap, int g_log, const int64_t* n_cand, const int64_t* cand_off,
                   const int64_t* s_hyp, const int64_t* s_row, const int64_t* s_cnt, const uint32_t* s_isum,
                   const int8_t* h_maxfz, int64_t* c_hyp, int64_t* c_row, int64_t* c_cnt, int32_t* c_row32,
                   int8_t* c_maxfz, uint32_t* c_isum, const float* h_M, const int8_t* h_z, const float* mass32,
                   const uint8_t* len, const uint8_t* missed, const float* mu, const float* sd,
                   __nv_bfloat16* feat) {
  const int64_t t = blockIdx.x * (int64_t)CF_THREADS + threadIdx.x;
  const int64_t s = t >> g_log;
  if (s >= n_spec) return;
  const int g = 1 << g_log;
  const int64_t m = min(n_cand[s], (int64_t)cap), dst0 = cand_off[s], src0 = s * cap;
  for (int64_t j = t & (g - 1); j < m; j += g) {
    const int64_t src = src0 + j, dst = dst0 + j;
    const int64_t h = s_hyp[src], r = s_row[src], c = s_cnt[src];
    const uint32_t is = s_isum[src];
    c_hyp[dst] = h;
    c_row[dst] = r;
    c_cnt[dst] = c;
    c_row32[dst] = (int32_t)r;
    c_maxfz[dst] = h_maxfz[h];
    c_isum[dst] = is;
    hit_features(h, r, c, is, h_M, h_z, mass32, len, missed, mu, sd, feat + dst * MLP_IN);
  }
}

// ------------------------------------------------------------------------------------------------ MLP inference
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16(float* c, const uint32_t* a, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__global__ void __launch_bounds__(INF_WARPS * 32)
mlp_infer_k(int64_t n, const int64_t* n_dev, const __nv_bfloat16* __restrict__ feat,
            const __nv_bfloat16* __restrict__ W1, const float* __restrict__ b1, const __nv_bfloat16* __restrict__ W2,
            const float* __restrict__ b2, const float* __restrict__ w3, float b3, float* __restrict__ logit) {
  extern __shared__ __align__(16) uint8_t mlp_smem[];
  __nv_bfloat16* sW2 = reinterpret_cast<__nv_bfloat16*>(mlp_smem);
  __nv_bfloat16* sW1 = sW2 + MLP_H * W2_STRIDE;
  float* sb1 = reinterpret_cast<float*>(sW1 + MLP_H * W1_STRIDE);
  float* sb2 = sb1 + MLP_H;
  float* sw3 = sb2 + MLP_H;
  for (int i = threadIdx.x; i < MLP_H * MLP_H; i += blockDim.x) sW2[(i / MLP_H) * W2_STRIDE + (i % MLP_H)] = W2[i];
  for (int i = threadIdx.x; i < MLP_H * MLP_IN; i += blockDim.x) sW1[(i / MLP_IN) * W1_STRIDE + (i % MLP_IN)] = W1[i];
  for (int i = threadIdx.x; i < MLP_H; i += blockDim.x) {
    sb1[i] = b1[i];
    sb2[i] = b2[i];
    sw3[i] = w3[i];
  }
  __syncthreads();
  if (n_dev) n = min(n, *n_dev);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int64_t n_tiles = (n + 15) >> 4;
  for (int64_t tile = (int64_t)blockIdx.x * INF_WARPS + warp; tile < n_tiles; tile += (int64_t)gridDim.x * INF_WARPS) {
    const int64_t r0 = tile << 4;
    // A fragment of the 16 x 16 input tile (rows beyond n read as zero)
    uint32_t a[4];
    {
      const int64_t ra = r0 + g, rb = r0 + g + 8;
      const uint32_t* fa = reinterpret_cast<const uint32_t*>(feat + ra * MLP_IN);
      const uint32_t* fb = reinterpret_cast<const uint32_t*>(feat + rb * MLP_IN);
      a[0] = ra < n ? fa[t] : 0u;
      a[1] = rb < n ? fb[t] : 0u;
      a[2] = ra < n ? fa[t + 4] : 0u;
      a[3] = rb < n ? fb[t + 4] : 0u;
    }
    // layer 1: 32 n-tiles of 8 outputs; ReLU; repacked as layer-2 A fragments (16 k-steps x 4 regs)
    uint32_t h1[16][4];
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
      const __nv_bfloat16* wrow = sW1 + (8 * j + g) * W1_STRIDE;
      const uint32_t b0 = *reinterpret_cast<const uint32_t*>(wrow + 2 * t);
      const uint32_t bb = *reinterpret_cast<const uint32_t*>(wrow + 8 + 2 * t);
      mma_bf16(c, a, b0, bb);
      const int col = 8 * j + 2 * t;
      const float x0 = fmaxf(c[0] + sb1[col], 0.f), x1 = fmaxf(c[1] + sb1[col + 1], 0.f);
      const float x2 = fmaxf(c[2] + sb1[col], 0.f), x3 = fmaxf(c[3] + sb1[col + 1], 0.f);
      const int kk = j >> 1;
      if ((j & 1) == 0) {
        h1[kk][0] = pack_bf16(x0, x1);
        h1[kk][1] = pack_bf16(x2, x3);
      } else {
        h1[kk][2] = pack_bf16(x0, x1);
        h1[kk][3] = pack_bf16(x2, x3);
      }
    }
    // layers 2 + 3 in chunks of 64 output columns
    float za = 0.f, zb = 0.f;   // partial logits of rows g and g + 8
#pragma unroll 1
    for (int ch = 0; ch < 4; ++ch) {
      float c[8][4];
#pragma unroll
      for (int j = 0; j < 8; ++j) c[j][0] = c[j][1] = c[j][2] = c[j][3] = 0.f;
#pragma unroll
      for (int kk = 0; kk < 16; ++kk) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const __nv_bfloat16* wrow = sW2 + (64 * ch + 8 * j + g) * W2_STRIDE + 16 * kk;
          const uint32_t b0 = *reinterpret_cast<const uint32_t*>(wrow + 2 * t);
          const uint32_t bb = *reinterpret_cast<const uint32_t*>(wrow + 8 + 2 * t);
          mma_bf16(c[j], h1[kk], b0, bb);
        }
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int col = 64 * ch + 8 * j + 2 * t;
        za += fmaxf(c[j][0] + sb2[col], 0.f) * sw3[col] + fmaxf(c[j][1] + sb2[col + 1], 0.f) * sw3[col + 1];
        zb += fmaxf(c[j][2] + sb2[col], 0.f) * sw3[col] + fmaxf(c[j][3] + sb2[col + 1], 0.f) * sw3[col + 1];
      }
    }
    za += __shfl_xor_sync(VK_FULL, za, 1);
    za += __shfl_xor_sync(VK_FULL, za, 2);
    zb += __shfl_xor_sync(VK_FULL, zb, 1);
    zb += __shfl_xor_sync(VK_FULL, zb, 2);
    if (t == 0) {
      if (r0 + g < n) logit[r0 + g] = za + b3;
      if (r0 + g + 8 < n) logit[r0 + g + 8] = zb + b3;
    }
  }
}

// ------------------------------------------------------------------------------------------------ selection
__device__ __forceinline__ uint32_t ord_f32(float x) {
  uint32_t u = __float_as_uint(x);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// ranking key of a hit: logit, count, row (all descending), hypothesis ascending
__device__ __forceinline__ unsigned long long prune_key_hi(float logit) { return ord_f32(logit); }

constexpr int PS_WARPS = 4;

__device__ __forceinline__ void warp_bitonic_u64(uint64_t* v, int n_pow2, int lane) {
  for (int k = 2; k <= n_pow2; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = lane; i < n_pow2; i += 32) {
        int p = i ^ j;
        if (p > i) {
          uint64_t a = v[i], b = v[p];
          bool up = (i & k) == 0;
          if ((a > b) == up) { v[i] = b; v[p] = a; }
        }
      }
      __syncwarp();
    }
}

// Per spectrum: rank hits by (logit, count, row) desc; keep those with logit >= tau or among the min_keep first,
// at most max_keep; add partners; sort by (row, hypothesis); merge duplicates (lowest hypothesis, highest count).
// The hits of spectrum s are [hit_off[s], hit_off[s+1]); hyp-local index = hit_hyp - first hypothesis of s.
__global__ void __launch_bounds__(PS_WARPS * 32)
select_pruned_k(int n_spec, const int64_t* spec_hyp_off, const int64_t* hit_off, const int64_t* hit_hyp,
                const int32_t* hit_row, const int64_t* hit_cnt, const float* logit, float tau, int min_keep,
                int max_keep, int pair_closure, const int64_t* partner, int cap, int sort_cap, int64_t* c_hyp,
                int64_t* c_row, int64_t* c_cnt, int64_t* n_cand) {
  extern __shared__ __align__(16) uint8_t ps_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int s = blockIdx.x * PS_WARPS + warp;
  if (s >= n_spec) return;
  const int list_cap = 2 * max_keep > 32 ? 2 * max_keep : 32;
  uint64_t* key = reinterpret_cast<uint64_t*>(ps_smem) + (size_t)warp * (sort_cap + list_cap);
  uint64_t* lst = key + sort_cap;          // (row << 34 | hl << 16 | idx) for the closure sort
  int32_t* lcnt = reinterpret_cast<int32_t*>(reinterpret_cast<uint64_t*>(ps_smem) +
                                             (size_t)PS_WARPS * (sort_cap + list_cap)) + (size_t)warp * list_cap;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t h0 = spec_hyp_off[s];
  const int64_t a = hit_off[s], b = hit_off[s + 1];
  const int n = (int)(b - a);
  // keys of the hits: ord(logit) << 32 | count(12 bits, saturated) << 20 | index (20 bits); the index order is
  // (hypothesis, row) ascending, so among equal (logit, count) the later index = higher row wins on "desc"; the
  // hypothesis tie (same row in two hypotheses) is resolved by the lower index first through the complement below
  int n_keep = 0;
  // the usual case needs no ranking: when every hit with logit >= tau is kept (their number is within
  // [min(min_keep, n), max_keep]) the selection is exactly those hits, since they rank above all others (keys are
  // ordered by logit first); NaN logits rank highest, so the shortcut is taken only when there is none
  int n_pass = 0;
  bool any_nan = false;
  for (int i0 = 0; i0 < n; i0 += 32) {
    const int i = i0 + lane;
    const float lg = i < n ? logit[a + i] : 0.f;
    n_pass += __popc(__ballot_sync(VK_FULL, i < n && lg >= tau));
    any_nan |= __any_sync(VK_FULL, i < n && isnan(lg));
  }
  const bool direct = n > 0 && !any_nan && n_pass <= max_keep && n_pass >= min(min_keep, n);
  if (direct) {
    for (int i0 = 0; i0 < n; i0 += 32) {
      const int i = i0 + lane;
      const bool take = i < n && logit[a + i] >= tau;
      const unsigned m = __ballot_sync(VK_FULL, take);
      if (take) {
        const int pos = n_keep + __popc(m & lt);
        lst[pos] = ((uint64_t)hit_row[a + i] << 34) | ((uint64_t)(hit_hyp[a + i] - h0) << 16) | (uint64_t)pos;
        lcnt[pos] = (int32_t)hit_cnt[a + i];
      }
      n_keep += __popc(m);
    }
  } else if (n > 0) {
    if (n > sort_cap) {
      // more hits than the sort buffer: keep those with logit >= tau by hit order, up to max_keep (rare)
      for (int i0 = 0; i0 < n && n_keep < max_keep; i0 += 32) {
        const int i = i0 + lane;
        const bool take = i < n && logit[a + i] >= tau;
        const unsigned m = __ballot_sync(VK_FULL, take);
        if (take) {
          const int pos = n_keep + __popc(m & lt);
          if (pos < max_keep) {
            lst[pos] = ((uint64_t)hit_row[a + i] << 34) | ((uint64_t)(hit_hyp[a + i] - h0) << 16) | (uint64_t)pos;
            lcnt[pos] = (int32_t)hit_cnt[a + i];
          }
        }
        n_keep = min(max_keep, n_keep + __popc(m));
      }
    } else {
      int n_pow2 = 32;
      while (n_pow2 < n) n_pow2 <<= 1;
      for (int i = lane; i < n_pow2; i += 32) {
        uint64_t k = 0ull;
        if (i < n) {
          const uint32_t c = (uint32_t)min(hit_cnt[a + i], (int64_t)4095);
          const uint32_t rowpart = (uint32_t)i;   // hits are in (hyp, row) order: later index = higher row
          k = (prune_key_hi(logit[a + i]) << 32) | ((uint64_t)c << 20) | (uint64_t)(rowpart & 0xfffff);
        }
        key[i] = k;
      }
      __syncwarp();
      warp_bitonic_u64(key, n_pow2, lane);   // ascending: best hit last
      for (int r0 = 0; r0 < n && r0 < max_keep; r0 += 32) {
        const int r = r0 + lane;   // rank, 0 = best
        bool take = false;
        int i = 0;
        if (r < n && r < max_keep) {
          const uint64_t k = key[n_pow2 - 1 - r];
          i = (int)(k & 0xfffff);
          take = r < min_keep || logit[a + i] >= tau;
        }
        const unsigned m = __ballot_sync(VK_FULL, take);
        if (take) {
          const int pos = n_keep + __popc(m & lt);
          lst[pos] = ((uint64_t)hit_row[a + i] << 34) | ((uint64_t)(hit_hyp[a + i] - h0) << 16) | (uint64_t)pos;
          lcnt[pos] = (int32_t)hit_cnt[a + i];
        }
        n_keep += __popc(m);
      }
    }
  }
  __syncwarp();
  int n_list = n_keep;
  if (pair_closure) {
    for (int i = lane; i < n_keep; i += 32) {
      const uint64_t k = lst[i];
      const int64_t r = (int64_t)(k >> 34);
      const uint64_t hl = (k >> 16) & 0x3ffff;
      lst[n_keep + i] = ((uint64_t)partner[r] << 34) | (hl << 16) | (uint64_t)(n_keep + i);
      lcnt[n_keep + i] = -1;
    }
    n_list = 2 * n_keep;
  }
  __syncwarp();
  const int64_t slot = (int64_t)s * cap;
  if (n_list <= 32) {
    // the usual short list: sorted across the lanes by a bitonic network of shuffles (ascending), each row's run
    // reduced to its highest count by a log-step segmented max (a row's entries are adjacent once sorted), and the
    // heads (lowest hypothesis of each row) written in order -- the shared-memory path's outputs
    uint64_t k = lane < n_list ? lst[lane] : ~0ull;
    for (int size = 2; size <= 32; size <<= 1)
      for (int st = size >> 1; st > 0; st >>= 1) {
        const uint64_t o = __shfl_xor_sync(VK_FULL, k, st);
        const bool want_min = ((lane & size) == 0) == ((lane & st) == 0);
        if (want_min ? o < k : o > k) k = o;
      }
    const bool valid = lane < n_list;
    const int64_t r = (int64_t)(k >> 34);
    const uint64_t kp = __shfl_up_sync(VK_FULL, k, 1);
    const bool head = valid && (lane == 0 || (int64_t)(kp >> 34) != r);
    int best = valid ? lcnt[k & 0xffff] : INT_MIN;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int b2 = __shfl_down_sync(VK_FULL, best, o);
      const uint64_t k2 = __shfl_down_sync(VK_FULL, k, o);
      if (lane + o < n_list && (int64_t)(k2 >> 34) == r) best = max(best, b2);
    }
    const unsigned hb = __ballot_sync(VK_FULL, head);
    if (head) {
      const int pos = __popc(hb & lt);
      c_hyp[slot + pos] = h0 + (int64_t)((k >> 16) & 0x3ffff);
      c_row[slot + pos] = r;
      c_cnt[slot + pos] = best;
    }
    if (lane == 0) n_cand[s] = __popc(hb);
    return;
  }
  int n_pow2 = 1;
  while (n_pow2 < n_list) n_pow2 <<= 1;
  for (int i = n_list + lane; i < n_pow2; i += 32) lst[i] = ~0ull;
  __syncwarp();
  warp_bitonic_u64(lst, n_pow2, lane);
  int n_out = 0;
  for (int i0 = 0; i0 < n_list; i0 += 32) {
    const int i = i0 + lane;
    bool head = false;
    int64_t r = 0;
    if (i < n_list) {
      r = (int64_t)(lst[i] >> 34);
      head = i == 0 || (int64_t)(lst[i - 1] >> 34) != r;
    }
    const unsigned m = __ballot_sync(VK_FULL, head);
    if (head) {
      int best = lcnt[lst[i] & 0xffff];
      for (int k = i + 1; k < n_list && (int64_t)(lst[k] >> 34) == r; ++k) best = max(best, lcnt[lst[k] & 0xffff]);
      const int pos = n_out + __popc(m & lt);
      c_hyp[slot + pos] = h0 + (int64_t)((lst[i] >> 16) & 0x3ffff);
      c_row[slot + pos] = r;
      c_cnt[slot + pos] = best;
    }
    n_out += __popc(m);
  }
  if (lane == 0) n_cand[s] = n_out;
}

}  // namespace

extern "C" {

int vk_cand_features(int64_t n, const int64_t* n_dev, const int64_t* c_hyp, const int64_t* c_row,
                     const int64_t* c_cnt, const int64_t* win_off, const int64_t* h_lo, const uint32_t* isum,
                     const float* h_M, const int8_t* h_z, const float* mass32, const uint8_t* len,
                     const uint8_t* missed, const float* mu, const float* sd, void* feat_bf16, void* stream) {
  if (n <= 0) return 0;
  if (!feat_bf16 || ((uintptr_t)feat_bf16 & 15)) return VK_E_ARG;
  cand_features_k<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      n, n_dev, c_hyp, c_row, c_cnt, win_off, h_lo, isum, h_M, h_z, mass32, len, missed, mu, sd,
      reinterpret_cast<__nv_bfloat16*>(feat_bf16));
  return vk_launch_status();
}

int vk_compact_hits_features(int n_spec, int cap, const int64_t* n_cand, const int64_t* cand_off,
                             const int64_t* s_hyp, const int64_t* s_row, const int64_t* s_cnt, const uint32_t* s_isum,
                             const int8_t* h_maxfz, int64_t* c_hyp, int64_t* c_row, int64_t* c_cnt, int32_t* c_row32,
                             int8_t* c_maxfz, uint32_t* c_isum, const float* h_M, const int8_t* h_z,
                             const float* mass32, const uint8_t* len, const uint8_t* missed, const float* mu,
                             const float* sd, void* feat_bf16, void* stream) {
  if (n_spec == 0) return 0;
  if (!s_isum || !c_isum || !mu || !sd || !feat_bf16 || ((uintptr_t)feat_bf16 & 15)) return VK_E_ARG;
  if (cap < 1) return VK_E_ARG;
  int g_log = 0;
  while ((1 << g_log) < cap && g_log < 5) ++g_log;
  const int64_t n_thr = (int64_t)n_spec << g_log;
  compact_features_k<<<(unsigned)((n_thr + CF_THREADS - 1) / CF_THREADS), CF_THREADS, 0, (cudaStream_t)stream>>>(
      n_spec, cap, g_log, n_cand, cand_off, s_hyp, s_row, s_cnt, s_isum, h_maxfz, c_hyp, c_row, c_cnt, c_row32,
      c_maxfz, c_isum, h_M, h_z, mass32, len, missed, mu, sd, reinterpret_cast<__nv_bfloat16*>(feat_bf16));
  return vk_launch_status();
}

int64_t vk_mlp_infer_smem(void) {
  return (int64_t)MLP_H * W2_STRIDE * 2 + (int64_t)MLP_H * W1_STRIDE * 2 + 3 * MLP_H * 4;
}

int vk_mlp_infer(int64_t n, const int64_t* n_dev, const void* feat_bf16, const void* W1_bf16, const float* b1,
                 const void* W2_bf16, const float* b2, const float* w3, float b3, float* logit, int grid,
                 void* stream) {
  if (n <= 0) return 0;
  if (grid < 1) return VK_E_ARG;
  size_t sh = (size_t)vk_mlp_infer_smem();
  cudaError_t e = cudaFuncSetAttribute(mlp_infer_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  if (e != cudaSuccess) return vk_err(e);
  mlp_infer_k<<<grid, INF_WARPS * 32, sh, (cudaStream_t)stream>>>(
      n, n_dev, reinterpret_cast<const __nv_bfloat16*>(feat_bf16), reinterpret_cast<const __nv_bfloat16*>(W1_bf16), b1,
      reinterpret_cast<const __nv_bfloat16*>(W2_bf16), b2, w3, b3, logit);
  return vk_launch_status();
}

int vk_select_pruned(int n_spec, const int64_t* spec_hyp_off, const int64_t* hit_off, const int64_t* hit_hyp,
                     const int32_t* hit_row, const int64_t* hit_cnt, const float* logit, float tau, int min_keep,
                     int max_keep, int pair_closure, const int64_t* partner, int cap, int max_hits, int64_t* c_hyp,
                     int64_t* c_row, int64_t* c_cnt, int64_t* n_cand, void* stream) {
  if (n_spec == 0) return 0;
  if (max_keep < 1 || min_keep < 0 || min_keep > max_keep || cap < (pair_closure ? 2 : 1) * max_keep) return VK_E_ARG;
  if (max_hits < 1 || max_hits > 4096) return VK_E_ARG;
  int sort_cap = 32;
  while (sort_cap < max_hits) sort_cap <<= 1;
  const int list_cap = 2 * max_keep > 32 ? 2 * max_keep : 32;
  int list_pow2 = 1;
  while (list_pow2 < list_cap) list_pow2 <<= 1;
  if (list_pow2 != list_cap) return VK_E_ARG;   // max_keep a power of two (>= 16)
  size_t sh = (size_t)PS_WARPS * (sort_cap + list_cap) * 8 + (size_t)PS_WARPS * list_cap * 4;
  if (sh > 200 * 1024) return VK_E_ARG;
  cudaError_t e = cudaFuncSetAttribute(select_pruned_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  if (e != cudaSuccess) return vk_err(e);
  select_pruned_k<<<(unsigned)((n_spec + PS_WARPS - 1) / PS_WARPS), PS_WARPS * 32, sh, (cudaStream_t)stream>>>(
      n_spec, spec_hyp_off, hit_off, hit_hyp, hit_row, hit_cnt, logit, tau, min_keep, max_keep, pair_closure, partner,
      cap, sort_cap, c_hyp, c_row, c_cnt, n_cand);
  return vk_launch_status();
}

}  // extern "C"
