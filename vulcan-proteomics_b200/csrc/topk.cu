// Per-spectrum top-K with pair closure (reference vulcan/gpu/engine.py:284-312), one warp per spectrum.
//
// The reference sorts every appended (hyp, row, count) of the run by a packed key
// (spectrum, 32767 - min(count, 32767), 2^28 - 1 - row) and keeps rank < topk per spectrum, then adds partner rows
// and merges duplicates of (spectrum, row) to the lowest hypothesis and highest count.  Here a warp reads its
// spectrum's dense K1 counts once (loads unrolled), computing the per-hypothesis scored/matched statistics and
// collecting the appended entries as unique 63-bit keys (min(count,32767), row, -hypothesis) in shared memory;
//   - if at most topk entries pass the threshold, takes them all;
//   - otherwise finds the topk-th largest key by an 8-bit radix select over the collected keys and keeps the keys
//     at or above it (keys are unique, so exactly topk);
// a spectrum with more appended entries than shared memory holds (key_cap) takes the same radix select over its
// counts in global memory and a second read to gather.  Then it appends the partners, sorts by (row, hypothesis)
// with a warp bitonic sort and merges duplicates.
#include "common.cuh"

namespace {

constexpr int TK_WARPS = 4;

struct WarpLists {
  uint64_t* key;   // sort keys
  int32_t* row;
  int32_t* hl;     // hypothesis index within the spectrum
  int32_t* cnt;
  uint32_t* hist;  // 256 radix counters
};

__device__ __forceinline__ uint64_t sel_key(int c, int64_t r, int hl) {
  uint64_t kc = (uint64_t)min(c, 32767);
  return (kc << 48) | ((uint64_t)r << 18) | (uint64_t)((1 << 18) - 1 - hl);
}

__device__ __forceinline__ void warp_bitonic_u64(uint64_t* v, int n_pow2, int lane) {
  for (int k = 2; k <= n_pow2; k <<= 1) {
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
}

// Digit selection of a radix select: with hist[256] the counts of the candidates' current digit, the digit d such
// that the candidates with a larger digit number < need <= those with digit >= d; need becomes the number still to
// take among the candidates with digit d.
__device__ __forceinline__ int radix_digit(const uint32_t* hist, long long& need, int lane) {
  long long above = 0;
  for (int d0 = 255; d0 >= 0; d0 -= 32) {
    const int d = d0 - lane;
    const long long v = hist[d];
    // inclusive scan from the top digit downwards across the lanes of this group of 32 digits
    const long long inc = vk::warp_incl_scan(v);
    const unsigned hit = __ballot_sync(VK_FULL, above + inc >= need);
    if (hit) {
      const int l = __ffs(hit) - 1;
      const long long inc_l = __shfl_sync(VK_FULL, inc, l);
      const long long v_l = __shfl_sync(VK_FULL, v, l);
      need -= above + inc_l - v_l;
      return d0 - l;
    }
    above += __shfl_sync(VK_FULL, inc, 31);
  }
  return 0;
}

// The k-th largest of n unique keys in shared memory (1 <= k <= n): an 8-bit radix select, most significant
// digit first, counting only the keys that match the digits chosen so far.  Up to KTH_SMALL keys (a short
// shortlist over few hits) are ranked by counting instead: each lane counts, for its keys, how many keys are
// larger (broadcast reads), and the key with k - 1 larger ones is the answer -- n reads per key against the radix
// select's eight histogram passes.
constexpr int KTH_SMALL = 64;

__device__ __forceinline__ uint64_t smem_kth_largest_radix(const uint64_t* key, int n, int k, uint32_t* hist,
                                                           int lane);

__device__ __forceinline__ uint64_t smem_kth_largest(const uint64_t* key, int n, int k, uint32_t* hist, int lane) {
  if (n <= KTH_SMALL) {
    uint64_t found = 0ull;
    bool have = false;
    for (int i = lane; i < n; i += 32) {
      const uint64_t v = key[i];
      int larger = 0;
      for (int j = 0; j < n; ++j) larger += key[j] > v;
      if (larger == k - 1) {
        found = v;
        have = true;
      }
    }
    const unsigned b = __ballot_sync(VK_FULL, have);
    if (b) return __shfl_sync(VK_FULL, found, __ffs(b) - 1);
    // unreachable for unique keys; the radix select below is the fallback
  }
  return smem_kth_largest_radix(key, n, k, hist, lane);
}

__device__ __forceinline__ uint64_t smem_kth_largest_radix(const uint64_t* key, int n, int k, uint32_t* hist,
                                                           int lane) {
  uint64_t prefix = 0, pmask = 0;
  long long need = k;
  for (int shift = 56; shift >= 0; shift -= 8) {
    for (int i = lane; i < 256; i += 32) hist[i] = 0;
    __syncwarp();
    for (int i = lane; i < n; i += 32) {
      const uint64_t v = key[i];
      if ((v & pmask) == prefix) atomicAdd(&hist[(v >> shift) & 255], 1u);
    }
    __syncwarp();
    prefix |= (uint64_t)radix_digit(hist, need, lane) << shift;
    pmask |= 255ull << shift;
    __syncwarp();
  }
  return prefix;
}

#ifndef TK_UNROLL
#define TK_UNROLL 8            // count loads in flight per lane
#endif

// rows of a hypothesis window, or 0 when its slice would end past the count buffer (cnt_cap entries)
__device__ __forceinline__ int64_t win_rows(int64_t w0, int64_t lo, int64_t hi, int64_t cnt_cap) {
  const int64_t n = hi > lo ? hi - lo : 0;
  return w0 + n <= cnt_cap ? n : 0;
}

__global__ void __launch_bounds__(TK_WARPS * 32)
select_topk_k(int n_spec, const int64_t* spec_hyp_off, const int64_t* h_lo, const int64_t* h_hi, const int64_t* win_off,
              const int32_t* cnt, int64_t cnt_cap, const int64_t* partner, int thr, int topk, int pair_closure, int cap,
              int list_pow2, int key_cap, int64_t* c_hyp, int64_t* c_row, int64_t* c_cnt, int64_t* n_cand,
              uint32_t* hyp_scored, uint64_t* hyp_matched, int64_t* spec_scored, int64_t* spec_matched) {
  extern __shared__ __align__(16) uint8_t tk_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int s = blockIdx.x * TK_WARPS + warp;
  if (s >= n_spec) return;
  const size_t per_warp = (size_t)key_cap * 8 + (size_t)list_pow2 * (4 + 4 + 4) + 256 * 4;
  uint8_t* base = tk_smem + per_warp * warp;
  WarpLists W;
  W.key = reinterpret_cast<uint64_t*>(base);
  W.row = reinterpret_cast<int32_t*>(base + (size_t)key_cap * 8);
  W.hl = W.row + list_pow2;
  W.cnt = W.hl + list_pow2;
  W.hist = reinterpret_cast<uint32_t*>(W.cnt + list_pow2);
  const unsigned lt_mask = (1u << lane) - 1u;

  const int64_t hb = spec_hyp_off[s], he = spec_hyp_off[s + 1];
  // one read of the counts: per-hypothesis statistics, and the appended keys into shared memory (as many as fit)
  long long n_app = 0, s_sc = 0, s_mt = 0;
  for (int64_t h = hb; h < he; ++h) {
    const int64_t w0 = win_off[h], lo = h_lo[h], n = win_rows(w0, lo, h_hi[h], cnt_cap);
    long long sc = 0, mt = 0;
    for (int64_t j0 = 0; j0 < n; j0 += 32 * TK_UNROLL) {
      int c[TK_UNROLL];
#pragma unroll
      for (int u = 0; u < TK_UNROLL; ++u) {
        const int64_t j = j0 + 32 * u + lane;
        c[u] = j < n ? cnt[w0 + j] : -1;
      }
#pragma unroll
      for (int u = 0; u < TK_UNROLL; ++u) {
        const int64_t j = j0 + 32 * u + lane;
        if (c[u] >= 0) {
          sc += c[u] > 0;
          mt += c[u];
        }
        const bool take = c[u] >= thr && j < n;
        const unsigned m = __ballot_sync(VK_FULL, take);
        const long long at = n_app + __popc(m & lt_mask);
        if (take && at < key_cap) W.key[at] = sel_key(c[u], lo + j, (int)(h - hb));
        n_app += __popc(m);
      }
    }
    sc = vk::warp_sum(sc);
    mt = vk::warp_sum(mt);
    if (lane == 0) {
      hyp_scored[h] = (uint32_t)sc;
      hyp_matched[h] = (uint64_t)mt;
    }
    s_sc += sc;
    s_mt += mt;
  }
  if (lane == 0 && spec_scored) {
    spec_scored[s] = s_sc;
    spec_matched[s] = s_mt;
  }
  __syncwarp();
  const bool limit = n_app > topk;
  int n_sel = 0;
  if (n_app <= key_cap) {
    // every appended key is in shared memory: threshold (if needed) and gather from there, in collection order
    const int n_k = (int)n_app;
    const uint64_t kth = limit ? smem_kth_largest(W.key, n_k, topk, W.hist, lane) : 0ull;
    for (int i0 = 0; i0 < n_k; i0 += 32) {
      const int i = i0 + lane;
      const uint64_t k = i < n_k ? W.key[i] : 0ull;
      const bool take = i < n_k && (!limit || k >= kth);
      const unsigned m = __ballot_sync(VK_FULL, take);
      if (take) {
        const int pos = n_sel + __popc(m & lt_mask);
        const int hl = (1 << 18) - 1 - (int)(k & 0x3ffff);
        const int64_t row = (int64_t)((k >> 18) & 0x3fffffffull);
        int c = (int)(k >> 48);
        if (c >= 32767) {   // the key holds min(count, 32767): the exact count from the dense slice
          const int64_t h = hb + hl;
          c = cnt[win_off[h] + (row - h_lo[h])];
        }
        W.row[pos] = (int32_t)row;
        W.hl[pos] = hl;
        W.cnt[pos] = c;
      }
      n_sel += __popc(m);
    }
  } else {
    // more appended entries than shared memory holds: radix select over the dense counts, then a second read
    uint64_t prefix = 0, pmask = 0;
    long long need = topk;
    for (int shift = 56; shift >= 0; shift -= 8) {
      for (int i = lane; i < 256; i += 32) W.hist[i] = 0;
      __syncwarp();
      for (int64_t h = hb; h < he; ++h) {
        const int64_t w0 = win_off[h], lo = h_lo[h], n = win_rows(w0, lo, h_hi[h], cnt_cap);
        for (int64_t j = lane; j < n; j += 32) {
          const int c = cnt[w0 + j];
          if (c < thr) continue;
          const uint64_t k = sel_key(c, lo + j, (int)(h - hb));
          if ((k & pmask) == prefix) atomicAdd(&W.hist[(k >> shift) & 255], 1u);
        }
      }
      __syncwarp();
      prefix |= (uint64_t)radix_digit(W.hist, need, lane) << shift;
      pmask |= 255ull << shift;
      __syncwarp();
    }
    const uint64_t kth = prefix;
    for (int64_t h = hb; h < he; ++h) {
      const int64_t w0 = win_off[h], lo = h_lo[h], n = win_rows(w0, lo, h_hi[h], cnt_cap);
      for (int64_t j0 = 0; j0 < n; j0 += 32) {
        const int64_t j = j0 + lane;
        const int c = j < n ? cnt[w0 + j] : -1;
        const bool take = j < n && c >= thr && sel_key(c, lo + j, (int)(h - hb)) >= kth;
        const unsigned m = __ballot_sync(VK_FULL, take);
        if (take) {
          const int pos = n_sel + __popc(m & lt_mask);
          W.row[pos] = (int32_t)(lo + j);
          W.hl[pos] = (int32_t)(h - hb);
          W.cnt[pos] = c;
        }
        n_sel += __popc(m);
      }
    }
  }
  __syncwarp();
  int n_list = n_sel;
  if (pair_closure) {
    for (int i = lane; i < n_sel; i += 32) {
      W.row[n_sel + i] = (int32_t)partner[W.row[i]];
      W.hl[n_sel + i] = W.hl[i];
      W.cnt[n_sel + i] = -1;
    }
    n_list = 2 * n_sel;
  }
  __syncwarp();
  // sort by (row, hypothesis); the low 16 bits carry the list index
  int n_pow2 = 1;
  while (n_pow2 < n_list) n_pow2 <<= 1;
  for (int i = lane; i < n_pow2; i += 32)
    W.key[i] = i < n_list ? (((uint64_t)W.row[i] << 34) | ((uint64_t)W.hl[i] << 16) | (uint64_t)i) : ~0ull;
  __syncwarp();
  warp_bitonic_u64(W.key, n_pow2, lane);
  // merge equal rows: head = first of a run of equal rows (lowest hypothesis); count = max over the run
  int n_out = 0;
  int64_t slot = (int64_t)s * cap;
  for (int i0 = 0; i0 < n_list; i0 += 32) {
    int i = i0 + lane;
    bool head = false;
    int64_t r = 0;
    if (i < n_list) {
      r = (int64_t)(W.key[i] >> 34);
      head = i == 0 || (int64_t)(W.key[i - 1] >> 34) != r;
    }
    unsigned m = __ballot_sync(VK_FULL, head);
    if (head) {
      int idx = (int)(W.key[i] & 0xffff);
      int best = W.cnt[idx];
      for (int k = i + 1; k < n_list && (int64_t)(W.key[k] >> 34) == r; ++k) best = max(best, W.cnt[W.key[k] & 0xffff]);
      int pos = n_out + __popc(m & lt_mask);
      c_hyp[slot + pos] = hb + (int)((W.key[i] >> 16) & 0x3ffff);
      c_row[slot + pos] = r;
      c_cnt[slot + pos] = best;
    }
    n_out += __popc(m);
  }
  if (lane == 0) n_cand[s] = n_out;
}

// Per-warp scratch of the hit reader: up to 32 hypotheses in visiting order and one chunk of 32 segments.
struct HitScratch {
  int64_t lo[32], region[32], t0[32];
  int32_t shift[32], hyp[32], seg_base[32];
  int64_t slot[32];
  int32_t pos[32], who[32];
};

// Visits the hits vk_k1_hits wrote for the hypotheses hb + S.hyp[0 .. nv) (nv <= 32, in that order): their segments
// (one per tile a window covers; a hypothesis with tile shift 0 ran no item and has none) in hypothesis order, tile
// order, and each segment's hits in row order.  Two parallel rounds per 32 segments: their hit counts (seg_cnt at
// the segment's first slot), then the hits themselves spread over the lanes.  f(ok, slot, value, local hypothesis)
// is called by the whole warp; lanes with ok hold a hit.
template <class F>
__device__ __forceinline__ void gather_hits(HitScratch& S, int nv, int64_t hb, const int64_t* h_lo, const int64_t* h_hi,
                                            const int64_t* win_off, const int8_t* hyp_shift, const uint32_t* seg_cnt,
                                            const uint64_t* rc, int lane, F&& f) {
  int nt = 0;
  if (lane < nv) {
    const int64_t h = hb + S.hyp[lane];
    const int64_t lo = h_lo[h], hi = h_hi[h];
    const int sh = hyp_shift[h];
    int64_t t0 = 0;
    if (hi > lo && sh > 0) {
      t0 = lo >> sh;
      nt = (int)(((hi - 1) >> sh) - t0 + 1);
    }
    S.lo[lane] = lo;
    S.region[lane] = win_off[h];
    S.t0[lane] = t0;
    S.shift[lane] = sh;
  }
  const int incl = (int)vk::warp_incl_scan(nt);
  S.seg_base[lane] = incl - nt;
  const int total = __shfl_sync(VK_FULL, incl, 31);
  __syncwarp();
  for (int k0 = 0; k0 < total; k0 += 32) {
    const int k = k0 + lane;
    uint32_t c = 0;
    int64_t slot = 0;
    int who = 0;
    if (k < total) {
      int a = 0, b = nv;            // the last hypothesis whose first segment is at or before k
      while (b - a > 1) {
        const int m = (a + b) >> 1;
        if (S.seg_base[m] <= k) a = m; else b = m;
      }
      who = a;
      const int sh = S.shift[who];
      const int64_t t = S.t0[who] + (k - S.seg_base[who]);
      const int64_t lo = S.lo[who];
      slot = S.region[who] + (max(lo, t << sh) - lo);
      c = seg_cnt[slot];
    }
    const int pincl = (int)vk::warp_incl_scan((long long)c);
    const int n_hits = __shfl_sync(VK_FULL, pincl, 31);
    __syncwarp();
    S.slot[lane] = slot;
    S.pos[lane] = pincl - (int)c;
    S.who[lane] = who;
    __syncwarp();
    for (int u0 = 0; u0 < n_hits; u0 += 32) {
      const int u = u0 + lane;
      const bool ok = u < n_hits;
      int64_t at = 0;
      uint64_t v = 0;
      int hl = 0;
      if (ok) {
        int a = 0, b = 32;          // the segment holding hit u
        while (b - a > 1) {
          const int m = (a + b) >> 1;
          if (S.pos[m] <= u) a = m; else b = m;
        }
        at = S.slot[a] + (u - S.pos[a]);
        v = rc[at];
        hl = S.hyp[S.who[a]];
      }
      f(ok, at, v, hl);
    }
    __syncwarp();
  }
}

__device__ __forceinline__ int hit_count(uint64_t v) { return (int)min(v >> 32, (uint64_t)INT32_MAX); }
__device__ __forceinline__ int64_t hit_row(uint64_t v) { return (int64_t)(uint32_t)v; }

// Shortlist from the hit lists of vk_k1_hits, one warp per spectrum: the hits of the spectrum's hypotheses ranked by
// (count desc, row desc, hypothesis asc) with the keys of select_topk_k, the first topk kept (all when fewer),
// optionally with pair closure, sorted by (row, hypothesis), duplicate rows merged to the lowest hypothesis (its
// intensity sum) and the highest count: the slots select_topk_k writes, plus c_isum.
//   Fast path (no closure, at most 32 hypotheses, their windows pairwise disjoint -- the usual case): the hypotheses
//   are visited in window order and each one's hits come in row order, so the collected hits are already sorted by
//   row with no duplicates; selection keeps that order and no sort is needed.
//   Otherwise: collect, select, add partners, bitonic sort and merge.  Spectra with more hits than shared memory
//   holds run the radix select over the hit lists in global memory and a second read.
__global__ void __launch_bounds__(TK_WARPS * 32)
select_hits_k(int n_spec, const int64_t* spec_hyp_off, const int64_t* h_lo, const int64_t* h_hi,
              const int64_t* win_off, const int8_t* hyp_shift, const uint32_t* seg_cnt, const uint64_t* rc,
              const uint32_t* hit_isum,
              const uint32_t* hyp_scored, const uint64_t* hyp_matched, int topk, int pair_closure,
              const int64_t* partner, int cap, int list_pow2, int key_cap, int64_t* c_hyp, int64_t* c_row,
              int64_t* c_cnt, uint32_t* c_isum, int64_t* n_cand, int64_t* spec_scored, int64_t* spec_matched) {
  extern __shared__ __align__(16) uint8_t tk_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int s = blockIdx.x * TK_WARPS + warp;
  if (s >= n_spec) return;
  const size_t per_warp = (size_t)key_cap * 12 + (size_t)list_pow2 * 16 + 256 * 4 + sizeof(HitScratch);
  uint8_t* base = tk_smem + per_warp * warp;
  HitScratch& S = *reinterpret_cast<HitScratch*>(base + per_warp - sizeof(HitScratch));
  uint64_t* key = reinterpret_cast<uint64_t*>(base);
  uint32_t* src = reinterpret_cast<uint32_t*>(base + (size_t)key_cap * 8);   // hit slot - win_off[hb]
  int32_t* row = reinterpret_cast<int32_t*>(src + key_cap);
  int32_t* hl = row + list_pow2;
  int32_t* cnt = hl + list_pow2;
  uint32_t* isum = reinterpret_cast<uint32_t*>(cnt + list_pow2);
  uint32_t* hist = isum + list_pow2;
  const unsigned lt_mask = (1u << lane) - 1u;
  const int64_t hb = spec_hyp_off[s], he = spec_hyp_off[s + 1];
  const int nhs = (int)(he - hb);
  const int64_t w_base = he > hb ? win_off[hb] : 0;
  const int64_t slot = (int64_t)s * cap;
  // per-spectrum statistics from K1's per-hypothesis totals
  long long sc = 0, mt = 0;
  for (int64_t h = hb + lane; h < he; h += 32) {
    sc += hyp_scored[h];
    mt += (long long)hyp_matched[h];
  }
  sc = vk::warp_sum(sc);
  mt = vk::warp_sum(mt);
  if (lane == 0 && spec_scored) {
    spec_scored[s] = sc;
    spec_matched[s] = mt;
  }
  // every hit of the spectrum's hypotheses in index order, 32 hypotheses at a time
  auto visit_all = [&](auto&& f) {
    for (int g0 = 0; g0 < nhs; g0 += 32) {
      __syncwarp();
      if (lane < min(32, nhs - g0)) S.hyp[lane] = g0 + lane;
      __syncwarp();
      gather_hits(S, min(32, nhs - g0), hb, h_lo, h_hi, win_off, hyp_shift, seg_cnt, rc, lane, f);
    }
  };

  // ---------------------------------------------------------------- fast path
  bool fast = !pair_closure && nhs <= 32;
  int my_rank = 0;
  if (fast) {
    const bool mine = lane < nhs;
    const int64_t my_lo = mine ? h_lo[hb + lane] : 0, my_hi = mine ? h_hi[hb + lane] : 0;
    const bool live = mine && my_hi > my_lo;
    bool overlap = false;
    for (int j = 0; j < nhs; ++j) {
      const int64_t lo_j = __shfl_sync(VK_FULL, my_lo, j), hi_j = __shfl_sync(VK_FULL, my_hi, j);
      const bool live_j = hi_j > lo_j;
      if (live && live_j && j != lane) {
        if (lo_j < my_lo || (lo_j == my_lo && j < lane)) ++my_rank;
        overlap |= lo_j < my_hi && my_lo < hi_j;
      }
      if (mine && !live && live_j) ++my_rank;   // empty windows after every live one
      if (mine && !live && !live_j && j < lane) ++my_rank;
    }
    fast = !__any_sync(VK_FULL, overlap);
  }
  if (fast) {
    long long n_app = 0;
    __syncwarp();
    if (lane < nhs) S.hyp[my_rank] = lane;     // the hypotheses in window order
    __syncwarp();
    gather_hits(S, nhs, hb, h_lo, h_hi, win_off, hyp_shift, seg_cnt, rc, lane,
                [&](bool ok, int64_t pos, uint64_t v, int hl_) {
      const unsigned m = __ballot_sync(VK_FULL, ok);
      const long long at = n_app + __popc(m & lt_mask);
      if (ok && at < key_cap) {
        key[at] = sel_key(hit_count(v), hit_row(v), hl_);
        src[at] = (uint32_t)(pos - w_base);
      }
      n_app += __popc(m);
    });
    __syncwarp();
    if (n_app <= key_cap) {
      const int n_k = (int)n_app;
      const bool limit = n_k > topk;
      const uint64_t kth = limit ? smem_kth_largest(key, n_k, topk, hist, lane) : 0ull;
      int n_out = 0;
      for (int i0 = 0; i0 < n_k; i0 += 32) {
        const int i = i0 + lane;
        const uint64_t k = i < n_k ? key[i] : 0ull;
        const bool take = i < n_k && (!limit || k >= kth);
        const unsigned m = __ballot_sync(VK_FULL, take);
        if (take) {
          const int64_t pos = w_base + src[i];
          const uint64_t v = rc[pos];
          const int64_t at = slot + n_out + __popc(m & lt_mask);
          c_hyp[at] = hb + ((1 << 18) - 1 - (int)(k & 0x3ffff));
          c_row[at] = hit_row(v);
          c_cnt[at] = hit_count(v);
          if (c_isum) c_isum[at] = hit_isum[pos];
        }
        n_out += __popc(m);
      }
      if (lane == 0) n_cand[s] = n_out;
      return;
    }
  }

  // ---------------------------------------------------------------- general path
  long long n_app = 0;
  visit_all([&](bool ok, int64_t pos, uint64_t v, int hl_) {
    const unsigned m = __ballot_sync(VK_FULL, ok);
    const long long at = n_app + __popc(m & lt_mask);
    if (ok && at < key_cap) {
      key[at] = sel_key(hit_count(v), hit_row(v), hl_);
      src[at] = (uint32_t)(pos - w_base);
    }
    n_app += __popc(m);
  });
  __syncwarp();
  const bool limit = n_app > topk;
  int n_sel = 0;
  auto take_hit = [&](bool take, int64_t pos_g, int h_local) {
    const unsigned m = __ballot_sync(VK_FULL, take);
    if (take) {
      const int at = n_sel + __popc(m & lt_mask);
      const uint64_t v = rc[pos_g];
      row[at] = (int32_t)hit_row(v);
      hl[at] = h_local;
      cnt[at] = hit_count(v);
      isum[at] = hit_isum ? hit_isum[pos_g] : 0u;
    }
    n_sel += __popc(m);
  };
  if (n_app <= key_cap) {
    const int n_k = (int)n_app;
    const uint64_t kth = limit ? smem_kth_largest(key, n_k, topk, hist, lane) : 0ull;
    for (int i0 = 0; i0 < n_k; i0 += 32) {
      const int i = i0 + lane;
      const uint64_t k = i < n_k ? key[i] : 0ull;
      const bool take = i < n_k && (!limit || k >= kth);
      take_hit(take, take ? w_base + src[i] : 0, (1 << 18) - 1 - (int)(k & 0x3ffff));
    }
  } else {
    uint64_t prefix = 0, pmask = 0;
    long long need = topk;
    for (int shift = 56; shift >= 0; shift -= 8) {
      for (int i = lane; i < 256; i += 32) hist[i] = 0;
      __syncwarp();
      visit_all([&](bool ok, int64_t, uint64_t v, int hl_) {
        if (!ok) return;
        const uint64_t k = sel_key(hit_count(v), hit_row(v), hl_);
        if ((k & pmask) == prefix) atomicAdd(&hist[(k >> shift) & 255], 1u);
      });
      __syncwarp();
      prefix |= (uint64_t)radix_digit(hist, need, lane) << shift;
      pmask |= 255ull << shift;
      __syncwarp();
    }
    visit_all([&](bool ok, int64_t pos, uint64_t v, int hl_) {
      const bool take = ok && sel_key(hit_count(v), hit_row(v), hl_) >= prefix;
      take_hit(take, pos, hl_);
    });
  }
  __syncwarp();
  // pair closure: the partner row of every kept hit, same hypothesis, count -1 (no intensity sum)
  int n_list = n_sel;
  if (pair_closure) {
    for (int i = lane; i < n_sel; i += 32) {
      row[n_sel + i] = (int32_t)partner[row[i]];
      hl[n_sel + i] = hl[i];
      cnt[n_sel + i] = -1;
      isum[n_sel + i] = 0u;
    }
    n_list = 2 * n_sel;
  }
  __syncwarp();
  // sort by (row, hypothesis); the low 16 bits carry the list index
  int n_pow2 = 1;
  while (n_pow2 < n_list) n_pow2 <<= 1;
  for (int i = lane; i < n_pow2; i += 32)
    key[i] = i < n_list ? (((uint64_t)row[i] << 34) | ((uint64_t)hl[i] << 16) | (uint64_t)i) : ~0ull;
  __syncwarp();
  warp_bitonic_u64(key, n_pow2, lane);
  int n_out = 0;
  for (int i0 = 0; i0 < n_list; i0 += 32) {
    const int i = i0 + lane;
    bool head = false;
    int64_t r = 0;
    if (i < n_list) {
      r = (int64_t)(key[i] >> 34);
      head = i == 0 || (int64_t)(key[i - 1] >> 34) != r;
    }
    const unsigned m = __ballot_sync(VK_FULL, head);
    if (head) {
      const int idx = (int)(key[i] & 0xffff);
      int best = cnt[idx];
      for (int k = i + 1; k < n_list && (int64_t)(key[k] >> 34) == r; ++k) best = max(best, cnt[key[k] & 0xffff]);
      const int pos = n_out + __popc(m & lt_mask);
      c_hyp[slot + pos] = hb + (int)((key[i] >> 16) & 0x3ffff);
      c_row[slot + pos] = r;
      c_cnt[slot + pos] = best;
      if (c_isum) c_isum[slot + pos] = isum[idx];
    }
    n_out += __popc(m);
  }
  if (lane == 0) n_cand[s] = n_out;
}

// select_hits_k for a short list without pair closure (topk <= 32), one warp per spectrum, with no per-warp key
// buffer: the running top (by the same 63-bit keys) is held in registers of the first lanes and merged with every
// batch of 32 hits as they are read.  topk <= 16: the batch is sorted across the lanes by a bitonic network of
// shuffles and its best tpow (the power of two >= topk) are merged with the running tpow by one bitonic merge;
// topk 17-32: each key's rank among the batch and the running list is counted with shuffles and lane r takes the
// key of rank r.  The kept hits are then ordered by (row, hypothesis) and rows reached by several hypotheses merged
// (lowest hypothesis and its intensity sum, highest count): the outputs of select_hits_k, bit for bit, from shared
// memory for the hit reader alone (more warps per SM).
__global__ void __launch_bounds__(TK_WARPS * 32)
select_hits_small_k(int n_spec, const int64_t* spec_hyp_off, const int64_t* h_lo, const int64_t* h_hi,
                    const int64_t* win_off, const int8_t* hyp_shift, const uint32_t* seg_cnt, const uint64_t* rc,
                    const uint32_t* hit_isum, const uint32_t* hyp_scored, const uint64_t* hyp_matched, int topk,
                    int cap, int64_t* c_hyp, int64_t* c_row, int64_t* c_cnt, uint32_t* c_isum, int64_t* n_cand,
                    int64_t* spec_scored, int64_t* spec_matched) {
  __shared__ HitScratch scratch[TK_WARPS];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int s = blockIdx.x * TK_WARPS + warp;
  if (s >= n_spec) return;
  HitScratch& S = scratch[warp];
  const int64_t hb = spec_hyp_off[s], he = spec_hyp_off[s + 1];
  const int nhs = (int)(he - hb);
  long long sc = 0, mt = 0;
  for (int64_t h = hb + lane; h < he; h += 32) {
    sc += hyp_scored[h];
    mt += (long long)hyp_matched[h];
  }
  sc = vk::warp_sum(sc);
  mt = vk::warp_sum(mt);
  if (lane == 0 && spec_scored) {
    spec_scored[s] = sc;
    spec_matched[s] = mt;
  }
  // running list: lane r < topk holds the key of rank r (0 = empty: a hit's key has its count >= 1 in the top bits);
  // for topk <= 16 the running list is the best tpow (the power of two >= topk), descending, in lanes 0 .. tpow-1
  uint64_t tk = 0ull;
  int64_t tp = 0;
  int tpow = 1;
  while (tpow < topk) tpow <<= 1;
  for (int g0 = 0; g0 < nhs; g0 += 32) {
    __syncwarp();
    if (lane < min(32, nhs - g0)) S.hyp[lane] = g0 + lane;
    __syncwarp();
    gather_hits(S, min(32, nhs - g0), hb, h_lo, h_hi, win_off, hyp_shift, seg_cnt, rc, lane,
                [&](bool ok, int64_t pos, uint64_t v, int hl_) {
      const uint64_t nk = ok ? sel_key(hit_count(v), hit_row(v), hl_) : 0ull;
      if (tpow <= 16) {
        // sort the batch descending across the lanes (bitonic, in registers; o = the lane the key came from), then
        // merge its first tpow with the running list (lanes 0 .. tpow-1, descending) brought in reversed behind
        // them: the first tpow lanes of the merged 2 x tpow hold the running list again
        uint64_t k = nk;
        uint32_t o = (uint32_t)lane;
        for (int size = 2; size <= 32; size <<= 1)
          for (int st = size >> 1; st > 0; st >>= 1) {
            const uint64_t ok2 = __shfl_xor_sync(VK_FULL, k, st);
            const uint32_t oo = __shfl_xor_sync(VK_FULL, o, st);
            const bool want_max = ((lane & size) == 0) == ((lane & st) == 0);
            if (want_max ? ok2 > k : ok2 < k) {
              k = ok2;
              o = oo;
            }
          }
        const int rl = 2 * tpow - 1 - lane;   // running key that lands in this lane, reversed
        const uint64_t rk = __shfl_sync(VK_FULL, tk, rl & 31);
        if (lane >= tpow) {
          k = lane < 2 * tpow ? rk : 0ull;
          o = 32u + (uint32_t)(rl & 31);
        }
        for (int st = tpow; st > 0; st >>= 1) {
          const uint64_t ok2 = __shfl_xor_sync(VK_FULL, k, st);
          const uint32_t oo = __shfl_xor_sync(VK_FULL, o, st);
          if (((lane & st) == 0) ? ok2 > k : ok2 < k) {
            k = ok2;
            o = oo;
          }
        }
        const int64_t pb = __shfl_sync(VK_FULL, pos, (int)(o & 31u));
        const int64_t pr = __shfl_sync(VK_FULL, tp, (int)(o & 31u));
        tk = lane < tpow ? k : 0ull;
        tp = lane < tpow ? (o < 32u ? pb : pr) : 0;
        return;
      }
      int rn = 0, rt = 0;   // ranks of this lane's new key and of its running key among all 32 + topk keys
#pragma unroll 4
      for (int j = 0; j < 32; ++j) {
        const uint64_t x = __shfl_sync(VK_FULL, nk, j);
        rn += x > nk;
        rt += x > tk;
      }
      for (int j = 0; j < topk; ++j) {
        const uint64_t x = __shfl_sync(VK_FULL, tk, j);
        rn += x > nk;
        rt += x > tk;
      }
      uint64_t nt = 0ull;
      int64_t np = 0;
      for (int r = 0; r < topk; ++r) {   // lane r takes the key of rank r, from the batch or the running list
        const unsigned bn = __ballot_sync(VK_FULL, nk != 0ull && rn == r);
        const unsigned bt = __ballot_sync(VK_FULL, lane < topk && tk != 0ull && rt == r);
        const int src = bn ? __ffs(bn) - 1 : (bt ? __ffs(bt) - 1 : 0);
        const uint64_t kx = __shfl_sync(VK_FULL, bn ? nk : tk, src);
        const int64_t px = __shfl_sync(VK_FULL, bn ? pos : tp, src);
        if (lane == r && (bn | bt)) {
          nt = kx;
          np = px;
        }
      }
      tk = nt;
      tp = np;
    });
  }
  // the kept hits ordered by (row, hypothesis); a row reached by several hypotheses keeps its lowest one
  if (lane >= topk) tk = 0ull;   // (tpow > topk: the list's tail beyond the first topk)
  const bool have = tk != 0ull;
  const int hl = have ? (1 << 18) - 1 - (int)(tk & 0x3ffff) : 0;
  const uint64_t v = have ? rc[tp] : 0ull;
  const int64_t row = hit_row(v);
  const int cnt = hit_count(v);
  int best = cnt;
  bool head = have;
  for (int j = 0; j < topk; ++j) {   // the whole warp shuffles: same row -> highest count, lowest hypothesis
    const bool hj = __shfl_sync(VK_FULL, have, j);
    const int64_t rj = __shfl_sync(VK_FULL, row, j);
    const int lj = __shfl_sync(VK_FULL, hl, j);
    const int cj = __shfl_sync(VK_FULL, cnt, j);
    if (have && hj && rj == row) {
      best = max(best, cj);
      if (lj < hl) head = false;
    }
  }
  int before = 0;   // the output position: the kept rows below this one, each counted once (at its head)
  for (int j = 0; j < topk; ++j) {
    const bool hj = __shfl_sync(VK_FULL, head, j);
    const int64_t rj = __shfl_sync(VK_FULL, row, j);
    if (head && hj && rj < row) ++before;
  }
  const int64_t slot = (int64_t)s * cap;
  if (head) {
    const int64_t at = slot + before;
    c_hyp[at] = hb + hl;
    c_row[at] = row;
    c_cnt[at] = best;
    if (c_isum) c_isum[at] = hit_isum[tp];
  }
  const unsigned heads = __ballot_sync(VK_FULL, head);
  if (lane == 0) n_cand[s] = __popc(heads);
}

// Each spectrum's n_cand[s] (<= cap) slots to [cand_off[s], ...).  A warp takes CP_GROUPS spectra: when each has
// at most 32 / CP_GROUPS candidates (the pruned lists) a group of 32 / CP_GROUPS lanes copies each one's, otherwise
// (the exhaustive top-k lists) the whole warp copies them one spectrum after the other.  A thread per slot of
// n_spec x cap would launch mostly idle threads (cap is a bound).
constexpr int CP_WARPS = 8;
constexpr int CP_GROUPS = 4;

__device__ __forceinline__ void compact_slot(int64_t src, int64_t dst, const int64_t* s_hyp, const int64_t* s_row,
                                             const int64_t* s_cnt, const int8_t* h_maxfz, int64_t* c_hyp,
                                             int64_t* c_row, int64_t* c_cnt, int32_t* c_row32, int8_t* c_maxfz,
                                             const uint32_t* s_isum, uint32_t* c_isum) {
  const int64_t h = s_hyp[src];
  c_hyp[dst] = h;
  c_row[dst] = s_row[src];
  c_cnt[dst] = s_cnt[src];
  c_row32[dst] = (int32_t)s_row[src];
  c_maxfz[dst] = h_maxfz[h];
  if (c_isum) c_isum[dst] = s_isum[src];
}

__global__ void __launch_bounds__(CP_WARPS * 32)
compact_k(int n_spec, int cap, const int64_t* n_cand, const int64_t* cand_off, const int64_t* s_hyp,
          const int64_t* s_row, const int64_t* s_cnt, const int8_t* h_maxfz, int64_t* c_hyp, int64_t* c_row,
          int64_t* c_cnt, int32_t* c_row32, int8_t* c_maxfz, const uint32_t* s_isum, uint32_t* c_isum) {
  constexpr int G = 32 / CP_GROUPS;
  const int lane = threadIdx.x & 31;
  const int64_t s0 = ((int64_t)blockIdx.x * CP_WARPS + (threadIdx.x >> 5)) * CP_GROUPS;
  if (s0 >= n_spec) return;   // uniform over the warp
  const int64_t s = s0 + lane / G;
  const int64_t m = s < n_spec ? min(n_cand[s], (int64_t)cap) : 0;
  if (__all_sync(VK_FULL, m <= G)) {
    if (lane % G < m) {
      const int64_t j = lane % G;
      compact_slot(s * cap + j, cand_off[s] + j, s_hyp, s_row, s_cnt, h_maxfz, c_hyp, c_row, c_cnt, c_row32, c_maxfz,
                   s_isum, c_isum);
    }
    return;
  }
  for (int g = 0; g < CP_GROUPS && s0 + g < n_spec; ++g) {
    const int64_t sg = s0 + g;
    const int64_t mg = __shfl_sync(VK_FULL, m, g * G), dst0 = cand_off[sg], src0 = sg * cap;
    for (int64_t j = lane; j < mg; j += 32)
      compact_slot(src0 + j, dst0 + j, s_hyp, s_row, s_cnt, h_maxfz, c_hyp, c_row, c_cnt, c_row32, c_maxfz, s_isum,
                   c_isum);
  }
}

}  // namespace

extern "C" {

int vk_select_topk(int n_spec, const int64_t* spec_hyp_off, const int64_t* h_lo, const int64_t* h_hi,
                   const int64_t* win_off, const int32_t* cnt, int64_t cnt_cap, const int64_t* partner, int thr,
                   int topk,
                   int pair_closure, int cap, int64_t* c_hyp, int64_t* c_row, int64_t* c_cnt, int64_t* n_cand,
                   uint32_t* hyp_scored, uint64_t* hyp_matched, int64_t* spec_scored, int64_t* spec_matched,
                   void* stream) {
  if (n_spec == 0) return 0;
  if (topk < 1 || topk > 8192 || cap < (pair_closure ? 2 : 1) * topk) return VK_E_ARG;
  int list_pow2 = 32;
  while (list_pow2 < (pair_closure ? 2 : 1) * topk) list_pow2 <<= 1;
  const int key_cap = list_pow2 > 512 ? list_pow2 : 512;   // sort path up to 512 appended entries
  size_t per_warp = (size_t)key_cap * 8 + (size_t)list_pow2 * 12 + 1024;
  size_t sh = per_warp * TK_WARPS;
  if (sh > 220 * 1024) return VK_E_ARG;
  cudaError_t e = cudaFuncSetAttribute(select_topk_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  if (e != cudaSuccess) return vk_err(e);
  select_topk_k<<<(unsigned)((n_spec + TK_WARPS - 1) / TK_WARPS), TK_WARPS * 32, sh, (cudaStream_t)stream>>>(
      n_spec, spec_hyp_off, h_lo, h_hi, win_off, cnt, cnt_cap, partner, thr, topk, pair_closure, cap, list_pow2,
      key_cap, c_hyp,
      c_row,
      c_cnt, n_cand, hyp_scored, hyp_matched, spec_scored, spec_matched);
  return vk_launch_status();
}

int vk_compact_cands(int n_spec, int cap, const int64_t* n_cand, const int64_t* cand_off, const int64_t* s_hyp,
                     const int64_t* s_row, const int64_t* s_cnt, const int8_t* h_maxfz, int64_t* c_hyp,
                     int64_t* c_row, int64_t* c_cnt, int32_t* c_row32, int8_t* c_maxfz, void* stream) {
  if (n_spec == 0) return 0;
  compact_k<<<(unsigned)((n_spec + CP_WARPS * CP_GROUPS - 1) / (CP_WARPS * CP_GROUPS)), CP_WARPS * 32, 0,
              (cudaStream_t)stream>>>(n_spec, cap, n_cand, cand_off, s_hyp, s_row, s_cnt, h_maxfz, c_hyp, c_row, c_cnt,
                                      c_row32, c_maxfz, nullptr, nullptr);
  return vk_launch_status();
}

int vk_compact_hits(int n_spec, int cap, const int64_t* n_cand, const int64_t* cand_off, const int64_t* s_hyp,
                    const int64_t* s_row, const int64_t* s_cnt, const uint32_t* s_isum, const int8_t* h_maxfz,
                    int64_t* c_hyp, int64_t* c_row, int64_t* c_cnt, int32_t* c_row32, int8_t* c_maxfz,
                    uint32_t* c_isum, void* stream) {
  if (n_spec == 0) return 0;
  if ((s_isum != nullptr) != (c_isum != nullptr)) return VK_E_ARG;
  compact_k<<<(unsigned)((n_spec + CP_WARPS * CP_GROUPS - 1) / (CP_WARPS * CP_GROUPS)), CP_WARPS * 32, 0,
              (cudaStream_t)stream>>>(n_spec, cap, n_cand, cand_off, s_hyp, s_row, s_cnt, h_maxfz, c_hyp, c_row, c_cnt,
                                      c_row32, c_maxfz, s_isum, c_isum);
  return vk_launch_status();
}

int vk_select_hits(int n_spec, const int64_t* spec_hyp_off, const int64_t* h_lo, const int64_t* h_hi,
                   const int64_t* win_off, const int8_t* hyp_shift, const uint32_t* seg_cnt, const uint64_t* hit_rc,
                   const uint32_t* hit_isum,
                   const uint32_t* hyp_scored, const uint64_t* hyp_matched, int topk, int pair_closure,
                   const int64_t* partner, int cap, int64_t* c_hyp, int64_t* c_row, int64_t* c_cnt, uint32_t* c_isum,
                   int64_t* n_cand, int64_t* spec_scored, int64_t* spec_matched, void* stream) {
  if (n_spec == 0) return 0;
  if (topk < 1 || topk > 8192 || cap < (pair_closure ? 2 : 1) * topk) return VK_E_ARG;
  if (!c_isum != !hit_isum || (pair_closure && !partner) || !h_lo || !h_hi || !hyp_shift || !seg_cnt) return VK_E_ARG;
  if (!pair_closure && topk <= 32) {   // a short list: kept in registers while the hits stream by
    select_hits_small_k<<<(unsigned)((n_spec + TK_WARPS - 1) / TK_WARPS), TK_WARPS * 32, 0,
                          (cudaStream_t)stream>>>(n_spec, spec_hyp_off, h_lo, h_hi, win_off, hyp_shift, seg_cnt,
                                                  hit_rc, hit_isum, hyp_scored, hyp_matched, topk, cap, c_hyp, c_row,
                                                  c_cnt, c_isum, n_cand, spec_scored, spec_matched);
    return vk_launch_status();
  }
  int list_pow2 = 32;
  while (list_pow2 < (pair_closure ? 2 : 1) * topk) list_pow2 <<= 1;
  const int key_cap = list_pow2 > 512 ? list_pow2 : 512;
  const size_t per_warp = (size_t)key_cap * 12 + (size_t)list_pow2 * 16 + 1024 + sizeof(HitScratch);
  const size_t sh = per_warp * TK_WARPS;
  if (sh > 220 * 1024) return VK_E_ARG;
  cudaError_t e = cudaFuncSetAttribute(select_hits_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  if (e != cudaSuccess) return vk_err(e);
  select_hits_k<<<(unsigned)((n_spec + TK_WARPS - 1) / TK_WARPS), TK_WARPS * 32, sh, (cudaStream_t)stream>>>(
      n_spec, spec_hyp_off, h_lo, h_hi, win_off, hyp_shift, seg_cnt, hit_rc, hit_isum, hyp_scored, hyp_matched, topk,
      pair_closure, partner, cap, list_pow2, key_cap, c_hyp, c_row, c_cnt, c_isum, n_cand, spec_scored,
      spec_matched);
  return vk_launch_status();
}

}  // extern "C"
