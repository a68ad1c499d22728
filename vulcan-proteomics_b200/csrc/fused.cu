// Fused persistent search: for every spectrum, K1 -> top-K + pair closure -> K2 -> PSM ranking in one CTA, all
// intermediate state in shared memory.
//
// The grid is persistent (a few CTAs per SM); CTAs take spectra from an atomic work counter, so spectra of
// uneven peak counts balance themselves.  Per spectrum:
//   1. the hypotheses' row windows are laid out back to back in a shared-memory count buffer;
//   2. K1: warps take the (hypothesis, tile) items; a warp stages the tile's postings and coarse-bin CSR into its
//      own shared buffer with two bulk (TMA) copies on its mbarrier (bounded wait), then runs the per-peak search
//      (k1_impl.cuh), adding into the count buffer;
//   3. per-hypothesis scored / matched, then top-K by (count desc, row desc, hypothesis asc) -- all entries when at
//      most topk pass the threshold, else a block radix select of the topk-th largest key -- pair closure, a block
//      bitonic sort by (row, hypothesis) and the merge of duplicate rows (lowest hypothesis, highest count): the
//      reference's select_topk (vulcan/gpu/engine.py:284-312);
//   4. K2 (k2_impl.cuh) of every candidate, one thread per candidate, peaks and bucket table in shared memory;
//   5. ranking by (hyperscore desc, row asc) among candidates with matched_b + matched_y >= min_matched, the first
//      `report` written with delta_next / delta_best (engine.py:366-392).
// Outputs equal the staged kernels' (same device functions, same order of every f32 operation).  A spectrum whose
// windows exceed the count buffer (or with more than FS_MAX_HYP hypotheses) is skipped with status bit 1; the
// caller searches it with the staged kernels.  Status bit 2: a tile copy did not complete within the bounded wait.
#include "common.cuh"
#include "k1_impl.cuh"
#include "k2_impl.cuh"

namespace {

constexpr int FS_MAX_HYP = 32;
constexpr uint32_t FS_WAIT_LIMIT = 1u << 22;
constexpr int FS_MAX_WARPS = 16;

struct FusedParams {
  vk_tindex ix;
  float tol_lo, tol_hi;
  int thr, topk, pair_closure, min_matched, report;
  int cnt_cap, cand_pow2, stage_words;
  int n_work;
  const int32_t* spec_ids;
  const int64_t* pk_off;
  const float* pk_mass;
  const float* pk_int;
  const int64_t* spec_hyp_off;
  const int64_t* h_lo;
  const int64_t* h_hi;
  const int8_t* h_maxfz;
  const int64_t* partner;
  const int64_t* seq_off;
  const uint8_t* len;
  const uint64_t* mask;
  const float* mass32;
  const uint8_t* res;
  unsigned int* work_counter;
  int32_t* status;
  int32_t* n_psm;
  int64_t* spec_scored;
  int64_t* spec_matched;
  vk_psm_out psm;
  vk_cand_out cand;
  uint32_t* hyp_scored;
  uint64_t* hyp_matched;
};

__device__ __forceinline__ uint64_t sel_key(int c, int64_t r, int hl) {
  uint64_t kc = (uint64_t)min(c, 32767);
  return (kc << 48) | ((uint64_t)r << 18) | (uint64_t)((1 << 18) - 1 - hl);
}

__device__ __forceinline__ void block_bitonic_u64(uint64_t* v, int n_pow2) {
  for (int k = 2; k <= n_pow2; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < n_pow2; i += blockDim.x) {
        int p = i ^ j;
        if (p > i) {
          uint64_t a = v[i], b = v[p];
          bool up = (i & k) == 0;
          if ((a > b) == up) { v[i] = b; v[p] = a; }
        }
      }
      __syncthreads();
    }
}

// hypothesis (local index) of a count-buffer position
__device__ __forceinline__ int hyp_of(const int* base, int nh, int idx) {
  int h = 0;
  while (h + 1 < nh && base[h + 1] <= idx) ++h;
  return h;
}

__device__ __forceinline__ bool before(double ha, int64_t ra, double hb, int64_t rb) {
  return ha > hb || (ha == hb && ra < rb);
}

__global__ void __launch_bounds__(FS_MAX_WARPS * 32) fused_search_k(FusedParams P, vk_frag_params fpv) {
  extern __shared__ __align__(16) uint8_t fs_smem[];
  __shared__ vk::SmemFrag fp;
  __shared__ __align__(8) uint64_t bars[FS_MAX_WARPS];
  __shared__ int h_base[FS_MAX_HYP + 1], h_tile[FS_MAX_HYP + 1];
  __shared__ int64_t h_lo_s[FS_MAX_HYP], h_hi_s[FS_MAX_HYP];
  __shared__ int h_mfz[FS_MAX_HYP];
  __shared__ int s_work, s_ok, s_nh, s_ntiles, s_W, s_napp, s_nsel, s_ncand;
  __shared__ unsigned long long s_sc, s_mt;
  __shared__ unsigned long long s_prefix, s_pmask;
  __shared__ long long s_need;
  __shared__ int s_warp_tot[FS_MAX_WARPS];

  const int nwarps = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const vk_tindex& ix = P.ix;
  const int T = 1 << ix.tile_shift;
  const int nb = 1 << ix.cbin_bits;
  const int cb_stride = (nb + 1 + 7) & ~7;
  const int tol_da = fpv.tol_da;

  // shared-memory carve-up
  uint8_t* q = fs_smem;
  float* sm = reinterpret_cast<float*>(q);
  q += VK_K2_MAXPK * 4;
  float* si = reinterpret_cast<float*>(q);
  q += VK_K2_MAXPK * 4;
  uint16_t* start = reinterpret_cast<uint16_t*>(q);
  q += vk::K2_BUCKETS * 2;
  uint32_t* counts = reinterpret_cast<uint32_t*>(q);
  q += (size_t)P.cnt_cap * 4;
  uint64_t* key = reinterpret_cast<uint64_t*>(q);
  q += (size_t)P.cand_pow2 * 8;
  double* khs = reinterpret_cast<double*>(q);
  q += (size_t)P.cand_pow2 * 8;
  int32_t* crow = reinterpret_cast<int32_t*>(q);
  int32_t* chl = crow + P.cand_pow2;
  int32_t* ccnt = chl + P.cand_pow2;
  int32_t* frow = ccnt + P.cand_pow2;
  int32_t* fhl = frow + P.cand_pow2;
  int32_t* fcnt = fhl + P.cand_pow2;
  float* ksb = reinterpret_cast<float*>(fcnt + P.cand_pow2);
  float* ksy = ksb + P.cand_pow2;
  float* kppm = ksy + P.cand_pow2;
  int16_t* kmb = reinterpret_cast<int16_t*>(kppm + P.cand_pow2);
  int16_t* kmy = kmb + P.cand_pow2;
  int16_t* klb = kmy + P.cand_pow2;
  int16_t* kly = klb + P.cand_pow2;
  q = reinterpret_cast<uint8_t*>(kly + P.cand_pow2);
  q = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(q) + 15) & ~uintptr_t(15));
  uint32_t* hist = reinterpret_cast<uint32_t*>(q);
  q += 256 * 4;
  const size_t stage_bytes = (size_t)P.stage_words * 4 + (size_t)cb_stride * 2;
  uint32_t* post = reinterpret_cast<uint32_t*>(q + stage_bytes * warp);
  uint16_t* cb = reinterpret_cast<uint16_t*>(q + stage_bytes * warp + (size_t)P.stage_words * 4);

  vk::load_frag(fp, fpv);
  if (lane == 0) vk::mbar_init(&bars[warp], 1);
  vk::fence_mbar_init();
  __syncthreads();
  uint32_t phase = 0;
  bool stalled = false;   // this warp's tile barrier gave up twice: it issues no more copies for the whole launch
  const vk::K2Out kout{khs, ksb, ksy, kppm, kmb, kmy, klb, kly};

  for (;;) {
    if (threadIdx.x == 0) s_work = (int)atomicAdd(P.work_counter, 1u);
    __syncthreads();
    const int wi = s_work;
    if (wi >= P.n_work) break;
    const int s = P.spec_ids ? P.spec_ids[wi] : wi;
    const int64_t hb = P.spec_hyp_off[s], he = P.spec_hyp_off[s + 1];
    const int64_t p0 = P.pk_off[s], p1 = P.pk_off[s + 1];
    if (threadIdx.x == 0) {
      int nh = (int)(he - hb);
      int ok = nh <= FS_MAX_HYP;
      int base = 0, nt = 0;
      for (int h = 0; ok && h < nh; ++h) {
        int64_t lo = P.h_lo[hb + h], hi = P.h_hi[hb + h];
        int64_t wl = hi > lo ? hi - lo : 0;
        h_lo_s[h] = lo;
        h_hi_s[h] = hi;
        h_mfz[h] = P.h_maxfz[hb + h];
        h_base[h] = base;
        h_tile[h] = nt;
        if ((int64_t)base + wl > P.cnt_cap) ok = 0;
        base += (int)wl;
        if (wl > 0) nt += (int)(((hi - 1) >> ix.tile_shift) - (lo >> ix.tile_shift) + 1);
      }
      if (ok) {
        h_base[nh] = base;
        h_tile[nh] = nt;
      }
      s_ok = ok;
      s_nh = nh;
      s_ntiles = nt;
      s_W = base;
      s_napp = 0;
      s_nsel = 0;
      s_sc = 0;
      s_mt = 0;
    }
    __syncthreads();
    if (!s_ok) {
      if (threadIdx.x == 0) {
        atomicOr(&P.status[s], 1);
        P.n_psm[s] = 0;
        if (P.cand.n_cand) P.cand.n_cand[s] = -1;
      }
      __syncthreads();
      continue;
    }
    const int nh = s_nh, W = s_W, ntiles = s_ntiles;
    const int np = (int)min((int64_t)VK_K2_MAXPK, p1 - p0);
    for (int j = threadIdx.x; j < np; j += blockDim.x) {
      sm[j] = P.pk_mass[p0 + j];
      si[j] = P.pk_int[p0 + j];
    }
    for (int j = threadIdx.x; j < W; j += blockDim.x) counts[j] = 0;
    __syncthreads();
    // ---------------------------------------------------------------- K1
    for (int it = warp; it < ntiles; it += nwarps) {
      int h = 0;
      while (h + 1 < nh && h_tile[h + 1] <= it) ++h;
      const int64_t lo = h_lo_s[h], hi = h_hi_s[h];
      const int64_t t = (lo >> ix.tile_shift) + (it - h_tile[h]);
      if (stalled) {   // copies of this warp may still be in flight: its buffers and barrier are not reused
        if (lane == 0) atomicOr(&P.status[s], VK_STATUS_WAIT_TIMEOUT << 1);
        continue;
      }
      const int64_t po = ix.tile_off[t];
      const uint32_t post_bytes = (uint32_t)((ix.tile_off[t + 1] - po) * 4);
      if (lane == 0) {
        vk::mbar_expect_tx(&bars[warp], post_bytes + (uint32_t)cb_stride * 2);
        if (post_bytes) vk::bulk_g2s(post, ix.postings + po, post_bytes, &bars[warp]);
        vk::bulk_g2s(cb, ix.cbin_off + t * cb_stride, (uint32_t)cb_stride * 2, &bars[warp]);
      }
      __syncwarp();
      // warp-uniform decisions: every lane waits, and the warp gives up only if a lane did
      if (!__all_sync(0xffffffffu, vk::mbar_wait(&bars[warp], phase, FS_WAIT_LIMIT))) {
        if (lane == 0) atomicOr(&P.status[s], VK_STATUS_WAIT_TIMEOUT << 1);
        if (!__all_sync(0xffffffffu, vk::mbar_wait(&bars[warp], phase, FS_WAIT_LIMIT))) {
          stalled = true;   // the staged tile is not read and no later copy targets these buffers
          continue;
        }
      }
      phase ^= 1u;
      const int64_t r0 = t << ix.tile_shift;
      const int rlo = (int)max(lo - r0, (int64_t)0), rhi = (int)min(hi - r0, (int64_t)T);
      vk::k1_item_per_peak(post, cb, counts, (int64_t)h_base[h] + r0 - lo, rlo, rhi, p0, p1, h_mfz[h], P.pk_mass,
                           P.tol_lo, P.tol_hi, tol_da, ix, lane);
      __syncwarp();
    }
    if (warp == 0) {
      // bucket table of the peaks for K2 (the staged search reads peaks from global memory)
      (void)vk::build_table(sm, si, start, np, lane);
    }
    __syncthreads();
    // ---------------------------------------------------------------- statistics, threshold count
    for (int h = warp; h < nh; h += nwarps) {
      long long sc = 0, mt = 0, ap = 0;
      for (int j = h_base[h] + lane; j < h_base[h + 1]; j += 32) {
        const int c = (int)counts[j];
        sc += c > 0;
        mt += c;
        ap += c >= P.thr;
      }
      sc = vk::warp_sum(sc);
      mt = vk::warp_sum(mt);
      ap = vk::warp_sum(ap);
      if (lane == 0) {
        if (P.hyp_scored) {
          P.hyp_scored[hb + h] = (uint32_t)sc;
          P.hyp_matched[hb + h] = (uint64_t)mt;
        }
        atomicAdd(&s_sc, (unsigned long long)sc);
        atomicAdd(&s_mt, (unsigned long long)mt);
        atomicAdd(&s_napp, (int)ap);
      }
    }
    if (threadIdx.x == 0) {
      s_prefix = 0;
      s_pmask = 0;
      s_need = P.topk;
    }
    __syncthreads();
    const bool limit = s_napp > P.topk;
    // ---------------------------------------------------------------- top-K threshold (radix select)
    if (limit) {
      for (int shift = 56; shift >= 0; shift -= 8) {
        for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
        __syncthreads();
        const uint64_t prefix = s_prefix, pmask = s_pmask;
        for (int j = threadIdx.x; j < W; j += blockDim.x) {
          const int c = (int)counts[j];
          if (c < P.thr) continue;
          const int h = hyp_of(h_base, nh, j);
          const uint64_t k = sel_key(c, h_lo_s[h] + (j - h_base[h]), h);
          if ((k & pmask) == prefix) atomicAdd(&hist[(k >> shift) & 255], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
          long long above = 0, need = s_need;
          int d = 255;
          for (; d > 0; --d) {
            if (above + hist[d] >= need) break;
            above += hist[d];
          }
          s_need = need - above;
          s_prefix = prefix | ((uint64_t)d << shift);
          s_pmask = pmask | (255ull << shift);
        }
        __syncthreads();
      }
    }
    const uint64_t kth = s_prefix;
    // ---------------------------------------------------------------- gather, closure
    for (int j = threadIdx.x; j < W; j += blockDim.x) {
      const int c = (int)counts[j];
      if (c < P.thr) continue;
      const int h = hyp_of(h_base, nh, j);
      const int64_t r = h_lo_s[h] + (j - h_base[h]);
      if (limit && sel_key(c, r, h) < kth) continue;
      const int pos = atomicAdd(&s_nsel, 1);
      crow[pos] = (int32_t)r;
      chl[pos] = h;
      ccnt[pos] = c;
    }
    __syncthreads();
    const int n_sel = s_nsel;
    int n_list = n_sel;
    if (P.pair_closure) {
      for (int j = threadIdx.x; j < n_sel; j += blockDim.x) {
        crow[n_sel + j] = (int32_t)P.partner[crow[j]];
        chl[n_sel + j] = chl[j];
        ccnt[n_sel + j] = -1;
      }
      n_list = 2 * n_sel;
    }
    int n_pow2 = 32;
    while (n_pow2 < n_list) n_pow2 <<= 1;
    __syncthreads();
    for (int j = threadIdx.x; j < n_pow2; j += blockDim.x)
      key[j] = j < n_list ? (((uint64_t)crow[j] << 34) | ((uint64_t)chl[j] << 16) | (uint64_t)j) : ~0ull;
    __syncthreads();
    block_bitonic_u64(key, n_pow2);
    // merge duplicate rows: ordered compaction of the run heads (block scan of warp ballots)
    {
      int total = 0;
      for (int i0 = 0; i0 < n_list; i0 += blockDim.x) {
        const int i = i0 + threadIdx.x;
        bool head = false;
        int64_t r = 0;
        if (i < n_list) {
          r = (int64_t)(key[i] >> 34);
          head = i == 0 || (int64_t)(key[i - 1] >> 34) != r;
        }
        const unsigned m = __ballot_sync(VK_FULL, head);
        if (lane == 0) s_warp_tot[warp] = __popc(m);
        __syncthreads();
        int before_w = 0, all = 0;
        for (int w = 0; w < nwarps; ++w) {
          if (w < warp) before_w += s_warp_tot[w];
          all += s_warp_tot[w];
        }
        if (head) {
          const int idx = (int)(key[i] & 0xffff);
          int best = ccnt[idx];
          for (int k = i + 1; k < n_list && (int64_t)(key[k] >> 34) == r; ++k) best = max(best, ccnt[key[k] & 0xffff]);
          const int pos = total + before_w + __popc(m & ((1u << lane) - 1u));
          frow[pos] = (int32_t)r;
          fhl[pos] = (int32_t)((key[i] >> 16) & 0x3ffff);
          fcnt[pos] = best;
        }
        total += all;
        __syncthreads();
      }
      if (threadIdx.x == 0) s_ncand = total;
    }
    __syncthreads();
    const int n_cand = s_ncand;
    // ---------------------------------------------------------------- K2
    {
      vk::PeakTable pt;
      pt.sm = sm;
      pt.si = si;
      pt.start = start;
      pt.np = np;
      pt.m0 = np > 0 ? sm[0] : 0.f;
      const float span = np > 0 ? __fsub_rn(sm[np - 1], pt.m0) : 0.f;
      pt.inv_w = span > 0.f ? __fdiv_rn((float)vk::K2_BUCKETS, span) : 0.f;
      for (int j = threadIdx.x; j < n_cand; j += blockDim.x)
        vk::k2_score<false>(fp, pt, frow[j], h_mfz[fhl[j]], P.seq_off, P.len, P.mask, P.mass32, P.res, P.tol_lo,
                            P.tol_hi, 0.f, kout, j);
    }
    __syncthreads();
    // ---------------------------------------------------------------- optional candidate outputs
    if (P.cand.n_cand) {
      const int64_t slot = (int64_t)s * P.cand.cap;
      for (int j = threadIdx.x; j < n_cand; j += blockDim.x) {
        P.cand.c_hyp[slot + j] = hb + fhl[j];
        P.cand.c_row[slot + j] = frow[j];
        P.cand.c_cnt[slot + j] = fcnt[j];
        if (P.cand.hs) {
          P.cand.hs[slot + j] = khs[j];
          P.cand.sb[slot + j] = ksb[j];
          P.cand.sy[slot + j] = ksy[j];
          P.cand.ppm[slot + j] = kppm[j];
          P.cand.mb[slot + j] = kmb[j];
          P.cand.my[slot + j] = kmy[j];
          P.cand.lb[slot + j] = klb[j];
          P.cand.ly[slot + j] = kly[j];
        }
      }
      if (threadIdx.x == 0) P.cand.n_cand[s] = n_cand;
    }
    // ---------------------------------------------------------------- ranking (warp 0)
    if (warp == 0) {
      double prev_h = 0.0, best_h = 0.0, cur_h = 0.0;
      int64_t prev_r = -1;
      int cur_j = -1;
      bool have_prev = false;
      int n = 0;
      for (int k = 0; k <= P.report; ++k) {
        double bh = 0.0;
        int64_t br = -1;
        int bj = -1;
        for (int j = lane; j < n_cand; j += 32) {
          if ((int)kmb[j] + (int)kmy[j] < P.min_matched) continue;
          const double h = khs[j];
          const int64_t r = frow[j];
          if (have_prev && !before(prev_h, prev_r, h, r)) continue;
          if (bj < 0 || before(h, r, bh, br)) { bh = h; br = r; bj = j; }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const double oh = __shfl_xor_sync(VK_FULL, bh, o);
          const int64_t orr = __shfl_xor_sync(VK_FULL, br, o);
          const int oj = __shfl_xor_sync(VK_FULL, bj, o);
          if (oj >= 0 && (bj < 0 || before(oh, orr, bh, br))) { bh = oh; br = orr; bj = oj; }
        }
        if (k > 0) {
          if (lane == 0) {
            const int64_t slot = (int64_t)s * P.report + (k - 1);
            P.psm.row[slot] = frow[cur_j];
            P.psm.hyp[slot] = hb + fhl[cur_j];
            P.psm.k1[slot] = fcnt[cur_j];
            P.psm.rank[slot] = k;
            P.psm.dnext[slot] = cur_h - (bj >= 0 ? bh : 0.0);
            P.psm.dbest[slot] = best_h - cur_h;
            P.psm.hs[slot] = khs[cur_j];
            P.psm.sb[slot] = ksb[cur_j];
            P.psm.sy[slot] = ksy[cur_j];
            P.psm.ppm[slot] = kppm[cur_j];
            P.psm.mb[slot] = kmb[cur_j];
            P.psm.my[slot] = kmy[cur_j];
            P.psm.lb[slot] = klb[cur_j];
            P.psm.ly[slot] = kly[cur_j];
          }
          ++n;
        }
        if (bj < 0) break;
        if (k == 0) best_h = bh;
        cur_h = bh;
        cur_j = bj;
        prev_h = bh;
        prev_r = br;
        have_prev = true;
      }
      if (lane == 0) {
        for (int k = n; k < P.report; ++k) P.psm.row[(int64_t)s * P.report + k] = -1;
        P.n_psm[s] = n;
        P.spec_scored[s] = (int64_t)s_sc;
        P.spec_matched[s] = (int64_t)s_mt;
      }
    }
    __syncthreads();
  }
}

}  // namespace

extern "C" {

int vk_search_fused_smem(const vk_tindex* ix, int warps, int topk, int pair_closure, int cnt_cap, int64_t* bytes) {
  if (!ix || !bytes || warps < 1 || warps > FS_MAX_WARPS || topk < 1 || cnt_cap < 32) return VK_E_ARG;
  int cap = (pair_closure ? 2 : 1) * topk;
  int cand_pow2 = 32;
  while (cand_pow2 < cap) cand_pow2 <<= 1;
  int stage_words = (ix->max_tile_postings + 3) & ~3;
  int cb_stride = ((1 << ix->cbin_bits) + 1 + 7) & ~7;
  int64_t b = (int64_t)VK_K2_MAXPK * 8 + vk::K2_BUCKETS * 2 + (int64_t)cnt_cap * 4 + (int64_t)cand_pow2 * (8 + 8) +
              (int64_t)cand_pow2 * (6 * 4 + 3 * 4 + 4 * 2) + 16 + 256 * 4 +
              (int64_t)warps * ((int64_t)stage_words * 4 + cb_stride * 2);
  *bytes = b;
  return 0;
}

int vk_search_fused(const vk_tindex* ix, const vk_frag_params* fp, const vk_fused_in* in, int warps, int cnt_cap,
                    int grid, unsigned int* work_counter, int32_t* status, int32_t* n_psm, int64_t* spec_scored,
                    int64_t* spec_matched, const vk_psm_out* psm, const vk_cand_out* cand, uint32_t* hyp_scored,
                    uint64_t* hyp_matched, void* stream) {
  if (!ix || !fp || !in || !psm || warps < 1 || warps > FS_MAX_WARPS || grid < 1) return VK_E_ARG;
  if (in->topk < 1 || in->report < 1 || cnt_cap < 32 || (ix->max_tile_postings & 3)) return VK_E_ARG;
  if (in->n_work <= 0) return 0;
  cudaStream_t st = (cudaStream_t)stream;
  FusedParams P;
  P.ix = *ix;
  P.tol_lo = in->tol_lo;
  P.tol_hi = in->tol_hi;
  P.thr = in->thr;
  P.topk = in->topk;
  P.pair_closure = in->pair_closure;
  P.min_matched = in->min_matched;
  P.report = in->report;
  P.cnt_cap = cnt_cap;
  int cap = (in->pair_closure ? 2 : 1) * in->topk;
  int cand_pow2 = 32;
  while (cand_pow2 < cap) cand_pow2 <<= 1;
  if (cand_pow2 > 65536) return VK_E_ARG;
  P.cand_pow2 = cand_pow2;
  P.stage_words = (ix->max_tile_postings + 3) & ~3;
  P.n_work = in->n_work;
  P.spec_ids = in->spec_ids;
  P.pk_off = in->pk_off;
  P.pk_mass = in->pk_mass;
  P.pk_int = in->pk_int;
  P.spec_hyp_off = in->spec_hyp_off;
  P.h_lo = in->h_lo;
  P.h_hi = in->h_hi;
  P.h_maxfz = in->h_maxfz;
  P.partner = in->partner;
  P.seq_off = in->seq_off;
  P.len = in->len;
  P.mask = in->mask;
  P.mass32 = in->mass32;
  P.res = in->res;
  P.work_counter = work_counter;
  P.status = status;
  P.n_psm = n_psm;
  P.spec_scored = spec_scored;
  P.spec_matched = spec_matched;
  P.psm = *psm;
  vk_cand_out none = {};
  P.cand = cand ? *cand : none;
  if (P.cand.n_cand && P.cand.cap < cap) return VK_E_ARG;
  P.hyp_scored = hyp_scored;
  P.hyp_matched = hyp_matched;
  int64_t sh = 0;
  int rc = vk_search_fused_smem(ix, warps, in->topk, in->pair_closure, cnt_cap, &sh);
  if (rc) return rc;
  if (sh > 225 * 1024) return VK_E_ARG;
  cudaError_t e = cudaFuncSetAttribute(fused_search_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  if (e != cudaSuccess) return vk_err(e);
  e = cudaMemsetAsync(work_counter, 0, sizeof(unsigned int), st);
  if (e != cudaSuccess) return vk_err(e);
  e = cudaMemsetAsync(status, 0, sizeof(int32_t) * (size_t)in->n_spec, st);
  if (e != cudaSuccess) return vk_err(e);
  fused_search_k<<<grid, warps * 32, (size_t)sh, st>>>(P, *fp);
  return vk_launch_status();
}

int vk_search_fused_grid(const vk_tindex* ix, int warps, int topk, int pair_closure, int cnt_cap, int* grid) {
  if (!grid) return VK_E_ARG;
  int64_t sh = 0;
  int rc = vk_search_fused_smem(ix, warps, topk, pair_closure, cnt_cap, &sh);
  if (rc) return rc;
  if (sh > 225 * 1024) return VK_E_ARG;
  cudaError_t e = cudaFuncSetAttribute(fused_search_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  if (e != cudaSuccess) return vk_err(e);
  int per_sm = 0, dev = 0, n_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fused_search_k, warps * 32, (size_t)sh);
  if (e != cudaSuccess) return vk_err(e);
  e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return vk_err(e);
  e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return vk_err(e);
  *grid = (per_sm > 0 ? per_sm : 1) * n_sm;
  return 0;
}

}  // extern "C"
