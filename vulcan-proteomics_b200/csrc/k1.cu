// K1 shared-peak counting on the tiled fragment index.
//
// Work items are (tile, hypothesis) pairs grouped by tile.  One CTA owns one tile: thread 0 stages the tile's
// postings, its coarse-bin CSR and its presence bitmap (a few bits per coarse bin) into shared memory with three bulk
// (TMA) copies completing on one mbarrier; then each warp takes the tile's hypotheses in turn (k1_impl.cuh,
// k1_item_filtered): lanes stride over the spectrum's peaks x fragment charges, read each tolerance window's filter
// word (computed once per pass by vk_k1_peak_keys), drop the windows whose bitmap bits are clear, and search the rest
// through the coarse bins and a binary search in the staged tile, one queued window per lane.
// Every posting in a window adds one to its row in a warp-private shared-memory histogram (rows of the hypothesis
// window only; with intensity sums, a second histogram adds the peak's fixed-point weight).  The histograms are
// written to the hypothesis' dense slices.
//
// Result = the reference's brute-force count (vulcan/gpu/kernels.cu:195-232) for every window row: a posting key
// compares exactly like its f32 fragment mass, so f == a and f == bd are both counted.
#include "common.cuh"
#include "k1_impl.cuh"

namespace {

constexpr int K1_MAX_WARPS = 16;
constexpr uint32_t WAIT_LIMIT = 1u << 22;

__global__ void plan_count_k(int64_t n_hyp, int shift, const int64_t* h_lo, const int64_t* h_hi,
                             unsigned long long* tile_items, int64_t* win_len) {
  int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (h >= n_hyp) return;
  int64_t lo = h_lo[h], hi = h_hi[h];
  win_len[h] = hi > lo ? hi - lo : 0;
  if (hi <= lo) return;
  for (int64_t t = lo >> shift; t <= (hi - 1) >> shift; ++t) atomicAdd(&tile_items[t], 1ull);
}

// item_cap bounds item_hyp: an item past it is not written and sets VK_STATUS_OVERFLOW
__global__ void plan_fill_k(int64_t n_hyp, int shift, const int64_t* h_lo, const int64_t* h_hi,
                            const int64_t* tile_item_off, unsigned long long* cursor, int32_t* item_hyp,
                            int64_t item_cap, int32_t* status) {
  int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (h >= n_hyp) return;
  int64_t lo = h_lo[h], hi = h_hi[h];
  if (hi <= lo) return;
  for (int64_t t = lo >> shift; t <= (hi - 1) >> shift; ++t) {
    unsigned long long pos = atomicAdd(&cursor[t], 1ull);
    const int64_t at = tile_item_off[t] + (int64_t)pos;
    if (at < item_cap) item_hyp[at] = (int32_t)h;
    else atomicOr(status, VK_STATUS_OVERFLOW);
  }
}

constexpr int K1_ITEMS = 64;   // item records staged per round

// Record of one (tile, hypothesis) item, read by the warp that takes it.
struct K1Rec {
  int64_t p0, base;   // first peak of the spectrum; cnt / isum index of the tile's row 0 for this hypothesis
  int32_t n, rows;    // peaks; local rows rlo | rhi << 16
  int32_t mfz;        // fragment charges + 1 (0: item skipped)
  float ws;           // intensity weight scale 2^24 / TIC
  int32_t h;          // hypothesis (the hit-list output appends to its region)
};

// Outputs of the hit-list form of K1 (vk_k1_hits): instead of a dense count per window row, each (tile, hypothesis)
// item writes the rows of its tile with count >= thr, in row order, to the start of its own segment of the
// hypothesis' region -- the slots of the window rows it covers -- as count << 32 | row (rc) and isum, and the number
// of those rows to seg_cnt at the segment's first slot; hyp_shift[h] gets the tiling's tile shift (the segment
// boundaries); per hypothesis the number of rows with a nonzero count and the sum of the counts (integer atomics).
// No atomic decides a position, so the layout does not depend on scheduling.
struct K1Hits {
  int thr;
  const int32_t* h_thr;   // per-hypothesis thresholds (NULL: thr for all)
  uint64_t* rc;
  uint32_t* isum;
  uint32_t* seg_cnt;
  int8_t* hyp_shift;
  uint32_t* hyp_scored;
  unsigned long long* hyp_matched;
};

// Loads the record of item `it` of the tile whose first row is r0; items and windows must lie inside the buffers the
// caller sized by bounds, anything else is skipped (mfz = 0) and sets VK_STATUS_OVERFLOW.
__device__ __forceinline__ K1Rec k1_record(int64_t it, int64_t r0, int T, const int32_t* item_hyp, int64_t n_hyp,
                                           const int32_t* h_spec, const int8_t* h_maxfz, const int64_t* h_lo,
                                           const int64_t* h_hi, const int64_t* win_off, int64_t cnt_cap,
                                           const int64_t* pk_off, const float* tic, bool want_ws, int32_t* status) {
  K1Rec r;
  r.mfz = 0;
  const int h = item_hyp[it];
  if (h < 0 || h >= n_hyp) {
    atomicOr(status, VK_STATUS_OVERFLOW);
    return r;
  }
  const int64_t lo = h_lo[h], hi = h_hi[h];
  if (hi <= lo) return r;
  if (win_off[h] + (hi - lo) > cnt_cap) {
    atomicOr(status, VK_STATUS_OVERFLOW);
    return r;
  }
  const int s = h_spec[h];
  r.h = h;
  r.p0 = pk_off[s];
  r.n = (int32_t)(pk_off[s + 1] - r.p0);
  r.base = win_off[h] + (r0 - lo);
  r.rows = (int32_t)max(lo - r0, (int64_t)0) | ((int32_t)min(hi - r0, (int64_t)T) << 16);
  const float ts = want_ws ? tic[s] : 0.f;
  r.ws = ts > 0.f ? __fdiv_rn(16777216.0f, ts) : 0.f;
  r.mfz = h_maxfz[h];
  return r;
}

// One CTA per tile with work.  Thread 0 issues the bulk copies of the tile's postings, coarse-bin CSR and bitmap;
// meanwhile the CTA loads the item records of the round (up to K1_ITEMS items) into shared memory, so that each
// item's chain of dependent loads (item -> hypothesis -> spectrum) overlaps the copy and the other items'.  Warp w
// then runs the filtered per-item search of items w, w + warps, ... (measured faster than items taken one at a time
// through a shared-memory counter).
// HITS: the hit-list form (K1Hits) instead of the dense counts.
template <bool HITS>
__global__ void __launch_bounds__(K1_MAX_WARPS * 32, 1)
k1_tiles_k(vk_tindex ix, float tol_lo, float tol_hi, int tol_da, int post_cap, const int64_t* tile_item_off,
           const int32_t* item_hyp, int64_t n_hyp, int64_t item_cap, const int32_t* h_spec, const int8_t* h_maxfz,
           const int64_t* h_lo, const int64_t* h_hi, const int64_t* win_off, int64_t cnt_cap, const int64_t* pk_off,
           const float* pk_mass, int32_t* cnt, int32_t* status, const float* pk_int, const float* tic,
           uint32_t* isum_out, const uint2* pk_keys, const uint32_t* pk_filt, int n_kz, int64_t kstride,
           K1Hits hits) {
  extern __shared__ __align__(16) uint8_t k1_smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ K1Rec rec[K1_ITEMS];
  const int64_t t = blockIdx.x;
  const int64_t i0 = min(tile_item_off[t], item_cap), i1 = min(tile_item_off[t + 1], item_cap);
  if (i0 == i1) return;
  const int n_warps = blockDim.x >> 5;
  const int T = 1 << ix.tile_shift;
  const int nb = 1 << ix.cbin_bits;
  const int stride = (nb + 1 + 7) & ~7;
  uint32_t* post = reinterpret_cast<uint32_t*>(k1_smem);
  uint16_t* cb = reinterpret_cast<uint16_t*>(k1_smem + (size_t)post_cap * 4);
  uint32_t* bm = reinterpret_cast<uint32_t*>(k1_smem + (size_t)post_cap * 4 + (size_t)stride * 2);
  uint32_t* hist = bm + nb * vk::K1_BM_WORDS;
  uint32_t* queue = hist + n_warps * T;   // per warp K1_QUEUE entries
  uint32_t* ihist = queue + n_warps * vk::K1_QUEUE;   // per warp T intensity sums (pruner features only)
  const int64_t po = ix.tile_off[t];
  const uint32_t post_bytes = (uint32_t)((ix.tile_off[t + 1] - po) * 4);
  const uint32_t cb_bytes = (uint32_t)stride * 2;
  const uint32_t bm_bytes = (uint32_t)nb * vk::K1_BM_WORDS * 4;
  if (threadIdx.x == 0) {
    vk::mbar_init(&bar, 1);
    vk::fence_mbar_init();
    vk::mbar_expect_tx(&bar, post_bytes + cb_bytes + bm_bytes);
    if (post_bytes) vk::bulk_g2s(post, ix.postings + po, post_bytes, &bar);
    vk::bulk_g2s(cb, ix.cbin_off + t * stride, cb_bytes, &bar);
    vk::bulk_g2s(bm, ix.bitmap + t * nb * vk::K1_BM_WORDS, bm_bytes, &bar);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* qw = queue + warp * vk::K1_QUEUE;
  uint32_t* hw = hist + warp * T;
  uint32_t* iw = isum_out ? ihist + warp * T : nullptr;
  const int64_t r0 = t << ix.tile_shift;
  bool staged = false;
  for (int64_t c0 = i0; c0 < i1; c0 += K1_ITEMS) {
    const int m = (int)min((int64_t)K1_ITEMS, i1 - c0);
    for (int j = threadIdx.x; j < m; j += blockDim.x)
      rec[j] = k1_record(c0 + j, r0, T, item_hyp, n_hyp, h_spec, h_maxfz, h_lo, h_hi, win_off, cnt_cap, pk_off,
                         tic, iw != nullptr, status);
    __syncthreads();
    if (!staged) {
      // CTA-uniform decision: later rounds begin with CTA barriers
      if (!__syncthreads_and(vk::mbar_wait(&bar, 0, WAIT_LIMIT))) {
        // give up on this tile, but do not leave while the copies may still land in shared memory
        if (threadIdx.x == 0) atomicOr(status, VK_STATUS_WAIT_TIMEOUT);
        vk::mbar_wait(&bar, 0, WAIT_LIMIT);
        return;
      }
      staged = true;
    }
    for (int j = warp; j < m; j += n_warps) {
      const K1Rec r = rec[j];
      if (r.mfz == 0) continue;
      const int rlo = r.rows & 0xffff, rhi = r.rows >> 16;
      for (int q = rlo + lane; q < rhi; q += 32) {
        hw[q] = 0;
        if (iw) iw[q] = 0;
      }
      __syncwarp();
      vk::k1_item_filtered(post, cb, bm, hw, iw, rlo, rhi, r.p0, r.p0 + r.n,
                           r.mfz, pk_keys, pk_filt, n_kz, kstride, pk_mass, tol_lo, tol_hi, tol_da, ix, lane, qw,
                           pk_int, r.ws);
      __syncwarp();
      if (HITS) {
        // the item's segment: the slots of the window rows rlo..rhi of this tile (r.base is the region index of
        // the tile's row 0); kept rows compacted to its start in row order, their number at its first slot
        const int64_t seg = r.base + rlo;
        const int thr_h = hits.h_thr ? hits.h_thr[r.h] : hits.thr;
        // per item at most T rows of at most (peaks x charges) counts each: 32-bit sums, one warp reduction each
        uint32_t sc = 0, mt = 0;
        int n_kept = 0;
        for (int q0 = rlo; q0 < rhi; q0 += 32) {
          const int q = q0 + lane;
          const uint32_t c = q < rhi ? hw[q] : 0u;
          sc += c > 0u;
          mt += c;
          const bool keep = q < rhi && (int)c >= thr_h;
          const unsigned bal = __ballot_sync(VK_FULL, keep);
          if (keep) {
            const int64_t at = seg + n_kept + __popc(bal & ((1u << lane) - 1u));
            hits.rc[at] = ((uint64_t)c << 32) | (uint64_t)(r0 + q);
            if (iw) hits.isum[at] = iw[q];
          }
          n_kept += __popc(bal);
        }
        sc = __reduce_add_sync(VK_FULL, sc);
        mt = __reduce_add_sync(VK_FULL, mt);
        if (lane == 0) {
          hits.seg_cnt[seg] = (uint32_t)n_kept;
          hits.hyp_shift[r.h] = (int8_t)ix.tile_shift;   // every item of h writes the same value
          if (sc) atomicAdd(&hits.hyp_scored[r.h], sc);
          if (mt) atomicAdd(&hits.hyp_matched[r.h], (unsigned long long)mt);
        }
      } else {
        for (int q = rlo + lane; q < rhi; q += 32) {
          cnt[r.base + q] = (int32_t)hw[q];
          if (iw) isum_out[r.base + q] = iw[q];
        }
      }
      __syncwarp();
    }
    if (c0 + K1_ITEMS < i1) __syncthreads();   // the records are overwritten by the next round
  }
}

// Window keys and filter words of every kept peak at fragment charges 1..n_kz; *n_peaks = the kept peak count.
__global__ void peak_keys_k(vk_tindex ix, float tol_lo, float tol_hi, int tol_da, const int64_t* n_peaks,
                            const float* pk_mass, int n_kz, int64_t kstride, uint2* keys, uint32_t* filt) {
  const int64_t n = min(*n_peaks, kstride);
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const float pm = pk_mass[p];
    for (int z = 1; z <= n_kz; ++z) {
      const uint2 k = vk::k1_window_keys(pm, z, tol_lo, tol_hi, tol_da, ix);
      keys[(int64_t)(z - 1) * kstride + p] = k;
      filt[(int64_t)(z - 1) * kstride + p] = vk::k1_filter_word(k, ix);
    }
  }
}

}  // namespace

extern "C" {

int vk_k1_plan_count(const vk_tindex* ix, int64_t n_hyp, const int64_t* h_lo, const int64_t* h_hi,
                     int64_t* tile_items, int64_t* win_len, void* stream) {
  if (!ix) return VK_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  if (ix->n_tiles > 0) {
    cudaError_t e = cudaMemsetAsync(tile_items, 0, sizeof(int64_t) * ix->n_tiles, st);
    if (e != cudaSuccess) return vk_err(e);
  }
  if (n_hyp == 0) return 0;
  plan_count_k<<<(unsigned)((n_hyp + 255) / 256), 256, 0, st>>>(n_hyp, ix->tile_shift, h_lo, h_hi,
                                                                 (unsigned long long*)tile_items, win_len);
  return vk_launch_status();
}

int vk_k1_plan_fill(const vk_tindex* ix, int64_t n_hyp, const int64_t* h_lo, const int64_t* h_hi,
                    const int64_t* tile_item_off, int64_t* cursor, int32_t* item_hyp, int64_t item_cap,
                    int32_t* status, void* stream) {
  if (!status || item_cap < 0) return VK_E_ARG;
  if (!ix) return VK_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  if (ix->n_tiles > 0) {
    cudaError_t e = cudaMemsetAsync(cursor, 0, sizeof(int64_t) * ix->n_tiles, st);
    if (e != cudaSuccess) return vk_err(e);
  }
  if (n_hyp == 0) return 0;
  plan_fill_k<<<(unsigned)((n_hyp + 255) / 256), 256, 0, st>>>(n_hyp, ix->tile_shift, h_lo, h_hi, tile_item_off,
                                                                (unsigned long long*)cursor, item_hyp, item_cap,
                                                                status);
  return vk_launch_status();
}

}  // extern "C"

namespace {

template <bool HITS>
int k1_tiles_launch(const vk_tindex* ix, const vk_frag_params* fp, float tol_lo, float tol_hi, int warps,
                    const int64_t* tile_item_off, const int32_t* item_hyp, int64_t n_hyp, int64_t item_cap,
                    const int32_t* h_spec, const int8_t* h_maxfz, const int64_t* h_lo, const int64_t* h_hi,
                    const int64_t* win_off, int64_t cnt_cap, const int64_t* pk_off, const float* pk_mass,
                    int32_t* cnt, int32_t* status, const float* pk_int, const float* tic, uint32_t* isum,
                    const uint32_t* pk_keys, const uint32_t* pk_filt, int n_kz, int64_t kstride, K1Hits hits,
                    void* stream) {
  if (!ix || !fp || !status) return VK_E_ARG;
  if (ix->n_tiles == 0) return 0;
  if ((ix->max_tile_postings & 3) || ix->max_tile_postings < 0 || warps < 1 || warps > K1_MAX_WARPS) return VK_E_ARG;
  if (!ix->bitmap || ((uintptr_t)ix->bitmap & 15)) return VK_E_ARG;
  if (n_kz < 0 || (n_kz > 0 && (!pk_keys || !pk_filt || kstride < 0 || ((uintptr_t)pk_keys & 7)))) return VK_E_ARG;
  const int T = 1 << ix->tile_shift;
  const int nb = 1 << ix->cbin_bits;
  const int stride = (nb + 1 + 7) & ~7;
  if (isum && (!pk_int || !tic)) return VK_E_ARG;
  const size_t sh = (size_t)ix->max_tile_postings * 4 + (size_t)stride * 2 + (size_t)nb * vk::K1_BM_WORDS * 4 +
                    (size_t)warps * (T * 4 * (isum ? 2 : 1) + vk::K1_QUEUE * 4);
  if (sh > 200 * 1024) return VK_E_TOO_LARGE;
  cudaError_t e = cudaFuncSetAttribute(k1_tiles_k<HITS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  if (e != cudaSuccess) return vk_err(e);
  k1_tiles_k<HITS><<<(unsigned)ix->n_tiles, warps * 32, sh, (cudaStream_t)stream>>>(
      *ix, tol_lo, tol_hi, fp->tol_da, ix->max_tile_postings, tile_item_off, item_hyp, n_hyp, item_cap, h_spec,
      h_maxfz, h_lo, h_hi, win_off, cnt_cap, pk_off, pk_mass, cnt, status, pk_int, tic, isum,
      reinterpret_cast<const uint2*>(pk_keys), pk_filt, n_kz > 0 ? n_kz : 0, kstride, hits);
  return vk_launch_status();
}

}  // namespace

extern "C" {

int vk_k1_tiles(const vk_tindex* ix, const vk_frag_params* fp, float tol_lo, float tol_hi, int warps,
                const int64_t* tile_item_off, const int32_t* item_hyp, int64_t n_hyp, int64_t item_cap,
                const int32_t* h_spec, const int8_t* h_maxfz, const int64_t* h_lo, const int64_t* h_hi,
                const int64_t* win_off, int64_t cnt_cap, const int64_t* pk_off, const float* pk_mass, int32_t* cnt,
                int32_t* status, const float* pk_int, const float* tic, uint32_t* isum, const uint32_t* pk_keys,
                const uint32_t* pk_filt, int n_kz, int64_t kstride, void* stream) {
  if (!cnt) return VK_E_ARG;
  return k1_tiles_launch<false>(ix, fp, tol_lo, tol_hi, warps, tile_item_off, item_hyp, n_hyp, item_cap, h_spec,
                                h_maxfz, h_lo, h_hi, win_off, cnt_cap, pk_off, pk_mass, cnt, status, pk_int, tic, isum,
                                pk_keys, pk_filt, n_kz, kstride, K1Hits{}, stream);
}

int vk_k1_hits(const vk_tindex* ix, const vk_frag_params* fp, float tol_lo, float tol_hi, int warps,
               const int64_t* tile_item_off, const int32_t* item_hyp, int64_t n_hyp, int64_t item_cap,
               const int32_t* h_spec, const int8_t* h_maxfz, const int64_t* h_lo, const int64_t* h_hi,
               const int64_t* win_off, int64_t cnt_cap, const int64_t* pk_off, const float* pk_mass, int thr,
               const int32_t* h_thr, uint64_t* hit_rc, uint32_t* hit_isum, uint32_t* seg_cnt, int8_t* hyp_shift,
               uint32_t* hyp_scored, uint64_t* hyp_matched, int32_t* status, const float* pk_int, const float* tic,
               const uint32_t* pk_keys, const uint32_t* pk_filt, int n_kz, int64_t kstride, void* stream) {
  if (!hit_rc || !seg_cnt || !hyp_shift || !hyp_scored || !hyp_matched || (!h_thr && thr < 1)) return VK_E_ARG;
  if ((hit_isum != nullptr) != (pk_int != nullptr)) return VK_E_ARG;
  K1Hits hits{thr, h_thr, hit_rc, hit_isum, seg_cnt, hyp_shift, hyp_scored,
              reinterpret_cast<unsigned long long*>(hyp_matched)};
  return k1_tiles_launch<true>(ix, fp, tol_lo, tol_hi, warps, tile_item_off, item_hyp, n_hyp, item_cap, h_spec,
                               h_maxfz, h_lo, h_hi, win_off, cnt_cap, pk_off, pk_mass, nullptr, status, pk_int, tic,
                               hit_isum, pk_keys, pk_filt, n_kz, kstride, hits, stream);
}

int vk_k1_peak_keys(const vk_tindex* ix, const vk_frag_params* fp, float tol_lo, float tol_hi, const int64_t* n_peaks,
                    const float* pk_mass, int n_kz, int64_t kstride, uint32_t* keys, uint32_t* filt, void* stream) {
  if (!ix || !fp || !n_peaks || n_kz < 0 || kstride < 0 || ((uintptr_t)keys & 7) || !filt) return VK_E_ARG;
  if (n_kz == 0 || kstride == 0) return 0;
  int dev = 0, n_sm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  const int64_t blocks = std::min<int64_t>((kstride + 255) / 256, (int64_t)n_sm * 8);
  peak_keys_k<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(*ix, tol_lo, tol_hi, fp->tol_da, n_peaks, pk_mass,
                                                                   n_kz, kstride, reinterpret_cast<uint2*>(keys),
                                                                   filt);
  return vk_launch_status();
}

}  // extern "C"
