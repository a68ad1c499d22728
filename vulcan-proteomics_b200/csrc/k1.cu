// K1 shared-peak counting on the tiled fragment index.
//
// Work items are (tile, hypothesis) pairs grouped by tile.  One CTA owns one tile: thread 0 stages the tile's
// postings and its coarse-bin CSR into shared memory with two bulk (TMA) copies completing on one mbarrier; then
// each warp takes the tile's hypotheses in turn.  A peak's tolerance window [a, bd] (Sage f32 arithmetic) is the
// posting key range [bits(a) - bits(fmin), bits(bd) - bits(fmin)] (the mass field of a posting).
//
// Merge join (default): the warp writes its spectrum's windows, in peak order, into shared memory (for sorted
// peaks both bounds are non-decreasing); each lane takes a contiguous slice of the tile's sorted postings, finds
// its first window with one binary search and then walks postings and windows together.  Every posting inside k
// windows adds k to its row's count in a warp-private shared-memory histogram (rows of the hypothesis window
// only).  Per-peak search (fallback when the windows are not monotone or the spectrum has more than max_win
// peaks): lanes stride over peaks, coarse-bin lookup + binary search in the staged tile, scan of the key range.
// The histogram is written to the hypothesis' dense count slice.
//
// Result = the reference's brute-force count (vulcan/gpu/kernels.cu:195-232) for every window row: a posting key
// compares exactly like its f32 fragment mass, so f == a and f == bd are both counted.
#include "common.cuh"
#include "k1_impl.cuh"

namespace {

constexpr int K1_WARPS = 4;
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

__global__ void plan_fill_k(int64_t n_hyp, int shift, const int64_t* h_lo, const int64_t* h_hi,
                            const int64_t* tile_item_off, unsigned long long* cursor, int32_t* item_hyp) {
  int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (h >= n_hyp) return;
  int64_t lo = h_lo[h], hi = h_hi[h];
  if (hi <= lo) return;
  for (int64_t t = lo >> shift; t <= (hi - 1) >> shift; ++t) {
    unsigned long long pos = atomicAdd(&cursor[t], 1ull);
    item_hyp[tile_item_off[t] + (int64_t)pos] = (int32_t)h;
  }
}

__global__ void __launch_bounds__(K1_WARPS * 32)
k1_tiles_k(vk_tindex ix, float tol_lo, float tol_hi, int tol_da, int post_cap, int max_win,
           const int64_t* tile_item_off, const int32_t* item_hyp, const int32_t* h_spec, const int8_t* h_maxfz,
           const int64_t* h_lo, const int64_t* h_hi, const int64_t* win_off, const int64_t* pk_off,
           const float* pk_mass, int32_t* cnt, int32_t* status, const float* pk_int, const float* tic,
           uint32_t* isum_out) {
  extern __shared__ __align__(16) uint8_t k1_smem[];
  __shared__ __align__(8) uint64_t bar;
  const int64_t t = blockIdx.x;
  const int64_t i0 = tile_item_off[t], i1 = tile_item_off[t + 1];
  if (i0 == i1) return;
  const int T = 1 << ix.tile_shift;
  const int nb = 1 << ix.cbin_bits;
  const int stride = (nb + 1 + 7) & ~7;
  uint32_t* post = reinterpret_cast<uint32_t*>(k1_smem);
  uint16_t* cb = reinterpret_cast<uint16_t*>(k1_smem + (size_t)post_cap * 4);
  uint32_t* hist = reinterpret_cast<uint32_t*>(k1_smem + (size_t)post_cap * 4 + (size_t)stride * 2);
  uint32_t* wins = hist + K1_WARPS * T;   // per warp: max_win window starts, then max_win window ends
  uint32_t* ihist = wins + (size_t)K1_WARPS * 2 * max_win;   // per warp T intensity sums (features only)
  const int64_t po = ix.tile_off[t];
  const uint32_t post_bytes = (uint32_t)((ix.tile_off[t + 1] - po) * 4);
  const uint32_t cb_bytes = (uint32_t)stride * 2;
  if (threadIdx.x == 0) {
    vk::mbar_init(&bar, 1);
    vk::fence_mbar_init();
    vk::mbar_expect_tx(&bar, post_bytes + cb_bytes);
    if (post_bytes) vk::bulk_g2s(post, ix.postings + po, post_bytes, &bar);
    vk::bulk_g2s(cb, ix.cbin_off + t * stride, cb_bytes, &bar);
  }
  __syncthreads();
  if (!vk::mbar_wait(&bar, 0, WAIT_LIMIT)) {
    // give up on this tile, but do not leave while the copies may still land in shared memory
    if (threadIdx.x == 0) atomicOr(status, VK_STATUS_WAIT_TIMEOUT);
    vk::mbar_wait(&bar, 0, WAIT_LIMIT);
    return;
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* hw = hist + warp * T;
  uint32_t* iw = isum_out ? ihist + warp * T : nullptr;
  uint32_t* wka = wins + (size_t)warp * 2 * max_win;
  uint32_t* wkb = wka + max_win;
  const int row_bits = ix.row_bits;
  const uint32_t rowmask = (1u << row_bits) - 1u;
  const float fmin = __uint_as_float(ix.fmin_bits), fmax = __uint_as_float(ix.fmax_bits);
  const uint32_t krange = ix.fmax_bits - ix.fmin_bits;
  const int n_post = cb[1 << ix.cbin_bits];   // real postings of the tile (the padding follows)
  const int64_t r0 = t << ix.tile_shift;
  const unsigned lt_mask = (1u << lane) - 1u;
  for (int64_t it = i0 + warp; it < i1; it += K1_WARPS) {
    const int h = item_hyp[it];
    const int64_t lo = h_lo[h], hi = h_hi[h];
    const int rlo = (int)max(lo - r0, (int64_t)0), rhi = (int)min(hi - r0, (int64_t)T);
    for (int j = lane; j < T; j += 32) {
      hw[j] = 0;
      if (iw) iw[j] = 0;
    }
    __syncwarp();
    const int s = h_spec[h], maxfz = h_maxfz[h];
    const int64_t p0 = pk_off[s], p1 = pk_off[s + 1];
    bool merged = (p1 - p0) <= max_win && !iw;   // the merge join does not accumulate intensities
    for (int z = 1; merged && z < maxfz; ++z) {
      // tolerance windows of this fragment charge, in key space, in peak (= mass) order; windows that miss
      // [fmin, fmax] are dropped, the others clamped to it
      int nw = 0;
      for (int64_t q0 = 0; q0 < p1 - p0; q0 += 32) {
        const int64_t p = p0 + q0 + lane;
        uint32_t ka = 0, kb = 0;
        bool keep = false;
        if (p < p1) {
          const float m = __fmul_rn(pk_mass[p], (float)z);
          const float a = vk::tol_bound(m, tol_lo, tol_da), bd = vk::tol_bound(m, tol_hi, tol_da);
          keep = bd >= fmin && a <= fmax;
          ka = a <= fmin ? 0u : __float_as_uint(a) - ix.fmin_bits;
          kb = bd >= fmax ? krange : __float_as_uint(bd) - ix.fmin_bits;
        }
        const unsigned mk = __ballot_sync(VK_FULL, keep);
        if (keep) {
          const int pos = nw + __popc(mk & lt_mask);
          wka[pos] = ka;
          wkb[pos] = kb;
        }
        nw += __popc(mk);
      }
      __syncwarp();
      // the merge needs both window bounds non-decreasing (they are for ppm and Da bounds of sorted peaks)
      bool mono = true;
      for (int j = 1 + lane; j < nw; j += 32) mono &= (wka[j] >= wka[j - 1]) && (wkb[j] >= wkb[j - 1]);
      if (!__all_sync(VK_FULL, mono)) {
        merged = false;
        break;
      }
      // merge join: lane takes a contiguous slice of the tile's sorted postings; the slice length is odd, so the
      // 32 lanes' current postings sit in 32 different shared-memory banks at every step
      const int slice = ((n_post + 31) >> 5) | 1;
      const int e0 = min(n_post, lane * slice), e1 = min(n_post, (lane + 1) * slice);
      if (e0 < e1 && nw > 0) {
        const uint32_t kf0 = post[e0] >> row_bits;
        int lo_w = 0, hi_w = nw;   // first window with end >= kf0
        while (lo_w < hi_w) {
          const int m = (lo_w + hi_w) >> 1;
          if (wkb[m] < kf0) lo_w = m + 1; else hi_w = m;
        }
        int j = lo_w;
        for (int e = e0; e < e1 && j < nw; ++e) {
          const uint32_t v = post[e];
          const uint32_t kf = v >> row_bits;
          while (j < nw && wkb[j] < kf) ++j;
          if (j < nw && wka[j] <= kf) {
            const int l = (int)(v & rowmask);
            if (l >= rlo && l < rhi) {
              int c = 1;
              for (int jj = j + 1; jj < nw && wka[jj] <= kf; ++jj) ++c;
              atomicAdd(&hw[l], (uint32_t)c);
            }
          }
        }
      }
      __syncwarp();
    }
    if (!merged) {
      // restart this item with the per-peak search (clears the partial histogram first)
      __syncwarp();
      for (int j = lane; j < T; j += 32) hw[j] = 0;
      __syncwarp();
      const float ts = iw ? tic[s] : 0.f;
      vk::k1_item_per_peak(post, cb, hw, 0, rlo, rhi, p0, p1, maxfz, pk_mass, tol_lo, tol_hi, tol_da, ix, lane, iw,
                           pk_int, ts > 0.f ? __fdiv_rn(16777216.0f, ts) : 0.f);
    }
    __syncwarp();
    const int64_t base = win_off[h] + (r0 - lo);
    for (int j = rlo + lane; j < rhi; j += 32) {
      cnt[base + j] = (int32_t)hw[j];
      if (iw) isum_out[base + j] = iw[j];
    }
    __syncwarp();
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
                    const int64_t* tile_item_off, int64_t* cursor, int32_t* item_hyp, void* stream) {
  if (!ix) return VK_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  if (ix->n_tiles > 0) {
    cudaError_t e = cudaMemsetAsync(cursor, 0, sizeof(int64_t) * ix->n_tiles, st);
    if (e != cudaSuccess) return vk_err(e);
  }
  if (n_hyp == 0) return 0;
  plan_fill_k<<<(unsigned)((n_hyp + 255) / 256), 256, 0, st>>>(n_hyp, ix->tile_shift, h_lo, h_hi, tile_item_off,
                                                                (unsigned long long*)cursor, item_hyp);
  return vk_launch_status();
}

int vk_k1_tiles(const vk_tindex* ix, const vk_frag_params* fp, float tol_lo, float tol_hi, int max_win,
                const int64_t* tile_item_off, const int32_t* item_hyp, const int32_t* h_spec,
                const int8_t* h_maxfz, const int64_t* h_lo, const int64_t* h_hi, const int64_t* win_off,
                const int64_t* pk_off, const float* pk_mass, int32_t* cnt, int32_t* status, const float* pk_int,
                const float* tic, uint32_t* isum, void* stream) {
  if (!ix || !fp || !status) return VK_E_ARG;
  if (ix->n_tiles == 0) return 0;
  if ((ix->max_tile_postings & 3) || ix->max_tile_postings < 0 || max_win < 0 || max_win > 4096) return VK_E_ARG;
  const int T = 1 << ix->tile_shift;
  const int stride = ((1 << ix->cbin_bits) + 1 + 7) & ~7;
  if (isum && (!pk_int || !tic)) return VK_E_ARG;
  size_t sh = (size_t)ix->max_tile_postings * 4 + (size_t)stride * 2 + (size_t)K1_WARPS * T * 4 +
              (size_t)K1_WARPS * 2 * max_win * 4 + (isum ? (size_t)K1_WARPS * T * 4 : 0);
  if (sh > 220 * 1024) return VK_E_ARG;
  cudaError_t e = cudaFuncSetAttribute(k1_tiles_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  if (e != cudaSuccess) return vk_err(e);
  k1_tiles_k<<<(unsigned)ix->n_tiles, K1_WARPS * 32, sh, (cudaStream_t)stream>>>(
      *ix, tol_lo, tol_hi, fp->tol_da, ix->max_tile_postings, max_win, tile_item_off, item_hyp, h_spec, h_maxfz,
      h_lo, h_hi, win_off, pk_off, pk_mass, cnt, status, pk_int, tic, isum);
  return vk_launch_status();
}

}  // extern "C"
