// K1 shared-peak counting on the tiled fragment index.
//
// Work items are (tile, hypothesis) pairs grouped by tile.  One CTA owns one tile: thread 0 stages the tile's
// postings and its coarse-bin CSR into shared memory with two bulk (TMA) copies completing on one mbarrier; then
// each warp takes the tile's hypotheses in turn and runs the per-peak search (k1_impl.cuh): lanes stride over the
// spectrum's peaks x fragment charges, each tolerance window is found through the coarse bins and a binary search
// in the staged tile, and every posting in it adds one to its row in a warp-private shared-memory histogram (rows
// of the hypothesis window only; with intensity sums, a second histogram adds the peak's fixed-point weight).  The
// histograms are written to the hypothesis' dense slices.
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

__global__ void __launch_bounds__(K1_MAX_WARPS * 32)
k1_tiles_k(vk_tindex ix, float tol_lo, float tol_hi, int tol_da, int post_cap, const int64_t* tile_item_off,
           const int32_t* item_hyp, int64_t n_hyp, int64_t item_cap, const int32_t* h_spec, const int8_t* h_maxfz,
           const int64_t* h_lo, const int64_t* h_hi, const int64_t* win_off, int64_t cnt_cap, const int64_t* pk_off,
           const float* pk_mass, int32_t* cnt, int32_t* status, const float* pk_int, const float* tic,
           uint32_t* isum_out) {
  extern __shared__ __align__(16) uint8_t k1_smem[];
  __shared__ __align__(8) uint64_t bar;
  const int64_t t = blockIdx.x;
  const int64_t i0 = min(tile_item_off[t], item_cap), i1 = min(tile_item_off[t + 1], item_cap);
  if (i0 == i1) return;
  const int n_warps = blockDim.x >> 5;
  const int T = 1 << ix.tile_shift;
  const int nb = 1 << ix.cbin_bits;
  const int stride = (nb + 1 + 7) & ~7;
  uint32_t* post = reinterpret_cast<uint32_t*>(k1_smem);
  uint16_t* cb = reinterpret_cast<uint16_t*>(k1_smem + (size_t)post_cap * 4);
  uint32_t* hist = reinterpret_cast<uint32_t*>(k1_smem + (size_t)post_cap * 4 + (size_t)stride * 2);
  uint32_t* ihist = hist + n_warps * T;   // per warp T intensity sums (pruner features only)
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
  const int64_t r0 = t << ix.tile_shift;
  for (int64_t it = i0 + warp; it < i1; it += n_warps) {
    const int h = item_hyp[it];
    // items and windows must lie inside the buffers the caller sized by bounds; anything else is skipped
    if (h < 0 || h >= n_hyp) {
      if (lane == 0) atomicOr(status, VK_STATUS_OVERFLOW);
      continue;
    }
    const int64_t lo = h_lo[h], hi = h_hi[h];
    if (hi <= lo || win_off[h] + (hi - lo) > cnt_cap) {
      if (lane == 0 && hi > lo) atomicOr(status, VK_STATUS_OVERFLOW);
      continue;
    }
    const int rlo = (int)max(lo - r0, (int64_t)0), rhi = (int)min(hi - r0, (int64_t)T);
    for (int j = rlo + lane; j < rhi; j += 32) {
      hw[j] = 0;
      if (iw) iw[j] = 0;
    }
    __syncwarp();
    const int s = h_spec[h];
    const float ts = iw ? tic[s] : 0.f;
    vk::k1_item_per_peak(post, cb, hw, 0, rlo, rhi, pk_off[s], pk_off[s + 1], h_maxfz[h], pk_mass, tol_lo, tol_hi,
                         tol_da, ix, lane, iw, pk_int, ts > 0.f ? __fdiv_rn(16777216.0f, ts) : 0.f);
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

int vk_k1_tiles(const vk_tindex* ix, const vk_frag_params* fp, float tol_lo, float tol_hi, int warps,
                const int64_t* tile_item_off, const int32_t* item_hyp, int64_t n_hyp, int64_t item_cap,
                const int32_t* h_spec, const int8_t* h_maxfz, const int64_t* h_lo, const int64_t* h_hi,
                const int64_t* win_off, int64_t cnt_cap, const int64_t* pk_off, const float* pk_mass, int32_t* cnt,
                int32_t* status, const float* pk_int, const float* tic, uint32_t* isum, void* stream) {
  if (!ix || !fp || !status) return VK_E_ARG;
  if (ix->n_tiles == 0) return 0;
  if ((ix->max_tile_postings & 3) || ix->max_tile_postings < 0 || warps < 1 || warps > K1_MAX_WARPS) return VK_E_ARG;
  const int T = 1 << ix->tile_shift;
  const int stride = ((1 << ix->cbin_bits) + 1 + 7) & ~7;
  if (isum && (!pk_int || !tic)) return VK_E_ARG;
  size_t sh = (size_t)ix->max_tile_postings * 4 + (size_t)stride * 2 + (size_t)warps * T * 4 * (isum ? 2 : 1);
  if (sh > 220 * 1024) return VK_E_TOO_LARGE;
  cudaError_t e = cudaFuncSetAttribute(k1_tiles_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  if (e != cudaSuccess) return vk_err(e);
  k1_tiles_k<<<(unsigned)ix->n_tiles, warps * 32, sh, (cudaStream_t)stream>>>(
      *ix, tol_lo, tol_hi, fp->tol_da, ix->max_tile_postings, tile_item_off, item_hyp, n_hyp, item_cap, h_spec,
      h_maxfz, h_lo, h_hi, win_off, cnt_cap, pk_off, pk_mass, cnt, status, pk_int, tic, isum);
  return vk_launch_status();
}

}  // extern "C"
