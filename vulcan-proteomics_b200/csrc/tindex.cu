// Tiled fragment index build and the device exclusive scan.
//
// Layout (vk_tindex in vulcan_b200.h): rows (mass-sorted peptidoforms) are cut into tiles of 2^tile_shift rows.
// A fragment's key is f32bits(f) - f32bits(fmin) (mass_bits wide).  For positive floats the bit pattern is monotone
// in the value, so sorting by key sorts fragments by their exact f32 mass, and a tolerance window [a, bd] is
// exactly the key range [bits(a) - base, bits(bd) - base]: no quantisation, no edge loss.  A tile's fragments are
// sorted by (key, row) and split into 2^cbin_bits coarse bins by the key's top cbin_bits bits (CSR cbin_off); the
// bin is implicit in a posting's position, so the u32 posting keeps only the low mass_bits - cbin_bits key bits
// and the local row: (key mod 2^(mass_bits - cbin_bits)) << row_bits | row.  Each tile's postings start at a
// multiple of 4 entries (16 bytes) so the search can stage a tile with one bulk copy; the padding entries are
// 0xffffffff, after the last bin.
#include <mutex>

#include "common.cuh"
#include "k1_impl.cuh"

namespace {

constexpr int TI_COUNT_WARPS = 4;

template <class F>
__device__ __forceinline__ int row_frag_count(const F& fp, const uint8_t* s, int L, uint64_t mk, float mass,
                                              int min_ion, float fmin, float fmax) {
  int c = 0;
  vk::row_ladder(fp, s, L, mk, mass, min_ion, fmin, fmax, [&](float) { ++c; });
  return c;
}

// One warp per tile: postings of the tile's rows (rounded up to a multiple of 4 for the 16-byte tile alignment).
__global__ void __launch_bounds__(TI_COUNT_WARPS * 32)
tindex_count_k(vk_tindex ix, vk_frag_params fpv, const int64_t* seq_off, const uint8_t* len, const uint64_t* mask,
               const float* mass32, const uint8_t* res, int64_t* tile_count) {
  __shared__ vk::SmemFrag fp;
  vk::load_frag(fp, fpv);
  __syncthreads();
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int64_t t = (int64_t)blockIdx.x * TI_COUNT_WARPS + warp;
  if (t >= ix.n_tiles) return;
  float fmin = __uint_as_float(ix.fmin_bits), fmax = __uint_as_float(ix.fmax_bits);
  int64_t r0 = t << ix.tile_shift, r1 = min(ix.n_rows, (t + 1) << ix.tile_shift);
  long long c = 0;
  for (int64_t r = r0 + lane; r < r1; r += 32)
    c += row_frag_count(fp, res + seq_off[r], len[r], mask[r], mass32[r], ix.min_ion_index, fmin, fmax);
  c = vk::warp_sum(c);
  if (lane == 0) tile_count[t] = (c + 3) & ~3ll;
}


__device__ __forceinline__ void bitonic_sort_u64(uint64_t* v, int n_pow2) {
  for (int k = 2; k <= n_pow2; k <<= 1) {
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
}

// One CTA per tile: generate the tile's (key << 16 | row) entries in shared memory, sort them, write the postings
// (low key bits and row) and the coarse-bin CSR.
__global__ void __launch_bounds__(512)
tindex_emit_k(vk_tindex ix, vk_frag_params fpv, const int64_t* seq_off, const uint8_t* len, const uint64_t* mask,
              const float* mass32, const uint8_t* res, uint32_t* postings, uint16_t* cbin_off, int n_pow2) {
  extern __shared__ uint64_t ti_smem[];
  __shared__ vk::SmemFrag fp;
  __shared__ int row_off[1025];
  __shared__ long long warp_tot[16];
  vk::load_frag(fp, fpv);
  __syncthreads();
  const int64_t t = blockIdx.x;
  const int T = 1 << ix.tile_shift;
  const float fmin = __uint_as_float(ix.fmin_bits), fmax = __uint_as_float(ix.fmax_bits);
  const int64_t r0 = t << ix.tile_shift;
  const int nr = (int)min((int64_t)T, ix.n_rows - r0);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // per-row counts and their exclusive scan (rows in chunks of blockDim)
  int base = 0;
  for (int c0 = 0; c0 < nr; c0 += blockDim.x) {
    int r = c0 + threadIdx.x;
    int c = 0;
    if (r < nr) {
      int64_t g = r0 + r;
      c = row_frag_count(fp, res + seq_off[g], len[g], mask[g], mass32[g], ix.min_ion_index, fmin, fmax);
    }
    long long inc = vk::warp_incl_scan(c);
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    long long wbase = 0;
    for (int w = 0; w < warp; ++w) wbase += warp_tot[w];
    if (r < nr) row_off[r] = base + (int)(wbase + inc - c);
    __syncthreads();
    long long tot = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += warp_tot[w];
    base += (int)tot;
    __syncthreads();
  }
  const int n_post = base;
  // emit keys
  for (int r = threadIdx.x; r < nr; r += blockDim.x) {
    int64_t g = r0 + r;
    uint64_t* o = ti_smem + row_off[r];
    vk::row_ladder(fp, res + seq_off[g], len[g], mask[g], mass32[g], ix.min_ion_index, fmin, fmax, [&](float f) {
      *o++ = ((uint64_t)(__float_as_uint(f) - ix.fmin_bits) << 16) | (uint64_t)r;
    });
  }
  for (int i = n_post + threadIdx.x; i < n_pow2; i += blockDim.x) ti_smem[i] = ~0ull;
  __syncthreads();
  bitonic_sort_u64(ti_smem, n_pow2);
  const int low_bits = ix.mass_bits - ix.cbin_bits;
  const uint64_t lowmask = (1ull << low_bits) - 1ull;
  const int64_t o0 = ix.tile_off[t];
  const int64_t o1 = ix.tile_off[t + 1];
  for (int64_t i = threadIdx.x; i < o1 - o0; i += blockDim.x) {
    uint32_t v = 0xffffffffu;
    if (i < n_post) {
      const uint64_t e = ti_smem[i];
      v = (uint32_t)(((e >> 16) & lowmask) << ix.row_bits) | (uint32_t)(e & 0xffffull);
    }
    postings[o0 + i] = v;
  }
  // coarse bins: CSR over the top cbin_bits key bits, offsets relative to the tile start
  const int nb = 1 << ix.cbin_bits;
  const int stride = (nb + 1 + 7) & ~7;
  for (int b = threadIdx.x; b <= nb; b += blockDim.x) {
    int pos;
    if (b == nb) {
      pos = n_post;
    } else {
      const uint64_t key = (uint64_t)b << low_bits;
      int lo = 0, hi = n_post;
      while (lo < hi) {
        int m = (lo + hi) >> 1;
        if ((ti_smem[m] >> 16) < key) lo = m + 1; else hi = m;
      }
      pos = lo;
    }
    cbin_off[t * stride + b] = (uint16_t)pos;
  }
}

// One CTA per tile: the tile's presence bitmap (2^K1_BM_LOG bits per coarse bin) from its postings and coarse-bin
// CSR.
__global__ void __launch_bounds__(256) tindex_bitmap_k(vk_tindex ix, uint32_t* bitmap) {
  const int64_t t = blockIdx.x;
  const int nb = 1 << ix.cbin_bits;
  const int stride = (nb + 1 + 7) & ~7;
  vk::k1_build_bitmap(ix.postings + ix.tile_off[t], ix.cbin_off + t * stride, nb, vk::k1_bm_bits(ix),
                      bitmap + t * nb * vk::K1_BM_WORDS);
}

// ------------------------------------------------------------------------------------------ exclusive scan
constexpr int SCAN_THREADS = 512;
constexpr int SCAN_PER_THREAD = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_PER_THREAD;

__device__ __forceinline__ long long block_excl_scan(long long v, long long* total) {
  __shared__ long long wsum[SCAN_THREADS / 32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  long long inc = vk::warp_incl_scan(v);
  if (lane == 31) wsum[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    long long w = lane < SCAN_THREADS / 32 ? wsum[lane] : 0;
    long long wi = vk::warp_incl_scan(w);
    if (lane < SCAN_THREADS / 32) wsum[lane] = wi - w;
    if (lane == SCAN_THREADS / 32 - 1) *total = wi;
  }
  __syncthreads();
  long long r = wsum[warp] + inc - v;
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(SCAN_THREADS) scan_reduce_k(const int64_t* in, int64_t n, int64_t* block_sums) {
  __shared__ long long tot;
  int64_t b0 = (int64_t)blockIdx.x * SCAN_TILE;
  long long s = 0;
  for (int i = 0; i < SCAN_PER_THREAD; ++i) {
    int64_t j = b0 + (int64_t)threadIdx.x * SCAN_PER_THREAD + i;
    if (j < n) s += in[j];
  }
  block_excl_scan(s, &tot);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(SCAN_THREADS) scan_blocks_k(int64_t* block_sums, int64_t nb) {
  __shared__ long long tot;
  long long carry = 0;
  for (int64_t c0 = 0; c0 < nb; c0 += SCAN_THREADS) {
    int64_t j = c0 + threadIdx.x;
    long long v = j < nb ? block_sums[j] : 0;
    long long e = block_excl_scan(v, &tot);
    if (j < nb) block_sums[j] = carry + e;
    carry += tot;
    __syncthreads();
  }
}

// in may alias out + 1: every element is read before the block's barrier and written after it.
// FOLD: block_sums holds the blocks' plain sums (scan_reduce_k's output, no scan_blocks_k), and each block adds up
// those before it itself (at most SCAN_FOLD_MAX_BLOCKS of them); with a single block nothing is read.
constexpr int64_t SCAN_FOLD_MAX_BLOCKS = 4 * SCAN_THREADS;

template <bool FOLD>
__global__ void __launch_bounds__(SCAN_THREADS)
scan_apply_k(const int64_t* in, int64_t n, const int64_t* block_sums, int64_t* out) {
  __shared__ long long tot;
  int64_t b0 = (int64_t)blockIdx.x * SCAN_TILE;
  long long v[SCAN_PER_THREAD];
  long long s = 0;
  for (int i = 0; i < SCAN_PER_THREAD; ++i) {
    int64_t j = b0 + (int64_t)threadIdx.x * SCAN_PER_THREAD + i;
    v[i] = j < n ? in[j] : 0;
    s += v[i];
  }
  long long base;
  if (FOLD) {
    long long pre = 0;
    for (int64_t j = threadIdx.x; j < (int64_t)blockIdx.x; j += SCAN_THREADS) pre += block_sums[j];
    block_excl_scan(pre, &tot);
    base = tot;   // read before the next scan's barriers (block_excl_scan ends with one)
  } else {
    base = block_sums[blockIdx.x];
  }
  long long e = block_excl_scan(s, &tot) + base;
  // grid-wide: the last element of the next block is read by that block only, so in/out aliasing is safe when
  // every block reads its own inputs before writing (done above, and out[j+1] belongs to in[j+1]'s block
  // except at the block edge, which is written by this block after its own reads only).
  for (int i = 0; i < SCAN_PER_THREAD; ++i) {
    int64_t j = b0 + (int64_t)threadIdx.x * SCAN_PER_THREAD + i;
    e += v[i];
    if (j < n) out[j + 1] = e;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) out[0] = 0;
}

// Scratch of vk_scan_i64_noalloc: the per-block partial sums, in a fixed device array instead of a caller buffer.
// 8192 blocks of SCAN_TILE (4096) elements: inputs of up to 33,554,432 values; 64 KiB held on every device that
// loads the library, until the process exits.
constexpr int64_t NOALLOC_SCAN_BLOCKS = 8192;
static __device__ __align__(256) int64_t g_scan_scratch[NOALLOC_SCAN_BLOCKS];

// Device address of g_scan_scratch per device.  In host code the array's name is only a stand-in; the address a
// kernel may use comes from cudaGetSymbolAddress, taken once per device with that device current.  The cached
// address is never refreshed, so it goes stale after a cudaDeviceReset of that device (documented in the header).
constexpr int NOALLOC_MAX_DEVICES = 64;
int64_t* g_scan_scratch_dev[NOALLOC_MAX_DEVICES] = {};
std::mutex g_scan_scratch_mu;

int scan_scratch_address(int64_t** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return vk_err(e);
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return VK_E_ARG;
  std::lock_guard<std::mutex> lock(g_scan_scratch_mu);
  if (!g_scan_scratch_dev[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scan_scratch);
    if (e != cudaSuccess) return vk_err(e);
    g_scan_scratch_dev[dev] = static_cast<int64_t*>(p);
  }
  *out = g_scan_scratch_dev[dev];
  return 0;
}

// Kernels of one scan of n > 0 values: one block -> the apply kernel alone; up to SCAN_FOLD_MAX_BLOCKS blocks ->
// block sums, then the apply kernel adding up the sums before its block; more -> block sums, their scan, apply.
int scan_kernels(int64_t n) {
  if (n <= 0) return 0;
  const int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  return nb == 1 ? 1 : (nb <= SCAN_FOLD_MAX_BLOCKS ? 2 : 3);
}

int scan_launch(const int64_t* in, int64_t n, int64_t* out, int64_t* bs, cudaStream_t st) {
  const int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  const int k = scan_kernels(n);
  if (k >= 2) scan_reduce_k<<<(unsigned)nb, SCAN_THREADS, 0, st>>>(in, n, bs);
  if (k == 3) {
    scan_blocks_k<<<1, SCAN_THREADS, 0, st>>>(bs, nb);
    scan_apply_k<false><<<(unsigned)nb, SCAN_THREADS, 0, st>>>(in, n, bs, out);
  } else {
    scan_apply_k<true><<<(unsigned)nb, SCAN_THREADS, 0, st>>>(in, n, bs, out);
  }
  return vk_launch_status();
}

}  // namespace

extern "C" {

int vk_tindex_layout(int64_t n_rows, int tile_rows, float fmin, float fmax, int min_ion_index, int cbin_bits,
                     vk_tindex* ix) {
  if (!ix || n_rows < 0 || !(fmin > 0.f) || !(fmax > fmin) || tile_rows < 32 || (tile_rows & (tile_rows - 1)))
    return VK_E_ARG;
  uint32_t lo = vk::f32_bits(fmin), hi = vk::f32_bits(fmax);
  uint32_t range = hi - lo;
  int mass_bits = 0;
  while (mass_bits < 32 && (range >> mass_bits) != 0) ++mass_bits;
  if (cbin_bits < 1 || cbin_bits >= mass_bits || cbin_bits > 12) return VK_E_ARG;
  // a posting keeps the low mass_bits - cbin_bits key bits; the row gets the rest
  int row_bits = 32 - (mass_bits - cbin_bits);
  int shift = 0;
  while ((1 << shift) < tile_rows) ++shift;
  // local rows must leave the all-ones posting (padding) unused, and fit the emit's 16-bit row field
  if (row_bits > 31 || shift >= row_bits || tile_rows > 1024) return VK_E_ARG;
  ix->n_rows = n_rows;
  ix->tile_shift = shift;
  ix->row_bits = row_bits;
  ix->mass_bits = mass_bits;
  ix->cbin_bits = cbin_bits;
  ix->fmin_bits = lo;
  ix->fmax_bits = hi;
  ix->min_ion_index = min_ion_index;
  ix->n_tiles = (n_rows + tile_rows - 1) / tile_rows;
  return 0;
}

int vk_tindex_count(const vk_tindex* ix, const vk_frag_params* fp, const int64_t* seq_off, const uint8_t* len,
                    const uint64_t* mask, const float* mass32, const uint8_t* res, int64_t* tile_count,
                    void* stream) {
  if (!ix || !fp) return VK_E_ARG;
  if (ix->n_tiles == 0) return 0;
  unsigned grid = (unsigned)((ix->n_tiles + TI_COUNT_WARPS - 1) / TI_COUNT_WARPS);
  tindex_count_k<<<grid, TI_COUNT_WARPS * 32, 0, (cudaStream_t)stream>>>(*ix, *fp, seq_off, len, mask, mass32, res,
                                                                         tile_count);
  return vk_launch_status();
}

int vk_tindex_emit(const vk_tindex* ix, const vk_frag_params* fp, const int64_t* seq_off, const uint8_t* len,
                   const uint64_t* mask, const float* mass32, const uint8_t* res, uint32_t* postings,
                   uint16_t* cbin_off, void* stream) {
  if (!ix || !fp || !ix->tile_off) return VK_E_ARG;
  if (ix->n_tiles == 0) return 0;
  if ((1 << ix->tile_shift) > 1024) return VK_E_ARG;
  if (ix->max_tile_postings > 16384) return VK_E_TOO_LARGE;   // the sort of a tile in shared memory
  int n_pow2 = 16;
  while (n_pow2 < ix->max_tile_postings) n_pow2 <<= 1;
  size_t sh = (size_t)n_pow2 * sizeof(uint64_t);
  cudaError_t e = cudaFuncSetAttribute(tindex_emit_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  if (e != cudaSuccess) return vk_err(e);
  tindex_emit_k<<<(unsigned)ix->n_tiles, 512, sh, (cudaStream_t)stream>>>(*ix, *fp, seq_off, len, mask, mass32, res,
                                                                          postings, cbin_off, n_pow2);
  return vk_launch_status();
}

int vk_tindex_bitmap(const vk_tindex* ix, uint32_t* bitmap, void* stream) {
  if (!ix || !ix->tile_off || !ix->cbin_off || !ix->postings || !bitmap || ((uintptr_t)bitmap & 15)) return VK_E_ARG;
  if (ix->n_tiles == 0) return 0;
  tindex_bitmap_k<<<(unsigned)ix->n_tiles, 256, 0, (cudaStream_t)stream>>>(*ix, bitmap);
  return vk_launch_status();
}

int64_t vk_tindex_bitmap_bytes(const vk_tindex* ix) {
  if (!ix) return -1;
  return ix->n_tiles * ((int64_t)1 << ix->cbin_bits) * vk::K1_BM_WORDS * 4;
}

int64_t vk_scan_noalloc_max_n(void) { return NOALLOC_SCAN_BLOCKS * SCAN_TILE; }

int vk_scan_i64_noalloc(const int64_t* in, int64_t n, int64_t* out, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (n < 0) return VK_E_ARG;
  if (n > NOALLOC_SCAN_BLOCKS * SCAN_TILE) return VK_E_TOO_LARGE;
  // an empty input needs no scratch: no address lookup, so this case works inside a stream capture too
  if (n == 0) return vk_err(cudaMemsetAsync(out, 0, sizeof(int64_t), st));
  int64_t* bs = nullptr;
  int rc = scan_scratch_address(&bs);
  if (rc != 0) return rc;
  // every block sum is written by scan_reduce_k before it is read: nothing in the scratch has to start at zero
  return scan_launch(in, n, out, bs, st);
}

int64_t vk_scan_tmp_bytes(int64_t n) { return ((n + SCAN_TILE - 1) / SCAN_TILE + 1) * (int64_t)sizeof(int64_t); }

int vk_scan_i64(const int64_t* in, int64_t n, int64_t* out, void* tmp, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (n < 0) return VK_E_ARG;
  if (n == 0) return vk_err(cudaMemsetAsync(out, 0, sizeof(int64_t), st));
  return scan_launch(in, n, out, (int64_t*)tmp, st);
}

int vk_scan_kernels(int64_t n) { return scan_kernels(n); }

}  // extern "C"
