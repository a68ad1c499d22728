// Reference-compatible entry points: the names and argument lists of the reference's ctypes binding
// (vulcan/gpu/_lib.py:22-35) with the results of its kernels (vulcan/gpu/kernels.cu), so that the reference's engine
// can bind this library.  What has to match is the interface and the arithmetic that defines the results (Sage f32
// fragment ladders, tolerance bounds, the log-ppm key format of the reference's CSR); the kernels are laid out for
// B200:
//   * vk_frag_count / vk_frag_emit: a CTA stages the residue bytes of its 256 consecutive rows into shared memory
//     with coalesced loads, then each thread walks its row's fragment ladder (vk::row_ladder, shared with the tiled
//     index build) out of shared memory;
//   * vk_k1: one warp per work item; the (peak, charge) windows that reach a non-empty bin of the item's chunk are
//     compacted into a per-warp queue (ballot), searched one window per lane, counted in a warp-private
//     shared-memory histogram; rows over the threshold are appended with one global atomic per 32 rows;
//   * vk_k1_brute: one warp per (hypothesis, row) pair; two lanes build the b and y ladders into shared memory,
//     then the lanes split the spectrum's peaks and compare their tolerance windows with every fragment;
//   * vk_k2 / vk_k2_shift: the shared K2 body (k2_impl.cuh) with the process-wide constants.
#include "common.cuh"
#include "k2_impl.cuh"

namespace {

// Process-wide fragment constants of the reference's binding (vk_set_params / vk_set_nterm / vk_set_tol_da).
struct ConstFrag {
  float mono[26];
  float stat[26];
  float var[26];
  float nterm;
  int tol_da;
};
__constant__ ConstFrag c_frag;

// Copy of the constants in shared memory, in the form the shared helpers take.
__device__ __forceinline__ void frag_from_const(vk::SmemFrag& s) {
  for (int i = threadIdx.x; i < 26; i += blockDim.x) {
    s.mono[i] = c_frag.mono[i];
    s.stat[i] = c_frag.stat[i];
    s.var[i] = c_frag.var[i];
  }
  if (threadIdx.x == 0) {
    s.nterm = c_frag.nterm;
    s.tol_da = c_frag.tol_da;
  }
}

// Quantised log-ppm position of fragment mass x in the reference's CSR: floor((ln x - ln fmin) * inv_logw * 2^16),
// evaluated in f64 in that order (a format: keys written by vk_frag_emit and read by vk_k1 must agree).
__device__ __forceinline__ int64_t log_pos(float x, double ln_fmin, double inv_logw) {
  return (int64_t)floor((log((double)x) - ln_fmin) * inv_logw * 65536.0);
}

// ------------------------------------------------------------------------------------------ fragment count / emit
constexpr int FE_ROWS = 256;                 // rows (threads) per CTA
constexpr int FE_STAGE = FE_ROWS * 64;       // residue bytes staged per CTA (rows of up to 64 residues on average)

// Residues of rows [r0, r0 + nr) (nr >= 1): staged into `stage` when their byte span fits; returns the first
// staged residue's global offset, or -1 when the rows are read from global memory instead.
__device__ __forceinline__ int64_t stage_residues(const int64_t* seq_off, const uint8_t* len, const uint8_t* res,
                                                  int64_t r0, int nr, uint8_t* stage, int64_t* s_lo,
                                                  int64_t* s_hi) {
  if (threadIdx.x == 0) {
    *s_lo = INT64_MAX;
    *s_hi = 0;
  }
  __syncthreads();
  if ((int)threadIdx.x < nr) {
    const int64_t o = seq_off[r0 + threadIdx.x];
    atomicMin((unsigned long long*)s_lo, (unsigned long long)o);
    atomicMax((unsigned long long*)s_hi, (unsigned long long)(o + len[r0 + threadIdx.x]));
  }
  __syncthreads();
  const int64_t lo = *s_lo, hi = *s_hi;
  if (hi - lo > FE_STAGE) return -1;
  for (int64_t i = threadIdx.x; i < hi - lo; i += blockDim.x) stage[i] = res[lo + i];
  __syncthreads();
  return lo;
}

__device__ __forceinline__ const uint8_t* row_residues(const uint8_t* stage, int64_t staged_lo, const uint8_t* res,
                                                       int64_t off) {
  return staged_lo >= 0 ? stage + (off - staged_lo) : res + off;
}

__global__ void __launch_bounds__(FE_ROWS)
frag_count_k(int64_t n, const int64_t* seq_off, const uint8_t* len, const uint64_t* mask, const float* mass32,
             const uint8_t* res, int min_ion, float fmin, float fmax, int32_t* count) {
  __shared__ vk::SmemFrag fp;
  __shared__ __align__(16) uint8_t stage[FE_STAGE];
  __shared__ int64_t s_lo, s_hi;
  frag_from_const(fp);
  const int64_t r0 = (int64_t)blockIdx.x * FE_ROWS;
  const int nr = (int)min((int64_t)FE_ROWS, n - r0);
  const int64_t staged_lo = stage_residues(seq_off, len, res, r0, nr, stage, &s_lo, &s_hi);
  if ((int)threadIdx.x >= nr) return;
  const int64_t r = r0 + threadIdx.x;
  const uint8_t* s = row_residues(stage, staged_lo, res, seq_off[r]);
  int c = 0;
  vk::row_ladder(fp, s, len[r], mask[r], mass32[r], min_ion, fmin, fmax, [&](float) { ++c; });
  count[r] = c;
}

// keys: chunk << 50 | (pos >> 16) << 32 | local row << 16 | (pos & 0xffff), the reference's CSR key format
__global__ void __launch_bounds__(FE_ROWS)
frag_emit_k(int64_t n, const int64_t* seq_off, const uint8_t* len, const uint64_t* mask, const float* mass32,
            const uint8_t* res, int min_ion, float fmin, float fmax, double inv_logw, int chunk_size, int64_t row0,
            const int64_t* out_off, int64_t* keys) {
  __shared__ vk::SmemFrag fp;
  __shared__ __align__(16) uint8_t stage[FE_STAGE];
  __shared__ int64_t s_lo, s_hi;
  frag_from_const(fp);
  const int64_t r0 = (int64_t)blockIdx.x * FE_ROWS;
  const int nr = (int)min((int64_t)FE_ROWS, n - r0);
  const int64_t staged_lo = stage_residues(seq_off, len, res, r0, nr, stage, &s_lo, &s_hi);
  if ((int)threadIdx.x >= nr) return;
  const int64_t r = r0 + threadIdx.x;
  const uint8_t* s = row_residues(stage, staged_lo, res, seq_off[r]);
  const int64_t g = row0 + r;
  const int64_t row_part = ((g / chunk_size) << 50) | ((g % chunk_size) << 16);
  const double ln_fmin = log((double)fmin);
  int64_t* o = keys + out_off[r];
  vk::row_ladder(fp, s, len[r], mask[r], mass32[r], min_ion, fmin, fmax, [&](float f) {
    const int64_t q = log_pos(f, ln_fmin, inv_logw);
    *o++ = row_part | ((q >> 16) << 32) | (q & 0xffff);
  });
}

// ------------------------------------------------------------------------------------------ K1 over the CSR
constexpr int KC_WARPS = 4;
constexpr int KC_QUEUE = 64;   // queued windows per warp

struct KcWindow {
  int64_t qlo, qhi;
  int32_t b0, b1;
};

// Counts, for one window (bins b0..b1 of the item's chunk, quantised range [qlo, qhi]), every entry whose local row
// lies in [lo, hi) into hist[row - lo].  A bin's entries are sorted by (local row, fine position).
__device__ __forceinline__ void kc_count_window(const KcWindow& w, const uint32_t* off, const uint32_t* entries,
                                                uint32_t lo_key, uint32_t hi_key, int lo, uint32_t* hist) {
  for (int b = w.b0; b <= w.b1; ++b) {
    uint32_t first = off[b];
    const uint32_t end = off[b + 1];
    uint32_t span = end - first;
    while (span > 0) {   // first entry with key >= lo_key
      const uint32_t half = span >> 1;
      if (entries[first + half] < lo_key) {
        first += half + 1;
        span -= half + 1;
      } else {
        span = half;
      }
    }
    for (uint32_t e = first; e < end; ++e) {
      const uint32_t v = entries[e];
      if (v >= hi_key) break;
      const int64_t q = ((int64_t)b << 16) | (v & 0xffffu);
      if (q >= w.qlo && q <= w.qhi) atomicAdd(&hist[(int)(v >> 16) - lo], 1u);
    }
  }
}

__global__ void __launch_bounds__(KC_WARPS * 32)
k1_csr_k(int n_items, const int32_t* it_hyp, const int32_t* it_chunk, const int32_t* it_lo, const int32_t* it_hi,
         const int32_t* hyp_spec, const int8_t* hyp_maxfz, const int64_t* pk_off, const float* pk_mass,
         const uint32_t* offsets, const uint32_t* entries, int n_bins, int chunk0, int chunk_size, int tile,
         float tol_lo, float tol_hi, float fmin, double inv_logw, int thr, int64_t cap, unsigned long long* n_out,
         int32_t* out_hyp, int32_t* out_row, int32_t* out_cnt, unsigned int* hyp_scored,
         unsigned long long* hyp_matched) {
  extern __shared__ __align__(16) uint8_t kc_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  KcWindow* queue = reinterpret_cast<KcWindow*>(kc_smem) + warp * KC_QUEUE;
  uint32_t* hist = reinterpret_cast<uint32_t*>(kc_smem + sizeof(KcWindow) * KC_QUEUE * KC_WARPS) + warp * tile;
  const int item = blockIdx.x * KC_WARPS + warp;
  if (item >= n_items) return;
  const int h = it_hyp[item], chunk = it_chunk[item], lo = it_lo[item], hi = it_hi[item];
  const int width = hi - lo;
  if (width <= 0 || width > tile) return;   // an item spans at most `tile` rows (the histogram's size)
  for (int j = lane; j < width; j += 32) hist[j] = 0;
  const int spec = hyp_spec[h], maxfz = hyp_maxfz[h];
  const int64_t p0 = pk_off[spec], n_pk = pk_off[spec + 1] - p0;
  const uint32_t* off = offsets + (int64_t)(chunk - chunk0) * n_bins;
  const int tol_da = c_frag.tol_da;
  const double ln_fmin = log((double)fmin);
  const uint32_t lo_key = (uint32_t)lo << 16, hi_key = (uint32_t)hi << 16;
  __syncwarp();
  // all (peak, charge) windows of the spectrum, 32 at a time; the ones reaching an entry of this chunk are queued
  const int64_t n_win = n_pk * (int64_t)max(maxfz - 1, 0);
  int nq = 0;
  for (int64_t base = 0; base < n_win; base += 32) {
    const int64_t i = base + lane;
    KcWindow w{0, -1, 0, -1};
    bool live = false;
    if (i < n_win) {
      const int64_t pk = i / (maxfz - 1);
      const int z = (int)(i % (maxfz - 1)) + 1;
      const float m = __fmul_rn(pk_mass[p0 + pk], (float)z);
      const float a = vk::tol_bound(m, tol_lo, tol_da), bd = vk::tol_bound(m, tol_hi, tol_da);
      if (bd >= fmin) {
        w.qlo = max(log_pos(a, ln_fmin, inv_logw), (int64_t)0);
        w.qhi = log_pos(bd, ln_fmin, inv_logw);
        w.b0 = (int32_t)min(w.qlo >> 16, (int64_t)n_bins);
        w.b1 = (int32_t)min(w.qhi >> 16, (int64_t)n_bins - 1);
        live = w.b0 <= w.b1 && off[w.b0] != off[w.b1 + 1];
      }
    }
    const unsigned bal = __ballot_sync(VK_FULL, live);
    if (live) queue[nq + __popc(bal & ((1u << lane) - 1u))] = w;
    nq += __popc(bal);
    if (nq >= 32) {   // a full round: one window per lane
      __syncwarp();
      kc_count_window(queue[lane], off, entries, lo_key, hi_key, lo, hist);
      __syncwarp();
      if (lane < nq - 32) queue[lane] = queue[lane + 32];
      __syncwarp();
      nq -= 32;
    }
  }
  __syncwarp();
  if (lane < nq) kc_count_window(queue[lane], off, entries, lo_key, hi_key, lo, hist);
  __syncwarp();
  // statistics and the threshold append: one atomic per 32 rows reserves the group's output slots
  unsigned int scored = 0;
  unsigned long long matched = 0;
  for (int j0 = 0; j0 < width; j0 += 32) {
    const int j = j0 + lane;
    const uint32_t c = j < width ? hist[j] : 0u;
    scored += c > 0u;
    matched += c;
    const bool app = j < width && (int)c >= thr;
    const unsigned bal = __ballot_sync(VK_FULL, app);
    if (!bal) continue;
    unsigned long long slot0 = 0;
    if (lane == 0) slot0 = atomicAdd(n_out, (unsigned long long)__popc(bal));
    slot0 = __shfl_sync(VK_FULL, slot0, 0);
    if (app) {
      const unsigned long long w = slot0 + __popc(bal & ((1u << lane) - 1u));
      if ((int64_t)w < cap) {
        out_hyp[w] = h;
        out_row[w] = chunk * chunk_size + lo + j;
        out_cnt[w] = (int32_t)c;
      }
    }
  }
  scored = (unsigned int)vk::warp_sum((long long)scored);
  matched = (unsigned long long)vk::warp_sum((long long)matched);
  if (lane == 0) {
    if (scored) atomicAdd(&hyp_scored[h], scored);
    if (matched) atomicAdd(&hyp_matched[h], matched);
  }
}

// ------------------------------------------------------------------------------------------ brute-force K1
constexpr int KB_WARPS = 4;
constexpr int KB_MAXF = 256;   // fragments per ladder (length <= 255)

__global__ void __launch_bounds__(KB_WARPS * 32)
k1_brute_k(int64_t n, const int32_t* c_hyp, const int32_t* c_row, const int32_t* hyp_spec, const int8_t* hyp_maxfz,
           const int64_t* pk_off, const float* pk_mass, const int64_t* seq_off, const uint8_t* len,
           const uint64_t* mask, const float* mass32, const uint8_t* res, int min_ion, float fmin, float fmax,
           float tol_lo, float tol_hi, int32_t* out_cnt) {
  __shared__ vk::SmemFrag fp;
  __shared__ float frag[KB_WARPS][2][KB_MAXF];   // b ladder, y ladder; NaN where the ion is not counted
  frag_from_const(fp);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t i = (int64_t)blockIdx.x * KB_WARPS + warp;
  if (i >= n) return;
  const int h = c_hyp[i], r = c_row[i];
  const int L = len[r];
  if (lane < 2) {   // lane 0 the b ions, lane 1 the y ions, each a running f32 sum in ladder order
    const uint8_t* s = res + seq_off[r];
    const uint64_t mk = mask[r];
    const float nt = vk::nterm_of(fp, mk);
    float acc = lane == 0 ? nt : __fsub_rn(mass32[r], nt);
    for (int k = 0; k + 1 < L; ++k) {
      const float rm = vk::resmass(fp, s[k], k, mk);
      acc = lane == 0 ? __fadd_rn(acc, rm) : __fsub_rn(acc, rm);
      const bool idx_ok = lane == 0 ? (k + 1 > min_ion) : (L - 1 - k > min_ion);
      frag[warp][lane][k] = (idx_ok && acc >= fmin && acc <= fmax) ? acc : __int_as_float(0x7fc00000);
    }
  }
  __syncwarp();
  const int spec = hyp_spec[h], maxfz = hyp_maxfz[h];
  const int64_t p0 = pk_off[spec], p1 = pk_off[spec + 1];
  const int tol_da = fp.tol_da;
  long long c = 0;
  for (int64_t p = p0 + lane; p < p1; p += 32) {
    const float pm = pk_mass[p];
    for (int z = 1; z < maxfz; ++z) {
      const float m = __fmul_rn(pm, (float)z);
      const float a = vk::tol_bound(m, tol_lo, tol_da), bd = vk::tol_bound(m, tol_hi, tol_da);
      for (int k = 0; k + 1 < L; ++k) {
        const float fb = frag[warp][0][k], fy = frag[warp][1][k];
        c += (fb >= a && fb <= bd);
        c += (fy >= a && fy <= bd);
      }
    }
  }
  c = vk::warp_sum(c);
  if (lane == 0) out_cnt[i] = (int32_t)c;
}

// ------------------------------------------------------------------------------------------ K2
template <bool SHIFT>
__global__ void __launch_bounds__(vk::K2_WARPS * 32)
k2_compat_k(int n_spec, const int64_t* cand_off, const int32_t* c_row, const int8_t* c_maxfz, const int32_t* spec_ids,
            const int64_t* pk_off, const float* pk_mass, const float* pk_int, const int64_t* seq_off,
            const uint8_t* len, const uint64_t* mask, const float* mass32, const uint8_t* res, float tol_lo,
            float tol_hi, const float* c_shift, vk::K2Out out) {
  __shared__ vk::SmemFrag sf;
  frag_from_const(sf);
  __syncthreads();
  vk::k2_body<SHIFT>(sf, n_spec, cand_off, c_row, c_maxfz, spec_ids, pk_off, pk_mass, pk_int, seq_off, len, mask,
                     mass32, res, tol_lo, tol_hi, c_shift, out);
}

int k2_compat(int n_spec, const int64_t* cand_off, const int32_t* c_row, const int8_t* c_maxfz,
              const int32_t* spec_ids, const int64_t* pk_off, const float* pk_mass, const float* pk_int,
              const int64_t* seq_off, const uint8_t* len, const uint64_t* mask, const float* mass32,
              const uint8_t* res, float tol_lo, float tol_hi, const float* c_shift, double* o_hs, float* o_sb,
              float* o_sy, float* o_ppm, int16_t* o_mb, int16_t* o_my, int16_t* o_lb, int16_t* o_ly,
              void* stream) {
  if (n_spec <= 0) return 0;
  vk::K2Out out{o_hs, o_sb, o_sy, o_ppm, o_mb, o_my, o_lb, o_ly};
  const unsigned grid = (unsigned)((n_spec + vk::K2_WARPS - 1) / vk::K2_WARPS);
  cudaStream_t st = (cudaStream_t)stream;
  if (c_shift)
    k2_compat_k<true><<<grid, vk::K2_WARPS * 32, 0, st>>>(n_spec, cand_off, c_row, c_maxfz, spec_ids, pk_off,
                                                           pk_mass, pk_int, seq_off, len, mask, mass32, res, tol_lo,
                                                           tol_hi, c_shift, out);
  else
    k2_compat_k<false><<<grid, vk::K2_WARPS * 32, 0, st>>>(n_spec, cand_off, c_row, c_maxfz, spec_ids, pk_off,
                                                            pk_mass, pk_int, seq_off, len, mask, mass32, res, tol_lo,
                                                            tol_hi, nullptr, out);
  return vk_launch_status();
}

}  // namespace

extern "C" {

int vk_set_params(const float* mono, const float* stat, const float* var) {
  if (!mono || !stat || !var) return VK_E_ARG;
  float tables[3][26];
  for (int i = 0; i < 26; ++i) {
    tables[0][i] = mono[i];
    tables[1][i] = stat[i];
    tables[2][i] = var[i];
  }
  // mono, stat and var are the first three members, contiguous
  return vk_err(cudaMemcpyToSymbol(c_frag, tables, sizeof(tables), 0));
}

int vk_set_nterm(float nterm) {
  return vk_err(cudaMemcpyToSymbol(c_frag, &nterm, sizeof(float), offsetof(ConstFrag, nterm)));
}

int vk_set_tol_da(int da) {
  return vk_err(cudaMemcpyToSymbol(c_frag, &da, sizeof(int), offsetof(ConstFrag, tol_da)));
}

int vk_frag_count(int64_t n, const int64_t* seq_off, const uint8_t* len, const uint64_t* mask, const float* mass32,
                  const uint8_t* res, int min_ion_index, float fmin, float fmax, int32_t* count, void* stream) {
  if (n < 0) return VK_E_ARG;
  if (n == 0) return 0;
  frag_count_k<<<(unsigned)((n + FE_ROWS - 1) / FE_ROWS), FE_ROWS, 0, (cudaStream_t)stream>>>(
      n, seq_off, len, mask, mass32, res, min_ion_index, fmin, fmax, count);
  return vk_launch_status();
}

int vk_frag_emit(int64_t n, const int64_t* seq_off, const uint8_t* len, const uint64_t* mask, const float* mass32,
                 const uint8_t* res, int min_ion_index, float fmin, float fmax, double inv_logw, int chunk_size,
                 int64_t row0, const int64_t* out_off, int64_t* keys, void* stream) {
  if (n < 0 || chunk_size <= 0) return VK_E_ARG;
  if (n == 0) return 0;
  frag_emit_k<<<(unsigned)((n + FE_ROWS - 1) / FE_ROWS), FE_ROWS, 0, (cudaStream_t)stream>>>(
      n, seq_off, len, mask, mass32, res, min_ion_index, fmin, fmax, inv_logw, chunk_size, row0, out_off, keys);
  return vk_launch_status();
}

int vk_k1(int n_items, const int32_t* it_hyp, const int32_t* it_chunk, const int32_t* it_lo, const int32_t* it_hi,
          const int32_t* hyp_spec, const int8_t* hyp_maxfz, const int64_t* pk_off, const float* pk_mass,
          const uint32_t* offsets, const uint32_t* entries, int n_bins, int chunk0, int chunk_size, int tile,
          float tol_lo, float tol_hi, float fmin, double inv_logw, int thr, int64_t cap,
          unsigned long long* n_out, int32_t* out_hyp, int32_t* out_row, int32_t* out_cnt,
          unsigned int* hyp_scored, unsigned long long* hyp_matched, void* stream) {
  if (n_items < 0) return VK_E_ARG;
  if (n_items == 0) return 0;
  if (tile <= 0 || n_bins <= 0) return VK_E_ARG;
  const size_t sh = sizeof(KcWindow) * KC_QUEUE * KC_WARPS + (size_t)KC_WARPS * tile * sizeof(uint32_t);
  if (sh > 200 * 1024) return VK_E_TOO_LARGE;
  cudaError_t e = cudaFuncSetAttribute(k1_csr_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  if (e != cudaSuccess) return vk_err(e);
  const unsigned grid = (unsigned)((n_items + KC_WARPS - 1) / KC_WARPS);
  k1_csr_k<<<grid, KC_WARPS * 32, sh, (cudaStream_t)stream>>>(
      n_items, it_hyp, it_chunk, it_lo, it_hi, hyp_spec, hyp_maxfz, pk_off, pk_mass, offsets, entries, n_bins,
      chunk0, chunk_size, tile, tol_lo, tol_hi, fmin, inv_logw, thr, cap, n_out, out_hyp, out_row, out_cnt,
      hyp_scored, hyp_matched);
  return vk_launch_status();
}

int vk_k1_brute(int64_t n, const int32_t* c_hyp, const int32_t* c_row, const int32_t* hyp_spec,
                const int8_t* hyp_maxfz, const int64_t* pk_off, const float* pk_mass, const int64_t* seq_off,
                const uint8_t* len, const uint64_t* mask, const float* mass32, const uint8_t* res,
                int min_ion_index, float fmin, float fmax, float tol_lo, float tol_hi, double inv_logw,
                int32_t* out_cnt, void* stream) {
  (void)inv_logw;   // part of the reference's argument list; the brute-force count does not quantise
  if (n < 0) return VK_E_ARG;
  if (n == 0) return 0;
  k1_brute_k<<<(unsigned)((n + KB_WARPS - 1) / KB_WARPS), KB_WARPS * 32, 0, (cudaStream_t)stream>>>(
      n, c_hyp, c_row, hyp_spec, hyp_maxfz, pk_off, pk_mass, seq_off, len, mask, mass32, res, min_ion_index, fmin,
      fmax, tol_lo, tol_hi, out_cnt);
  return vk_launch_status();
}

int vk_k2(int n_spec, const int64_t* cand_off, const int32_t* c_row, const int8_t* c_maxfz, const int32_t* spec_ids,
          const int64_t* pk_off, const float* pk_mass, const float* pk_int, const int64_t* seq_off,
          const uint8_t* len, const uint64_t* mask, const float* mass32, const uint8_t* res, float tol_lo,
          float tol_hi, double* o_hs, float* o_sb, float* o_sy, float* o_ppm, int16_t* o_mb, int16_t* o_my,
          int16_t* o_lb, int16_t* o_ly, int threads, void* stream) {
  (void)threads;   // the launch shape is this library's (one warp per spectrum)
  return k2_compat(n_spec, cand_off, c_row, c_maxfz, spec_ids, pk_off, pk_mass, pk_int, seq_off, len, mask, mass32,
                   res, tol_lo, tol_hi, nullptr, o_hs, o_sb, o_sy, o_ppm, o_mb, o_my, o_lb, o_ly, stream);
}

int vk_k2_shift(int n_spec, const int64_t* cand_off, const int32_t* c_row, const int8_t* c_maxfz,
                const int32_t* spec_ids, const int64_t* pk_off, const float* pk_mass, const float* pk_int,
                const int64_t* seq_off, const uint8_t* len, const uint64_t* mask, const float* mass32,
                const uint8_t* res, float tol_lo, float tol_hi, const float* c_shift, double* o_hs, float* o_sb,
                float* o_sy, float* o_ppm, int16_t* o_mb, int16_t* o_my, int16_t* o_lb, int16_t* o_ly,
                int threads, void* stream) {
  (void)threads;
  if (!c_shift) return VK_E_ARG;
  return k2_compat(n_spec, cand_off, c_row, c_maxfz, spec_ids, pk_off, pk_mass, pk_int, seq_off, len, mask, mass32,
                   res, tol_lo, tol_hi, c_shift, o_hs, o_sb, o_sy, o_ppm, o_mb, o_my, o_lb, o_ly, stream);
}

}  // extern "C"
