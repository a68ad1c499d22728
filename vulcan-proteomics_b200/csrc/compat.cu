// Reference-compatible entry points (names and argument lists of vulcan/gpu/_lib.py:22-35, semantics of
// vulcan/gpu/kernels.cu): process-wide fragment constants, the reference's log-ppm (chunk, bin) CSR index build and
// K1 count over it, the brute-force count, and K2 with the reference's candidate layout.
#include "common.cuh"
#include "k2_impl.cuh"

namespace {

struct ConstFrag {
  float mono[26];
  float stat[26];
  float var[26];
  float nterm;
  int tol_da;
};
__constant__ ConstFrag c_frag;

// View of the constant-memory constants with the field names the shared helpers use.
struct CView {
  const float* mono;
  const float* stat;
  const float* var;
  float nterm;
};

__device__ __forceinline__ float c_resmass(uint8_t r, int k, uint64_t mask) {
  int i = r - 'A';
  float d = ((mask >> k) & 1ull) ? c_frag.var[i] : c_frag.stat[i];
  return __fadd_rn(c_frag.mono[i], d);
}
__device__ __forceinline__ float c_nterm(uint64_t mask) { return (mask & VK_NTERM_BIT) ? c_frag.nterm : 0.f; }

// kernels.cu:53-71 -- one thread per row
__global__ void frag_count_k(int64_t n, const int64_t* seq_off, const uint8_t* len, const uint64_t* mask,
                             const float* mass32, const uint8_t* res, int min_ion, float fmin, float fmax,
                             int32_t* count) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint8_t* s = res + seq_off[i];
  int L = len[i];
  uint64_t mk = mask[i];
  float b = c_nterm(mk), y = __fsub_rn(mass32[i], c_nterm(mk));
  int c = 0;
  for (int k = 0; k + 1 < L; ++k) {
    float rm = c_resmass(s[k], k, mk);
    b = __fadd_rn(b, rm);
    y = __fsub_rn(y, rm);
    c += (k + 1 > min_ion && b >= fmin && b <= fmax);
    c += (L - 1 - k > min_ion && y >= fmin && y <= fmax);
  }
  count[i] = c;
}

__device__ __forceinline__ int64_t logq(float x, double lf, double inv_logw) {
  return (int64_t)floor((log((double)x) - lf) * inv_logw * 65536.0);
}

// kernels.cu:73-101 -- one thread per row, keys chunk<<50 | (q>>16)<<32 | local<<16 | (q & 0xffff)
__global__ void frag_emit_k(int64_t n, const int64_t* seq_off, const uint8_t* len, const uint64_t* mask,
                            const float* mass32, const uint8_t* res, int min_ion, float fmin, float fmax,
                            double inv_logw, int chunk_size, int64_t row0, const int64_t* out_off, int64_t* keys) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint8_t* s = res + seq_off[i];
  int L = len[i];
  uint64_t mk = mask[i];
  float b = c_nterm(mk), y = __fsub_rn(mass32[i], c_nterm(mk));
  int64_t g = row0 + i;
  int64_t hi_part = ((g / chunk_size) << 50) | ((g % chunk_size) << 16);
  int64_t o = out_off[i];
  double lf = log((double)fmin);
  for (int k = 0; k + 1 < L; ++k) {
    float rm = c_resmass(s[k], k, mk);
    b = __fadd_rn(b, rm);
    y = __fsub_rn(y, rm);
    if (k + 1 > min_ion && b >= fmin && b <= fmax) {
      int64_t q = logq(b, lf, inv_logw);
      keys[o++] = hi_part | ((q >> 16) << 32) | (q & 0xffff);
    }
    if (L - 1 - k > min_ion && y >= fmin && y <= fmax) {
      int64_t q = logq(y, lf, inv_logw);
      keys[o++] = hi_part | ((q >> 16) << 32) | (q & 0xffff);
    }
  }
}

__device__ __forceinline__ float c_tol(float m, float tol) { return vk::tol_bound(m, tol, c_frag.tol_da); }

// kernels.cu:112-190 semantics.  One warp per work item (hyp, chunk, [lo, hi)); warp-private shared counters;
// lanes stride over the spectrum's peaks x fragment charges; each (chunk, bin) list is searched for local >= lo.
constexpr int K1C_WARPS = 4;
__global__ void __launch_bounds__(K1C_WARPS * 32)
k1_compat_k(int n_items, const int32_t* it_hyp, const int32_t* it_chunk, const int32_t* it_lo, const int32_t* it_hi,
            const int32_t* hyp_spec, const int8_t* hyp_maxfz, const int64_t* pk_off, const float* pk_mass,
            const uint32_t* offsets, const uint32_t* entries, int n_bins, int chunk0, int chunk_size, int tile,
            float tol_lo, float tol_hi, float fmin, double inv_logw, int thr, int64_t cap,
            unsigned long long* n_out, int32_t* out_hyp, int32_t* out_row, int32_t* out_cnt,
            unsigned int* hyp_scored, unsigned long long* hyp_matched) {
  extern __shared__ uint32_t k1c_smem[];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int item = blockIdx.x * K1C_WARPS + warp;
  if (item >= n_items) return;
  uint32_t* cnt = k1c_smem + (size_t)warp * tile;
  int h = it_hyp[item], c = it_chunk[item], lo = it_lo[item], hi = it_hi[item];
  int n = hi - lo;
  for (int j = lane; j < n; j += 32) cnt[j] = 0;
  __syncwarp();
  int s = hyp_spec[h], maxfz = hyp_maxfz[h];
  int64_t p0 = pk_off[s], p1 = pk_off[s + 1];
  const uint32_t* off = offsets + (int64_t)(c - chunk0) * n_bins;
  double lf = log((double)fmin);
  uint32_t lo_key = (uint32_t)lo << 16, hi_key = (uint32_t)hi << 16;
  for (int64_t p = p0 + lane; p < p1; p += 32) {
    float pm = pk_mass[p];
    for (int z = 1; z < maxfz; ++z) {
      float m = __fmul_rn(pm, (float)z);
      float a = c_tol(m, tol_lo), bd = c_tol(m, tol_hi);
      if (bd < fmin) continue;
      int64_t qlo = logq(a, lf, inv_logw), qhi = logq(bd, lf, inv_logw);
      if (qlo < 0) qlo = 0;
      int64_t b0 = qlo >> 16, b1 = qhi >> 16;
      if (b1 >= n_bins) b1 = n_bins - 1;
      for (int64_t bb = b0; bb <= b1; ++bb) {
        uint32_t e0 = off[bb], e1 = off[bb + 1];
        uint32_t L = e0, R = e1;
        while (L < R) {
          uint32_t M = (L + R) >> 1;
          if (entries[M] < lo_key) L = M + 1; else R = M;
        }
        for (uint32_t e = L; e < e1; ++e) {
          uint32_t v = entries[e];
          if (v >= hi_key) break;
          int64_t q = (bb << 16) | (v & 0xffff);
          if (q >= qlo && q <= qhi) atomicAdd(&cnt[(v >> 16) - lo], 1u);
        }
      }
    }
  }
  __syncwarp();
  unsigned int scored = 0;
  unsigned long long matched = 0;
  for (int j = lane; j < n; j += 32) {
    uint32_t k = cnt[j];
    scored += (k > 0);
    matched += k;
    if ((int)k >= thr) {
      unsigned long long w = atomicAdd(n_out, 1ull);
      if ((int64_t)w < cap) {
        out_hyp[w] = h;
        out_row[w] = c * chunk_size + lo + j;
        out_cnt[w] = (int32_t)k;
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    scored += __shfl_xor_sync(VK_FULL, scored, o);
    matched += __shfl_xor_sync(VK_FULL, matched, o);
  }
  if (lane == 0) {
    if (scored) atomicAdd(&hyp_scored[h], scored);
    if (matched) atomicAdd(&hyp_matched[h], matched);
  }
}

// kernels.cu:195-232 -- one thread per (hyp, row) pair, plain f32 comparisons
__global__ void k1_brute_k(int64_t n, const int32_t* c_hyp, const int32_t* c_row, const int32_t* hyp_spec,
                           const int8_t* hyp_maxfz, const int64_t* pk_off, const float* pk_mass,
                           const int64_t* seq_off, const uint8_t* len, const uint64_t* mask, const float* mass32,
                           const uint8_t* res, int min_ion, float fmin, float fmax, float tol_lo, float tol_hi,
                           int32_t* out_cnt) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int h = c_hyp[i], r = c_row[i];
  int s = hyp_spec[h], maxfz = hyp_maxfz[h];
  int64_t p0 = pk_off[s], p1 = pk_off[s + 1];
  const uint8_t* sq = res + seq_off[r];
  int L = len[r];
  uint64_t mk = mask[r];
  float b = c_nterm(mk), y = __fsub_rn(mass32[r], c_nterm(mk));
  int cnt = 0;
  for (int k = 0; k + 1 < L; ++k) {
    float rm = c_resmass(sq[k], k, mk);
    b = __fadd_rn(b, rm);
    y = __fsub_rn(y, rm);
    for (int t = 0; t < 2; ++t) {
      float f = t == 0 ? b : y;
      bool ok = t == 0 ? (k + 1 > min_ion) : (L - 1 - k > min_ion);
      if (!ok || f < fmin || f > fmax) continue;
      for (int64_t p = p0; p < p1; ++p)
        for (int z = 1; z < maxfz; ++z) {
          float m = __fmul_rn(pk_mass[p], (float)z);
          if (f >= c_tol(m, tol_lo) && f <= c_tol(m, tol_hi)) ++cnt;
        }
    }
  }
  out_cnt[i] = cnt;
}

// K2 with the constant-memory fragment constants: copy them into shared memory and run the shared K2 body.
template <bool SHIFT>
__global__ void __launch_bounds__(vk::K2_WARPS * 32)
k2_compat_k(int n_spec, const int64_t* cand_off, const int32_t* c_row, const int8_t* c_maxfz, const int32_t* spec_ids,
            const int64_t* pk_off, const float* pk_mass, const float* pk_int, const int64_t* seq_off,
            const uint8_t* len, const uint64_t* mask, const float* mass32, const uint8_t* res, float tol_lo,
            float tol_hi, const float* c_shift, vk::K2Out out) {
  __shared__ vk::SmemFrag sf;
  for (int i = threadIdx.x; i < 26; i += blockDim.x) {
    sf.mono[i] = c_frag.mono[i];
    sf.stat[i] = c_frag.stat[i];
    sf.var[i] = c_frag.var[i];
  }
  if (threadIdx.x == 0) {
    sf.nterm = c_frag.nterm;
    sf.tol_da = c_frag.tol_da;
  }
  __syncthreads();
  vk::k2_body<SHIFT>(sf, n_spec, cand_off, c_row, c_maxfz, spec_ids, pk_off, pk_mass, pk_int, seq_off, len, mask,
                     mass32, res, tol_lo, tol_hi, c_shift, out);
}

}  // namespace

extern "C" {

int vk_set_params(const float* mono, const float* stat, const float* var) {
  ConstFrag f;
  cudaError_t e = cudaMemcpyFromSymbol(&f, c_frag, sizeof(ConstFrag));
  if (e != cudaSuccess) return vk_err(e);
  for (int i = 0; i < 26; ++i) {
    f.mono[i] = mono[i];
    f.stat[i] = stat[i];
    f.var[i] = var[i];
  }
  return vk_err(cudaMemcpyToSymbol(c_frag, &f, sizeof(ConstFrag)));
}

int vk_set_nterm(float nterm) {
  return vk_err(cudaMemcpyToSymbol(c_frag, &nterm, sizeof(float), offsetof(ConstFrag, nterm)));
}

int vk_set_tol_da(int da) {
  return vk_err(cudaMemcpyToSymbol(c_frag, &da, sizeof(int), offsetof(ConstFrag, tol_da)));
}

int vk_frag_count(int64_t n, const int64_t* seq_off, const uint8_t* len, const uint64_t* mask, const float* mass32,
                  const uint8_t* res, int min_ion_index, float fmin, float fmax, int32_t* count, void* stream) {
  if (n == 0) return 0;
  int bs = 256;
  frag_count_k<<<(unsigned)((n + bs - 1) / bs), bs, 0, (cudaStream_t)stream>>>(n, seq_off, len, mask, mass32, res,
                                                                              min_ion_index, fmin, fmax, count);
  return vk_launch_status();
}

int vk_frag_emit(int64_t n, const int64_t* seq_off, const uint8_t* len, const uint64_t* mask, const float* mass32,
                 const uint8_t* res, int min_ion_index, float fmin, float fmax, double inv_logw, int chunk_size,
                 int64_t row0, const int64_t* out_off, int64_t* keys, void* stream) {
  if (n == 0) return 0;
  int bs = 256;
  frag_emit_k<<<(unsigned)((n + bs - 1) / bs), bs, 0, (cudaStream_t)stream>>>(
      n, seq_off, len, mask, mass32, res, min_ion_index, fmin, fmax, inv_logw, chunk_size, row0, out_off, keys);
  return vk_launch_status();
}

int vk_k1(int n_items, const int32_t* it_hyp, const int32_t* it_chunk, const int32_t* it_lo, const int32_t* it_hi,
          const int32_t* hyp_spec, const int8_t* hyp_maxfz, const int64_t* pk_off, const float* pk_mass,
          const uint32_t* offsets, const uint32_t* entries, int n_bins, int chunk0, int chunk_size, int tile,
          float tol_lo, float tol_hi, float fmin, double inv_logw, int thr, int64_t cap,
          unsigned long long* n_out, int32_t* out_hyp, int32_t* out_row, int32_t* out_cnt,
          unsigned int* hyp_scored, unsigned long long* hyp_matched, void* stream) {
  if (n_items == 0) return 0;
  if (tile <= 0) return VK_E_ARG;
  size_t sh = (size_t)K1C_WARPS * tile * sizeof(uint32_t);
  if (sh > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k1_compat_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
    if (e != cudaSuccess) return vk_err(e);
  }
  unsigned grid = (unsigned)((n_items + K1C_WARPS - 1) / K1C_WARPS);
  k1_compat_k<<<grid, K1C_WARPS * 32, sh, (cudaStream_t)stream>>>(
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
  (void)inv_logw;
  if (n == 0) return 0;
  int bs = 128;
  k1_brute_k<<<(unsigned)((n + bs - 1) / bs), bs, 0, (cudaStream_t)stream>>>(
      n, c_hyp, c_row, hyp_spec, hyp_maxfz, pk_off, pk_mass, seq_off, len, mask, mass32, res, min_ion_index, fmin,
      fmax, tol_lo, tol_hi, out_cnt);
  return vk_launch_status();
}

static int k2_compat(int n_spec, const int64_t* cand_off, const int32_t* c_row, const int8_t* c_maxfz,
                     const int32_t* spec_ids, const int64_t* pk_off, const float* pk_mass, const float* pk_int,
                     const int64_t* seq_off, const uint8_t* len, const uint64_t* mask, const float* mass32,
                     const uint8_t* res, float tol_lo, float tol_hi, const float* c_shift, double* o_hs,
                     float* o_sb, float* o_sy, float* o_ppm, int16_t* o_mb, int16_t* o_my, int16_t* o_lb,
                     int16_t* o_ly, void* stream) {
  if (n_spec <= 0) return 0;
  vk::K2Out out{o_hs, o_sb, o_sy, o_ppm, o_mb, o_my, o_lb, o_ly};
  unsigned grid = (unsigned)((n_spec + vk::K2_WARPS - 1) / vk::K2_WARPS);
  if (c_shift)
    k2_compat_k<true><<<grid, vk::K2_WARPS * 32, 0, (cudaStream_t)stream>>>(
        n_spec, cand_off, c_row, c_maxfz, spec_ids, pk_off, pk_mass, pk_int, seq_off, len, mask, mass32, res, tol_lo,
        tol_hi, c_shift, out);
  else
    k2_compat_k<false><<<grid, vk::K2_WARPS * 32, 0, (cudaStream_t)stream>>>(
        n_spec, cand_off, c_row, c_maxfz, spec_ids, pk_off, pk_mass, pk_int, seq_off, len, mask, mass32, res, tol_lo,
        tol_hi, nullptr, out);
  return vk_launch_status();
}

int vk_k2(int n_spec, const int64_t* cand_off, const int32_t* c_row, const int8_t* c_maxfz, const int32_t* spec_ids,
          const int64_t* pk_off, const float* pk_mass, const float* pk_int, const int64_t* seq_off,
          const uint8_t* len, const uint64_t* mask, const float* mass32, const uint8_t* res, float tol_lo,
          float tol_hi, double* o_hs, float* o_sb, float* o_sy, float* o_ppm, int16_t* o_mb, int16_t* o_my,
          int16_t* o_lb, int16_t* o_ly, int threads, void* stream) {
  (void)threads;
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
