// K2 exact rescoring entry point with fragment constants by value (no process-wide state).
#include "k2_impl.cuh"

namespace {

template <bool SHIFT>
__global__ void __launch_bounds__(vk::K2_WARPS * 32)
k2_spectra_k(vk_frag_params fpv, int n_spec, const int64_t* cand_off, const int32_t* c_row, const int8_t* c_maxfz,
             const int64_t* pk_off, const float* pk_mass, const float* pk_int, const int64_t* seq_off,
             const uint8_t* len, const uint64_t* mask, const float* mass32, const uint8_t* res, float tol_lo,
             float tol_hi, const float* c_shift, vk::K2Out out) {
  __shared__ vk::SmemFrag sf;
  vk::load_frag(sf, fpv);
  __syncthreads();
  vk::k2_body<SHIFT>(sf, n_spec, cand_off, c_row, c_maxfz, nullptr, pk_off, pk_mass, pk_int, seq_off, len, mask,
                     mass32, res, tol_lo, tol_hi, c_shift, out);
}

// One thread per candidate (grid-stride over the run's candidates): the candidate's spectrum by binary search of
// cand_off, its peaks read in global memory (GlobalPeaks).  Same arithmetic as the warp-per-spectrum kernel.
__global__ void __launch_bounds__(256)
k2_cands_k(vk_frag_params fpv, int n_spec, const int64_t* cand_off, const int32_t* c_row, const int8_t* c_maxfz,
           const int64_t* pk_off, const float* pk_mass, const float* pk_int, const int64_t* seq_off,
           const uint8_t* len, const uint64_t* mask, const float* mass32, const uint8_t* res, float tol_lo,
           float tol_hi, vk::K2Out out) {
  __shared__ vk::SmemFrag sf;
  vk::load_frag(sf, fpv);
  __syncthreads();
  const int64_t n_c = cand_off[n_spec];
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n_c; c += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = n_spec;   // the spectrum s with cand_off[s] <= c < cand_off[s + 1]
    while (hi - lo > 1) {
      const int m = (lo + hi) >> 1;
      if (__ldg(cand_off + m) <= c) lo = m; else hi = m;
    }
    const int64_t p0 = pk_off[lo];
    const vk::GlobalPeaks pt{pk_mass + p0, pk_int + p0, (int)min((int64_t)VK_K2_MAXPK, pk_off[lo + 1] - p0)};
    vk::k2_score<false, vk::GlobalPeaks>(sf, pt, c_row[c], c_maxfz[c], seq_off, len, mask, mass32, res, tol_lo,
                                         tol_hi, 0.f, out, c);
  }
}

}  // namespace

extern "C" int vk_k2_cands(const vk_frag_params* fp, int n_spec, const int64_t* cand_off, const int32_t* c_row,
                           const int8_t* c_maxfz, const int64_t* pk_off, const float* pk_mass, const float* pk_int,
                           const int64_t* seq_off, const uint8_t* len, const uint64_t* mask, const float* mass32,
                           const uint8_t* res, float tol_lo, float tol_hi, double* o_hs, float* o_sb, float* o_sy,
                           float* o_ppm, int16_t* o_mb, int16_t* o_my, int16_t* o_lb, int16_t* o_ly, void* stream) {
  if (!fp) return VK_E_ARG;
  if (n_spec <= 0) return 0;
  vk::K2Out out{o_hs, o_sb, o_sy, o_ppm, o_mb, o_my, o_lb, o_ly};
  int per_sm = 0, dev = 0, n_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k2_cands_k, 256, 0);
  if (e == cudaSuccess) e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return vk_err(e);
  k2_cands_k<<<(unsigned)(std::max(per_sm, 1) * n_sm), 256, 0, (cudaStream_t)stream>>>(
      *fp, n_spec, cand_off, c_row, c_maxfz, pk_off, pk_mass, pk_int, seq_off, len, mask, mass32, res, tol_lo, tol_hi,
      out);
  return vk_launch_status();
}

extern "C" int vk_k2_spectra(const vk_frag_params* fp, int n_spec, const int64_t* cand_off, const int32_t* c_row,
                             const int8_t* c_maxfz, const int64_t* pk_off, const float* pk_mass, const float* pk_int,
                             const int64_t* seq_off, const uint8_t* len, const uint64_t* mask, const float* mass32,
                             const uint8_t* res, float tol_lo, float tol_hi, const float* c_shift, double* o_hs,
                             float* o_sb, float* o_sy, float* o_ppm, int16_t* o_mb, int16_t* o_my, int16_t* o_lb,
                             int16_t* o_ly, void* stream) {
  if (!fp) return VK_E_ARG;
  if (n_spec <= 0) return 0;
  vk::K2Out out{o_hs, o_sb, o_sy, o_ppm, o_mb, o_my, o_lb, o_ly};
  unsigned grid = (unsigned)((n_spec + vk::K2_WARPS - 1) / vk::K2_WARPS);
  cudaStream_t st = (cudaStream_t)stream;
  if (c_shift)
    k2_spectra_k<true><<<grid, vk::K2_WARPS * 32, 0, st>>>(*fp, n_spec, cand_off, c_row, c_maxfz, pk_off, pk_mass,
                                                           pk_int, seq_off, len, mask, mass32, res, tol_lo, tol_hi,
                                                           c_shift, out);
  else
    k2_spectra_k<false><<<grid, vk::K2_WARPS * 32, 0, st>>>(*fp, n_spec, cand_off, c_row, c_maxfz, pk_off, pk_mass,
                                                            pk_int, seq_off, len, mask, mass32, res, tol_lo, tol_hi,
                                                            nullptr, out);
  return vk_launch_status();
}
