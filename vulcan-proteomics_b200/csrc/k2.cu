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

}  // namespace

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
