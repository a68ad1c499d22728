// K1 per-peak search of one (tile, hypothesis) work item, shared by the staged K1 kernel and the fused search.
//
// The tile's postings (u32 keys: (f32bits(f) - f32bits(fmin)) << row_bits | local row, sorted) and its coarse-bin
// CSR are in shared memory.  Lanes stride over the spectrum's peaks x fragment charges: the tolerance window
// [a, bd] of peak mass p*z (Sage f32 bounds) is the key range [bits(a)-base, bits(bd)-base] (clamped to the
// fragment range), found through the coarse bins and a binary search; every posting in range whose row lies in
// [rlo, rhi) adds one to cnt[hoff + row].  Exactly the reference's brute-force count (kernels.cu:195-232).
#pragma once
#include "common.cuh"

namespace vk {

// cnt[hoff + l] is the count of tile row l (rows rlo <= l < rhi only).  With isum != nullptr, every match also adds
// the peak's weight round(intensity * wscale) (u32, wscale = 2^24 / TIC of the spectrum) to isum[hoff + l]: the
// summed matched intensity as a fixed-point fraction of the TIC, accumulated with integer atomics (deterministic).
__device__ __forceinline__ void k1_item_per_peak(const uint32_t* post, const uint16_t* cb, uint32_t* cnt, int64_t hoff,
                                                 int rlo, int rhi,
                                                 int64_t p0, int64_t p1, int maxfz, const float* pk_mass,
                                                 float tol_lo, float tol_hi, int tol_da, const vk_tindex& ix,
                                                 int lane, uint32_t* isum = nullptr, const float* pk_int = nullptr,
                                                 float wscale = 0.f) {
  const int row_bits = ix.row_bits;
  const uint32_t rowmask = (1u << row_bits) - 1u;
  const int sh = 32 - ix.cbin_bits;
  const float fmin = __uint_as_float(ix.fmin_bits), fmax = __uint_as_float(ix.fmax_bits);
  const uint32_t krange = ix.fmax_bits - ix.fmin_bits;
  const int64_t n_iter = (p1 - p0 + 31) & ~31ll;
  for (int64_t q = lane; q < n_iter; q += 32) {
    const int64_t p = p0 + q;
    const float pm = p < p1 ? pk_mass[p] : 0.f;
    const uint32_t wgt = (isum && p < p1) ? __float2uint_rn(__fmul_rn(pk_int[p], wscale)) : 0u;
    for (int z = 1; z < maxfz; ++z) {
      int e = 0, e1 = 0;
      uint32_t hi_key = 0;
      if (p < p1) {
        const float m = __fmul_rn(pm, (float)z);
        const float a = vk::tol_bound(m, tol_lo, tol_da), bd = vk::tol_bound(m, tol_hi, tol_da);
        if (bd >= fmin && a <= fmax) {
          const uint32_t ka = a <= fmin ? 0u : __float_as_uint(a) - ix.fmin_bits;
          const uint32_t kb = bd >= fmax ? krange : __float_as_uint(bd) - ix.fmin_bits;
          const uint32_t lo_key = ka << row_bits;
          hi_key = (kb << row_bits) | rowmask;
          e = cb[lo_key >> sh];
          e1 = cb[(hi_key >> sh) + 1];
          int R = e1;
          while (e < R) {
            int M = (e + R) >> 1;
            if (post[M] < lo_key) e = M + 1; else R = M;
          }
        }
      }
      for (; e < e1; ++e) {
        const uint32_t v = post[e];
        if (v > hi_key) break;
        const int l = (int)(v & rowmask);
        if (l >= rlo && l < rhi) {
          atomicAdd(&cnt[hoff + l], 1u);
          if (isum) atomicAdd(&isum[hoff + l], wgt);
        }
      }
    }
  }
}


}  // namespace vk
