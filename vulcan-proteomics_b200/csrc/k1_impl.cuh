// K1 per-peak search of one (tile, hypothesis) work item, shared by the staged K1 kernel and the fused search.
//
// The tile's postings and its coarse-bin CSR are in shared memory.  A fragment's key is f32bits(f) - f32bits(fmin)
// (mass_bits wide); its coarse bin is the top cbin_bits of the key, and the posting holds the remaining low key bits
// and the local row: (key mod 2^(mass_bits - cbin_bits)) << row_bits | row, sorted within each bin, the bin given
// by the posting's position (cbin_off).  Lanes stride over the spectrum's peaks x fragment charges: the tolerance
// window [a, bd] of peak mass p*z (Sage f32 bounds) is the key range [bits(a)-base, bits(bd)-base] (clamped to the
// fragment range); in each coarse bin it touches (one, or two at a bin edge) a binary search finds its first
// posting, and every posting in range whose row lies in [rlo, rhi) adds one to cnt[hoff + row].  Exactly the
// reference's brute-force count (kernels.cu:195-232).
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
  const int low_bits = ix.mass_bits - ix.cbin_bits;
  const uint32_t lowmask = (1u << low_bits) - 1u;
  const float fmin = __uint_as_float(ix.fmin_bits), fmax = __uint_as_float(ix.fmax_bits);
  const uint32_t krange = ix.fmax_bits - ix.fmin_bits;
  for (int64_t p = p0 + lane; p < p1; p += 32) {
    const float pm = pk_mass[p];
    const uint32_t wgt = isum ? __float2uint_rn(__fmul_rn(pk_int[p], wscale)) : 0u;
    for (int z = 1; z < maxfz; ++z) {
      const float m = __fmul_rn(pm, (float)z);
      const float a = vk::tol_bound(m, tol_lo, tol_da), bd = vk::tol_bound(m, tol_hi, tol_da);
      if (!(bd >= fmin && a <= fmax)) continue;
      const uint32_t ka = a <= fmin ? 0u : __float_as_uint(a) - ix.fmin_bits;
      const uint32_t kb = bd >= fmax ? krange : __float_as_uint(bd) - ix.fmin_bits;
      const uint32_t ba = ka >> low_bits, bb = kb >> low_bits;
      for (uint32_t bin = ba; bin <= bb; ++bin) {
        const uint32_t lo_key = bin == ba ? (ka & lowmask) << row_bits : 0u;
        const uint32_t hi_key = bin == bb ? ((kb & lowmask) << row_bits) | rowmask : 0xffffffffu;
        int e = cb[bin];
        const int e1 = cb[bin + 1];
        int R = e1;
        while (e < R) {
          const int M = (e + R) >> 1;
          if (post[M] < lo_key) e = M + 1; else R = M;
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
}


}  // namespace vk
