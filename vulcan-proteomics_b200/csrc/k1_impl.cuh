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

#ifndef K1_BM_LOG
#define K1_BM_LOG 6            // log2 of the presence-bitmap bits per coarse bin (6 or 7)
#endif
static_assert(K1_BM_LOG == 6 || K1_BM_LOG == 7, "64 or 128 bitmap bits per coarse bin");

namespace vk {

constexpr int K1_BM_WORDS = (1 << K1_BM_LOG) / 32;   // u32 words of a coarse bin's bitmap

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

// ---- filtered per-item search (staged K1) ----
//
// The tolerance window of a peak does not depend on the tile, so its key range is computed once per pass
// (k1_window_keys, by vk_k1_peak_keys) instead of once per (tile, hypothesis) item, together with a 32-bit filter
// word (k1_filter_word).  Every tile has a presence bitmap, built with the index (vk_tindex_bitmap) and staged with
// the tile: 2^K1_BM_LOG bits per coarse bin, bit s of bin b set when a posting of the bin has (low key) >>
// (low_bits - K1_BM_LOG) == s.  A window whose bits are all clear holds no posting and is dropped after one
// shared-memory word; the windows that may match are compacted into a per-warp queue (ballot) and searched
// exactly, one per lane, so the bin lookup and binary search run with every lane busy and only for them.  The
// counts are those of k1_item_per_peak: the bitmap only skips windows that hold no posting.

// Key range [ka, kb] of the tolerance window of fragment mass pm * z (Sage f32 bounds, both edges included), clamped
// to the index's fragment range; ka > kb when the window misses the range.
__device__ __forceinline__ uint2 k1_window_keys(float pm, int z, float tol_lo, float tol_hi, int tol_da,
                                                const vk_tindex& ix) {
  const float fmin = __uint_as_float(ix.fmin_bits), fmax = __uint_as_float(ix.fmax_bits);
  const float m = __fmul_rn(pm, (float)z);
  const float a = vk::tol_bound(m, tol_lo, tol_da), bd = vk::tol_bound(m, tol_hi, tol_da);
  if (!(bd >= fmin && a <= fmax)) return make_uint2(1u, 0u);
  const uint32_t ka = a <= fmin ? 0u : __float_as_uint(a) - ix.fmin_bits;
  const uint32_t kb = bd >= fmax ? ix.fmax_bits - ix.fmin_bits : __float_as_uint(bd) - ix.fmin_bits;
  return make_uint2(ka, kb);
}

// Bits per coarse bin actually used: 2^min(K1_BM_LOG, low_bits); a posting's bit is its top bits (row_bits +
// low_bits = 32).
__device__ __forceinline__ int k1_bm_bits(const vk_tindex& ix) {
  const int low_bits = ix.mass_bits - ix.cbin_bits;
  return low_bits < K1_BM_LOG ? low_bits : K1_BM_LOG;
}

// Bitmap position of key k: bin * 2^K1_BM_LOG + (low key >> (low_bits - bits)); monotone in k, below
// 2^(cbin_bits + K1_BM_LOG).
__device__ __forceinline__ uint32_t k1_bm_pos(uint32_t k, int low_bits, int bshift) {
  return ((k >> low_bits) << K1_BM_LOG) | ((k & ((1u << low_bits) - 1u)) >> bshift);
}

// One thread per coarse bin builds the bin's K1_BM_WORDS words in registers (the index build calls this per tile).
__device__ __forceinline__ void k1_build_bitmap(const uint32_t* post, const uint16_t* cb, int nb, int bits,
                                                uint32_t* bm) {
  const int top = 32 - bits;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    unsigned long long lo = 0ull, hi = 0ull;
    const int e1 = cb[b + 1];
    for (int e = cb[b]; e < e1; ++e) {
      const uint32_t s = post[e] >> top;
      if (s < 64u) lo |= 1ull << s; else hi |= 1ull << (s - 64u);
    }
    uint32_t* w = bm + (size_t)b * K1_BM_WORDS;
    w[0] = (uint32_t)lo;
    w[1] = (uint32_t)(lo >> 32);
    if (K1_BM_WORDS == 4) {
      w[2] = (uint32_t)hi;
      w[3] = (uint32_t)(hi >> 32);
    }
  }
}

// true when a bit in [ga, gb] (ga <= gb) is set
__device__ __forceinline__ bool k1_bm_any(const uint32_t* bm, uint32_t ga, uint32_t gb) {
  const uint32_t w0 = ga >> 5, w1 = gb >> 5;
  const uint32_t head = bm[w0] & (0xffffffffu << (ga & 31u));
  const uint32_t tail_mask = 0xffffffffu >> (31u - (gb & 31u));
  if (w0 == w1) return (head & tail_mask) != 0u;
  if (head) return true;
  for (uint32_t w = w0 + 1; w < w1; ++w)
    if (bm[w]) return true;
  return (bm[w1] & tail_mask) != 0u;
}

// Filter word of window [ka, kb]: the bitmap position of ka in bits 0..19 and the span to kb's position in bits
// 20..31, capped at 4095 (such wide windows always go to the exact search); K1_NO_WINDOW when ka > kb.
constexpr uint32_t K1_NO_WINDOW = 0xffffffffu;
__device__ __forceinline__ uint32_t k1_filter_word(uint2 k, const vk_tindex& ix) {
  if (k.x > k.y) return K1_NO_WINDOW;
  const int low_bits = ix.mass_bits - ix.cbin_bits;
  const int bshift = low_bits - k1_bm_bits(ix);
  const uint32_t ga = k1_bm_pos(k.x, low_bits, bshift), gb = k1_bm_pos(k.y, low_bits, bshift);
  return ga | (min(gb - ga, 4095u) << 20);
}

// true when the window of filter word f may hold a posting of the tile with bitmap bm
__device__ __forceinline__ bool k1_filter_pass(const uint32_t* bm, uint32_t f) {
  if (f == K1_NO_WINDOW) return false;
  const uint32_t ga = f & 0xfffffu, d = f >> 20;
  if (d == 4095u) return true;
  const uint32_t s = ga & 31u;
  if (s + d < 32u) return ((bm[ga >> 5] >> s) & ((2u << d) - 1u)) != 0u;
  return k1_bm_any(bm, ga, ga + d);
}

// Count the postings with key in [ka, kb] whose row lies in [rlo, rhi) (one lane, one window).
__device__ __forceinline__ void k1_count_range(const uint32_t* post, const uint16_t* cb, uint32_t* hw, uint32_t* iw,
                                               int rlo, int rhi, uint32_t ka, uint32_t kb, uint32_t wgt,
                                               const vk_tindex& ix) {
  const int row_bits = ix.row_bits;
  const uint32_t rowmask = (1u << row_bits) - 1u;
  const int low_bits = ix.mass_bits - ix.cbin_bits;
  const uint32_t lowmask = (1u << low_bits) - 1u;
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
        atomicAdd(&hw[l], 1u);
        if (iw) atomicAdd(&iw[l], wgt);
      }
    }
  }
}

constexpr int K1_QUEUE = 64;   // u32 entries per warp queue: (charge - 1) << 16 | peak index in the spectrum
#ifndef K1_UNROLL
#define K1_UNROLL 2            // filter-word loads in flight per lane
#endif

// One (tile, hypothesis) item by one warp.  For fragment charges z <= n_kz, keys[(z - 1) * kstride + p] holds the
// window keys of peak p and filt[...] its filter word; higher charges are computed here.  q: this warp's queue.
__device__ __forceinline__ void k1_item_filtered(const uint32_t* post, const uint16_t* cb, const uint32_t* bm,
                                                 uint32_t* hw, uint32_t* iw, int rlo, int rhi, int64_t p0,
                                                 int64_t p1, int maxfz, const uint2* __restrict__ keys,
                                                 const uint32_t* __restrict__ filt, int n_kz, int64_t kstride,
                                                 const float* pk_mass, float tol_lo, float tol_hi, int tol_da,
                                                 const vk_tindex& ix, int lane, uint32_t* q, const float* pk_int,
                                                 float wscale) {
  const int n = (int)(p1 - p0);
  int nq = 0;
  auto search = [&](uint32_t e) {
    const int zi = (int)(e >> 16);
    const int64_t p = p0 + (e & 0xffffu);
    const uint2 k = zi < n_kz ? keys[(int64_t)zi * kstride + p]
                              : k1_window_keys(pk_mass[p], zi + 1, tol_lo, tol_hi, tol_da, ix);
    const uint32_t wgt = iw ? __float2uint_rn(__fmul_rn(pk_int[p], wscale)) : 0u;
    k1_count_range(post, cb, hw, iw, rlo, rhi, k.x, k.y, wgt, ix);
  };
  auto push = [&](bool pass, uint32_t e) {
    const unsigned bal = __ballot_sync(0xffffffffu, pass);
    if (pass) q[nq + __popc(bal & ((1u << lane) - 1u))] = e;
    nq += __popc(bal);
    if (nq >= 32) {
      __syncwarp();
      search(q[lane]);
      __syncwarp();
      if (lane < nq - 32) q[lane] = q[lane + 32];
      __syncwarp();
      nq -= 32;
    }
  };
  for (int z = 1; z < maxfz; ++z) {
    const uint32_t zt = (uint32_t)(z - 1) << 16;
    if (z <= n_kz) {
      const uint32_t* __restrict__ fz = filt + (int64_t)(z - 1) * kstride + p0;
      for (int base = 0; base < n; base += 32 * K1_UNROLL) {
        uint32_t f[K1_UNROLL];
#pragma unroll
        for (int u = 0; u < K1_UNROLL; ++u) {   // the loads first: K1_UNROLL in flight per lane
          const int i = base + 32 * u + lane;
          f[u] = i < n ? __ldg(fz + i) : K1_NO_WINDOW;
        }
#pragma unroll
        for (int u = 0; u < K1_UNROLL; ++u) push(k1_filter_pass(bm, f[u]), zt | (uint32_t)(base + 32 * u + lane));
      }
    } else {
      for (int base = 0; base < n; base += 32) {
        const int i = base + lane;
        const uint32_t f = i < n ? k1_filter_word(k1_window_keys(pk_mass[p0 + i], z, tol_lo, tol_hi, tol_da, ix), ix)
                                 : K1_NO_WINDOW;
        push(k1_filter_pass(bm, f), zt | (uint32_t)i);
      }
    }
  }
  __syncwarp();
  if (lane < nq) search(q[lane]);
}


}  // namespace vk
