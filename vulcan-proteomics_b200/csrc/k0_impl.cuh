// Device helpers shared by the K0 peak-view kernels (global and window peak modes).
#pragma once
#include "common.cuh"

namespace {

__device__ __forceinline__ uint32_t ord_f32(float x) {
  uint32_t u = __float_as_uint(x);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float unord_f32(uint32_t o) {
  uint32_t u = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
  return __uint_as_float(u);
}
__device__ __forceinline__ bool in_range(float mz, float fmin, float fmax) {
  return mz >= fmin && mz <= fmax;   // false for NaN
}

// Ascending bitonic sort of v[0, n_pow2) by the whole CTA (n_pow2 a power of two; ends with a CTA barrier).
__device__ __forceinline__ void block_bitonic_u64(uint64_t* v, int n_pow2) {
  for (int k = 2; k <= n_pow2; k <<= 1)
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

constexpr int K0_THREADS = 512;

// Exclusive scan of one int per thread over the CTA (K0_THREADS threads); wsum: K0_THREADS / 32 ints of scratch.
__device__ __forceinline__ int k0_block_excl_scan(int v, int* wsum) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int inc = (int)vk::warp_incl_scan(v);
  if (lane == 31) wsum[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const int w = lane < K0_THREADS / 32 ? wsum[lane] : 0;
    const int wi = (int)vk::warp_incl_scan(w);
    if (lane < K0_THREADS / 32) wsum[lane] = wi - w;
  }
  __syncthreads();
  const int r = wsum[warp] + inc - v;
  __syncthreads();
  return r;
}

}  // namespace
