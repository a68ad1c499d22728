// K0 peak view, window peak mode (reference vulcan/gpu/engine.py:171-210 with peak_mode "window").
//
// The in-range peaks (fmin <= m/z <= fmax, not NaN) of a spectrum are grouped by window w = floor(m/z * inv), and
// the top window_k of every window by (intensity desc, mass desc) are kept, then ordered by mass ascending; equal
// masses keep the selection order (window ascending, then intensity descending).  There is no cap on the total
// (engine.py:195-196 does nothing).  The reference divides an f32 CUDA tensor by the Python float window_th, which
// the device evaluates as a product with the f32 reciprocal: inv = 1.0f / (float)window_th, and w is the floor of
// the f32 product.  Its group id is spectrum * 1000 + w, so the entry points require 0 <= floor(fmin * inv) and
// floor(fmax * inv) <= 999, where groups of different spectra never meet.
//
// The count kernel (a warp per spectrum, per-window counts in a warp-private histogram) gives each spectrum a code:
//   1  the raw peaks are already in the final order -- (mass, window', ~intensity) non-decreasing, where window'
//      places below-range peaks before and above-range peaks after every window -- with no NaN m/z and no window
//      over window_k: the view is the in-range subsequence (a copy).
//   2  the same order with a window over window_k and none over KW_SEL peaks: a warp per spectrum.  That order
//      makes the in-range peaks one contiguous run of the raw peaks and every window a contiguous run inside it;
//      windows with at most window_k peaks are copied, fuller ones are ranked in registers (shuffles).
//   0  the rest (shuffled input, NaN m/z, windows over KW_SEL peaks): one CTA per spectrum sorts (ord(m/z),
//      ~ord(intensity)) keys in shared memory -- which orders mass and window too, both being monotone in m/z --,
//      ranks every peak inside its window, and places the kept peaks by a scan; only runs of equal (mass, window)
//      with different m/z, where the sort's m/z order and the reference's intensity order can differ, take a
//      second look.
// Peaks with equal intensity and mass give equal outputs, so the reference's last tie order (input position) never
// shows.  TIC = f64 sum of the kept intensities, stored as f32.
#include "k0_impl.cuh"

namespace {

constexpr int KW_WARPS = 4;     // warps per CTA of the warp kernels
constexpr int KW_SEL = 128;     // largest window ranked in registers (4 keys per lane)
constexpr int KW_BINS = 1000;   // windows per spectrum at most (group ids spectrum * 1000 + w)

__device__ __forceinline__ int win_of(float mz, float inv) { return (int)floorf(__fmul_rn(mz, inv)); }

// selection key: ascending = intensity descending, then mass descending
__device__ __forceinline__ uint64_t win_sel_key(float mass, float it) {
  return ((uint64_t)(~ord_f32(it)) << 32) | (uint64_t)(~ord_f32(mass));
}

__global__ void __launch_bounds__(KW_WARPS * 32)
k0w_count_k(int n_spec, const int64_t* raw_off, const float* raw_mz, const float* raw_int, float fmin, float fmax,
            float inv, int w_lo, int n_bins, int wk, int64_t* kept, uint8_t* easy, int32_t* hard_list,
            int32_t* n_hard) {
  extern __shared__ uint32_t kw_hist[];
  const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (s >= n_spec) return;
  uint32_t* hist = kw_hist + (threadIdx.x >> 5) * n_bins;
  for (int b = lane; b < n_bins; b += 32) hist[b] = 0u;
  __syncwarp();
  const int64_t r0 = raw_off[s], r1 = raw_off[s + 1];
  bool sorted = true;
  uint32_t c_hi = 0u;   // key of the previous chunk's last peak
  uint64_t c_lo = 0ull;
  for (int64_t b0 = r0; b0 < r1; b0 += 32) {
    const int64_t i = b0 + lane;
    uint32_t hi = 0u;
    uint64_t lo = 0ull;
    if (i < r1) {
      const float mz = raw_mz[i], it = raw_int[i];
      sorted &= !isnan(mz);
      int wq;   // window' = 0 below the range, 1 + window inside, n_bins + 1 above
      if (in_range(mz, fmin, fmax)) {
        const int b = win_of(mz, inv) - w_lo;
        atomicAdd(&hist[b], 1u);
        wq = 1 + b;
      } else {
        wq = mz < fmin ? 0 : n_bins + 1;
      }
      hi = ord_f32(__fsub_rn(mz, VK_PROTON));
      lo = ((uint64_t)wq << 32) | (uint64_t)(~ord_f32(it));
    }
    uint32_t p_hi = __shfl_up_sync(VK_FULL, hi, 1);
    uint64_t p_lo = __shfl_up_sync(VK_FULL, lo, 1);
    if (lane == 0) {
      p_hi = c_hi;
      p_lo = c_lo;
    }
    if (i < r1 && i > r0) sorted &= p_hi < hi || (p_hi == hi && p_lo <= lo);
    c_hi = __shfl_sync(VK_FULL, hi, 31);
    c_lo = __shfl_sync(VK_FULL, lo, 31);
  }
  __syncwarp();
  long long k = 0;
  uint32_t mx = 0u;
  for (int b = lane; b < n_bins; b += 32) {
    const uint32_t c = hist[b];
    k += min(c, (uint32_t)wk);
    mx = max(mx, c);
  }
  k = vk::warp_sum(k);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(VK_FULL, mx, o));
  sorted = __all_sync(VK_FULL, sorted);
  if (lane == 0) {
    kept[s] = k;
    const int code = !sorted ? 0 : (mx <= (uint32_t)wk ? 1 : (mx <= (uint32_t)KW_SEL ? 2 : 0));
    easy[s] = (uint8_t)code;
    if (code == 0) hard_list[atomicAdd(n_hard, 1)] = s;
  }
}

// One over-full window of c (wk < c <= 32 * R) in-order peaks at mz / it: every lane ranks its R peaks against all
// of the window's selection keys (broadcast by shuffles; ties by position), and the peaks ranked below wk are
// written in input order from out_pos.  Returns the lane's sum of the written intensities.
template <int R>
__device__ __forceinline__ double rank_window(const float* mz, const float* it, int c, int wk, int out_pos, int n_out,
                                              float* pk_mass, float* pk_int) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  uint64_t key[R];
  int rank[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int t = lane + 32 * r;
    key[r] = t < c ? win_sel_key(__fsub_rn(mz[t], VK_PROTON), it[t]) : ~0ull;
    rank[r] = 0;
  }
#pragma unroll
  for (int r2 = 0; r2 < R; ++r2) {
    if (32 * r2 >= c) break;
    for (int src = 0; src < 32; ++src) {
      const uint64_t kj = __shfl_sync(VK_FULL, key[r2], src);
      const int j = src + 32 * r2;
#pragma unroll
      for (int r = 0; r < R; ++r) rank[r] += kj < key[r] || (kj == key[r] && j < lane + 32 * r);
    }
  }
  double part = 0.0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const bool take = lane + 32 * r < c && rank[r] < wk;
    const unsigned m = __ballot_sync(VK_FULL, take);
    const int pos = out_pos + __popc(m & lt);
    if (take && pos < n_out) {
      const float v = unord_f32(~(uint32_t)(key[r] >> 32));
      pk_mass[pos] = unord_f32(~(uint32_t)key[r]);
      pk_int[pos] = v;
      part += (double)v;
    }
    out_pos += __popc(m);
  }
  return part;
}

// Warp per spectrum of code 1 or 2.  Shared memory per warp: P[n_bins + 1] (in-range peaks before each window) and
// Q[n_bins + 1] (kept peaks before each window).
__global__ void __launch_bounds__(KW_WARPS * 32)
k0w_warp_k(int n_spec, const int64_t* raw_off, const float* raw_mz, const float* raw_int, float fmin, float fmax,
           float inv, int w_lo, int n_bins, int wk, int min_peaks, const int64_t* pk_off, float* pk_mass,
           float* pk_int, float* tic, uint8_t* valid, const uint8_t* easy) {
  extern __shared__ uint32_t kw_pq[];
  const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (s >= n_spec) return;
  const int code = easy[s];
  if (code != 1 && code != 2) return;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t r0 = raw_off[s], r1 = raw_off[s + 1], o0 = pk_off[s];
  const int n_out = (int)(pk_off[s + 1] - o0);
  double part = 0.0;
  if (code == 1) {   // every in-range peak, in input order
    int w = 0;
    for (int64_t b0 = r0; b0 < r1; b0 += 32) {
      const int64_t i = b0 + lane;
      const float mz = i < r1 ? raw_mz[i] : 0.f;
      const bool take = i < r1 && in_range(mz, fmin, fmax);
      const unsigned m = __ballot_sync(VK_FULL, take);
      const int pos = w + __popc(m & lt);
      if (take && pos < n_out) {
        const float it = raw_int[i];
        pk_mass[o0 + pos] = __fsub_rn(mz, VK_PROTON);
        pk_int[o0 + pos] = it;
        part += (double)it;
      }
      w += __popc(m);
    }
  } else {
    uint32_t* P = kw_pq + (threadIdx.x >> 5) * 2 * (n_bins + 1);
    uint32_t* Q = P + n_bins + 1;
    for (int b = lane; b < n_bins; b += 32) P[b] = 0u;
    __syncwarp();
    int below = 0;   // peaks before the in-range run (m/z < fmin)
    for (int64_t i = r0 + lane; i < r1; i += 32) {
      const float mz = raw_mz[i];
      if (in_range(mz, fmin, fmax)) atomicAdd(&P[win_of(mz, inv) - w_lo], 1u);
      else below += mz < fmin;
    }
    below = (int)vk::warp_sum((long long)below);
    __syncwarp();
    uint32_t cp = 0u, cq = 0u;   // running sums over the bins
    for (int b0 = 0; b0 < n_bins; b0 += 32) {
      const int b = b0 + lane;
      const uint32_t c = b < n_bins ? P[b] : 0u, ck = min(c, (uint32_t)wk);
      const uint32_t ip = (uint32_t)vk::warp_incl_scan((long long)c);
      const uint32_t iq = (uint32_t)vk::warp_incl_scan((long long)ck);
      if (b < n_bins) {
        P[b] = cp + ip - c;
        Q[b] = cq + iq - ck;
      }
      cp += __shfl_sync(VK_FULL, ip, 31);
      cq += __shfl_sync(VK_FULL, iq, 31);
    }
    if (lane == 0) {
      P[n_bins] = cp;
      Q[n_bins] = cq;
    }
    __syncwarp();
    const int64_t r_in = r0 + below;
    const int n_in = (int)cp;
    // windows with at most wk peaks: copied to their place
    for (int t = lane; t < n_in; t += 32) {
      const float mz = raw_mz[r_in + t];
      if (!in_range(mz, fmin, fmax)) continue;   // cannot happen in code-2 order; keeps P / Q indexes in bounds
      const int b = win_of(mz, inv) - w_lo;
      const int pb = (int)P[b];
      if ((int)P[b + 1] - pb <= wk) {
        const int pos = (int)Q[b] + t - pb;
        if (pos < n_out) {
          const float it = raw_int[r_in + t];
          pk_mass[o0 + pos] = __fsub_rn(mz, VK_PROTON);
          pk_int[o0 + pos] = it;
          part += (double)it;
        }
      }
    }
    // fuller windows (at most KW_SEL peaks): rank of every peak among its window's selection keys
    for (int b = 0; b < n_bins; ++b) {
      const int pb = (int)P[b], c = (int)P[b + 1] - pb;
      if (c <= wk) continue;
      const float *wm = raw_mz + r_in + pb, *wi = raw_int + r_in + pb;
      float *om = pk_mass + o0, *oi = pk_int + o0;
      if (c <= 32) part += rank_window<1>(wm, wi, c, wk, (int)Q[b], n_out, om, oi);
      else if (c <= 64) part += rank_window<2>(wm, wi, c, wk, (int)Q[b], n_out, om, oi);
      else part += rank_window<4>(wm, wi, c, wk, (int)Q[b], n_out, om, oi);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(VK_FULL, part, o);
  if (lane == 0) {
    tic[s] = (float)part;
    valid[s] = n_out >= min_peaks;
  }
}

// Window of the sorted key at j (keys carry ord(m/z) in the high half)
__device__ __forceinline__ int key_win(uint64_t k, float inv) { return win_of(unord_f32((uint32_t)(k >> 32)), inv); }
__device__ __forceinline__ uint32_t key_mass_ord(uint64_t k) {
  return ord_f32(__fsub_rn(unord_f32((uint32_t)(k >> 32)), VK_PROTON));
}

// CTA per code-0 spectrum.  Dynamic shared memory: keys[n_pow2] (u64) then keep[n_pow2] (u8).
__global__ void __launch_bounds__(K0_THREADS)
k0w_cta_k(const int32_t* hard_list, const int32_t* n_hard, const int64_t* raw_off, const float* raw_mz,
          const float* raw_int, float fmin, float fmax, float inv, int wk, int min_peaks, const int64_t* pk_off,
          float* pk_mass, float* pk_int, float* tic, uint8_t* valid) {
  extern __shared__ uint64_t kw_keys[];
  __shared__ double red[K0_THREADS / 32];
  __shared__ int wsum[K0_THREADS / 32], n_in_sh;
  const int n_work = *n_hard;
  for (int jw = blockIdx.x; jw < n_work; jw += gridDim.x) {
    const int s = hard_list[jw];
    const int64_t r0 = raw_off[s], o0 = pk_off[s];
    const int n = (int)(raw_off[s + 1] - r0), n_out = (int)(pk_off[s + 1] - o0);
    int n_pow2 = 1;
    while (n_pow2 < n) n_pow2 <<= 1;
    uint8_t* keep = reinterpret_cast<uint8_t*>(kw_keys + n_pow2);
    if (threadIdx.x == 0) n_in_sh = 0;
    __syncthreads();
    int my_in = 0;
    for (int i = threadIdx.x; i < n_pow2; i += blockDim.x) {
      uint64_t k = ~0ull;
      if (i < n) {
        const float mz = raw_mz[r0 + i];
        if (in_range(mz, fmin, fmax)) {
          k = ((uint64_t)ord_f32(mz) << 32) | (uint64_t)(~ord_f32(raw_int[r0 + i]));
          ++my_in;
        }
      }
      kw_keys[i] = k;
    }
    if (my_in) atomicAdd(&n_in_sh, my_in);
    __syncthreads();
    block_bitonic_u64(kw_keys, n_pow2);   // in-range peaks first, by (m/z asc, intensity desc)
    const int n_in = n_in_sh;
    // keep[i]: rank of peak i among its window (selection key, then sorted position) below wk
    for (int i = threadIdx.x; i < n_in; i += blockDim.x) {
      const uint64_t ki = kw_keys[i];
      const int w = key_win(ki, inv);
      int lo = 0, hi = n_in;   // first j with window >= w
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (key_win(kw_keys[mid], inv) < w) lo = mid + 1;
        else hi = mid;
      }
      const int a = lo;
      hi = n_in;   // first j with window > w
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (key_win(kw_keys[mid], inv) <= w) lo = mid + 1;
        else hi = mid;
      }
      const int b = lo;
      bool k = true;
      if (b - a > wk) {
        const float mi = unord_f32((uint32_t)(ki >> 32));
        const uint64_t si = win_sel_key(__fsub_rn(mi, VK_PROTON), unord_f32(~(uint32_t)ki));
        int rank = 0;
        for (int j = a; j < b && rank < wk; ++j) {
          const uint64_t kj = kw_keys[j];
          const uint64_t sj = win_sel_key(__fsub_rn(unord_f32((uint32_t)(kj >> 32)), VK_PROTON),
                                          unord_f32(~(uint32_t)kj));
          rank += sj < si || (sj == si && j < i);
        }
        k = rank < wk;
      }
      keep[i] = k;
    }
    __syncthreads();
    // output positions: a scan of keep over contiguous chunks per thread
    const int per = (n_in + K0_THREADS - 1) / K0_THREADS;
    const int c0 = min(n_in, (int)threadIdx.x * per), c1 = min(n_in, c0 + per);
    int cnt = 0;
    for (int i = c0; i < c1; ++i) cnt += keep[i];
    int pos = k0_block_excl_scan(cnt, wsum);
    double part = 0.0;
    for (int i = c0; i < c1; ++i) {
      if (!keep[i]) continue;
      const uint64_t ki = kw_keys[i];
      const float mz = unord_f32((uint32_t)(ki >> 32)), it = unord_f32(~(uint32_t)ki);
      int out = pos++;
      // run of equal (mass, window) around i: the sort put it in m/z order, the reference in intensity order
      const uint32_t mo = key_mass_ord(ki);
      const int w = win_of(mz, inv);
      int sa = i, sb = i + 1;
      while (sa > 0 && key_mass_ord(kw_keys[sa - 1]) == mo && key_win(kw_keys[sa - 1], inv) == w) --sa;
      while (sb < n_in && key_mass_ord(kw_keys[sb]) == mo && key_win(kw_keys[sb], inv) == w) ++sb;
      if ((uint32_t)(kw_keys[sa] >> 32) != (uint32_t)(kw_keys[sb - 1] >> 32)) {
        int before = 0, place = 0;   // kept peaks of the run before i (sorted order) / before i (final order)
        const uint32_t ii = ~(uint32_t)ki;
        for (int j = sa; j < sb; ++j) {
          if (!keep[j]) continue;
          const uint32_t ij = ~(uint32_t)kw_keys[j];
          before += j < i;
          place += ij < ii || (ij == ii && j < i);
        }
        out = out - before + place;
      }
      if (out < n_out) {
        pk_mass[o0 + out] = __fsub_rn(mz, VK_PROTON);
        pk_int[o0 + out] = it;
        part += (double)it;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(VK_FULL, part, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int q = 0; q < K0_THREADS / 32; ++q) t += red[q];
      tic[s] = (float)t;
      valid[s] = n_out >= min_peaks;
    }
    __syncthreads();
  }
}

// Host check of the window range: inv = 1 / window_th in f32, w_lo = floor(fmin * inv), bins = windows in range.
int win_setup(float fmin, float fmax, float window_th, float* inv, int* w_lo, int* n_bins) {
  if (!(window_th > 0.f) || !isfinite(window_th) || !isfinite(fmin) || !isfinite(fmax)) return VK_E_ARG;
  *inv = 1.0f / window_th;
  const float lo = floorf(fmin * *inv), hi = floorf(fmax * *inv);
  if (fmin > fmax) {   // nothing is in range
    *w_lo = 0;
    *n_bins = 1;
    return 0;
  }
  if (!(lo >= 0.f) || !(hi <= (float)(KW_BINS - 1))) return VK_E_ARG;
  *w_lo = (int)lo;
  *n_bins = (int)hi - (int)lo + 1;
  return 0;
}

}  // namespace

extern "C" {

int vk_k0w_count(int n_spec, const int64_t* raw_off, const float* raw_mz, const float* raw_int, float fmin,
                 float fmax, float window_th, int window_k, int64_t* kept, uint8_t* easy, int32_t* hard_list,
                 int32_t* n_hard, void* stream) {
  float inv;
  int w_lo, n_bins;
  if (int e = win_setup(fmin, fmax, window_th, &inv, &w_lo, &n_bins)) return e;
  cudaError_t e = cudaMemsetAsync(n_hard, 0, sizeof(int32_t), (cudaStream_t)stream);
  if (e != cudaSuccess) return vk_err(e);
  if (n_spec == 0) return 0;
  const int64_t threads = (int64_t)n_spec * 32;
  const size_t sh = (size_t)KW_WARPS * n_bins * sizeof(uint32_t);
  k0w_count_k<<<(unsigned)((threads + KW_WARPS * 32 - 1) / (KW_WARPS * 32)), KW_WARPS * 32, sh,
                (cudaStream_t)stream>>>(n_spec, raw_off, raw_mz, raw_int, fmin, fmax, inv, w_lo, n_bins,
                                        max(window_k, 0), kept, easy, hard_list, n_hard);
  return vk_launch_status();
}

int vk_k0w_fill(int n_spec, const int64_t* raw_off, const float* raw_mz, const float* raw_int, float fmin,
                float fmax, float window_th, int window_k, int min_peaks, const int64_t* pk_off, float* pk_mass,
                float* pk_int, float* tic, uint8_t* valid, int max_raw, const uint8_t* easy,
                const int32_t* hard_list, const int32_t* n_hard, void* stream) {
  float inv;
  int w_lo, n_bins;
  if (int e = win_setup(fmin, fmax, window_th, &inv, &w_lo, &n_bins)) return e;
  if (n_spec == 0) return 0;
  if (max_raw < 0 || max_raw > 16384) return VK_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const int wk = max(window_k, 0);
  const int64_t threads = (int64_t)n_spec * 32;
  const size_t sh_w = (size_t)KW_WARPS * 2 * (n_bins + 1) * sizeof(uint32_t);
  k0w_warp_k<<<(unsigned)((threads + KW_WARPS * 32 - 1) / (KW_WARPS * 32)), KW_WARPS * 32, sh_w, st>>>(
      n_spec, raw_off, raw_mz, raw_int, fmin, fmax, inv, w_lo, n_bins, wk, min_peaks, pk_off, pk_mass, pk_int, tic,
      valid, easy);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return vk_err(e);
  int dev = 0, n_sm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  int n_pow2 = 32;
  while (n_pow2 < max_raw) n_pow2 <<= 1;
  const size_t sh = (size_t)n_pow2 * (sizeof(uint64_t) + 1);
  e = cudaFuncSetAttribute(k0w_cta_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  if (e != cudaSuccess) return vk_err(e);
  const int grid = (int)min((int64_t)n_sm * 4, (int64_t)n_spec);
  k0w_cta_k<<<grid, K0_THREADS, sh, st>>>(hard_list, n_hard, raw_off, raw_mz, raw_int, fmin, fmax, inv, wk,
                                          min_peaks, pk_off, pk_mass, pk_int, tic, valid);
  return vk_launch_status();
}

}  // extern "C"
