// K0 peak view and precursor hypotheses on the device.
//
// K0 (reference vulcan/gpu/engine.py:171-210, global peak mode): peaks with fmin <= m/z <= fmax (not NaN), mass =
// m/z - PROTON in f32, the top max_peaks by (intensity desc, mass desc), then mass ascending.  Spectra whose raw
// peaks already come in that final order with at most max_peaks in range (the usual case) are copied by a warp
// with ballot compaction, no sort.  For the others one CTA sorts 64-bit keys that carry both values (no payload):
// (~ord(intensity), ~ord(mass)) for the selection and (ord(mass), ~ord(intensity)) for the final order, where
// ord() maps a float to an order-preserving u32.  Peaks with equal intensity and mass are indistinguishable, so the
// reference's remaining tie order (input position) cannot change any output.  TIC = f64 sum of the kept
// intensities (fixed-order tree), stored as f32.
//
// Hypotheses (reference vulcan/gpu/host.py:64-91): per valid spectrum with a finite precursor m/z, charges (the
// known one, else the configured range) x isotope errors in (charge, isotope) order, Sage f32 arithmetic, row
// window [lower_bound(lo), upper_bound(hi)) over the mass-sorted index masses.
#include "k0_impl.cuh"

namespace {

constexpr int K0_UNROLL = 4;   // raw-peak chunks of 32 loaded ahead per warp
constexpr int K0_WARP_SELECT = 512;   // in-order spectra up to this many raw peaks are selected by one warp

// mass-order key of a peak: ascending = mass ascending, then intensity descending
__device__ __forceinline__ uint64_t mass_key(float mz, float it) {
  return ((uint64_t)ord_f32(__fsub_rn(mz, VK_PROTON)) << 32) | (uint64_t)(~ord_f32(it));
}

// Warp per spectrum: kept = min(#in-range peaks, max_peaks); easy = the raw peaks are already in mass-key order
// (no NaN) and at most max_peaks are in range, so the peak view is the in-range subsequence as it is.  Spectra that
// are not easy are appended to hard_list (in any order: each is processed on its own).
__global__ void k0_count_k(int n_spec, const int64_t* raw_off, const float* raw_mz, const float* raw_int, float fmin,
                           float fmax, int max_peaks, int64_t* kept, uint8_t* easy, int32_t* hard_list,
                           int32_t* n_hard) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= n_spec) return;
  const int64_t r0 = raw_off[warp], r1 = raw_off[warp + 1];
  long long c = 0;
  bool sorted = true;
  uint64_t carry = 0;   // key of the previous chunk's last peak
  for (int64_t b0 = r0; b0 < r1; b0 += 32 * K0_UNROLL) {
    float mzv[K0_UNROLL], itv[K0_UNROLL];
#pragma unroll
    for (int u = 0; u < K0_UNROLL; ++u) {   // the loads first: K0_UNROLL chunks in flight per lane
      const int64_t i = b0 + 32 * u + lane;
      mzv[u] = i < r1 ? raw_mz[i] : 0.f;
      itv[u] = i < r1 ? raw_int[i] : 0.f;
    }
#pragma unroll
    for (int u = 0; u < K0_UNROLL; ++u) {
      const int64_t i = b0 + 32 * u + lane;
      uint64_t k = 0;
      if (i < r1) {
        c += in_range(mzv[u], fmin, fmax);
        sorted &= !isnan(mzv[u]);
        k = mass_key(mzv[u], itv[u]);
      }
      uint64_t prev = __shfl_up_sync(VK_FULL, k, 1);
      if (lane == 0) prev = carry;
      if (i < r1 && i > r0) sorted &= prev <= k;
      carry = __shfl_sync(VK_FULL, k, 31);
    }
  }
  c = vk::warp_sum(c);
  sorted = __all_sync(VK_FULL, sorted);
  if (lane == 0) {
    kept[warp] = min(c, (long long)max_peaks);
    // 1: in order, at most max_peaks in range (copy); 2: in order, more in range, at most K0_WARP_SELECT raw
    // peaks (warp selection); 3: the same with more raw peaks (CTA selection); 0: sort
    const int code = sorted ? (c <= max_peaks ? 1 : (r1 - r0 <= K0_WARP_SELECT ? 2 : 3)) : 0;
    easy[warp] = (uint8_t)code;
    if (code == 0 || code == 3) hard_list[atomicAdd(n_hard, 1)] = warp;
  }
}

// Warp per in-order spectrum of code 1 or 2 (codes 0 and 3 are the CTA kernel's).  Code 1 (at most max_peaks in
// range): the in-range peaks in input order (ballot compaction).  Code 2 (more in range): the kept peaks are the
// `kept` smallest selection keys (~ord(intensity), ~ord(mass)) -- an 8-bit radix select over the spectrum's peaks
// (re-read each pass, a warp-private histogram) -- taken in input order, which is the output order; keys equal to
// the threshold (equal peaks) in input order.  TIC as the f64 sum of lane partials (lane order, then a butterfly).
constexpr int KE_WARPS = 8;

__device__ __forceinline__ uint64_t k0_sel_key(float mz, float it) {
  return ((uint64_t)(~ord_f32(it)) << 32) | (uint64_t)(~ord_f32(__fsub_rn(mz, VK_PROTON)));
}

__global__ void __launch_bounds__(KE_WARPS * 32)
k0_easy_k(int n_spec, const int64_t* raw_off, const float* raw_mz, const float* raw_int, float fmin, float fmax,
          int min_peaks, const int64_t* pk_off, float* pk_mass, float* pk_int, float* tic, uint8_t* valid,
          const uint8_t* easy) {
  __shared__ uint32_t whist[KE_WARPS][256];
  const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (s >= n_spec) return;
  const int code = easy[s];
  if (code != 1 && code != 2) return;   // 0 and 3: the CTA kernel
  if (code == 2) {
    const unsigned lt = (1u << lane) - 1u;
    const int64_t r0 = raw_off[s], r1 = raw_off[s + 1], o0 = pk_off[s];
    const int kept = (int)(pk_off[s + 1] - o0);
    uint32_t* hist = whist[threadIdx.x >> 5];
    uint64_t prefix = 0ull, pmask = 0ull;
    int need = kept;   // the need-th smallest key among those matching the digits chosen so far
    for (int shift = 56; shift >= 0 && kept > 0; shift -= 8) {
      for (int q = lane; q < 256; q += 32) hist[q] = 0u;
      __syncwarp();
      for (int64_t i = r0 + lane; i < r1; i += 32) {
        const float m = raw_mz[i];
        const uint64_t k = in_range(m, fmin, fmax) ? k0_sel_key(m, raw_int[i]) : ~0ull;
        if ((k & pmask) == prefix) atomicAdd(&hist[(k >> shift) & 255], 1u);
      }
      __syncwarp();
      uint32_t c[8], tot = 0u;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        c[q] = hist[lane * 8 + q];
        tot += c[q];
      }
      const int inc = (int)vk::warp_incl_scan((long long)tot), exc = inc - (int)tot;
      const bool mine = exc < need && need <= inc;   // the lane whose digits hold the need-th key
      int d = 0, rem = 0;
      if (mine) {
        int cum = exc;
        d = lane * 8 + 7;
        for (int q = 0; q < 8; ++q) {
          if (cum + (int)c[q] >= need) {
            d = lane * 8 + q;
            break;
          }
          cum += (int)c[q];
        }
        rem = need - cum;
      }
      const unsigned who = __ballot_sync(VK_FULL, mine);
      const int src = who ? __ffs(who) - 1 : 0;
      d = __shfl_sync(VK_FULL, d, src);
      need = __shfl_sync(VK_FULL, rem, src);
      prefix |= (uint64_t)d << shift;
      pmask |= 255ull << shift;
      __syncwarp();
    }
    double part = 0.0;
    int w = 0, eq_seen = 0;
    for (int64_t i0 = r0; i0 < r1 && kept > 0; i0 += 32) {
      const int64_t i = i0 + lane;
      float m = 0.f, it = 0.f;
      uint64_t k = ~0ull;
      if (i < r1) {
        m = raw_mz[i];
        it = raw_int[i];
        if (in_range(m, fmin, fmax)) k = k0_sel_key(m, it);
      }
      const bool eq = i < r1 && k == prefix;
      const unsigned eqb = __ballot_sync(VK_FULL, eq);
      const bool take = i < r1 && (k < prefix || (eq && eq_seen + __popc(eqb & lt) < need));
      const unsigned tb = __ballot_sync(VK_FULL, take);
      const int pos = w + __popc(tb & lt);
      if (take && pos < kept) {
        pk_mass[o0 + pos] = __fsub_rn(m, VK_PROTON);
        pk_int[o0 + pos] = it;
        part += (double)it;
      }
      w += __popc(tb);
      eq_seen += __popc(eqb);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(VK_FULL, part, o);
    if (lane == 0) {
      tic[s] = (float)part;
      valid[s] = kept >= min_peaks;
    }
    return;
  }
  const unsigned lt_mask = (1u << lane) - 1u;
  const int64_t r0 = raw_off[s], r1 = raw_off[s + 1];
  const int64_t o0 = pk_off[s];
  const int n_out = (int)(pk_off[s + 1] - o0);   // the in-range count: every write stays in the slot
  double part = 0.0;
  int w = 0;
  for (int64_t b0 = r0; b0 < r1; b0 += 32 * K0_UNROLL) {
    float mzv[K0_UNROLL], itv[K0_UNROLL];
#pragma unroll
    for (int u = 0; u < K0_UNROLL; ++u) {   // the loads first: K0_UNROLL chunks in flight per lane
      const int64_t i = b0 + 32 * u + lane;
      mzv[u] = i < r1 ? raw_mz[i] : 0.f;
      itv[u] = i < r1 ? raw_int[i] : 0.f;
    }
#pragma unroll
    for (int u = 0; u < K0_UNROLL; ++u) {
      const int64_t i = b0 + 32 * u + lane;
      const bool take = i < r1 && in_range(mzv[u], fmin, fmax);
      const unsigned m = __ballot_sync(VK_FULL, take);
      const int pos = w + __popc(m & lt_mask);
      if (take && pos < n_out) {
        pk_mass[o0 + pos] = __fsub_rn(mzv[u], VK_PROTON);
        pk_int[o0 + pos] = itv[u];
        part += (double)itv[u];
      }
      w += __popc(m);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(VK_FULL, part, o);
  if (lane == 0) {
    tic[s] = (float)part;
    valid[s] = n_out >= min_peaks;
  }
}

// A spectrum whose raw peaks are in (mass asc, intensity desc) order but with more than max_peaks in range: the
// kept peaks are the `kept` smallest selection keys (~ord(intensity), ~ord(mass)), found by an 8-bit radix select in
// shared memory, and their output order is the input order, so a compaction replaces both sorts.  Keys equal to
// the threshold are taken in input order (equal keys are equal peaks).  Writes pk_mass / pk_int[o0, o0 + kept).
__device__ __forceinline__ void k0_select(uint64_t* keys, int n, int kept, const float* mz, const float* it,
                                          float fmin, float fmax, float* pk_mass, float* pk_int, int64_t o0,
                                          uint32_t* hist, int* wsum, int* bcast) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (kept <= 0) return;   // nothing kept (max_peaks 0): no selection (uniform over the CTA)
  for (int i = tid; i < n; i += K0_THREADS) {
    const float m = mz[i];
    keys[i] = in_range(m, fmin, fmax)
                  ? ((uint64_t)(~ord_f32(it[i])) << 32) | (uint64_t)(~ord_f32(__fsub_rn(m, VK_PROTON)))
                  : ~0ull;
  }
  uint64_t prefix = 0ull, pmask = 0ull;
  int need = kept;   // the need-th smallest key among those matching the digits chosen so far
  for (int shift = 56; shift >= 0; shift -= 8) {
    for (int i = tid; i < 256; i += K0_THREADS) hist[i] = 0u;
    __syncthreads();
    for (int i = tid; i < n; i += K0_THREADS) {
      const uint64_t k = keys[i];
      if ((k & pmask) == prefix) atomicAdd(&hist[(k >> shift) & 255], 1u);
    }
    __syncthreads();
    if (warp == 0) {
      uint32_t c[8], tot = 0u;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        c[q] = hist[lane * 8 + q];
        tot += c[q];
      }
      const int inc = (int)vk::warp_incl_scan((long long)tot);
      const int exc = inc - (int)tot;
      if (exc < need && need <= inc) {   // the lane whose digits hold the need-th key
        int cum = exc, d = lane * 8 + 7;
        for (int q = 0; q < 8; ++q) {
          if (cum + (int)c[q] >= need) {
            d = lane * 8 + q;
            break;
          }
          cum += (int)c[q];
        }
        bcast[0] = d;
        bcast[1] = need - cum;
      }
    }
    __syncthreads();
    prefix |= (uint64_t)bcast[0] << shift;
    pmask |= 255ull << shift;
    need = bcast[1];
    __syncthreads();
  }
  // compaction in input order: contiguous chunks per thread, keys below the threshold and the first `need` equal
  const int per = (n + K0_THREADS - 1) / K0_THREADS;
  const int a = min(n, tid * per), b = min(n, a + per);
  int eq = 0;
  for (int i = a; i < b; ++i) eq += keys[i] == prefix;
  const int eq_base = k0_block_excl_scan(eq, wsum);
  int cnt = 0, er = eq_base;
  for (int i = a; i < b; ++i) {
    const uint64_t k = keys[i];
    if (k < prefix) ++cnt;
    else if (k == prefix) cnt += er++ < need;
  }
  int pos = k0_block_excl_scan(cnt, wsum);
  er = eq_base;
  for (int i = a; i < b; ++i) {
    const uint64_t k = keys[i];
    const bool take = k < prefix || (k == prefix && er++ < need);
    if (take) {
      pk_int[o0 + pos] = unord_f32(~(uint32_t)(k >> 32));
      pk_mass[o0 + pos] = unord_f32(~(uint32_t)k);
      ++pos;
    }
  }
}

__global__ void __launch_bounds__(K0_THREADS)
k0_fill_k(const int32_t* hard_list, const int32_t* n_hard, const int64_t* raw_off, const float* raw_mz,
          const float* raw_int, float fmin, float fmax, int max_peaks, int min_peaks, const int64_t* pk_off,
          float* pk_mass, float* pk_int, float* tic, uint8_t* valid, const uint8_t* easy) {
  extern __shared__ uint64_t k0_keys[];
  __shared__ double red[K0_THREADS / 32];
  __shared__ uint32_t hist[256];
  __shared__ int wsum[K0_THREADS / 32], bcast[2];
  const int n_work = *n_hard;
  for (int j = blockIdx.x; j < n_work; j += gridDim.x) {
  const int s = hard_list[j];
  const int64_t r0 = raw_off[s];
  const int n = (int)(raw_off[s + 1] - r0);
  if (easy[s] == 3) {   // in order, too many peaks in range, a large spectrum: CTA selection
    const int64_t o0 = pk_off[s];
    const int kept = (int)(pk_off[s + 1] - o0);
    k0_select(k0_keys, n, kept, raw_mz + r0, raw_int + r0, fmin, fmax, pk_mass, pk_int, o0, hist, wsum, bcast);
    __syncthreads();   // the block's writes are visible to the TIC sum below
    double part = 0.0;
    for (int i = threadIdx.x; i < kept; i += blockDim.x) part += (double)pk_int[o0 + i];   // the sort path's order
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(VK_FULL, part, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < K0_THREADS / 32; ++w) t += red[w];
      tic[s] = (float)t;
      valid[s] = kept >= min_peaks;
    }
    __syncthreads();
    continue;
  }
  int n_pow2 = 1;
  while (n_pow2 < n) n_pow2 <<= 1;
  for (int i = threadIdx.x; i < n_pow2; i += blockDim.x) {
    uint64_t k = ~0ull;
    if (i < n) {
      float mz = raw_mz[r0 + i];
      if (in_range(mz, fmin, fmax)) {
        float mass = __fsub_rn(mz, VK_PROTON);
        k = ((uint64_t)(~ord_f32(raw_int[r0 + i])) << 32) | (uint64_t)(~ord_f32(mass));
      }
    }
    k0_keys[i] = k;
  }
  __syncthreads();
  block_bitonic_u64(k0_keys, n_pow2);   // in-range peaks first, by (intensity desc, mass desc)
  const int64_t o0 = pk_off[s];
  const int kept = (int)(pk_off[s + 1] - o0);
  int m_pow2 = 1;
  while (m_pow2 < kept) m_pow2 <<= 1;
  // re-key the kept peaks for the mass order (each thread rewrites only the elements it reads)
  for (int i = threadIdx.x; i < m_pow2; i += blockDim.x) {
    uint64_t k = ~0ull;
    if (i < kept) {
      uint64_t a = k0_keys[i];
      float it = unord_f32(~(uint32_t)(a >> 32));
      float mass = unord_f32(~(uint32_t)a);
      k = ((uint64_t)ord_f32(mass) << 32) | (uint64_t)(~ord_f32(it));
    }
    k0_keys[i] = k;
  }
  __syncthreads();
  block_bitonic_u64(k0_keys, m_pow2);
  double part = 0.0;
  for (int i = threadIdx.x; i < kept; i += blockDim.x) {
    uint64_t k = k0_keys[i];
    float mass = unord_f32((uint32_t)(k >> 32));
    float it = unord_f32(~(uint32_t)k);
    pk_mass[o0 + i] = mass;
    pk_int[o0 + i] = it;
    part += (double)it;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(VK_FULL, part, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < K0_THREADS / 32; ++w) t += red[w];
    tic[s] = (float)t;
    valid[s] = kept >= min_peaks;
  }
  __syncthreads();
  }
}

__global__ void hyp_count_k(int n_spec, const uint8_t* valid, const double* pmz, const int8_t* charge, int n_z,
                            int n_iso, int64_t* n_hyp) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_spec) return;
  bool ok = valid[s] && isfinite(pmz[s]);
  n_hyp[s] = ok ? (int64_t)(charge[s] > 0 ? 1 : n_z) * n_iso : 0;
}

__device__ __forceinline__ int64_t lower_bound_g(const float* a, int64_t n, float x) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t m = (lo + hi) >> 1;
    if (a[m] < x) lo = m + 1; else hi = m;
  }
  return lo;
}
__device__ __forceinline__ int64_t upper_bound_g(const float* a, int64_t n, float x) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t m = (lo + hi) >> 1;
    if (a[m] <= x) lo = m + 1; else hi = m;
  }
  return lo;
}

// Hypotheses of a spectrum (thread per spectrum): every column but the row window, in (charge, isotope) order.
__global__ void hyp_fill_k(int n_spec, const uint8_t* valid, const double* pmz, const int8_t* charge, int z_lo,
                           int z_hi, int iso_lo, int iso_hi, int mfc, const int64_t* hyp_off, int32_t* h_spec,
                           int8_t* h_z, int8_t* h_iso, float* h_pm, float* h_M, int8_t* h_maxfz) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_spec) return;
  if (!(valid[s] && isfinite(pmz[s]))) return;
  int64_t o = hyp_off[s];
  const int zk = charge[s];
  const int za = zk > 0 ? zk : z_lo, zb = zk > 0 ? zk : z_hi;
  const float mz = __fsub_rn(__double2float_rn(pmz[s]), VK_PROTON);
  for (int z = za; z <= zb; ++z) {
    const float pm = __fmul_rn(mz, (float)z);
    int mf = z;
    if (mfc > 0) mf = min(z, mfc + 1);
    mf = max(mf, 2);
    for (int iso = iso_lo; iso <= iso_hi; ++iso) {
      h_spec[o] = s;
      h_z[o] = (int8_t)z;
      h_iso[o] = (int8_t)iso;
      h_pm[o] = pm;
      h_M[o] = __fsub_rn(pm, __fmul_rn((float)iso, VK_NEUTRON));
      h_maxfz[o] = (int8_t)mf;
      ++o;
    }
  }
}

// Row windows: one thread per (hypothesis, bound) over the *n_hyp hypotheses, each an independent binary search
// of the index masses (all of them in flight at once instead of one after another per spectrum).
__global__ void hyp_window_k(const int64_t* n_hyp, const float* h_M, float ppm_lo, float ppm_hi,
                             const float* idx_mass32, int64_t n_rows, int64_t* h_lo, int64_t* h_hi) {
  const int64_t n2 = 2 * *n_hyp;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n2; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t h = t >> 1;
    const float M = h_M[h];
    if (t & 1) {
      const float hi = __fadd_rn(M, __fdiv_rn(__fmul_rn(M, ppm_hi), 1000000.0f));
      h_hi[h] = upper_bound_g(idx_mass32, n_rows, hi);
    } else {
      const float lo = __fadd_rn(M, __fdiv_rn(__fmul_rn(M, ppm_lo), 1000000.0f));
      h_lo[h] = lower_bound_g(idx_mass32, n_rows, lo);
    }
  }
}

}  // namespace

extern "C" {

int vk_k0_count(int n_spec, const int64_t* raw_off, const float* raw_mz, const float* raw_int, float fmin,
                float fmax, int max_peaks, int64_t* kept, uint8_t* easy, int32_t* hard_list, int32_t* n_hard,
                void* stream) {
  cudaError_t e = cudaMemsetAsync(n_hard, 0, sizeof(int32_t), (cudaStream_t)stream);
  if (e != cudaSuccess) return vk_err(e);
  if (n_spec == 0) return 0;
  int64_t threads = (int64_t)n_spec * 32;
  k0_count_k<<<(unsigned)((threads + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      n_spec, raw_off, raw_mz, raw_int, fmin, fmax, max_peaks, kept, easy, hard_list, n_hard);
  return vk_launch_status();
}

static int k0_fill_easy(int n_spec, const int64_t* raw_off, const float* raw_mz, const float* raw_int, float fmin,
                        float fmax, int min_peaks, const int64_t* pk_off, float* pk_mass, float* pk_int, float* tic,
                        uint8_t* valid, const uint8_t* easy, cudaStream_t st) {
  int64_t threads = (int64_t)n_spec * 32;
  k0_easy_k<<<(unsigned)((threads + KE_WARPS * 32 - 1) / (KE_WARPS * 32)), KE_WARPS * 32, 0, st>>>(
      n_spec, raw_off, raw_mz, raw_int, fmin, fmax, min_peaks, pk_off, pk_mass, pk_int, tic, valid, easy);
  return vk_launch_status();
}

// hard spectra (unsorted or NaN: sorted; in order with more than max_peaks in range and more than K0_WARP_SELECT raw
// peaks: selected): one CTA each, keys in shared memory
static int k0_fill_hard(int n_spec, const int64_t* raw_off, const float* raw_mz, const float* raw_int, float fmin,
                        float fmax, int max_peaks, int min_peaks, const int64_t* pk_off, float* pk_mass,
                        float* pk_int, float* tic, uint8_t* valid, int max_raw, const uint8_t* easy,
                        const int32_t* hard_list, const int32_t* n_hard, cudaStream_t st) {
  int dev = 0, n_sm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  int n_pow2 = 32;
  while (n_pow2 < max_raw) n_pow2 <<= 1;
  size_t sh = (size_t)n_pow2 * sizeof(uint64_t);
  cudaError_t e = cudaFuncSetAttribute(k0_fill_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  if (e != cudaSuccess) return vk_err(e);
  const int grid = (int)min((int64_t)n_sm * 8, (int64_t)n_spec);
  k0_fill_k<<<grid, K0_THREADS, sh, st>>>(hard_list, n_hard, raw_off, raw_mz, raw_int, fmin, fmax, max_peaks,
                                          min_peaks, pk_off, pk_mass, pk_int, tic, valid, easy);
  return vk_launch_status();
}

int vk_k0_fill(int n_spec, const int64_t* raw_off, const float* raw_mz, const float* raw_int, float fmin,
               float fmax, int max_peaks, int min_peaks, const int64_t* pk_off, float* pk_mass, float* pk_int,
               float* tic, uint8_t* valid, int max_raw, const uint8_t* easy, const int32_t* hard_list,
               const int32_t* n_hard, void* stream) {
  if (n_spec == 0) return 0;
  if (max_raw < 0 || max_raw > 16384) return VK_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const int r = k0_fill_easy(n_spec, raw_off, raw_mz, raw_int, fmin, fmax, min_peaks, pk_off, pk_mass, pk_int, tic,
                             valid, easy, st);
  if (r != 0) return r;
  return k0_fill_hard(n_spec, raw_off, raw_mz, raw_int, fmin, fmax, max_peaks, min_peaks, pk_off, pk_mass, pk_int,
                      tic, valid, max_raw, easy, hard_list, n_hard, st);
}

int vk_k0_fill_easy(int n_spec, const int64_t* raw_off, const float* raw_mz, const float* raw_int, float fmin,
                    float fmax, int max_peaks, int min_peaks, const int64_t* pk_off, float* pk_mass, float* pk_int,
                    float* tic, uint8_t* valid, int max_raw, const uint8_t* easy, const int32_t* hard_list,
                    const int32_t* n_hard, void* stream) {
  (void)max_peaks;
  (void)hard_list;
  (void)n_hard;
  if (n_spec == 0) return 0;
  if (max_raw < 0 || max_raw > 16384) return VK_E_ARG;
  return k0_fill_easy(n_spec, raw_off, raw_mz, raw_int, fmin, fmax, min_peaks, pk_off, pk_mass, pk_int, tic, valid,
                      easy, (cudaStream_t)stream);
}

int vk_k0_fill_hard(int n_spec, const int64_t* raw_off, const float* raw_mz, const float* raw_int, float fmin,
                    float fmax, int max_peaks, int min_peaks, const int64_t* pk_off, float* pk_mass, float* pk_int,
                    float* tic, uint8_t* valid, int max_raw, const uint8_t* easy, const int32_t* hard_list,
                    const int32_t* n_hard, void* stream) {
  if (n_spec == 0) return 0;
  if (max_raw < 0 || max_raw > 16384) return VK_E_ARG;
  return k0_fill_hard(n_spec, raw_off, raw_mz, raw_int, fmin, fmax, max_peaks, min_peaks, pk_off, pk_mass, pk_int,
                      tic, valid, max_raw, easy, hard_list, n_hard, (cudaStream_t)stream);
}

int vk_hyp_count(int n_spec, const uint8_t* valid, const double* precursor_mz, const int8_t* charge, int z_lo,
                 int z_hi, int iso_lo, int iso_hi, int64_t* n_hyp, void* stream) {
  if (n_spec == 0) return 0;
  if (z_hi < z_lo || iso_hi < iso_lo) return VK_E_ARG;
  hyp_count_k<<<(unsigned)((n_spec + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      n_spec, valid, precursor_mz, charge, z_hi - z_lo + 1, iso_hi - iso_lo + 1, n_hyp);
  return vk_launch_status();
}

int vk_hyp_fill(int n_spec, const uint8_t* valid, const double* precursor_mz, const int8_t* charge, int z_lo,
                int z_hi, int iso_lo, int iso_hi, float ppm_lo, float ppm_hi, int max_fragment_charge,
                const float* idx_mass32, int64_t n_rows, const int64_t* hyp_off, int32_t* h_spec, int8_t* h_z,
                int8_t* h_iso, float* h_pm, float* h_M, int64_t* h_lo, int64_t* h_hi, int8_t* h_maxfz,
                void* stream) {
  if (n_spec == 0) return 0;
  if (z_hi < z_lo || iso_hi < iso_lo) return VK_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  hyp_fill_k<<<(unsigned)((n_spec + 255) / 256), 256, 0, st>>>(n_spec, valid, precursor_mz, charge, z_lo, z_hi, iso_lo,
                                                                iso_hi, max_fragment_charge, hyp_off, h_spec, h_z,
                                                                h_iso, h_pm, h_M, h_maxfz);
  const int rc = vk_launch_status();
  if (rc != 0) return rc;
  int dev = 0, n_sm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  hyp_window_k<<<(unsigned)(n_sm * 8), 256, 0, st>>>(hyp_off + n_spec, h_M, ppm_lo, ppm_hi, idx_mass32, n_rows, h_lo,
                                                      h_hi);
  return vk_launch_status();
}

}  // extern "C"
