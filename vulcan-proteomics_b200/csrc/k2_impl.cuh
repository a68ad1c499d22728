// K2 exact rescoring body (Sage score_candidate semantics, reference vulcan/gpu/kernels.cu:240-376).
//
// B200 launch shape: one warp per spectrum, K2_WARPS spectra per CTA.  The warp stages its spectrum's first 512
// mass-sorted peaks in shared memory with a bucket table of start indices (one lookup + a short walk replaces the
// reference's binary search; same index found); each lane scores whole candidates (the f32 sums are sequential in
// ion order: b ions k ascending, fragment charge ascending, then y ions), so the per-candidate arithmetic is the
// reference's operation for operation and the outputs are bit-identical.
#pragma once
#include "common.cuh"

namespace vk {

constexpr int K2_WARPS = 8;

struct K2Out {
  double* hs;
  float* sb;
  float* sy;
  float* ppm;
  int16_t* mb;
  int16_t* my;
  int16_t* lb;
  int16_t* ly;
};

struct RunLen {
  int start, length, last, longest;
};

// Longest run of consecutive matched ion indices (kernels.cu:252-258)
__device__ __forceinline__ void run_matched(RunLen& r, int idx) {
  if (r.last == idx) return;
  if (r.start + r.length == idx) {
    r.length += 1;
  } else {
    r.start = idx;
    r.length = 1;
  }
  r.longest = max(r.longest, r.length);
  r.last = idx;
}

__device__ __forceinline__ int lower_bound_smem(const float* v, int n, float x) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int m = (lo + hi) >> 1;
    if (v[m] < x) lo = m + 1; else hi = m;
  }
  return lo;
}

// Bucket table of a spectrum's sorted peak masses: start[b] = first peak j with bucket(sm[j]) >= b, where
// bucket(x) = clamp((int)((x - m0) * inv_w), 0, K2_BUCKETS - 1) is monotone in x.  For a bound a with bucket b,
// every peak >= a has bucket >= b, so the first peak >= a is found by starting at start[b] and stepping while
// sm[j] < a: the same index the binary search returns, in one lookup and a short walk.
constexpr int K2_BUCKETS = 512;

struct PeakTable {
  const float* sm;
  const float* si;
  const uint16_t* start;
  int np;
  float m0, inv_w;

  __device__ __forceinline__ int bucket(float x) const {
    float t = __fmul_rn(__fsub_rn(x, m0), inv_w);
    int b = t <= 0.f ? 0 : (t >= (float)(K2_BUCKETS - 1) ? K2_BUCKETS - 1 : (int)t);
    return b;
  }
  __device__ __forceinline__ int first_ge(float a) const {
    int j = start[bucket(a)];
    while (j < np && sm[j] < a) ++j;
    return j;
  }
};

// Build the table for the warp's spectrum (peaks already in shared memory).
__device__ __forceinline__ PeakTable build_table(const float* sm, const float* si, uint16_t* start, int np, int lane) {
  PeakTable t;
  t.sm = sm;
  t.si = si;
  t.start = start;
  t.np = np;
  t.m0 = np > 0 ? sm[0] : 0.f;
  float span = np > 0 ? __fsub_rn(sm[np - 1], t.m0) : 0.f;
  t.inv_w = span > 0.f ? __fdiv_rn((float)K2_BUCKETS, span) : 0.f;
  for (int j = lane; j < np; j += 32) {
    int b = t.bucket(sm[j]);
    int bp = j > 0 ? t.bucket(sm[j - 1]) : -1;
    for (int q = bp + 1; q <= b; ++q) start[q] = (uint16_t)j;
  }
  int blast = np > 0 ? t.bucket(sm[np - 1]) : -1;
  for (int q = blast + 1 + lane; q < K2_BUCKETS; q += 32) start[q] = (uint16_t)np;
  __syncwarp();
  return t;
}

// A spectrum's mass-sorted peaks read where they lie (global memory); first_ge is the lower bound by binary search,
// the index the bucket table also finds.  For candidate-parallel scoring of sparse candidate lists.
struct GlobalPeaks {
  const float* sm;
  const float* si;
  int np;

  __device__ __forceinline__ int first_ge(float a) const {
    int lo = 0, hi = np;
    while (lo < hi) {
      const int m = (lo + hi) >> 1;
      if (__ldg(sm + m) < a) lo = m + 1; else hi = m;
    }
    return lo;
  }
};

template <bool SHIFT, class PT>
__device__ __forceinline__ void k2_score(const SmemFrag& fp, const PT& pt, int r,
                                         int maxfz, const int64_t* seq_off, const uint8_t* len,
                                         const uint64_t* mask, const float* mass32, const uint8_t* res,
                                         float tol_lo, float tol_hi, float shift, const K2Out& out, int64_t c) {
  const float* sm = pt.sm;
  const float* si = pt.si;
  const int np = pt.np;
  const uint8_t* sq = res + seq_off[r];
  int L = len[r];
  uint64_t mk = mask[r];
  float sb = 0.f, sy = 0.f, ppm = 0.f;
  int mb = 0, my = 0;
  RunLen rb = {0, 0, 0, 0}, ry = {0, 0, 0, 0};
  const int da = fp.tol_da;
  int n_alt = 1;
  // per ion kind and index: matched intensity and match count of the unshifted / shifted fragment
  float hit_u[2][SHIFT ? VK_K2_MAXLEN : 1], hit_s[2][SHIFT ? VK_K2_MAXLEN : 1];
  unsigned char cnt_u[2][SHIFT ? VK_K2_MAXLEN : 1], cnt_s[2][SHIFT ? VK_K2_MAXLEN : 1];
  if (SHIFT) {
    n_alt = shift != 0.f ? 2 : 1;
    if (n_alt == 2) {
      for (int k = 0; k < (SHIFT ? VK_K2_MAXLEN : 1); ++k) {
        hit_u[0][k] = hit_u[1][k] = hit_s[0][k] = hit_s[1][k] = 0.f;
        cnt_u[0][k] = cnt_u[1][k] = cnt_s[0][k] = cnt_s[1][k] = 0;
      }
    }
  }
  for (int kind = 0; kind < 2; ++kind) {
    float cum = kind == 0 ? nterm_of(fp, mk) : __fsub_rn(mass32[r], nterm_of(fp, mk));
    for (int k = 0; k + 1 < L; ++k) {
      float rm = resmass(fp, sq[k], k, mk);
      cum = kind == 0 ? __fadd_rn(cum, rm) : __fsub_rn(cum, rm);
      for (int z = 1; z < maxfz; ++z) {
        int best = -1;
        float mx = 0.f, best_mz = 0.f;
        for (int alt = 0; alt < n_alt; ++alt) {
          int best_a = -1;
          float mx_a = 0.f;
          float base = alt == 0 ? cum : __fadd_rn(cum, shift);
          float mz = z == 1 ? base : __fdiv_rn(base, (float)z);   // x / 1 == x exactly
          float a = tol_bound(mz, tol_lo, da), bd = tol_bound(mz, tol_hi, da);
          for (int j = pt.first_ge(a); j < np && sm[j] <= bd; ++j) {
            float it = si[j];
            if (it >= mx) { mx = it; best = j; best_mz = mz; }
            if (SHIFT && it >= mx_a) { mx_a = it; best_a = j; }
          }
          if (SHIFT && n_alt == 2 && best_a >= 0 && k < VK_K2_MAXLEN) {
            if (alt == 0) { hit_u[kind][k] = __fadd_rn(hit_u[kind][k], si[best_a]); cnt_u[kind][k] += 1; }
            else { hit_s[kind][k] = __fadd_rn(hit_s[kind][k], si[best_a]); cnt_s[kind][k] += 1; }
          }
        }
        if (best >= 0) {
          float pmass = sm[best], pint = si[best];
          float num = __fmul_rn(__fmul_rn(pint, fabsf(__fsub_rn(best_mz, pmass))), 2.0e6f);
          ppm = __fadd_rn(ppm, __fdiv_rn(num, __fadd_rn(best_mz, pmass)));
          if (kind == 0) { mb += 1; sb = __fadd_rn(sb, pint); run_matched(rb, k); }
          else { my += 1; sy = __fadd_rn(sy, pint); run_matched(ry, k); }
        }
      }
    }
  }
  if (SHIFT && n_alt == 2) {
    // best site of the delta (kernels.cu:343-363): b_k shifted iff k >= site, y_k iff k < site
    int Lk = min(L - 1, VK_K2_MAXLEN);
    float sum_bu = 0.f, sum_ys = 0.f, sum_bs = 0.f, sum_yu = 0.f;
    int n_bu = 0, n_ys = 0, n_bs = 0, n_yu = 0;
    for (int k = 0; k < Lk; ++k) {
      sum_bs = __fadd_rn(sum_bs, hit_s[0][k]); n_bs += cnt_s[0][k];
      sum_yu = __fadd_rn(sum_yu, hit_u[1][k]); n_yu += cnt_u[1][k];
    }
    double best_hs = -1e300;
    for (int site = 0; site < L; ++site) {
      if (site > 0 && site - 1 < Lk) {
        int k = site - 1;
        sum_bu = __fadd_rn(sum_bu, hit_u[0][k]); n_bu += cnt_u[0][k];
        sum_bs = __fsub_rn(sum_bs, hit_s[0][k]); n_bs -= cnt_s[0][k];
        sum_ys = __fadd_rn(sum_ys, hit_s[1][k]); n_ys += cnt_s[1][k];
        sum_yu = __fsub_rn(sum_yu, hit_u[1][k]); n_yu -= cnt_u[1][k];
      }
      float sb2 = __fadd_rn(sum_bu, sum_bs), sy2 = __fadd_rn(sum_yu, sum_ys);
      int mb2 = n_bu + n_bs, my2 = n_yu + n_ys;
      double h2 = log((double)__fadd_rn(fmaxf(sb2, 0.f), 1.0f) * (double)__fadd_rn(fmaxf(sy2, 0.f), 1.0f)) +
                  lnfact(mb2) + lnfact(my2);
      if (h2 > best_hs) { best_hs = h2; mb = mb2; my = my2; sb = fmaxf(sb2, 0.f); sy = fmaxf(sy2, 0.f); }
    }
  }
  double i2 = (double)__fadd_rn(sb, 1.0f) * (double)__fadd_rn(sy, 1.0f);
  double hs = log(i2) + lnfact(mb) + lnfact(my);
  if (!isfinite(hs)) hs = 255.0;
  out.hs[c] = hs;
  out.sb[c] = sb;
  out.sy[c] = sy;
  out.ppm[c] = __fdiv_rn(ppm, __fadd_rn(sb, sy));
  out.mb[c] = (int16_t)mb;
  out.my[c] = (int16_t)my;
  out.lb[c] = (int16_t)rb.longest;
  out.ly[c] = (int16_t)ry.longest;
}

// Warp-per-spectrum driver.  spec_ids == nullptr: spectrum bs uses peaks of spectrum bs.
template <bool SHIFT>
__device__ __forceinline__ void k2_body(const SmemFrag& fp, int n_spec, const int64_t* cand_off,
                                        const int32_t* c_row, const int8_t* c_maxfz, const int32_t* spec_ids,
                                        const int64_t* pk_off, const float* pk_mass, const float* pk_int,
                                        const int64_t* seq_off, const uint8_t* len, const uint64_t* mask,
                                        const float* mass32, const uint8_t* res, float tol_lo, float tol_hi,
                                        const float* c_shift, const K2Out& out) {
  __shared__ float s_mass[K2_WARPS][VK_K2_MAXPK];
  __shared__ float s_int[K2_WARPS][VK_K2_MAXPK];
  __shared__ uint16_t s_start[K2_WARPS][K2_BUCKETS];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int bs = blockIdx.x * K2_WARPS + warp; bs < n_spec; bs += gridDim.x * K2_WARPS) {
    int s = spec_ids ? spec_ids[bs] : bs;
    int64_t p0 = pk_off[s];
    int np = (int)min((int64_t)VK_K2_MAXPK, pk_off[s + 1] - p0);
    float* sm = s_mass[warp];
    float* si = s_int[warp];
    __syncwarp();
    for (int j = lane; j < np; j += 32) {
      sm[j] = pk_mass[p0 + j];
      si[j] = pk_int[p0 + j];
    }
    __syncwarp();
    const PeakTable pt = build_table(sm, si, s_start[warp], np, lane);
    int64_t c1 = cand_off[bs + 1];
    for (int64_t c = cand_off[bs] + lane; c < c1; c += 32) {
      float shift = SHIFT ? c_shift[c] : 0.f;
      k2_score<SHIFT, PeakTable>(fp, pt, c_row[c], c_maxfz[c], seq_off, len, mask, mass32, res, tol_lo, tol_hi,
                                 shift, out, c);
    }
  }
}

}  // namespace vk
