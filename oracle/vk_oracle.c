/* CPU oracle of the DDA search hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm load this library, and
 * only as the checker or the timed CPU baseline.  The product (vulcan-proteomics_b200/) never calls it.
 *
 * Plain C restatement of the reference's arithmetic (reference files cited per function):
 *   - fragment arithmetic                 vulcan/gpu/kernels.cu:47-51 (resmass), :61, :307 (b / y start values)
 *   - tolerance bound (ppm / Da)          vulcan/gpu/kernels.cu:36-38
 *   - index fragment count / emit keys    vulcan/gpu/kernels.cu:53-101
 *   - K1 brute-force counts               vulcan/gpu/kernels.cu:195-232
 *   - K1 per-hypothesis window counts     same semantics, faster search (sorted fragments per row)
 *   - K2 exact rescoring (+ shift mode)   vulcan/gpu/kernels.cu:240-376
 *   - K2 with FP64 accumulation           same matches, intensity sums and hyperscore in double (hyperscore oracle)
 *
 * Build: gcc -O2 -fopenmp -ffp-contract=off (no FMA contraction: every f32 operation rounds once, as the
 * reference's -fmad=false kernels and Sage's Rust code do).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
  float mono[26];
  float stat[26];
  float var[26];
  float nterm;
  int tol_da;
} or_params;

#define NTERM_BIT (1ull << 63)
#define K2_MAXPK 512
#define K2_MAXLEN 64

static inline float nterm_of(const or_params* P, uint64_t mask) { return (mask & NTERM_BIT) ? P->nterm : 0.f; }

/* kernels.cu:36-38 */
static inline float tol_bound(const or_params* P, float m, float tol) {
  if (P->tol_da) return m + tol;
  float t = m * tol;
  t = t / 1000000.0f;
  return m + t;
}

/* kernels.cu:47-51 */
static inline float resmass(const or_params* P, uint8_t r, int k, uint64_t mask) {
  int i = r - 'A';
  float d = ((mask >> k) & 1ull) ? P->var[i] : P->stat[i];
  return P->mono[i] + d;
}

static void set_threads(int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
}

/* kernels.cu:53-71 */
void or_frag_count(int64_t n, const int64_t* seq_off, const uint8_t* len, const uint64_t* mask, const float* mass32,
                   const uint8_t* res, int min_ion_index, float fmin, float fmax, int32_t* count,
                   const or_params* P) {
  for (int64_t i = 0; i < n; ++i) {
    const uint8_t* s = res + seq_off[i];
    int L = len[i];
    uint64_t mk = mask[i];
    float b = nterm_of(P, mk), y = mass32[i] - nterm_of(P, mk);
    int c = 0;
    for (int k = 0; k < L - 1; ++k) {
      float rm = resmass(P, s[k], k, mk);
      b = b + rm;
      y = y - rm;
      if (k + 1 > min_ion_index && b >= fmin && b <= fmax) ++c;
      if (L - 1 - k > min_ion_index && y >= fmin && y <= fmax) ++c;
    }
    count[i] = c;
  }
}

/* kernels.cu:73-101: int64 keys chunk<<50 | bin<<32 | local<<16 | fine, q = floor((log b - log fmin)*inv_logw*65536) */
void or_frag_emit(int64_t n, const int64_t* seq_off, const uint8_t* len, const uint64_t* mask, const float* mass32,
                  const uint8_t* res, int min_ion_index, float fmin, float fmax, double inv_logw, int chunk_size,
                  int64_t row0, const int64_t* out_off, int64_t* keys, const or_params* P) {
  double lf = log((double)fmin);
  for (int64_t i = 0; i < n; ++i) {
    const uint8_t* s = res + seq_off[i];
    int L = len[i];
    uint64_t mk = mask[i];
    float b = nterm_of(P, mk), y = mass32[i] - nterm_of(P, mk);
    int64_t g = row0 + i, chunk = g / chunk_size, local = g % chunk_size, o = out_off[i];
    for (int k = 0; k < L - 1; ++k) {
      float rm = resmass(P, s[k], k, mk);
      b = b + rm;
      y = y - rm;
      if (k + 1 > min_ion_index && b >= fmin && b <= fmax) {
        int64_t q = (int64_t)floor((log((double)b) - lf) * inv_logw * 65536.0);
        keys[o++] = (chunk << 50) | ((q >> 16) << 32) | (local << 16) | (q & 0xffff);
      }
      if (L - 1 - k > min_ion_index && y >= fmin && y <= fmax) {
        int64_t q = (int64_t)floor((log((double)y) - lf) * inv_logw * 65536.0);
        keys[o++] = (chunk << 50) | ((q >> 16) << 32) | (local << 16) | (q & 0xffff);
      }
    }
  }
}

/* Index fragments of one row (ion index > min_ion_index, fmin <= f <= fmax), in generation order. */
static int row_fragments(const or_params* P, const int64_t* seq_off, const uint8_t* len, const uint64_t* mask,
                         const float* mass32, const uint8_t* res, int64_t r, int min_ion_index, float fmin,
                         float fmax, float* out) {
  const uint8_t* s = res + seq_off[r];
  int L = len[r];
  uint64_t mk = mask[r];
  float b = nterm_of(P, mk), y = mass32[r] - nterm_of(P, mk);
  int c = 0;
  for (int k = 0; k < L - 1; ++k) {
    float rm = resmass(P, s[k], k, mk);
    b = b + rm;
    y = y - rm;
    if (k + 1 > min_ion_index && b >= fmin && b <= fmax) out[c++] = b;
    if (L - 1 - k > min_ion_index && y >= fmin && y <= fmax) out[c++] = y;
  }
  return c;
}

/* kernels.cu:195-232: count of (peak, fragment charge, index fragment) triples with a <= f <= bd. */
void or_k1_brute(int64_t n, const int32_t* c_hyp, const int32_t* c_row, const int32_t* hyp_spec,
                 const int8_t* hyp_maxfz, const int64_t* pk_off, const float* pk_mass, const int64_t* seq_off,
                 const uint8_t* len, const uint64_t* mask, const float* mass32, const uint8_t* res,
                 int min_ion_index, float fmin, float fmax, float tol_lo, float tol_hi, int32_t* out_cnt,
                 const or_params* P, int nthreads) {
  set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < n; ++i) {
    float fr[2 * K2_MAXLEN];
    int h = c_hyp[i], r = c_row[i];
    int s = hyp_spec[h], maxfz = hyp_maxfz[h];
    int64_t p0 = pk_off[s], p1 = pk_off[s + 1];
    int nf = row_fragments(P, seq_off, len, mask, mass32, res, r, min_ion_index, fmin, fmax, fr);
    int cnt = 0;
    for (int t = 0; t < nf; ++t) {
      float f = fr[t];
      for (int64_t p = p0; p < p1; ++p)
        for (int z = 1; z < maxfz; ++z) {
          float m = pk_mass[p] * (float)z;
          float a = tol_bound(P, m, tol_lo), bd = tol_bound(P, m, tol_hi);
          if (f >= a && f <= bd) ++cnt;
        }
    }
    out_cnt[i] = cnt;
  }
}

static int cmp_f32(const void* a, const void* b) {
  float x = *(const float*)a, y = *(const float*)b;
  return (x > y) - (x < y);
}

/* First index in sorted v[0,n) with v[i] >= x. */
static int lower_bound_f(const float* v, int n, float x) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int m = (lo + hi) >> 1;
    if (v[m] < x) lo = m + 1; else hi = m;
  }
  return lo;
}

/* K1 counts for every row of every hypothesis window (the exhaustive candidate set), dense layout:
 * cnt[win_off[h] + (row - lo[h])].  Same semantics as or_k1_brute; per row the index fragments are sorted and
 * each peak window [a, bd] is located by binary search.  scored[h] = #rows with count > 0, matched[h] = sum. */
void or_k1_windows(int64_t n_hyp, const int32_t* hyp_spec, const int8_t* hyp_maxfz, const int64_t* hyp_lo,
                   const int64_t* hyp_hi, const int64_t* win_off, const int64_t* pk_off, const float* pk_mass,
                   const int64_t* seq_off, const uint8_t* len, const uint64_t* mask, const float* mass32,
                   const uint8_t* res, int min_ion_index, float fmin, float fmax, float tol_lo, float tol_hi,
                   int32_t* cnt, uint32_t* scored, uint64_t* matched, const float* pk_int, const float* tic,
                   uint32_t* isum, const or_params* P, int nthreads) {
  set_threads(nthreads);
#pragma omp parallel
  {
    float fr[2 * K2_MAXLEN];
    int wcap = 0;
    float *wa = NULL, *wb = NULL;
    uint32_t* wg = NULL;
#pragma omp for schedule(dynamic, 16)
    for (int64_t h = 0; h < n_hyp; ++h) {
      int s = hyp_spec[h], maxfz = hyp_maxfz[h];
      int64_t p0 = pk_off[s], p1 = pk_off[s + 1];
      int nw = (int)((p1 - p0) * (maxfz > 1 ? maxfz - 1 : 0));
      if (nw > wcap) {
        wcap = nw * 2 + 16;
        wa = (float*)realloc(wa, sizeof(float) * wcap);
        wb = (float*)realloc(wb, sizeof(float) * wcap);
        wg = (uint32_t*)realloc(wg, sizeof(uint32_t) * wcap);
      }
      /* intensity weight of a peak: round-to-nearest-even of intensity * (2^24 / TIC) in f32 */
      float wscale = (isum && tic[s] > 0.f) ? 16777216.0f / tic[s] : 0.f;
      int w = 0;
      for (int64_t p = p0; p < p1; ++p)
        for (int z = 1; z < maxfz; ++z) {
          float m = pk_mass[p] * (float)z;
          wa[w] = tol_bound(P, m, tol_lo);
          wb[w] = tol_bound(P, m, tol_hi);
          wg[w] = isum ? (uint32_t)lrintf(pk_int[p] * wscale) : 0u;
          ++w;
        }
      uint32_t sc = 0;
      uint64_t mt = 0;
      for (int64_t r = hyp_lo[h]; r < hyp_hi[h]; ++r) {
        int nf = row_fragments(P, seq_off, len, mask, mass32, res, r, min_ion_index, fmin, fmax, fr);
        qsort(fr, nf, sizeof(float), cmp_f32);
        int c = 0;
        uint32_t is = 0;
        for (int j = 0; j < nw; ++j) {
          for (int t = lower_bound_f(fr, nf, wa[j]); t < nf && fr[t] <= wb[j]; ++t) {
            ++c;
            is += wg[j];
          }
        }
        cnt[win_off[h] + (r - hyp_lo[h])] = c;
        if (isum) isum[win_off[h] + (r - hyp_lo[h])] = is;
        if (c > 0) { ++sc; mt += (uint64_t)c; }
      }
      scored[h] = sc;
      matched[h] = mt;
    }
    free(wa);
    free(wb);
    free(wg);
  }
}

/* ------------------------------------------------------------------------------------------ K2 (f32) */
typedef struct { int start, length, last, longest; } run_t;

/* kernels.cu:252-258 */
static inline void run_matched(run_t* r, int idx) {
  if (r->last == idx) return;
  if (r->start + r->length == idx) {
    r->length += 1;
  } else {
    r->start = idx;
    r->length = 1;
  }
  if (r->length > r->longest) r->longest = r->length;
  r->last = idx;
}

/* kernels.cu:246-250: Stirling ln n!, lnfact(0) = 1 */
static inline double lnfact(int n) {
  if (n == 0) return 1.0;
  double x = (double)n;
  return x * log(x) - x + 0.5 * log(x) + 0.5 * log(2.0 * 3.141592653589793 * x);
}

/* kernels.cu:263-376.  One candidate per iteration; peaks of the spectrum truncated to the first 512. */
void or_k2(int n_spec, const int64_t* cand_off, const int32_t* c_row, const int8_t* c_maxfz, const int32_t* spec_ids,
           const int64_t* pk_off, const float* pk_mass, const float* pk_int, const int64_t* seq_off,
           const uint8_t* len, const uint64_t* mask, const float* mass32, const uint8_t* res, float tol_lo,
           float tol_hi, const float* c_shift, double* o_hs, float* o_sb, float* o_sy, float* o_ppm, int16_t* o_mb,
           int16_t* o_my, int16_t* o_lb, int16_t* o_ly, const or_params* P, int nthreads) {
  set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4)
  for (int bs = 0; bs < n_spec; ++bs) {
    int s = spec_ids[bs];
    int64_t p0 = pk_off[s];
    int np = (int)(pk_off[s + 1] - p0);
    if (np > K2_MAXPK) np = K2_MAXPK;
    const float* sm = pk_mass + p0;
    const float* si = pk_int + p0;
    for (int64_t c = cand_off[bs]; c < cand_off[bs + 1]; ++c) {
      int r = c_row[c];
      int maxfz = c_maxfz[c];
      const uint8_t* sq = res + seq_off[r];
      int L = len[r];
      uint64_t mk = mask[r];
      float sb = 0.f, sy = 0.f, ppm = 0.f;
      int mb = 0, my = 0;
      run_t rb = {0, 0, 0, 0}, ry = {0, 0, 0, 0};
      float shift = c_shift ? c_shift[c] : 0.f;
      int n_alt = (c_shift && shift != 0.f) ? 2 : 1;
      float iu[2][K2_MAXLEN], is_[2][K2_MAXLEN];
      unsigned char nu[2][K2_MAXLEN], ns[2][K2_MAXLEN];
      if (n_alt == 2) {
        memset(iu, 0, sizeof(iu));
        memset(is_, 0, sizeof(is_));
        memset(nu, 0, sizeof(nu));
        memset(ns, 0, sizeof(ns));
      }
      for (int kind = 0; kind < 2; ++kind) {
        float cum = kind == 0 ? nterm_of(P, mk) : mass32[r] - nterm_of(P, mk);
        for (int k = 0; k < L - 1; ++k) {
          float rm = resmass(P, sq[k], k, mk);
          cum = kind == 0 ? cum + rm : cum - rm;
          for (int z = 1; z < maxfz; ++z) {
            int best = -1;
            float mx = 0.f, mz = 0.f, best_mz = 0.f;
            for (int alt = 0; alt < n_alt; ++alt) {
              int best_a = -1;
              float mx_a = 0.f;
              float base = alt == 0 ? cum : cum + shift;
              mz = base / (float)z;
              float a = tol_bound(P, mz, tol_lo), bd = tol_bound(P, mz, tol_hi);
              int j = lower_bound_f(sm, np, a);
              for (; j < np && sm[j] <= bd; ++j) {
                if (si[j] >= mx) { mx = si[j]; best = j; best_mz = mz; }
                if (si[j] >= mx_a) { mx_a = si[j]; best_a = j; }
              }
              if (n_alt == 2 && best_a >= 0 && k < K2_MAXLEN) {
                if (alt == 0) { iu[kind][k] = iu[kind][k] + si[best_a]; nu[kind][k] += 1; }
                else { is_[kind][k] = is_[kind][k] + si[best_a]; ns[kind][k] += 1; }
              }
            }
            mz = best_mz;
            if (best >= 0) {
              float pmass = sm[best], pint = si[best];
              float num = (pint * fabsf(mz - pmass)) * 2.0e6f;
              ppm = ppm + num / (mz + pmass);
              if (kind == 0) { mb += 1; sb = sb + pint; run_matched(&rb, k); }
              else { my += 1; sy = sy + pint; run_matched(&ry, k); }
            }
          }
        }
      }
      if (n_alt == 2) {
        int Lk = L - 1 < K2_MAXLEN ? L - 1 : K2_MAXLEN;
        float b_u = 0.f, y_s = 0.f, b_s = 0.f, y_u = 0.f;
        int nb_u = 0, ny_s = 0, nb_s = 0, ny_u = 0;
        for (int k = 0; k < Lk; ++k) {
          b_s = b_s + is_[0][k]; nb_s += ns[0][k];
          y_u = y_u + iu[1][k]; ny_u += nu[1][k];
        }
        double best_hs = -1e300;
        for (int st = 0; st < L; ++st) {
          if (st > 0 && st - 1 < Lk) {
            int k = st - 1;
            b_u = b_u + iu[0][k]; nb_u += nu[0][k]; b_s = b_s - is_[0][k]; nb_s -= ns[0][k];
            y_s = y_s + is_[1][k]; ny_s += ns[1][k]; y_u = y_u - iu[1][k]; ny_u -= nu[1][k];
          }
          float sb2 = b_u + b_s, sy2 = y_u + y_s;
          int mb2 = nb_u + nb_s, my2 = ny_u + ny_s;
          float xb = (sb2 > 0.f ? sb2 : 0.f) + 1.0f, xy = (sy2 > 0.f ? sy2 : 0.f) + 1.0f;
          double h2 = log((double)xb * (double)xy) + lnfact(mb2) + lnfact(my2);
          if (h2 > best_hs) {
            best_hs = h2; mb = mb2; my = my2;
            sb = sb2 > 0.f ? sb2 : 0.f;
            sy = sy2 > 0.f ? sy2 : 0.f;
          }
        }
      }
      double i2 = (double)(sb + 1.0f) * (double)(sy + 1.0f);
      double hs = log(i2) + lnfact(mb) + lnfact(my);
      if (!isfinite(hs)) hs = 255.0;
      o_hs[c] = hs;
      o_sb[c] = sb;
      o_sy[c] = sy;
      o_ppm[c] = ppm / (sb + sy);
      o_mb[c] = (int16_t)mb;
      o_my[c] = (int16_t)my;
      o_lb[c] = (int16_t)rb.longest;
      o_ly[c] = (int16_t)ry.longest;
    }
  }
}

/* K2 closed mode with FP64 accumulation: the matches are decided exactly as the reference decides them (f32 ion
 * masses and tolerance bounds, most intense peak in the window, later peak on ties), then the matched intensities
 * are summed and the hyperscore evaluated in double precision.  The hyperscore oracle: it isolates the rounding of
 * the f32 accumulation from the (defined) f32 match semantics. */
void or_k2_f64(int n_spec, const int64_t* cand_off, const int32_t* c_row, const int8_t* c_maxfz,
               const int32_t* spec_ids, const int64_t* pk_off, const float* pk_mass, const float* pk_int,
               const int64_t* seq_off, const uint8_t* len, const uint64_t* mask, const float* mass32,
               const uint8_t* res, double tol_lo, double tol_hi, double* o_hs, int16_t* o_mb, int16_t* o_my,
               const or_params* P, int nthreads) {
  set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4)
  for (int bs = 0; bs < n_spec; ++bs) {
    int s = spec_ids[bs];
    int64_t p0 = pk_off[s];
    int np = (int)(pk_off[s + 1] - p0);
    if (np > K2_MAXPK) np = K2_MAXPK;
    const float* sm = pk_mass + p0;
    const float* si = pk_int + p0;
    for (int64_t c = cand_off[bs]; c < cand_off[bs + 1]; ++c) {
      int r = c_row[c], maxfz = c_maxfz[c];
      const uint8_t* sq = res + seq_off[r];
      int L = len[r];
      uint64_t mk = mask[r];
      double sb = 0.0, sy = 0.0;
      int mb = 0, my = 0;
      for (int kind = 0; kind < 2; ++kind) {
        float cum = kind == 0 ? nterm_of(P, mk) : mass32[r] - nterm_of(P, mk);
        for (int k = 0; k < L - 1; ++k) {
          float rm = resmass(P, sq[k], k, mk);
          cum = kind == 0 ? cum + rm : cum - rm;
          for (int z = 1; z < maxfz; ++z) {
            float mz = cum / (float)z;
            float a = tol_bound(P, mz, (float)tol_lo), bd = tol_bound(P, mz, (float)tol_hi);
            int best = -1;
            float mx = 0.f;
            for (int j = lower_bound_f(sm, np, a); j < np && sm[j] <= bd; ++j)
              if (si[j] >= mx) { mx = si[j]; best = j; }
            if (best >= 0) {
              if (kind == 0) { mb += 1; sb += (double)si[best]; }
              else { my += 1; sy += (double)si[best]; }
            }
          }
        }
      }
      double hs = log((sb + 1.0) * (sy + 1.0)) + lnfact(mb) + lnfact(my);
      if (!isfinite(hs)) hs = 255.0;
      o_hs[c] = hs;
      o_mb[c] = (int16_t)mb;
      o_my[c] = (int16_t)my;
    }
  }
}
