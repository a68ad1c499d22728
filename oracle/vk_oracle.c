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
 *   - K1 over a fragment index            vulcan/gpu/kernels.cu:112-190 (m/z-binned fragments, rows within a bin)
 *   - K0 view, global peak mode           vulcan/gpu/engine.py:171-210 (oracle.k0_view per spectrum)
 *   - top-K + pair closure over counts    vulcan/gpu/kernels.cu:170-180, engine.py:284-312 (oracle.select_topk)
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

/* ------------------------------------------------------------------------------------------ K1 over a fragment index
 * The reference's K1 (kernels.cu:112-190) searches a fragment index: every row's index fragments (row_fragments)
 * binned by m/z, each bin's entries in row order, and for a peak window the bins it touches, then the rows of the
 * hypothesis' window inside each bin.  This is that search on the host: bins of bin_w Th from fmin (bin(f) =
 * floor((f - fmin) / bin_w), monotone in f), entries (f32 mass, row) stored bin after bin, rows ascending within a
 * bin.  The counts are those of or_k1_windows (the same (peak, charge, fragment) triples with a <= f <= bd). */
static inline int64_t frag_bin(double f, double fmin, double inv_w, int64_t n_bins) {
  int64_t b = (int64_t)floor((f - fmin) * inv_w);
  return b < 0 ? 0 : (b >= n_bins ? n_bins - 1 : b);
}

/* bin_off[n_bins + 1] (entries before each bin), ent_mass / ent_row[bin_off[n_bins]] (the caller sizes them by the
 * sum of or_frag_count's counts).  Parallel over contiguous row blocks, each block's entries placed after the
 * lower blocks' in every bin, so rows stay ascending within a bin. */
void or_frag_index_build(int64_t n, const int64_t* seq_off, const uint8_t* len, const uint64_t* mask,
                         const float* mass32, const uint8_t* res, int min_ion_index, float fmin, float fmax,
                         double bin_w, int64_t n_bins, int64_t* bin_off, float* ent_mass, int32_t* ent_row,
                         const or_params* P, int nthreads) {
  set_threads(nthreads);
  int nt = 1;
#ifdef _OPENMP
  nt = omp_get_max_threads();
#endif
  const double inv_w = 1.0 / bin_w;
  int64_t* hist = (int64_t*)calloc((size_t)nt * (size_t)(n_bins + 1), sizeof(int64_t));
#pragma omp parallel num_threads(nt)
  {
    int t = 0;
#ifdef _OPENMP
    t = omp_get_thread_num();
#endif
    int64_t r0 = n * t / nt, r1 = n * (t + 1) / nt;
    int64_t* hc = hist + (size_t)t * (size_t)(n_bins + 1);
    float fr[512];   /* 2 (L - 1) fragments at most, L < 256 */
    for (int64_t r = r0; r < r1; ++r) {
      int nf = row_fragments(P, seq_off, len, mask, mass32, res, r, min_ion_index, fmin, fmax, fr);
      for (int i = 0; i < nf; ++i) ++hc[frag_bin(fr[i], fmin, inv_w, n_bins)];
    }
#pragma omp barrier
#pragma omp single
    {
      int64_t run = 0;
      for (int64_t b = 0; b < n_bins; ++b) {
        bin_off[b] = run;
        for (int u = 0; u < nt; ++u) {   /* hist becomes each block's first slot in the bin */
          int64_t c = hist[(size_t)u * (size_t)(n_bins + 1) + b];
          hist[(size_t)u * (size_t)(n_bins + 1) + b] = run;
          run += c;
        }
      }
      bin_off[n_bins] = run;
    }
    for (int64_t r = r0; r < r1; ++r) {
      int nf = row_fragments(P, seq_off, len, mask, mass32, res, r, min_ion_index, fmin, fmax, fr);
      for (int i = 0; i < nf; ++i) {
        int64_t at = hc[frag_bin(fr[i], fmin, inv_w, n_bins)]++;
        ent_mass[at] = fr[i];
        ent_row[at] = (int32_t)r;
      }
    }
  }
  free(hist);
}

/* First index in the row-sorted v[0,n) with v[i] >= x. */
static int64_t lower_bound_i32(const int32_t* v, int64_t n, int64_t x) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t m = (lo + hi) >> 1;
    if ((int64_t)v[m] < x) lo = m + 1; else hi = m;
  }
  return lo;
}

/* or_k1_windows' outputs (dense counts of every window row, scored / matched per hypothesis, optional intensity
 * sums) from the fragment index of or_frag_index_build. */
void or_k1_index(int64_t n_hyp, const int32_t* hyp_spec, const int8_t* hyp_maxfz, const int64_t* hyp_lo,
                 const int64_t* hyp_hi, const int64_t* win_off, const int64_t* pk_off, const float* pk_mass,
                 const int64_t* bin_off, const float* ent_mass, const int32_t* ent_row, float fmin, float fmax,
                 double bin_w, int64_t n_bins, float tol_lo, float tol_hi, int32_t* cnt, uint32_t* scored,
                 uint64_t* matched, const float* pk_int, const float* tic, uint32_t* isum, const or_params* P,
                 int nthreads) {
  set_threads(nthreads);
  const double inv_w = 1.0 / bin_w;
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t h = 0; h < n_hyp; ++h) {
    const int s = hyp_spec[h], maxfz = hyp_maxfz[h];
    const int64_t lo = hyp_lo[h], hi = hyp_hi[h], w0 = win_off[h];
    if (hi <= lo) {
      scored[h] = 0;
      matched[h] = 0;
      continue;
    }
    int32_t* c = cnt + w0;
    uint32_t* is = isum ? isum + w0 : NULL;
    memset(c, 0, sizeof(int32_t) * (size_t)(hi - lo));
    if (is) memset(is, 0, sizeof(uint32_t) * (size_t)(hi - lo));
    const float wscale = (isum && tic[s] > 0.f) ? 16777216.0f / tic[s] : 0.f;
    for (int64_t p = pk_off[s]; p < pk_off[s + 1]; ++p) {
      const uint32_t wg = isum ? (uint32_t)lrintf(pk_int[p] * wscale) : 0u;
      for (int z = 1; z < maxfz; ++z) {
        const float m = pk_mass[p] * (float)z;
        const float a = tol_bound(P, m, tol_lo), bd = tol_bound(P, m, tol_hi);
        if (!(bd >= fmin && a <= fmax)) continue;   /* every index fragment lies in [fmin, fmax] */
        const int64_t ba = frag_bin(a < fmin ? fmin : a, fmin, inv_w, n_bins);
        const int64_t bb = frag_bin(bd > fmax ? fmax : bd, fmin, inv_w, n_bins);
        for (int64_t b = ba; b <= bb; ++b) {
          const int64_t e0 = bin_off[b], e1 = bin_off[b + 1];
          for (int64_t e = e0 + lower_bound_i32(ent_row + e0, e1 - e0, lo); e < e1 && ent_row[e] < hi; ++e) {
            const float f = ent_mass[e];
            if (f >= a && f <= bd) {
              ++c[ent_row[e] - lo];
              if (is) is[ent_row[e] - lo] += wg;
            }
          }
        }
      }
    }
    uint32_t sc = 0;
    uint64_t mt = 0;
    for (int64_t r = 0; r < hi - lo; ++r)
      if (c[r] > 0) {
        ++sc;
        mt += (uint64_t)c[r];
      }
    scored[h] = sc;
    matched[h] = mt;
  }
}

/* ------------------------------------------------------------------------------------------ K0 view (global mode)
 * oracle.k0_view (engine.py:171-210) per spectrum: the peaks with fmin <= mz <= fmax (not NaN), mass = mz - PROTON
 * in f32, the top max_peaks by (intensity desc, mass desc, input order) -- NaN intensities after all others, as a
 * descending lexsort puts them -- then mass ascending (ties in that ranking order); TIC = the f64 sum of the kept
 * intensities in output order, as f32; valid = kept >= min_peaks.  out_off[n + 1] gets the offsets; out_mass /
 * out_int hold at most raw_off[n] peaks. */
typedef struct { float mass, it; int64_t idx; int32_t rank; } k0_peak;

static int k0_rank_cmp(const void* pa, const void* pb) {
  const k0_peak* a = (const k0_peak*)pa;
  const k0_peak* b = (const k0_peak*)pb;
  const int na = isnan(a->it), nb = isnan(b->it);
  if (na != nb) return na - nb;                      /* NaN intensities last */
  if (!na && a->it != b->it) return a->it > b->it ? -1 : 1;
  if (a->mass != b->mass) return a->mass > b->mass ? -1 : 1;
  return (a->idx > b->idx) - (a->idx < b->idx);
}

static int k0_mass_cmp(const void* pa, const void* pb) {
  const k0_peak* a = (const k0_peak*)pa;
  const k0_peak* b = (const k0_peak*)pb;
  if (a->mass != b->mass) return a->mass < b->mass ? -1 : 1;
  return (a->rank > b->rank) - (a->rank < b->rank);
}

void or_k0_global(int64_t n, const int64_t* raw_off, const float* raw_mz, const float* raw_int, float fmin,
                  float fmax, int max_peaks, int min_peaks, int64_t* out_off, float* out_mass, float* out_int,
                  float* tic, uint8_t* valid, int nthreads) {
  set_threads(nthreads);
  int32_t* kept = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
#pragma omp parallel
  {
    k0_peak* buf = NULL;
    int64_t cap = 0;
#pragma omp for schedule(dynamic, 64)
    for (int64_t s = 0; s < n; ++s) {
      int64_t c = 0;
      for (int64_t i = raw_off[s]; i < raw_off[s + 1]; ++i)
        if (raw_mz[i] >= fmin && raw_mz[i] <= fmax) ++c;   /* false for NaN */
      kept[s] = (int32_t)(c < max_peaks ? c : max_peaks);
    }
    /* offsets (one thread), then every spectrum's selection into its slot */
#pragma omp single
    {
      out_off[0] = 0;
      for (int64_t s = 0; s < n; ++s) out_off[s + 1] = out_off[s] + kept[s];
    }
#pragma omp for schedule(dynamic, 64)
    for (int64_t s = 0; s < n; ++s) {
      const int64_t r0 = raw_off[s], r1 = raw_off[s + 1];
      if (r1 - r0 > cap) {
        cap = (r1 - r0) * 2 + 16;
        buf = (k0_peak*)realloc(buf, sizeof(k0_peak) * (size_t)cap);
      }
      int64_t m = 0;
      for (int64_t i = r0; i < r1; ++i)
        if (raw_mz[i] >= fmin && raw_mz[i] <= fmax) {
          buf[m].mass = raw_mz[i] - 1.0072764f;
          buf[m].it = raw_int[i];
          buf[m].idx = i;
          ++m;
        }
      qsort(buf, (size_t)m, sizeof(k0_peak), k0_rank_cmp);
      const int64_t k = kept[s];
      for (int64_t j = 0; j < k; ++j) buf[j].rank = (int32_t)j;
      qsort(buf, (size_t)k, sizeof(k0_peak), k0_mass_cmp);
      double t = 0.0;
      const int64_t o = out_off[s];
      for (int64_t j = 0; j < k; ++j) {
        out_mass[o + j] = buf[j].mass;
        out_int[o + j] = buf[j].it;
        t += (double)buf[j].it;
      }
      tic[s] = (float)t;
      valid[s] = k >= min_peaks;
    }
    free(buf);
  }
  free(kept);
}

/* ------------------------------------------------------------------------------------------ top-K over window counts
 * oracle.k1_appended + oracle.select_topk (kernels.cu:170-180, engine.py:284-312) per spectrum: the window rows of
 * its hypotheses [spec_hyp_off[s], spec_hyp_off[s+1]) with count >= thr, the topk by (min(count, 32767) desc, row
 * desc, hypothesis asc), with pair closure the partner rows (same hypothesis, count -1), then one entry per row:
 * the lowest hypothesis and the highest count, rows ascending.  Spectrum s's list goes to slots [s * cap, ...),
 * its length to o_n[s] (cap >= topk, 2 topk with closure). */
typedef struct { int64_t h, r, c; } tk_ent;

static int tk_rank_cmp(const void* pa, const void* pb) {
  const tk_ent* a = (const tk_ent*)pa;
  const tk_ent* b = (const tk_ent*)pb;
  const int64_t ca = a->c < 32767 ? a->c : 32767, cb = b->c < 32767 ? b->c : 32767;
  if (ca != cb) return ca > cb ? -1 : 1;
  if (a->r != b->r) return a->r > b->r ? -1 : 1;
  return (a->h > b->h) - (a->h < b->h);
}

static int tk_row_cmp(const void* pa, const void* pb) {
  const tk_ent* a = (const tk_ent*)pa;
  const tk_ent* b = (const tk_ent*)pb;
  if (a->r != b->r) return a->r < b->r ? -1 : 1;
  return (a->h > b->h) - (a->h < b->h);
}

void or_topk_windows(int64_t n_spec, const int64_t* spec_hyp_off, const int64_t* hyp_lo, const int64_t* hyp_hi,
                     const int64_t* win_off, const int32_t* cnt, int thr, int topk, int closure,
                     const int64_t* partner, int cap, int64_t* o_h, int64_t* o_r, int64_t* o_c, int32_t* o_n,
                     int nthreads) {
  set_threads(nthreads);
#pragma omp parallel
  {
    tk_ent* buf = NULL;
    int64_t bcap = 0;
#pragma omp for schedule(dynamic, 64)
    for (int64_t s = 0; s < n_spec; ++s) {
      int64_t m = 0;
      for (int64_t h = spec_hyp_off[s]; h < spec_hyp_off[s + 1]; ++h) {
        const int64_t nw = hyp_hi[h] - hyp_lo[h];
        if (m + nw + 2 * (int64_t)topk > bcap) {
          bcap = (m + nw + 2 * (int64_t)topk) * 2 + 64;
          buf = (tk_ent*)realloc(buf, sizeof(tk_ent) * (size_t)bcap);
        }
        for (int64_t j = 0; j < nw; ++j) {
          const int32_t c = cnt[win_off[h] + j];
          if (c >= thr) {
            buf[m].h = h;
            buf[m].r = hyp_lo[h] + j;
            buf[m].c = c;
            ++m;
          }
        }
      }
      if (m + 2 * (int64_t)topk > bcap) {
        bcap = (m + 2 * (int64_t)topk) * 2 + 64;
        buf = (tk_ent*)realloc(buf, sizeof(tk_ent) * (size_t)bcap);
      }
      qsort(buf, (size_t)m, sizeof(tk_ent), tk_rank_cmp);
      int64_t k = m < topk ? m : topk;
      if (closure) {
        for (int64_t j = 0; j < k; ++j) {
          buf[k + j].h = buf[j].h;
          buf[k + j].r = partner[buf[j].r];
          buf[k + j].c = -1;
        }
        k *= 2;
      }
      qsort(buf, (size_t)k, sizeof(tk_ent), tk_row_cmp);
      int32_t w = 0;
      int64_t* oh = o_h + s * (int64_t)cap;
      int64_t* orr = o_r + s * (int64_t)cap;
      int64_t* oc = o_c + s * (int64_t)cap;
      for (int64_t j = 0; j < k; ++j) {
        if (w > 0 && orr[w - 1] == buf[j].r) {   /* same row: the lowest hypothesis came first; highest count */
          if (buf[j].c > oc[w - 1]) oc[w - 1] = buf[j].c;
          continue;
        }
        oh[w] = buf[j].h;
        orr[w] = buf[j].r;
        oc[w] = buf[j].c;
        ++w;
      }
      o_n[s] = w;
    }
    free(buf);
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
