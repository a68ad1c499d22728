// Host-side native core of the L1 index build: peptidoform expansion of target/decoy pairs.
//
// The reference does this in Rust (vulcan/rust/vulcan_core/src/lib.rs:271-399, `expand_pairs`): for every forward
// peptide, every set of variable-modification sites of size <= max_var is one peptidoform; the decoy side gets the
// same modifications carried through the pair's permutation; forms whose f64 mass is outside [min_mass, max_mass]
// are dropped; ids are xxh64(canonical string, id_seed) and masses are Sage's f32 sums.  This file restates that
// contract in C++ (plain C ABI, called through ctypes) and adds site limits on top of the global max_var: residue
// type r belongs to site group group_res[r], and a form may carry at most limit_group[g] sites of group g (255 = no
// own limit); e.g. S, T and Y in one group capped at 3 phospho sites, M in its own group capped at 1.
//
// xxh64 follows the published XXH64 specification (Yann Collet, xxHash); the tests compare it with the Python
// `xxhash` package.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr uint64_t P1 = 0x9E3779B185EBCA87ull, P2 = 0xC2B2AE3D27D4EB4Full, P3 = 0x165667B19E3779F9ull,
                   P4 = 0x85EBCA77C2B2AE63ull, P5 = 0x27D4EB2F165667C5ull;
constexpr uint64_t NTERM_BIT = 1ull << 63;

inline uint64_t rotl(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }
inline uint64_t rd64(const uint8_t* p) { uint64_t v; std::memcpy(&v, p, 8); return v; }
inline uint32_t rd32(const uint8_t* p) { uint32_t v; std::memcpy(&v, p, 4); return v; }
inline uint64_t round1(uint64_t acc, uint64_t lane) { acc += lane * P2; acc = rotl(acc, 31); return acc * P1; }
inline uint64_t merge(uint64_t acc, uint64_t v) { acc ^= round1(0, v); return acc * P1 + P4; }

uint64_t xxh64(const uint8_t* p, size_t n, uint64_t seed) {
  const uint8_t* end = p + n;
  uint64_t h;
  if (n >= 32) {
    uint64_t v1 = seed + P1 + P2, v2 = seed + P2, v3 = seed, v4 = seed - P1;
    const uint8_t* lim = end - 32;
    do {
      v1 = round1(v1, rd64(p)); v2 = round1(v2, rd64(p + 8));
      v3 = round1(v3, rd64(p + 16)); v4 = round1(v4, rd64(p + 24));
      p += 32;
    } while (p <= lim);
    h = rotl(v1, 1) + rotl(v2, 7) + rotl(v3, 12) + rotl(v4, 18);
    h = merge(h, v1); h = merge(h, v2); h = merge(h, v3); h = merge(h, v4);
  } else {
    h = seed + P5;
  }
  h += (uint64_t)n;
  while (p + 8 <= end) { h ^= round1(0, rd64(p)); h = rotl(h, 27) * P1 + P4; p += 8; }
  if (p + 4 <= end) { h ^= (uint64_t)rd32(p) * P1; h = rotl(h, 23) * P2 + P3; p += 4; }
  while (p < end) { h ^= (uint64_t)(*p) * P5; h = rotl(h, 11) * P1; ++p; }
  h ^= h >> 33; h *= P2; h ^= h >> 29; h *= P3; h ^= h >> 32;
  return h;
}

struct Cfg {
  const float* mono;        // 26 Sage f32 residue masses
  const double* res_f64;    // 26 Unimod f64 residue masses (mass filter)
  const double* stat;       // 26 static deltas (f64)
  const double* var;        // 26 variable deltas (f64), 0 = none
  double nterm;             // variable peptide-N-term delta, 0 = none
  float h2o32;
  double h2o64;
  int max_var;
  const uint8_t* group_res;   // 26: site group of each residue type
  const uint8_t* limit_group; // 26: site limit of each group (255 = none)
  char tag[26][24];         // "[+15.9949]" per residue
  char ntag[24];
};

void canonical(const Cfg& c, const uint8_t* s, int n, uint64_t mask, std::string& out) {
  out.clear();
  if (mask & NTERM_BIT) { out += c.ntag; out += '-'; }
  for (int k = 0; k < n; ++k) {
    out += (char)s[k];
    if ((mask >> k) & 1ull) out += c.tag[s[k] - 'A'];
  }
}

float mass32(const Cfg& c, const uint8_t* s, int n, uint64_t mask) {
  float m = c.h2o32;
  for (int k = 0; k < n; ++k) m = m + c.mono[s[k] - 'A'];
  float ms = 0.f;
  for (int k = 0; k < n; ++k) {
    int i = s[k] - 'A';
    float d = ((mask >> k) & 1ull) ? (float)c.var[i] : (float)c.stat[i];
    ms = ms + d;
  }
  if (mask & NTERM_BIT) ms = ms + (float)c.nterm;
  return m + ms;
}

double mass64(const Cfg& c, const uint8_t* s, int n, uint64_t mask) {
  double m = c.h2o64;
  for (int k = 0; k < n; ++k) {
    int i = s[k] - 'A';
    m += c.res_f64[i] + c.stat[i];
    if ((mask >> k) & 1ull) m += c.var[i];
  }
  if (mask & NTERM_BIT) m += c.nterm;
  return m;
}

// All site subsets of size <= max_var (respecting per-residue limits), as masks; sites sorted ascending, the
// N-term pseudo-site (bit 63) last.  Order: by size, then lexicographic (itertools.combinations order).
void forms_of(const Cfg& c, const uint8_t* s, int n, std::vector<uint64_t>& out) {
  out.clear();
  int sites[66];
  int ns = 0;
  for (int k = 0; k < n; ++k)
    if (c.var[s[k] - 'A'] != 0.0) sites[ns++] = k;
  if (c.nterm != 0.0) sites[ns++] = 63;
  int mv = c.max_var < ns ? c.max_var : ns;
  int idx[66];
  for (int r = 0; r <= mv; ++r) {
    for (int i = 0; i < r; ++i) idx[i] = i;
    while (true) {
      uint64_t m = 0;
      int per[26] = {0};
      bool ok = true;
      for (int i = 0; i < r; ++i) {
        int k = sites[idx[i]];
        m |= 1ull << k;
        if (k != 63) {
          int g = c.group_res[s[k] - 'A'];
          if (++per[g] > c.limit_group[g]) ok = false;
        }
      }
      if (ok) out.push_back(m);
      int i = r - 1;
      while (i >= 0 && idx[i] == ns - r + i) --i;
      if (i < 0) break;
      ++idx[i];
      for (int j = i + 1; j < r; ++j) idx[j] = idx[j - 1] + 1;
    }
  }
}

}  // namespace

extern "C" {

uint64_t vc_xxh64(const uint8_t* p, int64_t n, uint64_t seed) { return xxh64(p, (size_t)n, seed); }

// Expand pairs.  fwd/dec residues concatenated with offsets seq_off[n+1]; perm_flat/perm_off as in the reference
// (empty slice = pseudo-reverse).  Two calls: out arrays NULL -> returns the number of kept forms; otherwise fills
// them (capacity = that number) and returns it again.  Negative return: bad input (index of the pair, -1 - i).
int64_t vc_expand_pairs(int64_t n_pairs, const uint8_t* fwd, const uint8_t* dec, const int64_t* seq_off,
                        const uint8_t* perm_flat, const int64_t* perm_off, const float* mono, const double* res_f64,
                        const double* stat, const double* var, double nterm, int max_var, const uint8_t* group_res,
                        const uint8_t* limit_group,
                        double min_mass, double max_mass, uint64_t id_seed, int nthreads,
                        uint32_t* o_seq, uint64_t* o_mask_f, uint64_t* o_mask_d, double* o_mass, uint8_t* o_nvar,
                        uint64_t* o_id_f, uint64_t* o_id_d, float* o_m32f, float* o_m32d) {
  Cfg c;
  c.mono = mono; c.res_f64 = res_f64; c.stat = stat; c.var = var; c.nterm = nterm;
  c.h2o32 = 18.010565f; c.h2o64 = 18.010564684; c.max_var = max_var; c.group_res = group_res;
  c.limit_group = limit_group;
  for (int i = 0; i < 26; ++i) std::snprintf(c.tag[i], sizeof(c.tag[i]), "[%+.4f]", var[i]);
  std::snprintf(c.ntag, sizeof(c.ntag), "[%+.4f]", nterm);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  // pass 1: kept forms per pair
  std::vector<int64_t> cnt(n_pairs + 1, 0);
  int64_t bad = -1;
#pragma omp parallel
  {
    std::vector<uint64_t> forms;
#pragma omp for schedule(dynamic, 1024)
    for (int64_t i = 0; i < n_pairs; ++i) {
      const uint8_t* f = fwd + seq_off[i];
      int n = (int)(seq_off[i + 1] - seq_off[i]);
      if (n > 62 || n < 2) { bad = i; continue; }
      forms_of(c, f, n, forms);
      int64_t k = 0;
      for (uint64_t m : forms) {
        double ms = mass64(c, f, n, m);
        if (ms >= min_mass && ms <= max_mass) ++k;
      }
      cnt[i + 1] = k;
    }
  }
  if (bad >= 0) return -1 - bad;
  for (int64_t i = 0; i < n_pairs; ++i) cnt[i + 1] += cnt[i];
  int64_t total = cnt[n_pairs];
  if (!o_seq) return total;
#pragma omp parallel
  {
    std::vector<uint64_t> forms;
    std::string cs;
    int perm[64];
#pragma omp for schedule(dynamic, 1024)
    for (int64_t i = 0; i < n_pairs; ++i) {
      const uint8_t* f = fwd + seq_off[i];
      const uint8_t* d = dec + seq_off[i];
      int n = (int)(seq_off[i + 1] - seq_off[i]);
      int64_t a = perm_off[i], b = perm_off[i + 1];
      for (int j = 0; j < n; ++j) perm[j] = (a == b) ? (j + 1 < n ? n - 2 - j : n - 1) : (int)perm_flat[a + j];
      forms_of(c, f, n, forms);
      int64_t o = cnt[i];
      for (uint64_t m : forms) {
        double ms = mass64(c, f, n, m);
        if (!(ms >= min_mass && ms <= max_mass)) continue;
        uint64_t md = m & NTERM_BIT;
        for (int j = 0; j < n; ++j)
          if ((m >> perm[j]) & 1ull) md |= 1ull << j;
        o_seq[o] = (uint32_t)i;
        o_mask_f[o] = m;
        o_mask_d[o] = md;
        o_mass[o] = ms;
        o_nvar[o] = (uint8_t)__builtin_popcountll(m);
        canonical(c, f, n, m, cs);
        o_id_f[o] = xxh64((const uint8_t*)cs.data(), cs.size(), id_seed);
        canonical(c, d, n, md, cs);
        o_id_d[o] = xxh64((const uint8_t*)cs.data(), cs.size(), id_seed);
        o_m32f[o] = mass32(c, f, n, m);
        o_m32d[o] = mass32(c, d, n, md);
        ++o;
      }
    }
  }
  return total;
}

}  // extern "C"
