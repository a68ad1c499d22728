// PSM ranking per spectrum (reference vulcan/gpu/engine.py:366-392), one warp per spectrum.
//
// Candidates with matched_b + matched_y >= min_matched are ordered by (hyperscore desc, row asc); ranks 1..report
// are written with delta_next = hs - hs(next in that order, 0 if none) and delta_best = hs(rank 1) - hs.  The warp
// finds each next element with an arg-max reduction restricted to elements after the previous one in the order,
// so the cost is (report + 1) passes over the spectrum's candidates.
#include "common.cuh"

namespace {

constexpr int RK_WARPS = 4;

// (hs, row) ordered "before": higher hs, then lower row.
__device__ __forceinline__ bool before(double ha, int64_t ra, double hb, int64_t rb) {
  return ha > hb || (ha == hb && ra < rb);
}

// Spectrum s's ranking: pass k selects the k-th element of the order (k = 0..report) among the candidates with
// enough matched peaks, element k-1 is then written with its delta_next.  WARP: the 32 lanes of a warp scan the
// candidates and reduce (dense lists); otherwise one thread scans them in order (sparse lists).  Candidate rows are
// unique within a spectrum, so both find the same element.
template <bool WARP>
__device__ __forceinline__ void rank_spectrum(int s, int lane, const int64_t* cand_off, const int64_t* c_row,
                                              const double* hs, const int16_t* mb, const int16_t* my,
                                              int min_matched, int report, int64_t* psm_cand, int32_t* psm_rank,
                                              double* psm_dnext, double* psm_dbest, int32_t* n_psm) {
  const int64_t c0 = cand_off[s], c1 = cand_off[s + 1];
  double prev_h = 0.0, best_h = 0.0, cur_h = 0.0;
  int64_t prev_r = -1, cur_c = -1;
  bool have_prev = false;
  int n = 0;
  for (int k = 0; k <= report; ++k) {
    double bh = 0.0;
    int64_t br = -1, bc = -1;
    for (int64_t c = c0 + (WARP ? lane : 0); c < c1; c += (WARP ? 32 : 1)) {
      if ((int)mb[c] + (int)my[c] < min_matched) continue;
      double h = hs[c];
      int64_t r = c_row[c];
      if (have_prev && !before(prev_h, prev_r, h, r)) continue;
      if (bc < 0 || before(h, r, bh, br)) { bh = h; br = r; bc = c; }
    }
    if (WARP) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        double oh = __shfl_xor_sync(VK_FULL, bh, o);
        int64_t orr = __shfl_xor_sync(VK_FULL, br, o);
        int64_t oc = __shfl_xor_sync(VK_FULL, bc, o);
        if (oc >= 0 && (bc < 0 || before(oh, orr, bh, br))) { bh = oh; br = orr; bc = oc; }
      }
    }
    if (k > 0) {
      if (lane == 0) {
        int64_t slot = (int64_t)s * report + (k - 1);
        psm_cand[slot] = cur_c;
        psm_rank[slot] = k;
        psm_dnext[slot] = cur_h - (bc >= 0 ? bh : 0.0);
        psm_dbest[slot] = best_h - cur_h;
      }
      ++n;
    }
    if (bc < 0) break;
    if (k == 0) best_h = bh;
    cur_h = bh;
    cur_c = bc;
    prev_h = bh;
    prev_r = br;
    have_prev = true;
  }
  if (lane == 0) {
    for (int k = n; k < report; ++k) psm_cand[(int64_t)s * report + k] = -1;
    n_psm[s] = n;
  }
}

__global__ void __launch_bounds__(RK_WARPS * 32)
psm_rank_k(int n_spec, const int64_t* cand_off, const int64_t* c_row, const double* hs, const int16_t* mb,
           const int16_t* my, int min_matched, int report, int64_t* psm_cand, int32_t* psm_rank, double* psm_dnext,
           double* psm_dbest, int32_t* n_psm) {
  const int s = blockIdx.x * RK_WARPS + (threadIdx.x >> 5);
  if (s >= n_spec) return;
  rank_spectrum<true>(s, threadIdx.x & 31, cand_off, c_row, hs, mb, my, min_matched, report, psm_cand, psm_rank,
                      psm_dnext, psm_dbest, n_psm);
}

__global__ void __launch_bounds__(256)
psm_rank_seq_k(int n_spec, const int64_t* cand_off, const int64_t* c_row, const double* hs, const int16_t* mb,
               const int16_t* my, int min_matched, int report, int64_t* psm_cand, int32_t* psm_rank,
               double* psm_dnext, double* psm_dbest, int32_t* n_psm) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_spec) return;
  rank_spectrum<false>(s, 0, cand_off, c_row, hs, mb, my, min_matched, report, psm_cand, psm_rank, psm_dnext,
                       psm_dbest, n_psm);
}

// Column offsets of the packed PSM table, passed by value.
struct PackLayout {
  int64_t off[VK_PSM_COLS];
};

template <class T>
__device__ __forceinline__ void put(uint8_t* packed, const PackLayout& L, int c, int64_t j, T v) {
  reinterpret_cast<T*>(packed + L.off[c])[j] = v;
}

// One thread per PSM slot: the reference psm_table features (lnfact(0) = 1, Poisson term with +-inf -> 1e-325,
// which is 0 in f64), each operation rounded once (the library is built with -fmad=false).
__global__ void __launch_bounds__(256) pack_psms_k(vk_psm_pack_in in, int64_t slots, int report, PackLayout L,
                                                   const int64_t* row_pos, uint8_t* packed) {
  const int64_t slot = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (slot >= slots) return;
  if (row_pos && slot == 0) reinterpret_cast<int64_t*>(packed + L.off[0])[0] = row_pos[slots];
  const int64_t cand = in.psm_cand[slot];
  if (row_pos && cand < 0) return;   // compacted: filled slots only
  const int64_t j = row_pos ? row_pos[slot] : slot;   // output row
  const int64_t ci = cand < 0 ? 0 : cand;
  const int64_t s = slot / report;
  const int64_t hh = min(max(in.c_hyp[ci], (int64_t)0), in.n_hyp - 1);
  const int64_t row = min(max(in.c_row[ci], (int64_t)0), in.n_rows - 1);
  const int64_t mbk = in.mb[ci], myk = in.my[ci], kk = mbk + myk;
  const int64_t sc = in.spec_scored[s], mt = in.spec_matched[s];
  // Poisson term of the matched-peak count: lam^k e^-lam / e^lnfact(k), log10
  const double lam = (double)mt / (double)sc;
  const double x = (double)kk;
  const double lx = log(x);
  const double lnf = x == 0.0 ? 1.0 : ((x * lx - x) + 0.5 * lx) + 0.5 * log(6.283185307179586 * x);
  double pois = pow(lam, x) * exp(-lam) / exp(lnf);
  if (isinf(pois)) pois = 0.0;   // the reference's 1e-325, which is 0 in f64
  const int iso = in.h_iso[hh];
  const float pm = in.h_pm[hh];
  const float calc = in.mass32[row];
  const float ie = __fmul_rn((float)iso, 1.00335f);   // NEUTRON (an f32 value)
  const float dm = __fdiv_rn(__fmul_rn(fabsf(__fsub_rn(__fsub_rn(pm, calc), ie)), 2.0e6f),
                             __fadd_rn(__fsub_rn(pm, ie), calc));
  const float sbs = __fadd_rn(in.sb[ci], in.sy[ci]);
  const int plen = in.length[row];
  const int16_t ly = in.ly[ci];
  if (!row_pos) put<uint8_t>(packed, L, 0, j, cand >= 0 ? 1 : 0);
  put<int64_t>(packed, L, 1, j, s);
  put<int32_t>(packed, L, 2, j, in.psm_rank[slot]);
  put<int64_t>(packed, L, 3, j, row);
  put<int64_t>(packed, L, 4, j, in.pf_id[row]);
  put<int8_t>(packed, L, 5, j, in.h_z[hh]);
  put<int8_t>(packed, L, 6, j, (int8_t)iso);
  put<float>(packed, L, 7, j, pm);
  put<float>(packed, L, 8, j, calc);
  put<float>(packed, L, 9, j, dm);
  put<double>(packed, L, 10, j, in.hs[ci]);
  put<double>(packed, L, 11, j, in.dnext[slot]);
  put<double>(packed, L, 12, j, in.dbest[slot]);
  put<int16_t>(packed, L, 13, j, (int16_t)mbk);
  put<int16_t>(packed, L, 14, j, (int16_t)myk);
  put<int16_t>(packed, L, 15, j, (int16_t)kk);
  put<float>(packed, L, 16, j, sbs);
  put<float>(packed, L, 17, j, __fdiv_rn(__fmul_rn(100.0f, sbs), in.tic[s]));
  put<float>(packed, L, 18, j, in.ppm[ci]);
  put<int16_t>(packed, L, 19, j, in.lb[ci]);
  put<int16_t>(packed, L, 20, j, ly);
  put<float>(packed, L, 21, j, (float)((double)ly / (double)plen));
  put<int16_t>(packed, L, 22, j, (int16_t)plen);
  put<uint8_t>(packed, L, 23, j, in.missed[row]);
  put<uint8_t>(packed, L, 24, j, in.n_var[row]);
  put<int32_t>(packed, L, 25, j, (int32_t)in.c_cnt[ci]);
  put<int32_t>(packed, L, 26, j, (int32_t)sc);
  put<double>(packed, L, 27, j, log10(pois));
}

}  // namespace

extern "C" int vk_psm_rank(int n_spec, const int64_t* cand_off, const int64_t* c_row, const double* hs,
                           const int16_t* mb, const int16_t* my, int min_matched, int report, int64_t* psm_cand,
                           int32_t* psm_rank, double* psm_dnext, double* psm_dbest, int32_t* n_psm, void* stream) {
  if (n_spec == 0) return 0;
  if (report < 1) return VK_E_ARG;
  psm_rank_k<<<(unsigned)((n_spec + RK_WARPS - 1) / RK_WARPS), RK_WARPS * 32, 0, (cudaStream_t)stream>>>(
      n_spec, cand_off, c_row, hs, mb, my, min_matched, report, psm_cand, psm_rank, psm_dnext, psm_dbest, n_psm);
  return vk_launch_status();
}

extern "C" int vk_psm_rank_sparse(int n_spec, const int64_t* cand_off, const int64_t* c_row, const double* hs,
                                  const int16_t* mb, const int16_t* my, int min_matched, int report,
                                  int64_t* psm_cand, int32_t* psm_rank, double* psm_dnext, double* psm_dbest,
                                  int32_t* n_psm, void* stream) {
  if (n_spec == 0) return 0;
  if (report < 1) return VK_E_ARG;
  psm_rank_seq_k<<<(unsigned)((n_spec + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      n_spec, cand_off, c_row, hs, mb, my, min_matched, report, psm_cand, psm_rank, psm_dnext, psm_dbest, n_psm);
  return vk_launch_status();
}

extern "C" int vk_pack_psms(const vk_psm_pack_in* in, int64_t slots, int report, const int64_t* col_off,
                            const int64_t* row_pos, uint8_t* packed, void* stream) {
  if (!in || !col_off || !packed || report < 1 || in->n_hyp < 1 || in->n_rows < 1 || slots < 0) return VK_E_ARG;
  PackLayout L;
  for (int c = 0; c < VK_PSM_COLS; ++c) {
    if (col_off[c] < 0 || (col_off[c] & 7)) return VK_E_ARG;
    L.off[c] = col_off[c];
  }
  if (slots == 0) {   // no slots: a compacted buffer still states its (zero) rows
    if (!row_pos) return 0;
    const cudaError_t e = cudaMemsetAsync(packed + L.off[0], 0, sizeof(int64_t), (cudaStream_t)stream);
    return e == cudaSuccess ? 0 : vk_err(e);
  }
  pack_psms_k<<<(unsigned)((slots + 255) / 256), 256, 0, (cudaStream_t)stream>>>(*in, slots, report, L, row_pos,
                                                                                   packed);
  return vk_launch_status();
}
