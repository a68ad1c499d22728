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

__global__ void __launch_bounds__(RK_WARPS * 32)
psm_rank_k(int n_spec, const int64_t* cand_off, const int64_t* c_row, const double* hs, const int16_t* mb,
           const int16_t* my, int min_matched, int report, int64_t* psm_cand, int32_t* psm_rank, double* psm_dnext,
           double* psm_dbest, int32_t* n_psm) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int s = blockIdx.x * RK_WARPS + warp;
  if (s >= n_spec) return;
  const int64_t c0 = cand_off[s], c1 = cand_off[s + 1];
  double prev_h = 0.0, best_h = 0.0, cur_h = 0.0;
  int64_t prev_r = -1, cur_c = -1;
  bool have_prev = false;
  int n = 0;
  // pass k selects the k-th element of the order (k = 0..report); element k-1 is then written with its delta_next
  for (int k = 0; k <= report; ++k) {
    double bh = 0.0;
    int64_t br = -1, bc = -1;
    for (int64_t c = c0 + lane; c < c1; c += 32) {
      if ((int)mb[c] + (int)my[c] < min_matched) continue;
      double h = hs[c];
      int64_t r = c_row[c];
      if (have_prev && !before(prev_h, prev_r, h, r)) continue;
      if (bc < 0 || before(h, r, bh, br)) { bh = h; br = r; bc = c; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double oh = __shfl_xor_sync(VK_FULL, bh, o);
      int64_t orr = __shfl_xor_sync(VK_FULL, br, o);
      int64_t oc = __shfl_xor_sync(VK_FULL, bc, o);
      if (oc >= 0 && (bc < 0 || before(oh, orr, bh, br))) { bh = oh; br = orr; bc = oc; }
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
