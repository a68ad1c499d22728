// Training GEMMs of the candidate pruner on the 5th-generation tensor cores (tcgen05, FP32 accumulation in TMEM).
//
// C[m, n] = sum_k A(m, k) B(k, n) (+ bias[n]) (ReLU) (rounded to BF16 values), with A(m, k) = A[m*sam + k*sak]
// (FP32) and B(k, n) = B[k*sbk + n*sbn] (BF16, or FP32); strides make every transpose of the backward pass free.
// Both operands are rounded to BF16 (round to nearest) as they are staged into shared memory -- the weights, the
// features and the BF16-rounded layer-1 activations are BF16 values already, so only the backward gradients lose
// bits -- and the products are summed in FP32 by the tensor core (an order of its own: not the fixed order of the
// SIMT kernel in mlp_train.cu, which stays the bit-exact reference of the oracle test).
//
// CTA: 128 threads, tile 128 (M) x Nt (N <= 256, a multiple of 16), K in chunks of 64 staged into the canonical
// K-major layout (tc_common.cuh) by all threads (coalesced along whichever of m / k, n / k is contiguous), then
// four UMMAs (K 16 each) by one thread, committed to an mbarrier that every thread waits on before the next chunk
// overwrites the operands.  Weight gradients reduce over the batch (K = batch rows): the K range is split over
// blockIdx.z, each split writes its partial tile to a workspace, and tc_gemm_reduce_k sums the splits in split
// order (deterministic) and applies bias / ReLU / rounding.  Waits are bounded: on a timeout the CTA records
// VK_STATUS_WAIT_TIMEOUT, stops issuing, waits (bounded) for its last commit and frees its TMEM.
#include <cuda_bf16.h>

#include "common.cuh"
#include "tc_common.cuh"

namespace {

constexpr int TG_M = 128;
constexpr int TG_NMAX = 256;
constexpr int TG_KC = 64;
constexpr int TG_THREADS = 128;
constexpr uint32_t TG_WAIT = 1u << 24;
constexpr int TG_SMEM_A = TG_M * TG_KC * 2;        // 16 KB
constexpr int TG_SMEM_B = TG_NMAX * TG_KC * 2;     // 32 KB
// requested dynamic shared memory: the operands, padded so that at most two CTAs share an SM (2 x 256 TMEM columns)
constexpr int TG_SMEM = 96 * 1024;
static_assert(TG_SMEM_A + TG_SMEM_B + 128 <= TG_SMEM, "operand tiles and alignment slack fit");

template <typename T>
__device__ __forceinline__ float ld_f(const T* p, int64_t i);
template <>
__device__ __forceinline__ float ld_f<float>(const float* p, int64_t i) { return p[i]; }
template <>
__device__ __forceinline__ float ld_f<__nv_bfloat16>(const __nv_bfloat16* p, int64_t i) { return __bfloat162float(p[i]); }

// rows r0.. (R of them) x K chunk [k0, k0 + TG_KC) of X(r, k) = X[r*sr + k*sk] into the canonical layout at dst
template <typename T>
__device__ __forceinline__ void stage(uint8_t* dst, const T* X, int64_t sr, int64_t sk, int r0, int R, int nr,
                                      int k0, int K) {
  const bool k_fast = sk == 1;
  for (int idx = threadIdx.x; idx < R * TG_KC; idx += TG_THREADS) {
    const int r = k_fast ? idx / TG_KC : idx % R;
    const int k = k_fast ? idx % TG_KC : idx / R;
    const int gr = r0 + r, gk = k0 + k;
    const float v = (gr < nr && gk < K) ? ld_f<T>(X, (int64_t)gr * sr + (int64_t)gk * sk) : 0.f;
    *reinterpret_cast<__nv_bfloat16*>(dst + canon_off(r, k, TG_KC)) = __float2bfloat16_rn(v);
  }
}

__device__ __forceinline__ float tg_out(float v, const float* bias, int n, int relu, int round_bf16) {
  if (bias) v = __fadd_rn(v, bias[n]);
  if (relu) v = fmaxf(v, 0.f);
  if (round_bf16) v = __bfloat162float(__float2bfloat16_rn(v));
  return v;
}

template <typename TB>
__global__ void __launch_bounds__(TG_THREADS)
tc_gemm_k(int M, int N, int K, int k_split, const float* __restrict__ A, int64_t sam, int64_t sak,
          const TB* __restrict__ B, int64_t sbk, int64_t sbn, const float* __restrict__ bias, int relu,
          int round_bf16, float* __restrict__ C, int64_t scm, int64_t scn, float* __restrict__ ws,
          int32_t* status) {
  extern __shared__ uint8_t tg_raw[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(tg_raw) + 127) & ~uintptr_t(127));
  uint8_t* sA = sm;
  uint8_t* sB = sm + TG_SMEM_A;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * TG_M;
  const int n0 = blockIdx.y * TG_NMAX;
  const int Nt = min(TG_NMAX, N - n0);            // a multiple of 16
  const int kb = blockIdx.z * k_split, ke = min(K, kb + k_split);
  if (tid == 0) {
    abort_flag = 0;
    vk::mbar_init(&bar, 1);
    vk::fence_mbar_init();
  }
  if (warp == 0) tmem_alloc_warp(&tmem_slot, TG_NMAX);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  const uint32_t sA_addr = (uint32_t)__cvta_generic_to_shared(sA), sB_addr = (uint32_t)__cvta_generic_to_shared(sB);
  const uint32_t idesc = instr_desc(TG_M, Nt);
  uint32_t phase = 0;
  bool issued = false;
  for (int k0 = kb; k0 < ke; k0 += TG_KC) {
    stage<float>(sA, A, sam, sak, m0, TG_M, M, k0, ke);
    stage<TB>(sB, B, sbn, sbk, n0, Nt, N, k0, ke);
    async_proxy_fence();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int ks = 0; ks < TG_KC / 16; ++ks) {
        const uint64_t dA = smem_desc(sA_addr + ks * 256, 128, (TG_KC / 8) * 128);
        const uint64_t dB = smem_desc(sB_addr + ks * 256, 128, (TG_KC / 8) * 128);
        umma_bf16(tmem, dA, dB, idesc, (k0 > kb || ks > 0) ? 1u : 0u);
      }
      umma_commit(&bar);
    }
    issued = true;
    // the operands are overwritten by the next chunk only after these MMAs completed
    if (vk::mbar_wait(&bar, phase, TG_WAIT)) phase ^= 1u;
    else atomicOr(&abort_flag, 1);
    tc_fence_after();
    __syncthreads();
    if (abort_flag) break;
  }
  if (abort_flag) {
    if (tid == 0) {
      atomicOr(status, VK_STATUS_WAIT_TIMEOUT);
      vk::mbar_wait(&bar, phase, TG_WAIT);   // the MMAs in flight, once more (bounded), before TMEM is freed
    }
  } else if (issued) {
    // epilogue: warp w holds rows 32w.. of the tile (its TMEM lane quarter)
    const int row = m0 + warp * 32 + lane;
    const uint32_t lane_off = (uint32_t)(warp * 32) << 16;
    const bool split = gridDim.z > 1;
    for (int c0 = 0; c0 < Nt; c0 += 16) {
      uint32_t v[16];
      tmem_ld16(tmem + lane_off + (uint32_t)c0, v);
      tmem_wait_ld();
      if (row < M) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int n = n0 + c0 + j;
          const float x = __uint_as_float(v[j]);
          if (split)
            ws[((int64_t)blockIdx.z * M + row) * N + n] = x;
          else
            C[(int64_t)row * scm + (int64_t)n * scn] = tg_out(x, bias, n, relu, round_bf16);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc_warp(tmem, TG_NMAX);
  }
}

// C[m, n] = out(sum over the splits z, in order, of ws[z][m][n])
__global__ void tc_gemm_reduce_k(int M, int N, int splits, const float* __restrict__ ws, const float* bias, int relu,
                                 int round_bf16, float* __restrict__ C, int64_t scm, int64_t scn) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= (int64_t)M * N) return;
  const int m = (int)(i / N), n = (int)(i % N);
  float s = 0.f;
  for (int z = 0; z < splits; ++z) s = __fadd_rn(s, ws[(int64_t)z * M * N + i]);
  C[(int64_t)m * scm + (int64_t)n * scn] = tg_out(s, bias, n, relu, round_bf16);
}

// K per split: splits only when the output tiles alone would leave most SMs idle
int tc_gemm_k_split(int M, int N, int K) {
  const int tiles = ((M + TG_M - 1) / TG_M) * ((N + TG_NMAX - 1) / TG_NMAX);
  if (tiles >= 64 || K <= 4 * TG_KC) return K;
  int splits = (128 + tiles - 1) / tiles;
  int ks = (K + splits - 1) / splits;
  ks = (ks + TG_KC - 1) / TG_KC * TG_KC;
  return ks < TG_KC ? TG_KC : ks;
}

}  // namespace

extern "C" {

int64_t vk_tc_gemm_ws_floats(int M, int N, int K) {
  if (M <= 0 || N <= 0 || K <= 0) return 0;
  const int ks = tc_gemm_k_split(M, N, K);
  const int splits = (K + ks - 1) / ks;
  return splits > 1 ? (int64_t)splits * M * N : 0;
}

int vk_tc_gemm(int M, int N, int K, const float* A, int64_t sam, int64_t sak, const void* B, int b_bf16, int64_t sbk,
               int64_t sbn, const float* bias, int relu, int round_bf16, float* C, int64_t scm, int64_t scn,
               float* ws, int64_t ws_floats, int32_t* status, void* stream) {
  if (M <= 0 || N <= 0) return 0;
  if (K <= 0 || (N % 16) != 0 || !A || !B || !C || !status) return VK_E_ARG;
  const int ks = tc_gemm_k_split(M, N, K);
  const int splits = (K + ks - 1) / ks;
  if (splits > 1 && (!ws || ws_floats < (int64_t)splits * M * N)) return VK_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  dim3 grid((unsigned)((M + TG_M - 1) / TG_M), (unsigned)((N + TG_NMAX - 1) / TG_NMAX), (unsigned)splits);
  cudaError_t e;
  if (b_bf16) {
    e = cudaFuncSetAttribute(tc_gemm_k<__nv_bfloat16>, cudaFuncAttributeMaxDynamicSharedMemorySize, TG_SMEM);
    if (e != cudaSuccess) return vk_err(e);
    tc_gemm_k<__nv_bfloat16><<<grid, TG_THREADS, TG_SMEM, st>>>(
        M, N, K, ks, A, sam, sak, reinterpret_cast<const __nv_bfloat16*>(B), sbk, sbn, bias, relu, round_bf16, C, scm,
        scn, ws, status);
  } else {
    e = cudaFuncSetAttribute(tc_gemm_k<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, TG_SMEM);
    if (e != cudaSuccess) return vk_err(e);
    tc_gemm_k<float><<<grid, TG_THREADS, TG_SMEM, st>>>(M, N, K, ks, A, sam, sak, reinterpret_cast<const float*>(B),
                                                        sbk, sbn, bias, relu, round_bf16, C, scm, scn, ws, status);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return vk_err(e);
  if (splits > 1) {
    const int64_t n = (int64_t)M * N;
    tc_gemm_reduce_k<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(M, N, splits, ws, bias, relu, round_bf16, C, scm,
                                                                  scn);
  }
  return vk_launch_status();
}

}  // extern "C"
