// Candidate-pruner MLP inference on the 5th-generation tensor cores (tcgen05 / UMMA, TMEM accumulators).
//
// Network: logit = w3 . relu(W2 relu(W1 x + b1) + b2) + b3; x 16 BF16 features, W1 [256 x 16], W2 [256 x 256] BF16,
// b1, b2, w3 FP32.  The layer-1 activations are rounded to BF16 (the layer-2 operand), everything else stays FP32.
//
// Persistent CTAs of 16 warps, one per SM (the weights fill most of the shared memory).  Warp w reads TMEM lanes
// 32*(w%4).. (hit rows; a warp may only touch its lane quarter) and columns 64*(w/4).. .  Per tile of 128 hits:
//   1. the 128 x 16 feature tile (loaded into registers one tile ahead) is stored into shared memory in the UMMA
//      canonical K-major layout;
//   2. one thread issues D = X W1^T (M 128, N 256, K 16) into the tile's 256 TMEM columns and commits to an
//      mbarrier;
//   3. epilogue 1: every warp reads its 32 rows x 64 columns with tcgen05.ld, adds b1 (packed f32x2 adds),
//      applies ReLU and rounds to BF16 in one cvt per pair, and writes them into shared memory as the layer-2 A
//      operand;
//   4. one thread issues D = H1 W2^T (K 256: 16 UMMAs) into the same TMEM columns and commits;
//   5. epilogue 2 (done while the next tile's layer 2 runs): ReLU(D + b2) . w3 over the warp's 64 columns (packed
//      f32x2 adds and fused multiply-adds into four partial sums), the four column quarters of a row summed in a
//      fixed order through shared memory, + b3, written to `logit`.
// Shared-memory operands use the no-swizzle canonical layout: 8-row x 16-byte core matrices (128 contiguous bytes),
// the two 16-byte K chunks of one UMMA K-step 128 bytes apart (leading byte offset), 8-row groups a whole K-row of
// core matrices apart (stride byte offset).  Every mbarrier wait is bounded: on a timeout the CTA records
// VK_STATUS_WAIT_TIMEOUT, waits once more for its own MMAs, frees its TMEM and stops.
#include <cuda_bf16.h>

#include "common.cuh"
#include "tc_common.cuh"

namespace {

constexpr int TC_M = 128;          // hits per tile (UMMA M)
constexpr int TC_IN = 16;          // features (UMMA K of layer 1)
constexpr int TC_H = 256;          // hidden width (UMMA N; K of layer 2)
constexpr int TC_THREADS = 512;
constexpr int TC_COLS_PER_WARP = 64;
constexpr uint32_t TC_TMEM_COLS = 256;
constexpr uint32_t TC_WAIT = 1u << 24;

// shared-memory map (bytes)
constexpr int OFF_W2 = 0;                                  // 256 x 256 bf16, K-major canonical: 128 KB
constexpr int OFF_W1 = OFF_W2 + TC_H * TC_H * 2;           // 256 x 16: 8 KB
constexpr int OFF_X = OFF_W1 + TC_H * TC_IN * 2;           // 128 x 16: 4 KB
constexpr int OFF_H = OFF_X + TC_M * TC_IN * 2;            // 128 x 256: 64 KB
constexpr int OFF_B1 = OFF_H + TC_M * TC_H * 2;
constexpr int OFF_B2 = OFF_B1 + TC_H * 4;
constexpr int OFF_W3 = OFF_B2 + TC_H * 4;
constexpr int OFF_PART = OFF_W3 + TC_H * 4;                // 4 column quarters x 128 rows of partial logits
constexpr int TC_SMEM = OFF_PART + 4 * TC_M * 4;           // + 128 for alignment slack at launch

// Pairs of f32 in one 64-bit register (element 2j in the low half), added / fused-multiply-added with the
// packed-f32x2 instructions: two IEEE round-to-nearest operations each, half the instruction count.
__device__ __forceinline__ uint64_t f2(uint32_t lo, uint32_t hi) {
  uint64_t d;
  asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "r"(lo), "r"(hi));
  return d;
}
__device__ __forceinline__ uint64_t add_f2(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t fma_f2(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ float lo_f(uint64_t a) { return __uint_as_float((uint32_t)a); }
__device__ __forceinline__ float hi_f(uint64_t a) { return __uint_as_float((uint32_t)(a >> 32)); }
__device__ __forceinline__ uint64_t relu_f2(uint64_t a) {
  return f2(__float_as_uint(fmaxf(lo_f(a), 0.f)), __float_as_uint(fmaxf(hi_f(a), 0.f)));
}
// BF16 pair of relu(lo), relu(hi) rounded to nearest (lo in the low half): rounding keeps the sign, so this is
// the rounding of the ReLU output
__device__ __forceinline__ uint32_t relu_bf16x2(uint64_t a) {
  uint32_t d;
  asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi_f(a)), "f"(lo_f(a)));
  return d;
}

// Epilogue 1 of 32 accumulator columns c0.. of this thread's row: BF16(relu(D + b1)) into the layer-2 operand
// (four 16-byte K chunks, 128 bytes apart).
__device__ __forceinline__ void epi1_cols(const uint32_t* v, const float* sb1, int c0, uint8_t* dst) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const ulonglong2 ba = *reinterpret_cast<const ulonglong2*>(sb1 + c0 + 8 * q);       // 16-byte aligned
    const ulonglong2 bb = *reinterpret_cast<const ulonglong2*>(sb1 + c0 + 8 * q + 4);
    uint4 w;
    w.x = relu_bf16x2(add_f2(f2(v[8 * q + 0], v[8 * q + 1]), ba.x));
    w.y = relu_bf16x2(add_f2(f2(v[8 * q + 2], v[8 * q + 3]), ba.y));
    w.z = relu_bf16x2(add_f2(f2(v[8 * q + 4], v[8 * q + 5]), bb.x));
    w.w = relu_bf16x2(add_f2(f2(v[8 * q + 6], v[8 * q + 7]), bb.y));
    *reinterpret_cast<uint4*>(dst + q * 128) = w;
  }
}

// Epilogue 2 of 32 accumulator columns c0..: relu(D + b2) . w3 accumulated into two f32 pairs (four partial
// sums: columns c = 0, 1, 2, 3 mod 4).
__device__ __forceinline__ void epi2_cols(const uint32_t* v, const float* sb2, const float* sw3, int c0,
                                          uint64_t& za, uint64_t& zb) {
#pragma unroll
  for (int j = 0; j < 32; j += 4) {
    const ulonglong2 b = *reinterpret_cast<const ulonglong2*>(sb2 + c0 + j);
    const ulonglong2 w = *reinterpret_cast<const ulonglong2*>(sw3 + c0 + j);
    za = fma_f2(relu_f2(add_f2(f2(v[j + 0], v[j + 1]), b.x)), w.x, za);
    zb = fma_f2(relu_f2(add_f2(f2(v[j + 2], v[j + 3]), b.y)), w.y, zb);
  }
}

// This thread's share of a row's logit from the 64 columns col0.. of TMEM buffer pbuf (layer-2 accumulators).
__device__ __forceinline__ float epi2_share(uint32_t pbuf, uint32_t lane_off, int col0, const float* sb2,
                                            const float* sw3) {
  uint64_t za = 0ull, zb = 0ull;   // +0.0f pairs
#pragma unroll 1
  for (int c0 = col0; c0 < col0 + TC_COLS_PER_WARP; c0 += 32) {
    uint32_t v[32];
    tmem_ld32(pbuf + lane_off + (uint32_t)c0, v);
    tmem_wait_ld();
    epi2_cols(v, sb2, sw3, c0, za, zb);
  }
  return (lo_f(za) + hi_f(za)) + (lo_f(zb) + hi_f(zb));
}

// Two TMEM accumulators of 256 columns (tile i uses buffer i % 2 for both layers), so that the layer-2 UMMAs of
// tile i run while the warps finish tile i-1 (epilogue 2), and the layer-1 UMMA of tile i+1 is issued before the
// epilogue of tile i.  tcgen05.commit tracks every earlier MMA of the issuing thread, so the wait for tile i's
// layer 1 also covers tile i-1's layer 2 (which reads H1 in shared memory and tile i-1's TMEM buffer).
__global__ void __launch_bounds__(TC_THREADS, 1)
mlp_infer_tc_k(int64_t n, const int64_t* n_dev, const __nv_bfloat16* __restrict__ feat,
               const __nv_bfloat16* __restrict__ W1, const float* __restrict__ b1,
               const __nv_bfloat16* __restrict__ W2, const float* __restrict__ b2, const float* __restrict__ w3,
               float b3, float* __restrict__ logit, int32_t* status) {
  extern __shared__ uint8_t tc_raw[];
  __shared__ __align__(8) uint64_t bar1[2], bar2[2];
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(tc_raw) + 127) & ~uintptr_t(127));
  const int tid = threadIdx.x, warp = tid >> 5;
  if (n_dev) n = min(n, *n_dev);
  // weights into the canonical layouts (16-byte chunks), biases and w3; W2's 16 chunks per thread are loaded in two
  // batches of 8 independent loads before they are stored, so that the loads of a batch are in flight together
  constexpr int W2_PER = TC_H * TC_H / 8 / TC_THREADS;   // 16
  static_assert(W2_PER % 8 == 0, "W2 chunks per thread");
#pragma unroll
  for (int u0 = 0; u0 < W2_PER; u0 += 8) {
    uint4 v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int c = tid + (u0 + u) * TC_THREADS;
      const int r = c / (TC_H / 8), k = (c % (TC_H / 8)) * 8;
      v[u] = __ldg(reinterpret_cast<const uint4*>(W2 + (size_t)r * TC_H + k));
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int c = tid + (u0 + u) * TC_THREADS;
      const int r = c / (TC_H / 8), k = (c % (TC_H / 8)) * 8;
      *reinterpret_cast<uint4*>(sm + OFF_W2 + canon_off(r, k, TC_H)) = v[u];
    }
  }
  for (int c = tid; c < TC_H * TC_IN / 8; c += TC_THREADS) {
    const int r = c / (TC_IN / 8), k = (c % (TC_IN / 8)) * 8;
    *reinterpret_cast<uint4*>(sm + OFF_W1 + canon_off(r, k, TC_IN)) =
        *reinterpret_cast<const uint4*>(W1 + (size_t)r * TC_IN + k);
  }
  float* sb1 = reinterpret_cast<float*>(sm + OFF_B1);
  float* sb2 = reinterpret_cast<float*>(sm + OFF_B2);
  float* sw3 = reinterpret_cast<float*>(sm + OFF_W3);
  for (int i = tid; i < TC_H; i += TC_THREADS) {
    sb1[i] = b1[i];
    sb2[i] = b2[i];
    sw3[i] = w3[i];
  }
  if (tid == 0) {
    abort_flag = 0;
    for (int q = 0; q < 2; ++q) {
      vk::mbar_init(&bar1[q], 1);
      vk::mbar_init(&bar2[q], 1);
    }
    vk::fence_mbar_init();
  }
  if (warp == 0) {
    const uint32_t slot = (uint32_t)__cvta_generic_to_shared(&tmem_slot);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot),
                 "r"(2 * TC_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  const int64_t n_tiles = (n + TC_M - 1) / TC_M;
  const int64_t G = gridDim.x;
  // feature rows: threads < 256 each hold one 16-byte half row of the next tile
  const int fr = tid >> 1, fk = (tid & 1) * 8;
  auto load_feat = [&](int64_t tile) {
    uint4 v = make_uint4(0, 0, 0, 0);
    if (tid < 2 * TC_M && tile < n_tiles) {
      const int64_t row = tile * TC_M + fr;
      if (row < n) v = *reinterpret_cast<const uint4*>(feat + row * TC_IN + fk);
    }
    return v;
  };
  uint4 fv = load_feat(blockIdx.x);
  async_proxy_fence();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  const uint32_t s_base = (uint32_t)__cvta_generic_to_shared(sm);
  const uint32_t id_l = instr_desc(TC_M, TC_H);
  const uint64_t dW1 = smem_desc(s_base + OFF_W1, 128, (TC_IN / 8) * 128);
  const uint64_t dX = smem_desc(s_base + OFF_X, 128, (TC_IN / 8) * 128);
  const int rq = warp & 3, cq = warp >> 2;                 // lane (row) quarter, column quarter
  const int my_row = rq * 32 + (threadIdx.x & 31);
  const int col0 = cq * TC_COLS_PER_WARP;
  const uint32_t lane_off = (uint32_t)(rq * 32) << 16;
  float* part = reinterpret_cast<float*>(sm + OFF_PART);
  uint32_t ph1 = 0u, ph2 = 0u;                   // phase bit q of bar1[q] / bar2[q] to wait for next
  uint64_t* last_bar = nullptr;                   // the latest commit (it covers every earlier MMA) ...
  uint32_t last_ph = 0u;                          // ... and the phase it completes
  int64_t tile = blockIdx.x, prev = -1;
  int k = 0;
  // prologue: tile 0's features and its layer 1
  if (tile < n_tiles) {
    if (tid < 2 * TC_M) *reinterpret_cast<uint4*>(sm + OFF_X + canon_off(fr, fk, TC_IN)) = fv;
    async_proxy_fence();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      umma_bf16(tmem, dX, dW1, id_l, 0u);
      umma_commit(&bar1[0]);
    }
    last_bar = &bar1[0];
    last_ph = 0u;
    fv = load_feat(tile + G);
  }
  while (tile < n_tiles) {
    const int b = k & 1;
    const uint32_t buf = tmem + (uint32_t)b * TC_TMEM_COLS;
    // layer 1 of this tile (and everything issued before it) is done
    if (!vk::mbar_wait(&bar1[b], (ph1 >> b) & 1u, TC_WAIT)) atomicOr(&abort_flag, 1);
    ph1 ^= 1u << b;
    tc_fence_after();
    // epilogue 1: H1 = bf16(relu(D + b1)) into the layer-2 operand
#pragma unroll 1
    for (int c0 = col0; c0 < col0 + TC_COLS_PER_WARP; c0 += 32) {
      uint32_t v[32];
      tmem_ld32(buf + lane_off + (uint32_t)c0, v);
      tmem_wait_ld();
      epi1_cols(v, sb1, c0, sm + OFF_H + canon_off(my_row, c0, TC_H));
    }
    async_proxy_fence();
    tc_fence_before();
    __syncthreads();
    if (abort_flag) break;
    // layer 2 of this tile into the same buffer (K = 256 in 16 steps)
    if (tid == 0) {
      tc_fence_after();
#pragma unroll 1
      for (int ks = 0; ks < TC_H / 16; ++ks) {
        const uint64_t dA = smem_desc(s_base + OFF_H + ks * 256, 128, (TC_H / 8) * 128);
        const uint64_t dB = smem_desc(s_base + OFF_W2 + ks * 256, 128, (TC_H / 8) * 128);
        umma_bf16(buf, dA, dB, id_l, ks > 0 ? 1u : 0u);
      }
      umma_commit(&bar2[b]);
    }
    last_bar = &bar2[b];
    last_ph = (ph2 >> b) & 1u;
    // epilogue 2 of the previous tile (its buffer), overlapping this tile's layer 2
    if (prev >= 0) {
      const int pb = b ^ 1;
      if (!vk::mbar_wait(&bar2[pb], (ph2 >> pb) & 1u, TC_WAIT)) atomicOr(&abort_flag, 1);
      ph2 ^= 1u << pb;
      tc_fence_after();
      part[cq * TC_M + my_row] = epi2_share(tmem + (uint32_t)pb * TC_TMEM_COLS, lane_off, col0, sb2, sw3);
    }
    // the next tile's features (layer 1 of this tile is done with the feature buffer)
    const int64_t nt = tile + G;
    if (nt < n_tiles && tid < 2 * TC_M) *reinterpret_cast<uint4*>(sm + OFF_X + canon_off(fr, fk, TC_IN)) = fv;
    async_proxy_fence();
    tc_fence_before();
    __syncthreads();
    if (prev >= 0 && tid < TC_M) {
      const int64_t row = prev * TC_M + tid;
      if (row < n) logit[row] = ((part[tid] + part[TC_M + tid]) + (part[2 * TC_M + tid] + part[3 * TC_M + tid])) + b3;
    }
    if (abort_flag) break;
    // layer 1 of the next tile into the other buffer (epilogue 2 above has finished reading it)
    if (nt < n_tiles) {
      if (tid == 0) {
        tc_fence_after();
        umma_bf16(tmem + (uint32_t)(b ^ 1) * TC_TMEM_COLS, dX, dW1, id_l, 0u);
        umma_commit(&bar1[b ^ 1]);
      }
      last_bar = &bar1[b ^ 1];
      last_ph = (ph1 >> (b ^ 1)) & 1u;
      fv = load_feat(nt + G);
    }
    prev = tile;
    tile = nt;
    ++k;
  }
  // epilogue 2 of the last tile
  if (!abort_flag && prev >= 0) {
    const int pb = (k - 1) & 1;
    if (!vk::mbar_wait(&bar2[pb], (ph2 >> pb) & 1u, TC_WAIT)) atomicOr(&abort_flag, 1);
    ph2 ^= 1u << pb;
    tc_fence_after();
    part[cq * TC_M + my_row] = epi2_share(tmem + (uint32_t)pb * TC_TMEM_COLS, lane_off, col0, sb2, sw3);
    tc_fence_before();
    __syncthreads();
    if (tid < TC_M) {
      const int64_t row = prev * TC_M + tid;
      if (row < n) logit[row] = ((part[tid] + part[TC_M + tid]) + (part[2 * TC_M + tid] + part[3 * TC_M + tid])) + b3;
    }
  }
  __syncthreads();
  if (abort_flag) {
    if (tid == 0) {
      atomicOr(status, VK_STATUS_WAIT_TIMEOUT);
      // the MMAs in flight, once more, bounded: the latest commit covers every earlier MMA
      if (last_bar) vk::mbar_wait(last_bar, last_ph, TC_WAIT);
    }
    __syncthreads();
  }
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * TC_TMEM_COLS));
  }
}

}  // namespace

extern "C" {

int64_t vk_mlp_infer_tc_smem(void) { return (int64_t)TC_SMEM + 128; }

int vk_mlp_infer_tc(int64_t n, const int64_t* n_dev, const void* feat_bf16, const void* W1_bf16, const float* b1,
                    const void* W2_bf16, const float* b2, const float* w3, float b3, float* logit, int grid,
                    int32_t* status, void* stream) {
  if (n <= 0) return 0;
  if (grid < 1 || !status) return VK_E_ARG;
  const size_t sh = (size_t)vk_mlp_infer_tc_smem();
  cudaError_t e = cudaFuncSetAttribute(mlp_infer_tc_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  if (e != cudaSuccess) return vk_err(e);
  mlp_infer_tc_k<<<grid, TC_THREADS, sh, (cudaStream_t)stream>>>(
      n, n_dev, reinterpret_cast<const __nv_bfloat16*>(feat_bf16), reinterpret_cast<const __nv_bfloat16*>(W1_bf16), b1,
      reinterpret_cast<const __nv_bfloat16*>(W2_bf16), b2, w3, b3, logit, status);
  return vk_launch_status();
}

}  // extern "C"
