// Training kernels of the candidate pruner's MLP (x -> 256 -> 256 -> 1; BF16 weights, FP32 accumulation).
//
// One tiled GEMM serves the forward pass and both backward products of every layer:
//   forward      Y[n x o]  = X[n x i] * W[o x i]^T + b    (optionally ReLU, optionally rounded to BF16 values)
//   input grad   dX[n x i] = dY[n x o] * W[o x i]
//   weight grad  dW[o x i] = dY^T[o x n] * X[n x i]
// Operands are addressed through strides, so transposes cost nothing; W is read as BF16 (the weights the
// inference kernel uses), activations and gradients are FP32.  Every output element is summed over k in a fixed
// order by one thread: results are deterministic, run to run.  Then BCE-with-logits loss/gradient, the ReLU mask of
// a backward gradient, the bias gradient (column sums) and an Adam step on the FP32 master weights that also writes
// their BF16 copy.
#include <cuda_bf16.h>

#include "common.cuh"

namespace {

constexpr int GT = 64;    // output tile (GT x GT) per CTA
constexpr int GK = 16;    // k tile
constexpr int GTHR = 256; // threads: each computes a 4 x 4 sub-tile

template <typename TB>
__device__ __forceinline__ float ld(const TB* p, int64_t i);
template <>
__device__ __forceinline__ float ld<float>(const float* p, int64_t i) { return p[i]; }
template <>
__device__ __forceinline__ float ld<__nv_bfloat16>(const __nv_bfloat16* p, int64_t i) { return __bfloat162float(p[i]); }

// C[m, n] = sum_k A[m*sam + k*sak] * B[k*sbk + n*sbn]  (+ bias[n]) (ReLU) (BF16 rounding)
template <typename TB>
__global__ void __launch_bounds__(GTHR)
gemm_k(int M, int N, int K, const float* __restrict__ A, int64_t sam, int64_t sak, const TB* __restrict__ B,
       int64_t sbk, int64_t sbn, const float* __restrict__ bias, int relu, int round_bf16, float* __restrict__ C,
       int64_t scm, int64_t scn) {
  __shared__ float As[GK][GT + 1];
  __shared__ float Bs[GK][GT + 1];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int m0 = blockIdx.y * GT, n0 = blockIdx.x * GT;
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
  for (int k0 = 0; k0 < K; k0 += GK) {
    for (int e = threadIdx.x; e < GK * GT; e += GTHR) {
      const int kk = e / GT, mm = e % GT;
      const int m = m0 + mm, k = k0 + kk;
      As[kk][mm] = (m < M && k < K) ? A[m * sam + k * sak] : 0.f;
      const int nn = mm, n = n0 + nn;
      Bs[kk][nn] = (n < N && k < K) ? ld<TB>(B, k * sbk + n * sbn) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GK; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = __fadd_rn(acc[i][j], __fmul_rn(a[i], b[j]));
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty * 4 + i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = n0 + tx * 4 + j;
      if (n >= N) continue;
      float v = acc[i][j];
      if (bias) v = __fadd_rn(v, bias[n]);
      if (relu) v = fmaxf(v, 0.f);
      if (round_bf16) v = __bfloat162float(__float2bfloat16_rn(v));
      C[m * scm + n * scn] = v;
    }
  }
}

// Column sums db[j] = sum_i dY[i, j] (v[i] dY[i, j] when v is given: the weighted sum of layer 3's weight
// gradient), in a fixed order: rows in chunks of CS_ROWS, each chunk summed sequentially (colsum_chunk_k, one thread
// per (chunk, column)), the chunk sums added in chunk order (colsum_total_k).
constexpr int CS_ROWS = 64;

__global__ void colsum_chunk_k(int n, int o, const float* dY, const float* v, float* part) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (j >= o) return;
  const int i1 = min(n, (c + 1) * CS_ROWS);
  float s = 0.f;
  for (int i = c * CS_ROWS; i < i1; ++i) {
    const float x = dY[(int64_t)i * o + j];
    s = __fadd_rn(s, v ? __fmul_rn(x, v[i]) : x);
  }
  part[(int64_t)c * o + j] = s;
}

__global__ void colsum_total_k(int chunks, int o, const float* part, float* db) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= o) return;
  float s = 0.f;
  for (int c = 0; c < chunks; ++c) s = __fadd_rn(s, part[(int64_t)c * o + j]);
  db[j] = s;
}

// dY *= (Y > 0)
__global__ void relu_mask_k(int64_t n, const float* Y, float* dY) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n && !(Y[i] > 0.f)) dY[i] = 0.f;
}

// Weighted BCE with logits: dz = w (sigmoid(z) - y) / sum_w; per-block loss partial sums (fixed order).
__global__ void bce_k(int n, const float* z, const float* y, const float* w, float inv_wsum, float* dz,
                      float* loss_part) {
  __shared__ float red[256];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  if (i < n) {
    const float zi = z[i], yi = y[i], wi = w[i];
    const float p = 1.f / (1.f + expf(-zi));
    dz[i] = wi * (p - yi) * inv_wsum;
    // log(1 + exp(-|z|)) + max(z, 0) - z*y
    l = wi * (log1pf(expf(-fabsf(zi))) + fmaxf(zi, 0.f) - zi * yi) * inv_wsum;
  }
  red[threadIdx.x] = l;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) loss_part[blockIdx.x] = red[0];
}

__global__ void adam_k(int64_t n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2,
                       float eps, float c1, float c2, float wd, __nv_bfloat16* p_bf16) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i] + wd * p[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  p[i] = pi;
  if (p_bf16) p_bf16[i] = __float2bfloat16_rn(pi);
}

__global__ void to_bf16_k(int64_t n, const float* x, __nv_bfloat16* y) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) y[i] = __float2bfloat16_rn(x[i]);
}

__global__ void bf16_to_f32_k(int64_t n, const __nv_bfloat16* x, float* y) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) y[i] = __bfloat162float(x[i]);
}

}  // namespace

extern "C" {

// b_bf16 != 0: B holds BF16 values, else FP32.
int vk_gemm(int M, int N, int K, const float* A, int64_t sam, int64_t sak, const void* B, int b_bf16, int64_t sbk,
            int64_t sbn, const float* bias, int relu, int round_bf16, float* C, int64_t scm, int64_t scn,
            void* stream) {
  if (M <= 0 || N <= 0) return 0;
  dim3 grid((unsigned)((N + GT - 1) / GT), (unsigned)((M + GT - 1) / GT));
  cudaStream_t st = (cudaStream_t)stream;
  if (b_bf16)
    gemm_k<__nv_bfloat16><<<grid, GTHR, 0, st>>>(M, N, K, A, sam, sak, reinterpret_cast<const __nv_bfloat16*>(B), sbk,
                                                 sbn, bias, relu, round_bf16, C, scm, scn);
  else
    gemm_k<float><<<grid, GTHR, 0, st>>>(M, N, K, A, sam, sak, reinterpret_cast<const float*>(B), sbk, sbn, bias,
                                         relu, round_bf16, C, scm, scn);
  return vk_launch_status();
}

int64_t vk_colsum_ws_floats(int n, int o) {
  return n > 0 && o > 0 ? (int64_t)((n + CS_ROWS - 1) / CS_ROWS) * o : 0;
}

int vk_colsum(int n, int o, const float* dY, const float* v, float* ws, int64_t ws_floats, float* db, void* stream) {
  if (o <= 0) return 0;
  cudaStream_t st = (cudaStream_t)stream;
  const int chunks = n > 0 ? (n + CS_ROWS - 1) / CS_ROWS : 0;
  if (chunks > 0 && (!ws || ws_floats < vk_colsum_ws_floats(n, o))) return VK_E_ARG;
  if (chunks > 0) {
    dim3 grid((unsigned)((o + 127) / 128), (unsigned)chunks);
    colsum_chunk_k<<<grid, 128, 0, st>>>(n, o, dY, v, ws);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return vk_err(e);
  }
  colsum_total_k<<<(unsigned)((o + 255) / 256), 256, 0, st>>>(chunks, o, ws, db);
  return vk_launch_status();
}

int vk_relu_mask(int64_t n, const float* Y, float* dY, void* stream) {
  if (n <= 0) return 0;
  relu_mask_k<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(n, Y, dY);
  return vk_launch_status();
}

int vk_bce(int n, const float* z, const float* y, const float* w, float inv_wsum, float* dz, float* loss_part,
           void* stream) {
  if (n <= 0) return 0;
  bce_k<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(n, z, y, w, inv_wsum, dz, loss_part);
  return vk_launch_status();
}

int vk_adam(int64_t n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2, float eps,
            int step, float wd, void* p_bf16, void* stream) {
  if (n <= 0) return 0;
  float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  adam_k<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      n, p, g, m, v, lr, b1, b2, eps, c1, c2, wd, reinterpret_cast<__nv_bfloat16*>(p_bf16));
  return vk_launch_status();
}

int vk_to_bf16(int64_t n, const float* x, void* y, void* stream) {
  if (n <= 0) return 0;
  to_bf16_k<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(n, x, reinterpret_cast<__nv_bfloat16*>(y));
  return vk_launch_status();
}

int vk_bf16_to_f32(int64_t n, const void* x, float* y, void* stream) {
  if (n <= 0) return 0;
  bf16_to_f32_k<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      n, reinterpret_cast<const __nv_bfloat16*>(x), y);
  return vk_launch_status();
}

}  // extern "C"
