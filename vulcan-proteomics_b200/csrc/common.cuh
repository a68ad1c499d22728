// Shared device helpers of the search kernels (sm_100a).
//
// Fragment arithmetic is Sage's f32 arithmetic (reference vulcan/gpu/kernels.cu:11-12, :36-51): every operation
// is an explicitly rounded intrinsic (__fadd_rn, __fmul_rn, __fdiv_rn), and the library is built with
// -fmad=false, so nothing is contracted into an FMA.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "vulcan_b200.h"

#define VK_FULL 0xffffffffu
#define VK_NTERM_BIT (1ull << 63)
#define VK_K2_MAXPK 512      // K2 scores against the first 512 mass-sorted peaks (kernels.cu:260, :277-278)
#define VK_K2_MAXLEN 64      // ion-index bound of the shifted (open / offset) scoring (kernels.cu:261)
#define VK_PROTON 1.0072764f
#define VK_NEUTRON 1.00335f

// Status bits written by kernels that wait on asynchronous copies (bounded waits).
#define VK_STATUS_WAIT_TIMEOUT 1
#define VK_STATUS_OVERFLOW 2

namespace vk {

// Fragment constants copied into shared memory by kernels that index them per lane.
struct SmemFrag {
  float mono[26];
  float stat[26];
  float var[26];
  float nterm;
  int tol_da;
};

__device__ __forceinline__ void load_frag(SmemFrag& s, const vk_frag_params& p) {
  for (int i = threadIdx.x; i < 26; i += blockDim.x) {
    s.mono[i] = p.mono[i];
    s.stat[i] = p.stat[i];
    s.var[i] = p.var[i];
  }
  if (threadIdx.x == 0) {
    s.nterm = p.nterm;
    s.tol_da = p.tol_da;
  }
}

// Sage Tolerance bound: ppm  m + (m * tol) / 1e6 ; Da  m + tol   (kernels.cu:36-38)
__device__ __forceinline__ float tol_bound(float m, float tol, int da) {
  return da ? __fadd_rn(m, tol) : __fadd_rn(m, __fdiv_rn(__fmul_rn(m, tol), 1000000.0f));
}

// Residue mass of residue r at position k: mono + (variable delta if mask bit k else static delta)
template <class F>
__device__ __forceinline__ float resmass(const F& fp, uint8_t r, int k, uint64_t mask) {
  int i = r - 'A';
  float d = ((mask >> k) & 1ull) ? fp.var[i] : fp.stat[i];
  return __fadd_rn(fp.mono[i], d);
}

template <class F>
__device__ __forceinline__ float nterm_of(const F& fp, uint64_t mask) {
  return (mask & VK_NTERM_BIT) ? fp.nterm : 0.f;
}

// Fragment ladder of one peptidoform row in Sage f32 arithmetic (reference kernels.cu:53-71): for k = 0 .. L-2,
// the b ion after residue k (a running sum from the N-terminal modification) and the y ion (the row's mass minus
// that sum); visit(mass) is called for each ion whose ion index exceeds min_ion and whose mass lies in
// [fmin, fmax], b before y at every k.  Shared by the tiled index build and the reference-layout CSR build.
template <class F, class V>
__device__ __forceinline__ void row_ladder(const F& fp, const uint8_t* s, int L, uint64_t mk, float mass,
                                           int min_ion, float fmin, float fmax, V&& visit) {
  const float nt = nterm_of(fp, mk);
  float b = nt, y = __fsub_rn(mass, nt);
  for (int k = 0; k + 1 < L; ++k) {
    const float rm = resmass(fp, s[k], k, mk);
    b = __fadd_rn(b, rm);
    y = __fsub_rn(y, rm);
    if (k + 1 > min_ion && b >= fmin && b <= fmax) visit(b);
    if (L - 1 - k > min_ion && y >= fmin && y <= fmax) visit(y);
  }
}

__device__ __forceinline__ double lnfact(int n) {
  // Stirling's approximation of ln n!, with lnfact(0) = 1 as in Sage (kernels.cu:246-250)
  if (n == 0) return 1.0;
  double x = (double)n;
  return x * log(x) - x + 0.5 * log(x) + 0.5 * log(2.0 * 3.141592653589793 * x);
}

__host__ __device__ __forceinline__ uint32_t f32_bits(float x) {
#ifdef __CUDA_ARCH__
  return __float_as_uint(x);
#else
  union { float f; uint32_t u; } v;
  v.f = x;
  return v.u;
#endif
}

// Bounded wait on an mbarrier phase (try_wait in a loop with an iteration limit).  Returns false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, uint32_t limit) {
  uint32_t addr = (uint32_t)__cvta_generic_to_shared(bar);
  for (uint32_t it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  uint32_t addr = (uint32_t)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(addr), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  uint32_t addr = (uint32_t)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(addr), "r"(bytes) : "memory");
}

// 1-D bulk (TMA) copy global -> shared, completion on an mbarrier.  dst, src 16-byte aligned; bytes % 16 == 0.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
  asm volatile("cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(d),
               "l"(src), "r"(bytes), "r"(b)
               : "memory");
}

// Inclusive warp scan (int64)
__device__ __forceinline__ long long warp_incl_scan(long long v) {
  int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    long long t = __shfl_up_sync(VK_FULL, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

__device__ __forceinline__ long long warp_sum(long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(VK_FULL, v, o);
  return v;
}

}  // namespace vk

static inline int vk_err(cudaError_t e) { return (int)e; }
static inline int vk_launch_status() { return (int)cudaGetLastError(); }
