// Shared device helpers for the Diff-FVR B200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include "fvr_b200.h"

#define FVR_RETURN_IF(cond, code) \
  do {                            \
    if (cond) return (code);      \
  } while (0)

#define FVR_LAUNCH_CHECK()                        \
  do {                                            \
    cudaError_t e_ = cudaGetLastError();          \
    if (e_ != cudaSuccess) return FVR_ERR_CUDA;   \
  } while (0)

namespace fvr {

constexpr int kWarp = 32;

// ---- bounds-checked debug build --------------------------------------------
// Built with -DFVR_CHECK (libfvr_b200_check.so), every global or shared
// access guarded by fvr_checked(index, extent, site) whose index falls
// outside [0, extent) is skipped (the guarded load reads zero, the guarded
// store or atomic does nothing), and the first such event of each
// translation unit is recorded in that unit's check word: the site code in
// bits 40-63, the low 40 bits of the index below.  fvr_check_words reads and
// clears the words.  The normal build compiles every guard to `true`.
#ifdef FVR_CHECK
static __device__ unsigned long long g_fvr_check_word;

__device__ __forceinline__ bool fvr_checked(long long i, long long n, unsigned site) {
  if (i >= 0 && i < n) return true;
  atomicCAS(&g_fvr_check_word, 0ull,
            (static_cast<unsigned long long>(site) << 40) | (static_cast<unsigned long long>(i) & 0xffffffffffull));
  return false;
}

// Host side of one translation unit's check word (read, then optionally clear).
#define FVR_CHECK_ACCESSOR(name)                                                              \
  namespace fvr {                                                                             \
  int name(unsigned long long* out, int clear) {                                              \
    if (cudaMemcpyFromSymbol(out, g_fvr_check_word, sizeof(*out)) != cudaSuccess) return 1;   \
    if (clear) {                                                                              \
      const unsigned long long zero = 0ull;                                                   \
      if (cudaMemcpyToSymbol(g_fvr_check_word, &zero, sizeof(zero)) != cudaSuccess) return 1; \
    }                                                                                         \
    return 0;                                                                                 \
  }                                                                                           \
  }
#else
__device__ __forceinline__ constexpr bool fvr_checked(long long, long long, unsigned) { return true; }
#define FVR_CHECK_ACCESSOR(name)
#endif

// Checked read-only load / atomic add of element i of an n-element buffer.
__device__ __forceinline__ float ldg_in(const float* p, long long i, long long n, unsigned site) {
  return fvr_checked(i, n, site) ? __ldg(p + i) : 0.f;
}
__device__ __forceinline__ void atomic_add_in(float* p, long long i, long long n, unsigned site, float v) {
  if (fvr_checked(i, n, site)) atomicAdd(p + i, v);
}

// Site codes of the checked accesses.
enum : unsigned {
  kSiteStencilEntry = 1,  // stencil entry gather
  kSiteStencilScale,      // f16 brick scale
  kSiteSnccTarget,        // spectral-NCC target / high-pass sample
  kSitePlanar,            // planar drop-in gather
  kSiteNpGather,          // NumPy-convention fp64 gather
  kSiteWarpTap,           // PoU warp image tap (per-pixel paths)
  kSiteWarpGrad,          // PoU warp adjoint image-gradient atomic
  kSiteWarpStrip,         // PoU warp row-strip shared-memory access
  kSiteWarpStripRow,      // PoU warp row-strip image row read
  kSiteWarpFused,         // fused PoU warp adjoint: detector-row buffer and column-map reads
};

template <typename T>
struct Cx {
  T x, y;
};

template <typename T>
__host__ __device__ __forceinline__ Cx<T> cmul(Cx<T> a, Cx<T> b) {
  return Cx<T>{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename T>
__host__ __device__ __forceinline__ Cx<T> cadd(Cx<T> a, Cx<T> b) {
  return Cx<T>{a.x + b.x, a.y + b.y};
}
template <typename T>
__host__ __device__ __forceinline__ Cx<T> csub(Cx<T> a, Cx<T> b) {
  return Cx<T>{a.x - b.x, a.y - b.y};
}

// Scalar loads of one storage element as float (read-only path).
__device__ __forceinline__ float ldf(const float* p) { return __ldg(p); }
__device__ __forceinline__ float ldf(const __nv_bfloat16* p) {
  unsigned short b = __ldg(reinterpret_cast<const unsigned short*>(p));
  return __uint_as_float(static_cast<unsigned int>(b) << 16);
}
__device__ __forceinline__ float ldf(const __half* p) {
  unsigned short b = __ldg(reinterpret_cast<const unsigned short*>(p));
  return __half2float(__ushort_as_half(b));
}

// Round-to-nearest-even float -> storage element.
__device__ __forceinline__ void stf(float* p, float v) { *p = v; }
__device__ __forceinline__ void stf(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
__device__ __forceinline__ void stf(__half* p, float v) { *p = __float2half_rn(v); }

// bf16 pair packed in a 32-bit word -> two floats (exact).
__device__ __forceinline__ float bf_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf_hi(uint32_t w) { return __uint_as_float(w & 0xffff0000u); }
__device__ __forceinline__ float h_lo(uint32_t w) {
  return __half2float(__ushort_as_half(static_cast<unsigned short>(w & 0xffffu)));
}
__device__ __forceinline__ float h_hi(uint32_t w) {
  return __half2float(__ushort_as_half(static_cast<unsigned short>(w >> 16)));
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Reduce NV per-thread float accumulators over the CTA; warp stage in fp32,
// cross-warp stage in fp64.  Thread m < NV of warp 0 returns the CTA total of
// value m in `out`.  `red` must hold NV * (blockDim.x / 32) doubles.
template <int NV>
__device__ __forceinline__ void block_reduce_to_f64(float (&acc)[NV], double* red, double* out_m) {
  const int lane = threadIdx.x & 31;
  const int wid = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
#pragma unroll
  for (int m = 0; m < NV; ++m) {
    float v = warp_sum(acc[m]);
    if (lane == 0) red[m * nw + wid] = static_cast<double>(v);
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += red[threadIdx.x * nw + w];
    *out_m = s;
  }
}

// torch.linspace(start, end, steps) element i, evaluated the way torch does
// (symmetric halves from both ends, float arithmetic).
__host__ __device__ __forceinline__ float linspace_f32(float start, float end, int steps, int i) {
  if (steps == 1) return start;
  const float step = (end - start) / static_cast<float>(steps - 1);
  const int halfway = steps / 2;
  return (i < halfway) ? start + step * static_cast<float>(i)
                       : end - step * static_cast<float>(steps - i - 1);
}

__host__ __device__ __forceinline__ int64_t cdiv64(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace fvr
