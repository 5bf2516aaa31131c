// Stencil spectrum build (+ f16 brick scales) and small elementwise helpers
// (high-pass table, linspace, complex-by-table product, ReLU adjoint mask).
#include "fvr_stencil.cuh"

namespace fvr {

// ----------------------------------------------------------------------------
// stencil build
// ----------------------------------------------------------------------------

// master spectrum: planar [2][D][H][W] (the reference's f_vol_5d[0]) or
// interleaved [D][H][W][2]
template <typename MT>
__device__ __forceinline__ float2 master_load(const MT* m, int64_t idx, int64_t plane) {
  return plane ? make_float2(ldf(m + idx), ldf(m + plane + idx)) : make_float2(ldf(m + 2 * idx), ldf(m + 2 * idx + 1));
}

template <typename MT>
__device__ __forceinline__ void entry_values(const MT* m, int64_t plane, int D, int H, int W, int ez, int ey, int ex,
                                             float (&re)[8], float (&im)[8]) {
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int z = ez - 1 + (c >> 2), y = ey - 1 + ((c >> 1) & 1), x = ex - 1 + (c & 1);
    if (z >= 0 && z < D && y >= 0 && y < H && x >= 0 && x < W) {
      float2 v = master_load(m, (static_cast<int64_t>(z) * H + y) * W + x, plane);
      re[c] = v.x;
      im[c] = v.y;
    } else {
      re[c] = 0.f;
      im[c] = 0.f;
    }
  }
}

// atomicMax of non-negative float bits into table[idx], one atomic per group
// of lanes that share idx (consecutive entries mostly share their brick, so
// the lanes of a warp merge their maxima first instead of all contending for
// one address).
__device__ __forceinline__ void group_atomic_max(unsigned int* table, long long idx, unsigned int bits) {
  const unsigned grp = __match_any_sync(__activemask(), idx);
  const unsigned m = __reduce_max_sync(grp, bits);
  if ((threadIdx.x & 31) == static_cast<unsigned>(__ffs(grp) - 1)) atomicMax(table + idx, m);
}

template <typename MT>
__global__ void stencil_brick_max_kernel(const MT* __restrict__ m0, int64_t plane, int64_t items, int D, int H,
                                         int W, unsigned int* bmax0) {
  const int64_t n1 = static_cast<int64_t>(D + 1) * (H + 1) * (W + 1);
  const int64_t n = n1 * items;
  const int bx = (W + 1 + kBrick - 1) / kBrick, by = (H + 1 + kBrick - 1) / kBrick;
  const int64_t nb1 = static_cast<int64_t>(bx) * by * ((D + 1 + kBrick - 1) / kBrick);
  for (int64_t ee = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; ee < n;
       ee += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t item = ee / n1, e = ee - item * n1;
    const MT* m = m0 + item * 2 * static_cast<int64_t>(D) * H * W;
    const int ex = static_cast<int>(e % (W + 1));
    const int ey = static_cast<int>((e / (W + 1)) % (H + 1));
    const int ez = static_cast<int>(e / (static_cast<int64_t>(W + 1) * (H + 1)));
    float re[8], im[8];
    entry_values(m, plane, D, H, W, ez, ey, ex, re, im);
    float mx = 0.f;
#pragma unroll
    for (int c = 0; c < 8; ++c) mx = fmaxf(mx, fmaxf(fabsf(re[c]), fabsf(im[c])));
    const int64_t b = (static_cast<int64_t>(ez / kBrick) * by + ey / kBrick) * bx + ex / kBrick;
    group_atomic_max(bmax0, item * nb1 + b, __float_as_uint(mx));  // non-negative floats order like their bits
  }
}

// scale = 2^e with max/scale <= 2^15 (half max is 65504); exact to apply.
__global__ void stencil_scale_kernel(const unsigned int* bmax, float* scales, int64_t nb) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= nb) return;
  const float mx = __uint_as_float(bmax[i]);
  float sc = 1.f;
  if (mx > 0.f && isfinite(mx)) {
    int e;
    frexpf(mx, &e);  // mx = f * 2^e, f in [0.5, 1)
    sc = ldexpf(1.f, e - 15);
  }
  scales[i] = sc;
}

template <typename MT, int DT>
__global__ void stencil_build_kernel(const MT* __restrict__ m0, int64_t plane, int64_t items, int D, int H, int W,
                                     void* __restrict__ out0, const float* __restrict__ scales0) {
  const int64_t n1 = static_cast<int64_t>(D + 1) * (H + 1) * (W + 1);
  const int64_t n = n1 * items;
  const int bx = (W + 1 + kBrick - 1) / kBrick, by = (H + 1 + kBrick - 1) / kBrick;
  const int64_t nb1 = static_cast<int64_t>(bx) * by * ((D + 1 + kBrick - 1) / kBrick);
  for (int64_t ee = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; ee < n;
       ee += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t item = ee / n1, e = ee - item * n1;
    const MT* m = m0 + item * 2 * static_cast<int64_t>(D) * H * W;
    const float* scales = scales0 ? scales0 + item * nb1 : nullptr;
    void* out = static_cast<char*>(out0) + item * n1 * (DT == FVR_F32 ? 64 : 32);
    const int ex = static_cast<int>(e % (W + 1));
    const int ey = static_cast<int>((e / (W + 1)) % (H + 1));
    const int ez = static_cast<int>(e / (static_cast<int64_t>(W + 1) * (H + 1)));
    float re[8], im[8];
    entry_values(m, plane, D, H, W, ez, ey, ex, re, im);
    if constexpr (DT == FVR_F32) {
      float4* p = static_cast<float4*>(out) + e * 4;
#pragma unroll
      for (int i = 0; i < 4; ++i) p[i] = make_float4(re[2 * i], im[2 * i], re[2 * i + 1], im[2 * i + 1]);
    } else {
      uint32_t w[8];
      if constexpr (DT == FVR_BF16) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const uint32_t lo = __bfloat16_as_ushort(__float2bfloat16_rn(re[c]));
          const uint32_t hi = __bfloat16_as_ushort(__float2bfloat16_rn(im[c]));
          w[c] = lo | (hi << 16);
        }
      } else {
        const float inv = 1.f / scales[(static_cast<int64_t>(ez / kBrick) * by + ey / kBrick) * bx + ex / kBrick];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const uint32_t lo = __half_as_ushort(__float2half_rn(re[c] * inv));
          const uint32_t hi = __half_as_ushort(__float2half_rn(im[c] * inv));
          w[c] = lo | (hi << 16);
        }
      }
      uint4* p = static_cast<uint4*>(out) + e * 2;
      p[0] = make_uint4(w[0], w[1], w[2], w[3]);
      p[1] = make_uint4(w[4], w[5], w[6], w[7]);
    }
  }
}

// ---- x-pair layout (16-bit): entry (ez, ey, ex) = the 4 complex values of
// voxel column x = ex - 1 at (y, z) = (ey - 1 + dy, ez - 1 + dz), k = dz*2 + dy.
template <typename MT>
__device__ __forceinline__ void pair_values(const MT* m, int64_t plane, int D, int H, int W, int ez, int ey, int ex,
                                            float (&re)[4], float (&im)[4]) {
  const int x = ex - 1;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int z = ez - 1 + (k >> 1), y = ey - 1 + (k & 1);
    if (z >= 0 && z < D && y >= 0 && y < H && x >= 0 && x < W) {
      const float2 v = master_load(m, (static_cast<int64_t>(z) * H + y) * W + x, plane);
      re[k] = v.x;
      im[k] = v.y;
    } else {
      re[k] = 0.f;
      im[k] = 0.f;
    }
  }
}

// f16 scale slabs: kBrick x kBrick (z, y) entry rows over the whole x extent,
// so the two entries of every sample share one scale.
struct PairGrid {
  int ew, eh, ed;  // entries along x, y, z: W + 2, H + 1, D + 1
  int by;          // slabs along y
  __device__ __forceinline__ int64_t slab(int ez, int ey) const {
    return static_cast<int64_t>(ez / kBrick) * by + ey / kBrick;
  }
};

__host__ __device__ inline PairGrid pair_grid(int D, int H, int W) {
  PairGrid g;
  g.ew = W + 2;
  g.eh = H + 1;
  g.ed = D + 1;
  g.by = (g.eh + kBrick - 1) / kBrick;
  return g;
}

template <typename MT>
__global__ void pair_slab_max_kernel(const MT* __restrict__ m0, int64_t plane, int64_t items, int D, int H, int W,
                                     unsigned int* __restrict__ smax0) {
  const PairGrid g = pair_grid(D, H, W);
  const int64_t n1 = static_cast<int64_t>(g.ed) * g.eh * g.ew;
  const int64_t nb1 = static_cast<int64_t>((g.ed + kBrick - 1) / kBrick) * g.by;
  for (int64_t ee = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; ee < n1 * items;
       ee += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t item = ee / n1, e = ee - item * n1;
    const MT* m = m0 + item * 2 * static_cast<int64_t>(D) * H * W;
    const int ex = static_cast<int>(e % g.ew), ey = static_cast<int>((e / g.ew) % g.eh);
    const int ez = static_cast<int>(e / (static_cast<int64_t>(g.ew) * g.eh));
    float re[4], im[4];
    pair_values(m, plane, D, H, W, ez, ey, ex, re, im);
    float mx = 0.f;
#pragma unroll
    for (int k = 0; k < 4; ++k) mx = fmaxf(mx, fmaxf(fabsf(re[k]), fabsf(im[k])));
    group_atomic_max(smax0, item * nb1 + g.slab(ez, ey), __float_as_uint(mx));  // non-negative floats order like their bits
  }
}

template <typename MT, int DT>
__global__ void pair_build_kernel(const MT* __restrict__ m0, int64_t plane, int64_t items, int D, int H, int W,
                                  void* __restrict__ out0, const float* __restrict__ scales0) {
  const PairGrid g = pair_grid(D, H, W);
  const int64_t n1 = static_cast<int64_t>(g.ed) * g.eh * g.ew;
  const int64_t nb1 = static_cast<int64_t>((g.ed + kBrick - 1) / kBrick) * g.by;
  for (int64_t ee = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; ee < n1 * items;
       ee += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t item = ee / n1, e = ee - item * n1;
    const MT* m = m0 + item * 2 * static_cast<int64_t>(D) * H * W;
    const int ex = static_cast<int>(e % g.ew), ey = static_cast<int>((e / g.ew) % g.eh);
    const int ez = static_cast<int>(e / (static_cast<int64_t>(g.ew) * g.eh));
    float re[4], im[4];
    pair_values(m, plane, D, H, W, ez, ey, ex, re, im);
    if constexpr (DT == FVR_F32_PAIR) {
      float4* p = static_cast<float4*>(out0) + (item * n1 + e) * 2;
      p[0] = make_float4(re[0], im[0], re[1], im[1]);
      p[1] = make_float4(re[2], im[2], re[3], im[3]);
    } else {
      uint32_t w[4];
      if constexpr (DT == FVR_BF16_PAIR) {
#pragma unroll
        for (int k = 0; k < 4; ++k)
          w[k] = static_cast<uint32_t>(__bfloat16_as_ushort(__float2bfloat16_rn(re[k]))) |
                 (static_cast<uint32_t>(__bfloat16_as_ushort(__float2bfloat16_rn(im[k]))) << 16);
      } else {
        const float inv = 1.f / scales0[item * nb1 + g.slab(ez, ey)];
#pragma unroll
        for (int k = 0; k < 4; ++k)
          w[k] = static_cast<uint32_t>(__half_as_ushort(__float2half_rn(re[k] * inv))) |
                 (static_cast<uint32_t>(__half_as_ushort(__float2half_rn(im[k] * inv))) << 16);
      }
      static_cast<uint4*>(out0)[item * n1 + e] = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

// relu mask of the saved image, as complex: G = (img > 0) * g
__global__ void relu_mask_kernel(const float* __restrict__ img, const float* __restrict__ g, float* __restrict__ out,
                                 int64_t n) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  out[i] = img[i] > 0.f ? g[i] : 0.f;
}

// complex * real table (per image), e.g. the high-pass filter of a target spectrum
__global__ void cmul_table_kernel(float2* __restrict__ x, const float* __restrict__ t, int64_t per, int64_t n) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const float w = t[i % per];
  x[i] = make_float2(x[i].x * w, x[i].y * w);
}

// HP = 1 - exp(-r^2 / (2 sigma^2)) on linspace(-H/2, H/2, H) x linspace(-W/2, W/2, W)
// (torch_engine.py:123-136), evaluated in fp64.
__global__ void hp_filter_kernel(float* __restrict__ out, int H, int W, double sigma) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= H * W) return;
  const int r = i / W, c = i - r * W;
  const double y = H > 1 ? -0.5 * H + r * (static_cast<double>(H) / (H - 1)) : -0.5 * H;
  const double x = W > 1 ? -0.5 * W + c * (static_cast<double>(W) / (W - 1)) : -0.5 * W;
  out[i] = static_cast<float>(1.0 - exp(-(x * x + y * y) / (2.0 * sigma * sigma)));
}

__global__ void linspace_kernel(float* out, float start, float end, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = linspace_f32(start, end, n, i);
}

}  // namespace fvr

using namespace fvr;

extern "C" {

int64_t fvr_stencil_bytes(int64_t D, int64_t H, int64_t W, int dtype) {
  const int64_t n = (D + 1) * (H + 1) * (W + 1);
  if (dtype == FVR_F32) return n * 64;
  if (dtype == FVR_BF16 || dtype == FVR_F16) return n * 32;
  return -1;
}

int64_t fvr_stencil_scale_count(int64_t D, int64_t H, int64_t W) {
  return fvr::cdiv64(D + 1, kBrick) * fvr::cdiv64(H + 1, kBrick) * fvr::cdiv64(W + 1, kBrick);
}

int fvr_stencil_build(const void* master, int master_dtype, int master_planar, int64_t items, int64_t D, int64_t H,
                      int64_t W, int out_dtype, void* out, float* scales, unsigned int* scratch_max, void* stream) {
  if (!master || !out || D < 1 || H < 1 || W < 1 || D > 8192 || H > 8192 || W > 8192) return FVR_ERR_ARG;
  if ((reinterpret_cast<uintptr_t>(out) & 15) != 0) return FVR_ERR_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (items < 1) return FVR_ERR_ARG;
  const int64_t n = (D + 1) * (H + 1) * (W + 1) * items;
  const int64_t nblk = cdiv64(n, 256);
  const unsigned grid = static_cast<unsigned>(nblk < 148 * 64 ? nblk : 148 * 64);
  const int d = (int)D, h = (int)H, w = (int)W;
  const int64_t plane = master_planar ? D * H * W : 0;
  if (out_dtype == FVR_F16) {
    if (!scales || !scratch_max) return FVR_ERR_ARG;
    const int64_t nb = fvr_stencil_scale_count(D, H, W) * items;
    if (cudaMemsetAsync(scratch_max, 0, nb * sizeof(unsigned int), s) != cudaSuccess) return FVR_ERR_CUDA;
    if (master_dtype == FVR_F32)
      stencil_brick_max_kernel<float>
          <<<grid, 256, 0, s>>>(static_cast<const float*>(master), plane, items, d, h, w, scratch_max);
    else if (master_dtype == FVR_BF16)
      stencil_brick_max_kernel<__nv_bfloat16>
          <<<grid, 256, 0, s>>>(static_cast<const __nv_bfloat16*>(master), plane, items, d, h, w, scratch_max);
    else if (master_dtype == FVR_F16)
      stencil_brick_max_kernel<__half>
          <<<grid, 256, 0, s>>>(static_cast<const __half*>(master), plane, items, d, h, w, scratch_max);
    else
      return FVR_ERR_DTYPE;
    stencil_scale_kernel<<<static_cast<unsigned>(cdiv64(nb, 256)), 256, 0, s>>>(scratch_max, scales, nb);
  }
#define FVR_BUILD(MT, DT)                                                                                  \
  stencil_build_kernel<MT, DT><<<grid, 256, 0, s>>>(static_cast<const MT*>(master), plane, items, d, h, w, out, \
                                                    scales);                                                    \
  break;
  if (master_dtype == FVR_F32) {
    switch (out_dtype) {
      case FVR_F32: FVR_BUILD(float, FVR_F32)
      case FVR_BF16: FVR_BUILD(float, FVR_BF16)
      case FVR_F16: FVR_BUILD(float, FVR_F16)
      default: return FVR_ERR_DTYPE;
    }
  } else if (master_dtype == FVR_BF16) {
    switch (out_dtype) {
      case FVR_F32: FVR_BUILD(__nv_bfloat16, FVR_F32)
      case FVR_BF16: FVR_BUILD(__nv_bfloat16, FVR_BF16)
      case FVR_F16: FVR_BUILD(__nv_bfloat16, FVR_F16)
      default: return FVR_ERR_DTYPE;
    }
  } else if (master_dtype == FVR_F16) {
    switch (out_dtype) {
      case FVR_F32: FVR_BUILD(__half, FVR_F32)
      case FVR_BF16: FVR_BUILD(__half, FVR_BF16)
      case FVR_F16: FVR_BUILD(__half, FVR_F16)
      default: return FVR_ERR_DTYPE;
    }
  } else {
    return FVR_ERR_DTYPE;
  }
#undef FVR_BUILD
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int64_t fvr_stencil_pair_bytes(int64_t D, int64_t H, int64_t W, int dtype) {
  if (D < 1 || H < 1 || W < 1) return 0;
  const int64_t n = (D + 1) * (H + 1) * (W + 2);
  if (dtype == FVR_BF16_PAIR || dtype == FVR_F16_PAIR) return n * 16;
  if (dtype == FVR_F32_PAIR) return n * 32;
  return 0;
}

int64_t fvr_stencil_pair_scale_count(int64_t D, int64_t H, int64_t W) {
  if (D < 1 || H < 1 || W < 1) return 0;
  return cdiv64(D + 1, kBrick) * cdiv64(H + 1, kBrick);
}

int fvr_stencil_pair_build(const void* master, int master_dtype, int master_planar, int64_t items, int64_t D,
                           int64_t H, int64_t W, int out_dtype, void* out, float* scales, unsigned int* scratch_max,
                           void* stream) {
  if (!master || !out || items < 1 || D < 1 || H < 1 || W < 1 || D > 8192 || H > 8192 || W > 8192)
    return FVR_ERR_ARG;
  if ((reinterpret_cast<uintptr_t>(out) & 31) != 0) return FVR_ERR_ARG;
  if (out_dtype != FVR_BF16_PAIR && out_dtype != FVR_F16_PAIR && out_dtype != FVR_F32_PAIR) return FVR_ERR_DTYPE;
  if (master_dtype != FVR_F32 && master_dtype != FVR_BF16 && master_dtype != FVR_F16) return FVR_ERR_DTYPE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t n = (D + 1) * (H + 1) * (W + 2) * items;
  const int64_t nblk = cdiv64(n, 256);
  const unsigned grid = static_cast<unsigned>(nblk < 148 * 64 ? nblk : 148 * 64);
  const int d = (int)D, h = (int)H, w = (int)W;
  const int64_t plane = master_planar ? D * H * W : 0;
  if (out_dtype == FVR_F16_PAIR) {
    if (!scales || !scratch_max) return FVR_ERR_ARG;
    const int64_t nb = fvr_stencil_pair_scale_count(D, H, W) * items;
    if (cudaMemsetAsync(scratch_max, 0, nb * sizeof(unsigned int), s) != cudaSuccess) return FVR_ERR_CUDA;
    if (master_dtype == FVR_F32)
      pair_slab_max_kernel<float>
          <<<grid, 256, 0, s>>>(static_cast<const float*>(master), plane, items, d, h, w, scratch_max);
    else if (master_dtype == FVR_BF16)
      pair_slab_max_kernel<__nv_bfloat16>
          <<<grid, 256, 0, s>>>(static_cast<const __nv_bfloat16*>(master), plane, items, d, h, w, scratch_max);
    else
      pair_slab_max_kernel<__half>
          <<<grid, 256, 0, s>>>(static_cast<const __half*>(master), plane, items, d, h, w, scratch_max);
    stencil_scale_kernel<<<static_cast<unsigned>(cdiv64(nb, 256)), 256, 0, s>>>(scratch_max, scales, nb);
  }
#define FVR_PAIR(MT)                                                                                          \
  switch (out_dtype) {                                                                                        \
    case FVR_F16_PAIR:                                                                                        \
      pair_build_kernel<MT, FVR_F16_PAIR>                                                                     \
          <<<grid, 256, 0, s>>>(static_cast<const MT*>(master), plane, items, d, h, w, out, scales);           \
      break;                                                                                                  \
    case FVR_BF16_PAIR:                                                                                       \
      pair_build_kernel<MT, FVR_BF16_PAIR>                                                                    \
          <<<grid, 256, 0, s>>>(static_cast<const MT*>(master), plane, items, d, h, w, out, nullptr);          \
      break;                                                                                                  \
    default:                                                                                                  \
      pair_build_kernel<MT, FVR_F32_PAIR>                                                                     \
          <<<grid, 256, 0, s>>>(static_cast<const MT*>(master), plane, items, d, h, w, out, nullptr);          \
      break;                                                                                                  \
  }
  if (master_dtype == FVR_F32) {
    FVR_PAIR(float)
  } else if (master_dtype == FVR_BF16) {
    FVR_PAIR(__nv_bfloat16)
  } else {
    FVR_PAIR(__half)
  }
#undef FVR_PAIR
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_relu_mask(const float* img, const float* g, float* out, int64_t n, void* stream) {
  if (!img || !g || !out || n < 1) return FVR_ERR_ARG;
  relu_mask_kernel<<<static_cast<unsigned>(cdiv64(n, 256)), 256, 0, static_cast<cudaStream_t>(stream)>>>(img, g,
                                                                                                          out, n);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_cmul_table(void* x, const float* table, int64_t per, int64_t n, void* stream) {
  if (!x || !table || per < 1 || n < 1) return FVR_ERR_ARG;
  cmul_table_kernel<<<static_cast<unsigned>(cdiv64(n, 256)), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<float2*>(x), table, per, n);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_hp_filter(float* out, int64_t H, int64_t W, double sigma, void* stream) {
  if (!out || H < 1 || W < 1 || H * W > (int64_t)1 << 30) return FVR_ERR_ARG;
  hp_filter_kernel<<<static_cast<unsigned>(cdiv64(H * W, 256)), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      out, (int)H, (int)W, sigma);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_linspace(float* out, float start, float end, int64_t n, void* stream) {
  if (!out || n < 1 || n > (int64_t)1 << 30) return FVR_ERR_ARG;
  linspace_kernel<<<static_cast<unsigned>(cdiv64(n, 256)), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      out, start, end, (int)n);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

}  // extern "C"
