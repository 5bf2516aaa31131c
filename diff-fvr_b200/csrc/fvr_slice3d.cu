// Drop-in trilinear Fourier-slice gather on the reference's planar layout
// vol[B][2][D][H][W] (src/fvr/triton_slice.py:37-339): forward and the
// adjoint to the slice axes u, v.  Sample positions are formed in FP64.
#include "fvr_stencil.cuh"

namespace fvr {

// ----------------------------------------------------------------------------
// drop-in planar gather  (triton_slice.py:46-143, 145-271)
// ----------------------------------------------------------------------------

template <typename VT>
__device__ __forceinline__ float planar_at(const VT* ch, int D, int H, int W, int z, int y, int x) {
  if (z < 0 || z >= D || y < 0 || y >= H || x < 0 || x >= W) return 0.f;
  const int64_t i = (static_cast<int64_t>(z) * H + y) * W + x;
  return fvr_checked(i, static_cast<int64_t>(D) * H * W, kSitePlanar) ? ldf(ch + i) : 0.f;
}

template <typename VT>
__device__ __forceinline__ void planar_corners(const VT* base, int64_t vol_dhw, int D, int H, int W, double px,
                                               double py, double pz, Sample8& v, float& tx, float& ty, float& tz) {
  const double fx = floor(px), fy = floor(py), fz = floor(pz);
  tx = static_cast<float>(px - fx);
  ty = static_cast<float>(py - fy);
  tz = static_cast<float>(pz - fz);
  // clamp the integer base far outside the volume (all corners then read as 0)
  const double lo = -2.0;
  const int ix = static_cast<int>(fmin(fmax(fx, lo), static_cast<double>(W)));
  const int iy = static_cast<int>(fmin(fmax(fy, lo), static_cast<double>(H)));
  const int iz = static_cast<int>(fmin(fmax(fz, lo), static_cast<double>(D)));
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int z = iz + (c >> 2), y = iy + ((c >> 1) & 1), x = ix + (c & 1);
    v.re[c] = planar_at(base, D, H, W, z, y, x);
    v.im[c] = planar_at(base + vol_dhw, D, H, W, z, y, x);
  }
}

template <typename VT>
__global__ void __launch_bounds__(256) slice3d_fwd_kernel(const VT* __restrict__ vol, int D, int H, int W,
                                                          const float* __restrict__ u, const float* __restrict__ v,
                                                          int N, const float* __restrict__ fx,
                                                          const float* __restrict__ fy, int K, float cx, float cy,
                                                          float cz, VT* __restrict__ out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int bn = blockIdx.y;
  if (q >= K) return;
  const int b = bn / N, n = bn - b * N;
  const float a = __ldg(fx + q), bb = __ldg(fy + q);
  const double px = fma((double)bb, (double)__ldg(v + 3 * n + 0), fma((double)a, (double)__ldg(u + 3 * n + 0), (double)cx));
  const double py = fma((double)bb, (double)__ldg(v + 3 * n + 1), fma((double)a, (double)__ldg(u + 3 * n + 1), (double)cy));
  const double pz = fma((double)bb, (double)__ldg(v + 3 * n + 2), fma((double)a, (double)__ldg(u + 3 * n + 2), (double)cz));
  const int64_t dhw = static_cast<int64_t>(D) * H * W;
  Sample8 s;
  float tx, ty, tz;
  planar_corners(vol + static_cast<int64_t>(b) * 2 * dhw, dhw, D, H, W, px, py, pz, s, tx, ty, tz);
  Interp o;
  trilerp<false>(s, tx, ty, tz, o);
  VT* dst = out + static_cast<int64_t>(bn) * 2 * K;
  stf(dst + q, o.sr);
  stf(dst + K + q, o.si);
}

// Per (pose, tile) partial sums of dL/du, dL/dv (6 values) in fp64.
template <typename VT, typename GT>
__global__ void __launch_bounds__(256) slice3d_bwd_kernel(const VT* __restrict__ vol, int B, int D, int H, int W,
                                                          const GT* __restrict__ go, const float* __restrict__ u,
                                                          const float* __restrict__ v, int N,
                                                          const float* __restrict__ fx, const float* __restrict__ fy,
                                                          int K, float cx, float cy, float cz,
                                                          double* __restrict__ partial) {
  __shared__ double red[6 * 8];
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = blockIdx.y;
  float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (q < K) {
    const float a = __ldg(fx + q), bb = __ldg(fy + q);
    const double px = fma((double)bb, (double)__ldg(v + 3 * n + 0), fma((double)a, (double)__ldg(u + 3 * n + 0), (double)cx));
    const double py = fma((double)bb, (double)__ldg(v + 3 * n + 1), fma((double)a, (double)__ldg(u + 3 * n + 1), (double)cy));
    const double pz = fma((double)bb, (double)__ldg(v + 3 * n + 2), fma((double)a, (double)__ldg(u + 3 * n + 2), (double)cz));
    const int64_t dhw = static_cast<int64_t>(D) * H * W;
    float gx = 0.f, gy = 0.f, gz = 0.f;
    for (int b = 0; b < B; ++b) {
      Sample8 s;
      float tx, ty, tz;
      planar_corners(vol + static_cast<int64_t>(b) * 2 * dhw, dhw, D, H, W, px, py, pz, s, tx, ty, tz);
      Interp o;
      trilerp<true>(s, tx, ty, tz, o);
      const GT* g = go + (static_cast<int64_t>(b) * N + n) * 2 * K;
      const float gr = ldf(g + q), gi = ldf(g + K + q);
      gx = fmaf(gr, o.dxr, fmaf(gi, o.dxi, gx));
      gy = fmaf(gr, o.dyr, fmaf(gi, o.dyi, gy));
      gz = fmaf(gr, o.dzr, fmaf(gi, o.dzi, gz));
    }
    acc[0] = gx * a;
    acc[1] = gy * a;
    acc[2] = gz * a;
    acc[3] = gx * bb;
    acc[4] = gy * bb;
    acc[5] = gz * bb;
  }
  double tot;
  block_reduce_to_f64<6>(acc, red, &tot);
  if (threadIdx.x < 6) partial[(static_cast<int64_t>(n) * gridDim.x + blockIdx.x) * 6 + threadIdx.x] = tot;
}

__global__ void slice3d_bwd_finalize_kernel(const double* __restrict__ partial, int N, int tiles, float* gu,
                                            float* gv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N * 6) return;
  const int n = i / 6, m = i - n * 6;
  double s = 0.0;
  for (int t = 0; t < tiles; ++t) s += partial[(static_cast<int64_t>(n) * tiles + t) * 6 + m];
  if (m < 3)
    gu[n * 3 + m] = static_cast<float>(s);
  else
    gv[n * 3 + m - 3] = static_cast<float>(s);
}

}  // namespace fvr

using namespace fvr;

extern "C" {

int fvr_slice3d_fwd(const void* vol, int dtype, int64_t B, int64_t D, int64_t H, int64_t W, const float* u,
                    const float* v, int64_t N, const float* fx, const float* fy, int64_t K, float cx, float cy,
                    float cz, void* out, void* stream) {
  if (!vol || !u || !v || !fx || !fy || !out) return FVR_ERR_ARG;
  if (B < 1 || N < 1 || K < 1 || D < 1 || H < 1 || W < 1) return FVR_ERR_ARG;
  if (B * N > 65535 || K > (int64_t)1 << 30) return FVR_ERR_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  dim3 grid(static_cast<unsigned>(cdiv64(K, 256)), static_cast<unsigned>(B * N));
  switch (dtype) {
    case FVR_F32:
      slice3d_fwd_kernel<float><<<grid, 256, 0, s>>>(static_cast<const float*>(vol), (int)D, (int)H, (int)W, u, v,
                                                     (int)N, fx, fy, (int)K, cx, cy, cz, static_cast<float*>(out));
      break;
    case FVR_BF16:
      slice3d_fwd_kernel<__nv_bfloat16><<<grid, 256, 0, s>>>(static_cast<const __nv_bfloat16*>(vol), (int)D, (int)H,
                                                             (int)W, u, v, (int)N, fx, fy, (int)K, cx, cy, cz,
                                                             static_cast<__nv_bfloat16*>(out));
      break;
    case FVR_F16:
      slice3d_fwd_kernel<__half><<<grid, 256, 0, s>>>(static_cast<const __half*>(vol), (int)D, (int)H, (int)W, u, v,
                                                      (int)N, fx, fy, (int)K, cx, cy, cz, static_cast<__half*>(out));
      break;
    default:
      return FVR_ERR_DTYPE;
  }
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int64_t fvr_slice3d_bwd_workspace(int64_t N, int64_t K) { return N * cdiv64(K, 256) * 6 * (int64_t)sizeof(double); }

int fvr_slice3d_bwd(const void* vol, int dtype, int64_t B, int64_t D, int64_t H, int64_t W, const void* grad_out,
                    const float* u, const float* v, int64_t N, const float* fx, const float* fy, int64_t K, float cx,
                    float cy, float cz, float* gu, float* gv, void* workspace, int64_t ws_bytes, void* stream) {
  if (!vol || !grad_out || !u || !v || !fx || !fy || !gu || !gv || !workspace) return FVR_ERR_ARG;
  if (B < 1 || N < 1 || K < 1 || D < 1 || H < 1 || W < 1 || N > 65535) return FVR_ERR_ARG;
  if (ws_bytes < fvr_slice3d_bwd_workspace(N, K)) return FVR_ERR_WORKSPACE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int tiles = static_cast<int>(cdiv64(K, 256));
  dim3 grid(static_cast<unsigned>(tiles), static_cast<unsigned>(N));
  double* part = static_cast<double*>(workspace);
  switch (dtype) {
    case FVR_F32:
      slice3d_bwd_kernel<float, float><<<grid, 256, 0, s>>>(static_cast<const float*>(vol), (int)B, (int)D, (int)H,
                                                            (int)W, static_cast<const float*>(grad_out), u, v, (int)N,
                                                            fx, fy, (int)K, cx, cy, cz, part);
      break;
    case FVR_BF16:
      slice3d_bwd_kernel<__nv_bfloat16, __nv_bfloat16><<<grid, 256, 0, s>>>(
          static_cast<const __nv_bfloat16*>(vol), (int)B, (int)D, (int)H, (int)W,
          static_cast<const __nv_bfloat16*>(grad_out), u, v, (int)N, fx, fy, (int)K, cx, cy, cz, part);
      break;
    case FVR_F16:
      slice3d_bwd_kernel<__half, __half><<<grid, 256, 0, s>>>(static_cast<const __half*>(vol), (int)B, (int)D,
                                                              (int)H, (int)W, static_cast<const __half*>(grad_out), u,
                                                              v, (int)N, fx, fy, (int)K, cx, cy, cz, part);
      break;
    default:
      return FVR_ERR_DTYPE;
  }
  FVR_LAUNCH_CHECK();
  slice3d_bwd_finalize_kernel<<<static_cast<unsigned>(cdiv64(N * 6, 256)), 256, 0, s>>>(part, (int)N, tiles, gu, gv);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

}  // extern "C"

FVR_CHECK_ACCESSOR(check_word_slice3d)
