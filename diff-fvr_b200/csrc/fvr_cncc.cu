// Spectral NCC between two batches of centred 2D spectra, forward + adjoint.
// Image-domain loss TorchDiffFVREngine.spectral_ncc_loss
// (src/fvr/torch_engine.py:309-337): F = fftshift(fft2(img)), both sides
// multiplied by the high-pass table, ncc_b = Re sum Fp conj(Ft) /
// (sqrt(Ep Et) + 1e-8), loss = 1 - mean_b ncc_b.
#include "fvr_common.cuh"

namespace fvr {

// partial[b][tile][3] = (cross, Ep, Et) over one tile of one image pair
__global__ void __launch_bounds__(256) cncc_moments_kernel(const float2* __restrict__ Fp,
                                                           const float2* __restrict__ Ft, int64_t t_stride,
                                                           const float* __restrict__ hp, int64_t n,
                                                           double* __restrict__ partial) {
  __shared__ double red[3 * 8];
  const int b = blockIdx.y;
  float acc[3] = {0.f, 0.f, 0.f};
  for (int64_t i = blockIdx.x * 1024LL + threadIdx.x, e = 0; e < 4; ++e, i += 256) {
    if (i >= n) break;
    const float h = hp ? __ldg(hp + i) : 1.f;
    const float2 p = __ldg(Fp + b * n + i), t = __ldg(Ft + b * t_stride + i);
    const float pr = h * p.x, pi = h * p.y, tr = h * t.x, ti = h * t.y;
    acc[0] = fmaf(pr, tr, fmaf(pi, ti, acc[0]));
    acc[1] = fmaf(pr, pr, fmaf(pi, pi, acc[1]));
    acc[2] = fmaf(tr, tr, fmaf(ti, ti, acc[2]));
  }
  double tot;
  block_reduce_to_f64<3>(acc, red, &tot);
  if (threadIdx.x < 3) partial[(static_cast<int64_t>(b) * gridDim.x + blockIdx.x) * 3 + threadIdx.x] = tot;
}

__global__ void __launch_bounds__(256) cncc_finalize_kernel(const double* __restrict__ partial, int B, int tiles,
                                                            double* __restrict__ mom, float* __restrict__ loss) {
  __shared__ double red[8];
  double nsum = 0.0;
  for (int b = threadIdx.x; b < B; b += blockDim.x) {
    double v[3] = {0.0, 0.0, 0.0};
    for (int t = 0; t < tiles; ++t)
      for (int m = 0; m < 3; ++m) v[m] += partial[(static_cast<int64_t>(b) * tiles + t) * 3 + m];
    for (int m = 0; m < 3; ++m) mom[b * 3 + m] = v[m];
    nsum += v[0] / (sqrt(v[1] * v[2]) + 1e-8);
  }
  nsum = warp_sum(nsum);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = nsum;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (blockDim.x >> 5); ++w) s += red[w];
    *loss = static_cast<float>(1.0 - s / B);
  }
}

// X = dL/dFp (before the high-pass) = gc hp^2 (a Ft + 2 b Fp)
__global__ void cncc_grad_kernel(const float2* __restrict__ Fp, const float2* __restrict__ Ft, int64_t t_stride,
                                 const float* __restrict__ hp, int64_t n, int B, const double* __restrict__ mom,
                                 const float* __restrict__ g, float2* __restrict__ X) {
  const int b = blockIdx.y;
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const double cross = mom[3 * b], ep = mom[3 * b + 1], et = mom[3 * b + 2];
  const double s = sqrt(ep * et);
  const double aa = 1.0 / (s + 1e-8);
  const double bb = s > 0.0 ? -cross * et / (2.0 * s * (s + 1e-8) * (s + 1e-8)) : 0.0;
  const double gc = -static_cast<double>(*g) / B;
  const float h = hp ? hp[i] : 1.f;
  const float ca = static_cast<float>(gc * aa) * h * h, cb = static_cast<float>(gc * 2.0 * bb) * h * h;
  const float2 p = Fp[b * n + i], t = Ft[b * t_stride + i];
  X[b * n + i] = make_float2(ca * t.x + cb * p.x, ca * t.y + cb * p.y);
}

}  // namespace fvr

using namespace fvr;

extern "C" {

int64_t fvr_cncc_workspace(int64_t B, int64_t n) { return B * cdiv64(n, 1024) * 3 * (int64_t)sizeof(double); }

int fvr_cncc_forward(const void* Fp, const void* Ft, int64_t B, int64_t Bt, int64_t n, const float* hp,
                     void* workspace, int64_t ws_bytes, double* mom, float* loss, void* stream) {
  if (!Fp || !Ft || !workspace || !mom || !loss || B < 1 || n < 1 || B > 65535) return FVR_ERR_ARG;
  if (Bt != 1 && Bt != B) return FVR_ERR_ARG;
  if (ws_bytes < fvr_cncc_workspace(B, n)) return FVR_ERR_WORKSPACE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int tiles = static_cast<int>(cdiv64(n, 1024));
  cncc_moments_kernel<<<dim3(tiles, (unsigned)B), 256, 0, s>>>(
      static_cast<const float2*>(Fp), static_cast<const float2*>(Ft), Bt == 1 ? 0 : n, hp, n,
      static_cast<double*>(workspace));
  FVR_LAUNCH_CHECK();
  cncc_finalize_kernel<<<1, 256, 0, s>>>(static_cast<double*>(workspace), (int)B, tiles, mom, loss);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_cncc_backward(const void* Fp, const void* Ft, int64_t B, int64_t Bt, int64_t n, const float* hp,
                      const double* mom, const float* g, void* X, void* stream) {
  if (!Fp || !Ft || !mom || !g || !X || B < 1 || n < 1 || B > 65535) return FVR_ERR_ARG;
  if (Bt != 1 && Bt != B) return FVR_ERR_ARG;
  cncc_grad_kernel<<<dim3((unsigned)cdiv64(n, 256), (unsigned)B), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const float2*>(Fp), static_cast<const float2*>(Ft), Bt == 1 ? 0 : n, hp, n, (int)B, mom, g,
      static_cast<float2*>(X));
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

}  // extern "C"
