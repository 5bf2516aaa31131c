// SE(3) exponential map for batched pose parameters, fp64 inside, sm_100a.
//
// theta[n] = (w_x, w_y, w_z, t_x, t_y, t_z) (rad, mm) -> 4x4 rigid matrix
// [[R(w), t], [0, 1]] with R(w) = exp([w]x) (Rodrigues:
// I + A [w]x + B [w]x^2, A = sin(a)/a, B = (1 - cos a)/a^2, a = |w|), the map
// the reference builds with torch.matrix_exp of the skew matrix
// (experiments/exp30_gpu_multistart_registration.py:42-55,
// tests/test_cone_beam_fvr.py:221-229).  The adjoint maps dL/dT to dL/dtheta
// with dR/dw_i = (w_i [w]x + [w x (I - R) e_i]x) R / a^2 (series below a
// small angle).
#include "fvr_common.cuh"

namespace fvr {

struct M3 {
  double m[3][3];
};

__device__ __forceinline__ M3 skew(double x, double y, double z) {
  return M3{{{0.0, -z, y}, {z, 0.0, -x}, {-y, x, 0.0}}};
}

__device__ __forceinline__ M3 mul(const M3& a, const M3& b) {
  M3 r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j] + a.m[i][2] * b.m[2][j];
  return r;
}

// R(w) and a^2 = |w|^2
__device__ __forceinline__ M3 so3_exp(const double w[3], double* a2_out) {
  const double a2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  double A, B;
  if (a2 < 1e-10) {  // Taylor to the rounding level at |w| < 1e-5
    A = 1.0 - a2 / 6.0;
    B = 0.5 - a2 / 24.0;
  } else {
    const double a = sqrt(a2);
    double s, c;
    sincos(a, &s, &c);
    A = s / a;
    B = (1.0 - c) / a2;
  }
  const M3 K = skew(w[0], w[1], w[2]);
  const M3 K2 = mul(K, K);
  M3 R;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) R.m[i][j] = (i == j ? 1.0 : 0.0) + A * K.m[i][j] + B * K2.m[i][j];
  *a2_out = a2;
  return R;
}

__global__ void se3_exp_kernel(const float* __restrict__ theta, int64_t N, float* __restrict__ mats) {
  const int64_t n = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const float* p = theta + 6 * n;
  const double w[3] = {p[0], p[1], p[2]};
  double a2;
  const M3 R = so3_exp(w, &a2);
  float* o = mats + 16 * n;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) o[4 * i + j] = static_cast<float>(R.m[i][j]);
    o[4 * i + 3] = p[3 + i];
  }
  o[12] = o[13] = o[14] = 0.f;
  o[15] = 1.f;
}

__global__ void se3_exp_bwd_kernel(const float* __restrict__ theta, const float* __restrict__ gmats, int64_t N,
                                   float* __restrict__ gtheta) {
  const int64_t n = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const float* p = theta + 6 * n;
  const float* g = gmats + 16 * n;
  const double w[3] = {p[0], p[1], p[2]};
  double a2;
  const M3 R = so3_exp(w, &a2);
  const M3 K = skew(w[0], w[1], w[2]);
  float* o = gtheta + 6 * n;
  for (int i = 0; i < 3; ++i) {
    M3 dR;
    const M3 Ei = skew(i == 0, i == 1, i == 2);
    if (a2 < 1e-10) {
      // d/dw_i of I + K + K^2/2: E_i + (E_i K + K E_i) / 2
      const M3 EK = mul(Ei, K), KE = mul(K, Ei);
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) dR.m[r][c] = Ei.m[r][c] + 0.5 * (EK.m[r][c] + KE.m[r][c]);
    } else {
      // (w_i K + [w x (I - R) e_i]x) R / a^2
      const double ce[3] = {(i == 0) - R.m[0][i], (i == 1) - R.m[1][i], (i == 2) - R.m[2][i]};
      const double x[3] = {w[1] * ce[2] - w[2] * ce[1], w[2] * ce[0] - w[0] * ce[2], w[0] * ce[1] - w[1] * ce[0]};
      const M3 S = skew(x[0], x[1], x[2]);
      M3 L;
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) L.m[r][c] = (w[i] * K.m[r][c] + S.m[r][c]) / a2;
      dR = mul(L, R);
    }
    double s = 0.0;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) s += static_cast<double>(g[4 * r + c]) * dR.m[r][c];
    o[i] = static_cast<float>(s);
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) o[3 + i] = g[4 * i + 3];
}

}  // namespace fvr

using namespace fvr;

extern "C" {

int fvr_se3_exp(const float* theta, int64_t N, float* mats, void* stream) {
  if (!theta || !mats || N < 1) return FVR_ERR_ARG;
  se3_exp_kernel<<<static_cast<unsigned>(cdiv64(N, 128)), 128, 0, static_cast<cudaStream_t>(stream)>>>(theta, N,
                                                                                                       mats);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_se3_exp_backward(const float* theta, const float* grad_mats, int64_t N, float* grad_theta, void* stream) {
  if (!theta || !grad_mats || !grad_theta || N < 1) return FVR_ERR_ARG;
  se3_exp_bwd_kernel<<<static_cast<unsigned>(cdiv64(N, 128)), 128, 0, static_cast<cudaStream_t>(stream)>>>(
      theta, grad_mats, N, grad_theta);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

}  // extern "C"
