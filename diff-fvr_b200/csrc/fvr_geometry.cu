// Geometry tables of the PoU-FVR pinhole path and the spine phantom, in FP64
// (lattice) and exact float32 (phantom) on sm_100a.
//
// Pinhole lattice.  A pixel (row r, column c) of an H x W detector looks
// along the camera-frame direction d = K^-1 (c + 1/2, r + 1/2, 1); its
// detector point is q = d * sdd / max(d_z, 1e-6), on the plane z = sdd.  The
// detector's axes are the unit vectors along its first row (u0) and first
// column (v0); its normal n0 is the unit v0 x u0, turned so that it points
// from the source (the camera origin) towards the lattice's centroid.  Each
// pixel then carries three SE(3)-invariant ray numbers: with the unit ray
// r = q / |q|, ic = 1 / max(r.n0, 0.1) (obliquity), rx = (r.u0) ic and
// ry = (r.v0) ic (the ray's in-plane slopes).  Everything is formed in
// FP64 and stored as float32.  Replaces the lattice and ray cache of
// PerspectiveSlabFVR (src/fvr/cone_beam_fvr.py:523-545, 575-596, 705-728).
//
// Spine phantom.  Every voxel evaluates the phantom's shape tests in the
// order the reference draws them (later shapes overwrite earlier ones), each
// test in float32 with round-to-nearest operations and no contraction, so
// the HU labels equal those of the NumPy float32 construction bit for bit.
// Replaces create_spine_phantom (src/fvr/dicom_loader.py:114-176).

#include "fvr_common.cuh"

namespace fvr {
namespace {

struct Mat3 {
  double m[9];
};

__device__ __forceinline__ void pinhole_point(const Mat3& k, double sdd, int r, int c, double q[3]) {
  const double px = c + 0.5, py = r + 0.5;
  double d[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) d[i] = fma(k.m[3 * i], px, fma(k.m[3 * i + 1], py, k.m[3 * i + 2]));
  const double s = sdd / fmax(d[2], 1e-6);
#pragma unroll
  for (int i = 0; i < 3; ++i) q[i] = d[i] * s;
}

__device__ __forceinline__ void unit3(double v[3]) {
  const double inv = 1.0 / (sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) + 1e-12);
  v[0] *= inv;
  v[1] *= inv;
  v[2] *= inv;
}

// One CTA: centroid of the detector points (FP64 block sum), then the basis.
__global__ void __launch_bounds__(256) pinhole_basis_kernel(Mat3 k, double sdd, int H, int W, double* basis) {
  __shared__ double red[3][8];
  double acc[3] = {0.0, 0.0, 0.0};
  const int64_t n = static_cast<int64_t>(H) * W;
  for (int64_t p = threadIdx.x; p < n; p += blockDim.x) {
    double q[3];
    pinhole_point(k, sdd, static_cast<int>(p / W), static_cast<int>(p % W), q);
    acc[0] += q[0];
    acc[1] += q[1];
    acc[2] += q[2];
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const double v = warp_sum(acc[i]);
    if (lane == 0) red[i][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  double cen[3];
  for (int i = 0; i < 3; ++i) {
    double s = 0.0;
    for (int w = 0; w < 8; ++w) s += red[i][w];
    cen[i] = s / static_cast<double>(n);
  }
  double q00[3], q0w[3], qh0[3];
  pinhole_point(k, sdd, 0, 0, q00);
  pinhole_point(k, sdd, 0, W - 1, q0w);
  pinhole_point(k, sdd, H - 1, 0, qh0);
  double u[3], v[3], nn[3];
  for (int i = 0; i < 3; ++i) {
    u[i] = q0w[i] - q00[i];
    v[i] = qh0[i] - q00[i];
  }
  unit3(u);
  unit3(v);
  nn[0] = v[1] * u[2] - v[2] * u[1];
  nn[1] = v[2] * u[0] - v[0] * u[2];
  nn[2] = v[0] * u[1] - v[1] * u[0];
  unit3(nn);
  const double side = cen[0] * nn[0] + cen[1] * nn[1] + cen[2] * nn[2];
  if (side < 0.0) {
    nn[0] = -nn[0];
    nn[1] = -nn[1];
    nn[2] = -nn[2];
  }
  for (int i = 0; i < 3; ++i) {
    basis[i] = u[i];
    basis[3 + i] = v[i];
    basis[6 + i] = nn[i];
  }
}

__global__ void __launch_bounds__(256) pinhole_rays_kernel(Mat3 k, double sdd, int H, int W,
                                                           const double* __restrict__ basis, float* __restrict__ trg,
                                                           float* __restrict__ rx, float* __restrict__ ry,
                                                           float* __restrict__ ic) {
  const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= static_cast<int64_t>(H) * W) return;
  double q[3];
  pinhole_point(k, sdd, static_cast<int>(p / W), static_cast<int>(p % W), q);
  const double inv_len = 1.0 / sqrt(fmax(q[0] * q[0] + q[1] * q[1] + q[2] * q[2], 1e-12));
  double dots[3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
    dots[a] = (q[0] * __ldg(basis + 3 * a) + q[1] * __ldg(basis + 3 * a + 1) + q[2] * __ldg(basis + 3 * a + 2)) *
              inv_len;
  const double inv_cos = 1.0 / fmax(dots[2], 0.1);
  trg[3 * p] = static_cast<float>(q[0]);
  trg[3 * p + 1] = static_cast<float>(q[1]);
  trg[3 * p + 2] = static_cast<float>(q[2]);
  rx[p] = static_cast<float>(dots[0] * inv_cos);
  ry[p] = static_cast<float>(dots[1] * inv_cos);
  ic[p] = static_cast<float>(inv_cos);
}

// ------------------------------------------------------------ phantom ----
constexpr int kVertebrae = 5;

struct PhantomConst {
  float center, torso_ax, torso_ay;  // centre, torso semi-axes (x, y)
  float body_y, body_r2, inner_r2;   // vertebral body centre y, radius^2, trabecular radius^2
  float canal_y, canal_r2;           // spinal canal centre y, radius^2
  float spin_hw, spin_top;           // spinous process half-width, posterior end (y)
  float tr_hw, tr_out, tr_in;        // transverse process half-height (y), outer / inner |x - c|
  float vz[kVertebrae], half_h[kVertebrae], tr_half_h[kVertebrae];
};

__device__ __forceinline__ float sq_rn(float a) { return __fmul_rn(a, a); }

__global__ void __launch_bounds__(256) spine_phantom_kernel(PhantomConst pc, int n, float* __restrict__ out) {
  const int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t nn = static_cast<int64_t>(n) * n;
  if (idx >= nn * n) return;
  const float z = static_cast<float>(idx / nn);
  const float y = static_cast<float>((idx / n) % n);
  const float x = static_cast<float>(idx % n);
  float hu = -1000.0f;
  const float dx = __fsub_rn(x, pc.center);
  if (__fadd_rn(sq_rn(__fdiv_rn(dx, pc.torso_ax)), sq_rn(__fdiv_rn(__fsub_rn(y, pc.center), pc.torso_ay))) <= 1.0f)
    hu = 40.0f;
  const float body_d2 = __fadd_rn(sq_rn(dx), sq_rn(__fsub_rn(y, pc.body_y)));
  const float canal_d2 = __fadd_rn(sq_rn(dx), sq_rn(__fsub_rn(y, pc.canal_y)));
  const float adx = fabsf(dx);
  const float ady_canal = fabsf(__fsub_rn(y, pc.canal_y));
#pragma unroll
  for (int i = 0; i < kVertebrae; ++i) {
    const float adz = fabsf(__fsub_rn(z, pc.vz[i]));
    if (adz <= pc.half_h[i]) {
      if (body_d2 <= pc.body_r2) hu = 1100.0f;
      if (body_d2 <= pc.inner_r2) hu = 400.0f;
      if (canal_d2 <= pc.canal_r2) hu = 15.0f;
      if (adx <= pc.spin_hw && y >= pc.canal_y && y <= pc.spin_top) hu = 900.0f;
    }
    if (ady_canal <= pc.tr_hw && adx <= pc.tr_out && adx >= pc.tr_in && adz <= pc.tr_half_h[i]) hu = 850.0f;
  }
  out[idx] = hu;
}

}  // namespace
}  // namespace fvr

using namespace fvr;

extern "C" {

int fvr_pou_pinhole_lattice(const double* k_inv, double sdd_mm, int64_t H, int64_t W, float* trg0, float* rx,
                            float* ry, float* ic, double* basis, void* stream) {
  if (!k_inv || !trg0 || !rx || !ry || !ic || !basis || H < 1 || W < 1 || H * W > (int64_t)1 << 30)
    return FVR_ERR_ARG;
  Mat3 k;
  for (int i = 0; i < 9; ++i) k.m[i] = k_inv[i];
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  pinhole_basis_kernel<<<1, 256, 0, s>>>(k, sdd_mm, (int)H, (int)W, basis);
  FVR_LAUNCH_CHECK();
  pinhole_rays_kernel<<<static_cast<unsigned>(cdiv64(H * W, 256)), 256, 0, s>>>(k, sdd_mm, (int)H, (int)W, basis,
                                                                                 trg0, rx, ry, ic);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_spine_phantom(int64_t n, float* out, void* stream) {
  if (!out || n < 1 || n > 2048) return FVR_ERR_ARG;
  // The reference forms these constants in double precision; each one meets
  // the float32 voxel coordinates as a float32 operand.
  const double sz = static_cast<double>(n), c = sz / 2.0, period = sz / kVertebrae;
  const double r_body = 0.12 * sz, r_canal = 0.055 * sz;
  PhantomConst pc;
  pc.center = static_cast<float>(c);
  pc.torso_ax = static_cast<float>(0.38 * sz);
  pc.torso_ay = static_cast<float>(0.32 * sz);
  pc.body_y = static_cast<float>(c - 0.06 * sz);
  pc.body_r2 = static_cast<float>(r_body * r_body);
  pc.inner_r2 = static_cast<float>((r_body * 0.75) * (r_body * 0.75));
  pc.canal_y = static_cast<float>(c + 0.08 * sz);
  pc.canal_r2 = static_cast<float>(r_canal * r_canal);
  pc.spin_hw = static_cast<float>(0.03 * sz);
  pc.spin_top = static_cast<float>(c + 0.22 * sz);
  pc.tr_hw = static_cast<float>(0.04 * sz);
  pc.tr_out = static_cast<float>(0.24 * sz);
  pc.tr_in = static_cast<float>(0.07 * sz);
  for (int i = 0; i < kVertebrae; ++i) {
    const double height = period * 0.72;
    pc.vz[i] = static_cast<float>((i + 0.5) * period);
    pc.half_h[i] = static_cast<float>(height / 2.0);
    pc.tr_half_h[i] = static_cast<float>(height * 0.35);
  }
  const int64_t total = n * n * n;
  spine_phantom_kernel<<<static_cast<unsigned>(cdiv64(total, 256)), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      pc, (int)n, out);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

}  // extern "C"
