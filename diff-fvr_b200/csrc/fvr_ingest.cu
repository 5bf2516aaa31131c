// Volume ingest on the GPU (src/fvr/dicom_loader.py:11-30, 179-188): a CT
// (HU, float32 [Z][Y][X], anisotropic spacing) is resampled into an isotropic
// target_res^3 cube that keeps its whole physical field of view centred
// (scipy.ndimage.affine_transform with a diagonal matrix, order 1, mode
// 'constant', cval -1000 HU: air outside), optionally converted to linear
// attenuation mu = max(0, (HU + 1000) / 1000) in the same pass, ready for the
// spectrum precompute.
#include "fvr_common.cuh"

namespace fvr {

struct IngestArgs {
  const float* hu;
  int Z, Y, X, N;
  double ratio[3], offset[3];  // input coordinate = ratio * output index + offset, per (Z, Y, X)
  int to_mu;
  float* out;  // [N][N][N]
};

// Linear interpolation with scipy 'constant' semantics: cval unless
// 0 <= c <= n - 1 on every axis; inside, the upper neighbour is clamped.
__global__ void __launch_bounds__(256) ingest_resample_kernel(IngestArgs a) {
  const int64_t n3 = static_cast<int64_t>(a.N) * a.N * a.N;
  for (int64_t q = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; q < n3;
       q += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int ox = static_cast<int>(q % a.N), oy = static_cast<int>((q / a.N) % a.N),
              oz = static_cast<int>(q / (static_cast<int64_t>(a.N) * a.N));
    // offset + matrix row . index, summed as scipy sums it (no fused multiply-add)
    const double cz = __dadd_rn(a.offset[0], __dmul_rn(a.ratio[0], static_cast<double>(oz)));
    const double cy = __dadd_rn(a.offset[1], __dmul_rn(a.ratio[1], static_cast<double>(oy)));
    const double cx = __dadd_rn(a.offset[2], __dmul_rn(a.ratio[2], static_cast<double>(ox)));
    double v = -1000.0;
    if (cz >= 0.0 && cz <= a.Z - 1 && cy >= 0.0 && cy <= a.Y - 1 && cx >= 0.0 && cx <= a.X - 1) {
      const double fz = floor(cz), fy = floor(cy), fx = floor(cx);
      const int iz = static_cast<int>(fz), iy = static_cast<int>(fy), ix = static_cast<int>(fx);
      const int iz1 = min(iz + 1, a.Z - 1), iy1 = min(iy + 1, a.Y - 1), ix1 = min(ix + 1, a.X - 1);
      const double tz = cz - fz, ty = cy - fy, tx = cx - fx;
      const int zs[2] = {iz, iz1}, ys[2] = {iy, iy1}, xs[2] = {ix, ix1};
      const double wz[2] = {1.0 - tz, tz}, wy[2] = {1.0 - ty, ty}, wx[2] = {1.0 - tx, tx};
      v = 0.0;
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int k = 0; k < 2; ++k)
            v += wz[i] * wy[j] * wx[k] *
                 static_cast<double>(__ldg(a.hu + (static_cast<int64_t>(zs[i]) * a.Y + ys[j]) * a.X + xs[k]));
    }
    float h = static_cast<float>(v);
    if (a.to_mu) h = fmaxf(0.f, __fdiv_rn(__fadd_rn(h, 1000.f), 1000.f));  // float32 as the reference computes it
    a.out[q] = h;
  }
}

__global__ void __launch_bounds__(256) hu_to_mu_kernel(const float* __restrict__ hu, int64_t n, float* __restrict__ out) {
  for (int64_t q = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; q < n;
       q += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[q] = fmaxf(0.f, __fdiv_rn(__fadd_rn(__ldg(hu + q), 1000.f), 1000.f));
}

}  // namespace fvr

using namespace fvr;

extern "C" {

int fvr_ingest_resample(const float* hu, int64_t Z, int64_t Y, int64_t X, double sz, double sy, double sx,
                        int64_t target_res, int to_mu, float* out, double* voxel_mm, void* stream) {
  if (!hu || !out || Z < 2 || Y < 2 || X < 2 || target_res < 2 || target_res > 4096) return FVR_ERR_ARG;
  if (!(sz > 0.0) || !(sy > 0.0) || !(sx > 0.0)) return FVR_ERR_ARG;
  const double ext[3] = {static_cast<double>(Z) * sz, static_cast<double>(Y) * sy, static_cast<double>(X) * sx};
  const double vmm = fmax(fmax(ext[0], ext[1]), ext[2]) / static_cast<double>(target_res);
  const double sp[3] = {sz, sy, sx};
  const int64_t shp[3] = {Z, Y, X};
  IngestArgs a{};
  a.hu = hu;
  a.Z = static_cast<int>(Z);
  a.Y = static_cast<int>(Y);
  a.X = static_cast<int>(X);
  a.N = static_cast<int>(target_res);
  for (int k = 0; k < 3; ++k) {
    a.ratio[k] = vmm / sp[k];
    a.offset[k] = static_cast<double>(shp[k] - 1) / 2.0 - a.ratio[k] * static_cast<double>(target_res - 1) / 2.0;
  }
  a.to_mu = to_mu ? 1 : 0;
  a.out = out;
  const int64_t n3 = target_res * target_res * target_res;
  const int64_t nb = cdiv64(n3, 256);
  const unsigned blocks = static_cast<unsigned>(nb < 148 * 16 ? nb : 148 * 16);
  ingest_resample_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(a);
  FVR_LAUNCH_CHECK();
  if (voxel_mm) *voxel_mm = vmm;
  return FVR_OK;
}

int fvr_hu_to_attenuation(const float* hu, int64_t n, float* out, void* stream) {
  if (!hu || !out || n < 1) return FVR_ERR_ARG;
  const int64_t nb = cdiv64(n, 256);
  const unsigned blocks = static_cast<unsigned>(nb < 148 * 16 ? nb : 148 * 16);
  hu_to_mu_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(hu, n, out);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

}  // extern "C"
