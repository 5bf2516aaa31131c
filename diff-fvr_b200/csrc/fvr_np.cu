// NumPy-convention Diff-FVR kernels (src/fvr/diff_fvr.py, src/fvr/gradients.py), fp64, sm_100a.
//
// A batch of (pose, view) items is sliced from the fp64 centred spectrum with
// scipy map_coordinates(order=1, mode='constant') semantics (zero unless
// 0 <= coordinate <= n-1 on every axis), phase-ramped, and either written out
// or reduced against per-item target spectra into the moments the spectral
// NCC and its closed-form translation gradient need.
#include "fvr_common.cuh"

namespace fvr {

struct NpItem {
  double yaw, pitch, roll;  // degrees
  double tx, ty;            // in-plane translation, voxels
  int view;                 // 0 lateral, 1 ap, 2 axial
  int sh, sw;               // slice rows, columns
  int pad_;
  long long off;            // element offset of the item's slice / target
};

// basis of diff_fvr.py:56-104: rot = rz(yaw) . ry(roll) . rx(pitch) on (Z, Y, X)
__device__ __forceinline__ void np_basis(const NpItem& it, double u[3], double v[3]) {
  double sy, cy, sp, cp, sr, cr;
  sincospi(it.yaw / 180.0, &sy, &cy);
  sincospi(it.pitch / 180.0, &sp, &cp);
  sincospi(it.roll / 180.0, &sr, &cr);
  const double rz[3][3] = {{1, 0, 0}, {0, cy, -sy}, {0, sy, cy}};
  const double ry[3][3] = {{cr, 0, sr}, {0, 1, 0}, {-sr, 0, cr}};
  const double rx[3][3] = {{cp, -sp, 0}, {sp, cp, 0}, {0, 0, 1}};
  double t[3][3], r[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) t[i][j] = ry[i][0] * rx[0][j] + ry[i][1] * rx[1][j] + ry[i][2] * rx[2][j];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r[i][j] = rz[i][0] * t[0][j] + rz[i][1] * t[1][j] + rz[i][2] * t[2][j];
  // u_base / v_base per view (diff_fvr.py:90-100)
  const int ui = it.view == 0 ? 1 : 2;  // lateral: wy, ap / axial: wx
  const int vi = it.view == 2 ? 1 : 0;  // axial: wy, else wz
  for (int k = 0; k < 3; ++k) {
    u[k] = r[k][ui];
    v[k] = r[k][vi];
  }
}

// map_coordinates order 1, mode 'constant' on interleaved complex f3d[D][H][W]
__device__ __forceinline__ double2 np_sample(const double2* __restrict__ f, int D, int H, int W, double z, double y,
                                             double x) {
  if (!(z >= 0.0 && z <= D - 1 && y >= 0.0 && y <= H - 1 && x >= 0.0 && x <= W - 1)) return make_double2(0.0, 0.0);
  const double fz = floor(z), fy = floor(y), fx = floor(x);
  const int iz = static_cast<int>(fz), iy = static_cast<int>(fy), ix = static_cast<int>(fx);
  const double tz = z - fz, ty = y - fy, tx = x - fx;
  const int iz1 = min(iz + 1, D - 1), iy1 = min(iy + 1, H - 1), ix1 = min(ix + 1, W - 1);
  const int zs[2] = {iz, iz1}, ys[2] = {iy, iy1}, xs[2] = {ix, ix1};
  const double wz[2] = {1.0 - tz, tz}, wy[2] = {1.0 - ty, ty}, wx[2] = {1.0 - tx, tx};
  double re = 0.0, im = 0.0;
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const double w = wz[a] * wy[b] * wx[c];
        const int64_t e = (static_cast<int64_t>(zs[a]) * H + ys[b]) * W + xs[c];
        const double2 v = fvr_checked(e, static_cast<int64_t>(D) * H * W, kSiteNpGather) ? __ldg(f + e)
                                                                                          : make_double2(0.0, 0.0);
        re += w * v.x;
        im += w * v.y;
      }
  return make_double2(re, im);
}

// Phase-ramped slice value at (row i, column j) of an item (diff_fvr.py:120-150)
__device__ __forceinline__ double2 np_slice_value(const double2* __restrict__ f, int D, int H, int W,
                                                  const NpItem& it, const double u[3], const double v[3], int i,
                                                  int j, double& uu, double& vv) {
  // linspace(-n/2, n/2, n, endpoint=False): step 1
  uu = -0.5 * it.sw + j;
  vv = -0.5 * it.sh + i;
  const double z = uu * u[0] + vv * v[0] + 0.5 * D;
  const double y = uu * u[1] + vv * v[1] + 0.5 * H;
  const double x = uu * u[2] + vv * v[2] + 0.5 * W;
  double2 s = np_sample(f, D, H, W, z, y, x);
  if (it.tx != 0.0 || it.ty != 0.0) {
    double sn, cs;
    sincospi(-2.0 * (uu * it.tx / it.sw + vv * it.ty / it.sh), &sn, &cs);
    s = make_double2(s.x * cs - s.y * sn, s.x * sn + s.y * cs);
  }
  return s;
}

__global__ void __launch_bounds__(256) np_slice_kernel(const double2* __restrict__ f, int D, int H, int W,
                                                       const NpItem* __restrict__ items, double2* __restrict__ out) {
  const NpItem it = items[blockIdx.y];
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= it.sh * it.sw) return;
  double u[3], v[3];
  np_basis(it, u, v);
  double uu, vv;
  out[it.off + q] = np_slice_value(f, D, H, W, it, u, v, q / it.sw, q % it.sw, uu, vv);
}

// per (item, tile): cross = Re sum S conj T, ES = sum |S|^2, ET = sum |T|^2,
// IU = sum u Im(S conj T), IV = sum v Im(S conj T)
__global__ void __launch_bounds__(256) np_ncc_kernel(const double2* __restrict__ f, int D, int H, int W,
                                                     const NpItem* __restrict__ items,
                                                     const double2* __restrict__ targets, int tiles,
                                                     double* __restrict__ partial) {
  __shared__ double red[5 * 8];
  const NpItem it = items[blockIdx.y];
  double acc[5] = {0, 0, 0, 0, 0};
  double u[3], v[3];
  np_basis(it, u, v);
  const int n = it.sh * it.sw;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += tiles * blockDim.x) {
    double uu, vv;
    const double2 s = np_slice_value(f, D, H, W, it, u, v, q / it.sw, q % it.sw, uu, vv);
    const double2 t = __ldg(targets + it.off + q);
    const double cr = s.x * t.x + s.y * t.y, ci = s.y * t.x - s.x * t.y;  // S conj T
    acc[0] += cr;
    acc[1] += s.x * s.x + s.y * s.y;
    acc[2] += t.x * t.x + t.y * t.y;
    acc[3] += uu * ci;
    acc[4] += vv * ci;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int m = 0; m < 5; ++m) {
    const double s = warp_sum(acc[m]);
    if (lane == 0) red[m * nw + wid] = s;
  }
  __syncthreads();
  if (threadIdx.x < 5) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += red[threadIdx.x * nw + w];
    partial[(static_cast<int64_t>(blockIdx.y) * tiles + blockIdx.x) * 5 + threadIdx.x] = s;
  }
}

__global__ void np_ncc_finalize_kernel(const double* __restrict__ partial, int n_items, int tiles,
                                       double* __restrict__ mom) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_items * 5) return;
  const int item = i / 5, m = i % 5;
  double s = 0.0;
  for (int t = 0; t < tiles; ++t) s += partial[(static_cast<int64_t>(item) * tiles + t) * 5 + m];
  mom[i] = s;
}

constexpr int kNpTiles = 64;

// Articulated (multi-segment) spectrum: output o is the sum, in segment order,
// of the phase-ramped slices of segment spectra f[s] at item (o, s)
// (articulated_spine.py:39-71, Fourier linearity); every segment spectrum has
// the same padded shape.  Items are [n_out][n_seg]; output o is written at
// the offset of item (o, 0).
constexpr int kMaxSegments = 16;
struct SegSpectra {
  const double2* f[kMaxSegments];
};

__global__ void __launch_bounds__(256) np_segment_sum_kernel(const __grid_constant__ SegSpectra sp, int n_seg, int D,
                                                             int H, int W, const NpItem* __restrict__ items,
                                                             double2* __restrict__ out) {
  __shared__ NpItem s_it[kMaxSegments];
  __shared__ double s_uv[kMaxSegments][6];
  const int o = blockIdx.y;
  if (threadIdx.x < n_seg) {
    const NpItem it = items[static_cast<int64_t>(o) * n_seg + threadIdx.x];
    double u[3], v[3];
    np_basis(it, u, v);
    s_it[threadIdx.x] = it;
    for (int k = 0; k < 3; ++k) {
      s_uv[threadIdx.x][k] = u[k];
      s_uv[threadIdx.x][3 + k] = v[k];
    }
  }
  __syncthreads();
  const int sh = s_it[0].sh, sw = s_it[0].sw;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= sh * sw) return;
  const int i = q / sw, j = q - (q / sw) * sw;
  double2 sum = make_double2(0.0, 0.0);
  for (int s = 0; s < n_seg; ++s) {
    const double u[3] = {s_uv[s][0], s_uv[s][1], s_uv[s][2]}, v[3] = {s_uv[s][3], s_uv[s][4], s_uv[s][5]};
    double uu, vv;
    const double2 x = np_slice_value(sp.f[s], D, H, W, s_it[s], u, v, i, j, uu, vv);
    sum.x += x.x;
    sum.y += x.y;
  }
  out[s_it[0].off + q] = sum;
}

// Moments of two complex fp64 [sh][sw] arrays on the slice grid
// u = j - sw/2, v = i - sh/2: (Re sum a conj b, sum |a|^2, sum |b|^2,
// sum u Im(a conj b), sum v Im(a conj b))
__global__ void __launch_bounds__(256) np_pair_kernel(const double2* __restrict__ a, const double2* __restrict__ b,
                                                      int sh, int sw, double* __restrict__ partial) {
  __shared__ double red[5 * 8];
  double acc[5] = {0, 0, 0, 0, 0};
  const int64_t n = static_cast<int64_t>(sh) * sw;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double2 x = __ldg(a + i), y = __ldg(b + i);
    const double ci = x.y * y.x - x.x * y.y;
    acc[0] += x.x * y.x + x.y * y.y;
    acc[1] += x.x * x.x + x.y * x.y;
    acc[2] += y.x * y.x + y.y * y.y;
    acc[3] += (static_cast<double>(i % sw) - 0.5 * sw) * ci;
    acc[4] += (static_cast<double>(i / sw) - 0.5 * sh) * ci;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int m = 0; m < 5; ++m) {
    const double s = warp_sum(acc[m]);
    if (lane == 0) red[m * nw + wid] = s;
  }
  __syncthreads();
  if (threadIdx.x < 5) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += red[threadIdx.x * nw + w];
    partial[blockIdx.x * 5 + threadIdx.x] = s;
  }
}
}  // namespace fvr

using namespace fvr;

extern "C" {

int64_t fvr_np_item_bytes(void) { return sizeof(NpItem); }

int fvr_np_slices(const void* f3d, int64_t D, int64_t H, int64_t W, const void* items, int64_t n_items,
                  int64_t max_n, void* out, void* stream) {
  if (!f3d || !items || !out || n_items < 1 || n_items > 65535 || max_n < 1 || D < 2 || H < 2 || W < 2)
    return FVR_ERR_ARG;
  np_slice_kernel<<<dim3((unsigned)cdiv64(max_n, 256), (unsigned)n_items), 256, 0,
                    static_cast<cudaStream_t>(stream)>>>(static_cast<const double2*>(f3d), (int)D, (int)H, (int)W,
                                                        static_cast<const NpItem*>(items),
                                                        static_cast<double2*>(out));
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_np_segment_slices(const void* const* f3ds, int64_t n_seg, int64_t D, int64_t H, int64_t W, const void* items,
                          int64_t n_out, int64_t max_n, void* out, void* stream) {
  if (!f3ds || !items || !out || n_seg < 1 || n_seg > kMaxSegments || n_out < 1 || n_out > 65535 || max_n < 1 ||
      D < 2 || H < 2 || W < 2)
    return FVR_ERR_ARG;
  SegSpectra sp{};
  for (int64_t k = 0; k < n_seg; ++k) {
    if (!f3ds[k]) return FVR_ERR_ARG;
    sp.f[k] = static_cast<const double2*>(f3ds[k]);
  }
  np_segment_sum_kernel<<<dim3((unsigned)cdiv64(max_n, 256), (unsigned)n_out), 256, 0,
                          static_cast<cudaStream_t>(stream)>>>(sp, (int)n_seg, (int)D, (int)H, (int)W,
                                                               static_cast<const NpItem*>(items),
                                                               static_cast<double2*>(out));
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int64_t fvr_np_ncc_workspace(int64_t n_items) { return n_items * kNpTiles * 5 * (int64_t)sizeof(double); }

int fvr_np_ncc_moments(const void* f3d, int64_t D, int64_t H, int64_t W, const void* items, int64_t n_items,
                       const void* targets, void* workspace, int64_t ws_bytes, double* mom, void* stream) {
  if (!f3d || !items || !targets || !workspace || !mom || n_items < 1 || n_items > 65535 || D < 2 || H < 2 || W < 2)
    return FVR_ERR_ARG;
  if (ws_bytes < fvr_np_ncc_workspace(n_items)) return FVR_ERR_WORKSPACE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* part = static_cast<double*>(workspace);
  np_ncc_kernel<<<dim3(kNpTiles, (unsigned)n_items), 256, 0, s>>>(static_cast<const double2*>(f3d), (int)D, (int)H,
                                                                  (int)W, static_cast<const NpItem*>(items),
                                                                  static_cast<const double2*>(targets), kNpTiles, part);
  FVR_LAUNCH_CHECK();
  np_ncc_finalize_kernel<<<(unsigned)cdiv64(n_items * 5, 128), 128, 0, s>>>(part, (int)n_items, kNpTiles, mom);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int64_t fvr_np_pair_workspace(void) { return kNpTiles * 5 * (int64_t)sizeof(double); }

int fvr_np_pair_moments(const void* a, const void* b, int64_t sh, int64_t sw, void* workspace, int64_t ws_bytes,
                        double* mom, void* stream) {
  if (!a || !b || !workspace || !mom || sh < 1 || sw < 1) return FVR_ERR_ARG;
  if (ws_bytes < fvr_np_pair_workspace()) return FVR_ERR_WORKSPACE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* part = static_cast<double*>(workspace);
  np_pair_kernel<<<kNpTiles, 256, 0, s>>>(static_cast<const double2*>(a), static_cast<const double2*>(b), (int)sh,
                                          (int)sw, part);
  FVR_LAUNCH_CHECK();
  np_ncc_finalize_kernel<<<1, 128, 0, s>>>(part, 1, kNpTiles, mom);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

}  // extern "C"

FVR_CHECK_ACCESSOR(check_word_np)
