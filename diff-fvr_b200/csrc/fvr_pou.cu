// PoU-FVR cone-beam kernels (src/fvr/cone_beam_fvr.py, src/fvr/triton_slice.py:341-591), sm_100a.
//
// Precompute: partition-of-unity block extraction (window product, centring
// in an M^3 cube, trilinear resize to block_res^3, sinc^2 pre-compensation,
// zero pad to P^3) straight from the volume on the device; the block spectra
// then come from the batched 3D FFT and are stored in the stencil layout.
//
// Per step, for N poses and B blocks:
//   pose kernel     rigid matrices -> source / detector axes (fp64), slice
//                   axes and per-(block, pose) offsets d_b, cu, cv (fp64)
//   slice kernel    every block sliced along the pose's detector plane, written
//                   in ifftshift order -> batched 2D IFFT -> real block images
//   warp kernel     per detector pixel, sum over blocks of the bilinear sample
//                   of each block image at its magnified position, x 1/cos
// and the adjoint chain warp -> IFFT -> slice -> pose.
#include "fvr_pose.cuh"
#include "fvr_stencil.cuh"
#include "fvr_wfft.cuh"

namespace fvr {

// ----------------------------------------------------------------------------
// block extraction  (cone_beam_fvr.py:208-290)
// ----------------------------------------------------------------------------

struct PouAxisTables {
  const float* w;    // windows [k][n] (float32, as the reference builds them)
  const int* sup;    // supports [k][2]: first index, length
  int k, n;
};

// Sum over the support of vol * w0 * w1 * w2 (fp64) for candidate block
// kb = blockIdx.x: one warp per (z, y) row of the support, lanes along x (no
// division per voxel), then warps in order.
constexpr int kBlockSumThreads = 1024;

__global__ void __launch_bounds__(kBlockSumThreads) pou_block_sums_kernel(const float* __restrict__ vol,
                                                                          PouAxisTables a0, PouAxisTables a1,
                                                                          PouAxisTables a2, double* __restrict__ sums) {
  __shared__ double red[kBlockSumThreads / 32];
  const int kb = blockIdx.x;
  const int i0 = kb / (a1.k * a2.k), i1 = (kb / a2.k) % a1.k, i2 = kb % a2.k;
  const int s0 = a0.sup[2 * i0], l0 = a0.sup[2 * i0 + 1];
  const int s1 = a1.sup[2 * i1], l1 = a1.sup[2 * i1 + 1];
  const int s2 = a2.sup[2 * i2], l2 = a2.sup[2 * i2 + 1];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const float* w2 = a2.w + i2 * a2.n + s2;
  double acc = 0.0;
  for (int zy = wid; zy < l0 * l1; zy += nw) {
    const int z = zy / l1, y = zy - z * l1;
    const int gz = s0 + z, gy = s1 + y;
    const float wzy = a0.w[i0 * a0.n + gz] * a1.w[i1 * a1.n + gy];
    const float* row = vol + (static_cast<int64_t>(gz) * a1.n + gy) * a2.n + s2;
    for (int x = lane; x < l2; x += 32) acc += static_cast<double>(row[x] * (wzy * w2[x]));
  }
  acc = warp_sum(acc);
  if (lane == 0) red[wid] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double sum = 0.0;
    for (int w = 0; w < nw; ++w) sum += red[w];
    sums[kb] = sum;
  }
}

struct PouBuildArgs {
  const float* vol;
  PouAxisTables ax[3];
  const int* blocks;  // [B] candidate block index kb of each active block
  const float* w3;    // [block_res] sinc^2 pre-compensation (cone_beam_fvr.py:64-68)
  int M, br, P, pad_b;
  float ds;           // ds_block (resize intensity factor)
  float* out;         // [B][P][P][P]
};

// windowed sub-volume value at M-cube index (z, y, x) of block kb
__device__ __forceinline__ float pou_cube(const PouBuildArgs& a, const int (&ib)[3], const int (&s)[3],
                                          const int (&l)[3], const int (&m)[3], int z, int y, int x) {
  const int c[3] = {z - m[0], y - m[1], x - m[2]};
  if (c[0] < 0 || c[0] >= l[0] || c[1] < 0 || c[1] >= l[1] || c[2] < 0 || c[2] >= l[2]) return 0.f;
  const int g0 = s[0] + c[0], g1 = s[1] + c[1], g2 = s[2] + c[2];
  const float wv = a.ax[0].w[ib[0] * a.ax[0].n + g0] * a.ax[1].w[ib[1] * a.ax[1].n + g1] *
                   a.ax[2].w[ib[2] * a.ax[2].n + g2];
  return a.vol[(static_cast<int64_t>(g0) * a.ax[1].n + g1) * a.ax[2].n + g2] * wv;
}

// F.interpolate(..., mode='trilinear', align_corners=False) source index along one axis
__device__ __forceinline__ void resize_src(int dst, int in, int out, int& i0, int& i1, float& lam) {
  const float scale = static_cast<float>(in) / static_cast<float>(out);
  float src = scale * (static_cast<float>(dst) + 0.5f) - 0.5f;
  if (src < 0.f) src = 0.f;
  i0 = static_cast<int>(src);
  i1 = i0 < in - 1 ? i0 + 1 : i0;
  lam = src - static_cast<float>(i0);
}

__global__ void __launch_bounds__(256) pou_block_build_kernel(PouBuildArgs a, int64_t total) {
  const int64_t P3 = static_cast<int64_t>(a.P) * a.P * a.P;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int b = static_cast<int>(e / P3);
    const int64_t r = e - b * P3;
    const int z = static_cast<int>(r / (static_cast<int64_t>(a.P) * a.P)) - a.pad_b;
    const int y = static_cast<int>((r / a.P) % a.P) - a.pad_b;
    const int x = static_cast<int>(r % a.P) - a.pad_b;
    float val = 0.f;
    if (z >= 0 && z < a.br && y >= 0 && y < a.br && x >= 0 && x < a.br) {
      const int kb = a.blocks[b];
      const int ib[3] = {kb / (a.ax[1].k * a.ax[2].k), (kb / a.ax[2].k) % a.ax[1].k, kb % a.ax[2].k};
      int s[3], l[3], m[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        s[d] = a.ax[d].sup[2 * ib[d]];
        l[d] = a.ax[d].sup[2 * ib[d] + 1];
        m[d] = (a.M - l[d]) / 2;
      }
      float cube;
      if (a.M == a.br) {
        cube = pou_cube(a, ib, s, l, m, z, y, x);
      } else {
        int z0, z1, y0, y1, x0, x1;
        float lz, ly, lx;
        resize_src(z, a.M, a.br, z0, z1, lz);
        resize_src(y, a.M, a.br, y0, y1, ly);
        resize_src(x, a.M, a.br, x0, x1, lx);
        const float c000 = pou_cube(a, ib, s, l, m, z0, y0, x0), c001 = pou_cube(a, ib, s, l, m, z0, y0, x1);
        const float c010 = pou_cube(a, ib, s, l, m, z0, y1, x0), c011 = pou_cube(a, ib, s, l, m, z0, y1, x1);
        const float c100 = pou_cube(a, ib, s, l, m, z1, y0, x0), c101 = pou_cube(a, ib, s, l, m, z1, y0, x1);
        const float c110 = pou_cube(a, ib, s, l, m, z1, y1, x0), c111 = pou_cube(a, ib, s, l, m, z1, y1, x1);
        const float mz = 1.f - lz, my = 1.f - ly, mx = 1.f - lx;
        cube = mz * (my * (mx * c000 + lx * c001) + ly * (mx * c010 + lx * c011)) +
               lz * (my * (mx * c100 + lx * c101) + ly * (mx * c110 + lx * c111));
      }
      val = cube * a.ds * (a.w3[z] * a.w3[y] * a.w3[x]);
    }
    a.out[e] = val;
  }
}

// ----------------------------------------------------------------------------
// pose geometry  (cone_beam_fvr.py:485-488, 507-521, 670-682)
// ----------------------------------------------------------------------------

constexpr int kGeo = 18;  // per pose: src[3], u[3], v[3], n[3], u_xyz[3], v_xyz[3]

struct PouBase {
  double src0[3], u0[3], v0[3], n0[3];
};

__global__ void pou_pose_kernel(const float* __restrict__ mats, const float* __restrict__ vecs, int N, PouBase base,
                                double vscale, const float* __restrict__ centers, int B, double* __restrict__ geo,
                                double* __restrict__ offs) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  double g[kGeo];
  if (mats) {
    const float* M = mats + 16 * n;
    double R[3][3], t[3];
    for (int i = 0; i < 3; ++i) {
      for (int j = 0; j < 3; ++j) R[i][j] = M[4 * i + j];
      t[i] = M[4 * i + 3];
    }
    for (int i = 0; i < 3; ++i) {
      g[i] = R[i][0] * base.src0[0] + R[i][1] * base.src0[1] + R[i][2] * base.src0[2] + t[i];
      g[3 + i] = R[i][0] * base.u0[0] + R[i][1] * base.u0[1] + R[i][2] * base.u0[2];
      g[6 + i] = R[i][0] * base.v0[0] + R[i][1] * base.v0[1] + R[i][2] * base.v0[2];
      g[9 + i] = R[i][0] * base.n0[0] + R[i][1] * base.n0[1] + R[i][2] * base.n0[2];
    }
  } else {  // explicit source / detector axes [N][12] = (s, u, v, n)
    for (int k = 0; k < 12; ++k) g[k] = vecs[12 * n + k];
  }
  // slice axes in (x, y, z) voxel order = world (axis2, axis1, axis0), scaled by P * ds
  for (int i = 0; i < 3; ++i) {
    g[12 + i] = g[3 + 2 - i] * vscale;
    g[15 + i] = g[6 + 2 - i] * vscale;
  }
  for (int k = 0; k < kGeo; ++k) geo[n * kGeo + k] = g[k];
  for (int b = 0; b < B; ++b) {
    const double d0 = centers[3 * b] - g[0], d1 = centers[3 * b + 1] - g[1], d2 = centers[3 * b + 2] - g[2];
    double* o = offs + 3 * (static_cast<int64_t>(b) * N + n);
    o[0] = d0 * g[9] + d1 * g[10] + d2 * g[11];  // d_b  = (c_b - s) . n0
    o[1] = d0 * g[3] + d1 * g[4] + d2 * g[5];    // cu   = (c_b - s) . u
    o[2] = d0 * g[6] + d1 * g[7] + d2 * g[8];    // cv   = (c_b - s) . v
  }
}

// Explicit rays (cone_beam_fvr.py:451-457): per pose and pixel
// rx = (r.u)/cos, ry = (r.v)/cos, ic = 1/cos with r the unit ray, cos = max(r.n, 0.1).
__global__ void pou_rays_prep_kernel(const float* __restrict__ trg, const double* __restrict__ geo, int N, int K,
                                     float* __restrict__ rx, float* __restrict__ ry, float* __restrict__ ic) {
  const int n = blockIdx.y;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= K) return;
  const double* g = geo + n * kGeo;
  const float* t = trg + (static_cast<int64_t>(n) * K + q) * 3;
  const double r0 = t[0] - g[0], r1 = t[1] - g[1], r2 = t[2] - g[2];
  const double inv = 1.0 / sqrt(fmax(r0 * r0 + r1 * r1 + r2 * r2, 1e-12));
  const double h0 = r0 * inv, h1 = r1 * inv, h2 = r2 * inv;
  const double c = fmax(h0 * g[9] + h1 * g[10] + h2 * g[11], 0.1);
  const double icv = 1.0 / c;
  const int64_t o = static_cast<int64_t>(n) * K + q;
  rx[o] = static_cast<float>((h0 * g[3] + h1 * g[4] + h2 * g[5]) * icv);
  ry[o] = static_cast<float>((h0 * g[6] + h1 * g[7] + h2 * g[8]) * icv);
  ic[o] = static_cast<float>(icv);
}

// ----------------------------------------------------------------------------
// block slices  (cone_beam_fvr.py:480-505; triton_slice.py:46-143)
// ----------------------------------------------------------------------------

struct PouSliceArgs {
  Stencil st;            // block 0; block b at data + b*item_bytes, scales + b*item_scales
  int64_t item_bytes, item_scales;
  const double* geo;     // [N][18]
  const float* freqs;    // [P] fftshift(fftfreq(P, d=ds))
  int P, N;
  double c;              // P // 2
};

__device__ __forceinline__ Stencil pou_block_stencil(const PouSliceArgs& a, int b) {
  Stencil s = a.st;
  s.data = static_cast<const char*>(a.st.data) + b * a.item_bytes;
  if (a.st.scales) s.scales = a.st.scales + b * a.item_scales;
  return s;
}

template <int DT>
__global__ void __launch_bounds__(256) pou_slice_kernel(PouSliceArgs a, float2* __restrict__ out) {
  const int n = blockIdx.y, b = blockIdx.z, P = a.P;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= P * P) return;
  const int i = q / P, j = q - (q / P) * P;  // i: fy index (rows), j: fx index
  const double* g = a.geo + n * kGeo;
  const double fx = __ldg(a.freqs + j), fy = __ldg(a.freqs + i);
  const Stencil st = pou_block_stencil(a, b);
  Interp o;
  stencil_sample_d<DT, false, false>(st, fma(fy, g[15], fma(fx, g[12], a.c)), fma(fy, g[16], fma(fx, g[13], a.c)),
                                     fma(fy, g[17], fma(fx, g[14], a.c)), o);
  // ifftshift position for the IFFT input
  const int h = P / 2;
  int ii = i - h, jj = j - h;
  if (ii < 0) ii += P;
  if (jj < 0) jj += P;
  out[(static_cast<int64_t>(b) * a.N + n) * P * P + ii * P + jj] = make_float2(o.sr, o.si);
}

// Slice adjoint: G[b][n][P*P] (natural order) -> partial[n][b][tile][6] = sums
// of (fx, fy) x <G, dS/dp_k> over the tile.
template <int DT>
__global__ void __launch_bounds__(256) pou_slice_adjoint_kernel(PouSliceArgs a, const float2* __restrict__ G,
                                                                double* __restrict__ partial) {
  __shared__ double red[6 * 8];
  const int n = blockIdx.y, b = blockIdx.z, P = a.P;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (q < P * P) {
    const int i = q / P, j = q - (q / P) * P;
    const double* g = a.geo + n * kGeo;
    const float fxf = __ldg(a.freqs + j), fyf = __ldg(a.freqs + i);
    const double fx = fxf, fy = fyf;
    const Stencil st = pou_block_stencil(a, b);
    Interp o;
    stencil_sample_d<DT, true, false>(st, fma(fy, g[15], fma(fx, g[12], a.c)), fma(fy, g[16], fma(fx, g[13], a.c)),
                                      fma(fy, g[17], fma(fx, g[14], a.c)), o);
    const float2 gg = __ldg(G + (static_cast<int64_t>(b) * a.N + n) * P * P + q);
    const float e0 = gg.x * o.dxr + gg.y * o.dxi, e1 = gg.x * o.dyr + gg.y * o.dyi, e2 = gg.x * o.dzr + gg.y * o.dzi;
    acc[0] = fxf * e0;
    acc[1] = fxf * e1;
    acc[2] = fxf * e2;
    acc[3] = fyf * e0;
    acc[4] = fyf * e1;
    acc[5] = fyf * e2;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int m = 0; m < 6; ++m) {
    const double v = warp_sum(static_cast<double>(acc[m]));
    if (lane == 0) red[m * nw + wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += red[threadIdx.x * nw + w];
    partial[((static_cast<int64_t>(n) * gridDim.z + b) * gridDim.x + blockIdx.x) * 6 + threadIdx.x] = s;
  }
}
// ----------------------------------------------------------------------------
// fused block image: slice + 2D inverse FFT in shared memory (forward), and
// 2D FFT + slice adjoint (backward), one CTA per (pose, block), P = 32 M.
// ----------------------------------------------------------------------------
constexpr int kPouImgThreads = 512;

// Row / column split-position tables of one (pose, block) image: entry j < P
// is the column part fx_j u, entry P + i the row part c + fy_i v (fp64, split
// into integer cell and float fraction; .w = the frequency).
__device__ __forceinline__ void pou_image_tables(const AxisTables& t, const PouSliceArgs& a, const double* g) {
  for (int e = threadIdx.x; e < 2 * a.P; e += blockDim.x) {
    const bool col = e < a.P;
    const float kf = __ldg(a.freqs + (col ? e : e - a.P));
    const double k = kf;
    const double px = col ? k * g[12] : fma(k, g[15], a.c);
    const double py = col ? k * g[13] : fma(k, g[16], a.c);
    const double pz = col ? k * g[14] : fma(k, g[17], a.c);
    const double fx = floor(px), fy = floor(py), fz = floor(pz);
    t.idx[e] = make_int4(static_cast<int>(fx), static_cast<int>(fy), static_cast<int>(fz), 0);
    t.frac[e] = make_float4(static_cast<float>(px - fx), static_cast<float>(py - fy), static_cast<float>(pz - fz), kf);
  }
}

template <int DT, bool DERIV>
__device__ __forceinline__ void pou_table_sample(const Stencil& st, const Raw<DT>& raw, const float4& fa,
                                                 const float4& fb, Interp& o) {
  float tx = fa.x + fb.x, ty = fa.y + fb.y, tz = fa.z + fb.z;
  if (tx >= 1.f) tx -= 1.f;
  if (ty >= 1.f) ty -= 1.f;
  if (tz >= 1.f) tz -= 1.f;
  Sample8 sm;
  tab_decode<DT>(raw, sm);
  trilerp<DERIV>(sm, tx, ty, tz, o);
  const float sc = raw_scale(raw);
  if (DT == FVR_F16) {
    o.sr *= sc;
    o.si *= sc;
    if (DERIV) {
      o.dxr *= sc;
      o.dxi *= sc;
      o.dyr *= sc;
      o.dyi *= sc;
      o.dzr *= sc;
      o.dzi *= sc;
    }
  }
}

// Smem layout of the fused forward image kernel: the P x (P + 1) complex
// image, then the 2P-entry tables.
__host__ __device__ constexpr int64_t pou_image_smem(int P) {
  return static_cast<int64_t>(P) * (P + 1) * 8 + 40 * 2 * static_cast<int64_t>(P) + 16;
}

// Hermitian pairing of slice samples.  A block is real, so its centred
// spectrum obeys F[c + m] = conj F[c - m] for |m| < P/2 in every axis (grid
// indices 1 .. P-1; index 0, the Nyquist plane, has no partner).  A slice
// sample at c + k whose trilinear cell [i, i + 1] lies inside 1 .. P-1 in all
// three axes therefore has the mirror sample S(c - k) = conj S(c + k), and the
// spectrum's gradient there is -conj of the gradient at c + k.  The gradient
// relation also needs the sample off the cell faces: on a face the trilinear
// derivative is one-sided, and the side flips under the mirror, so the
// adjoint pairs only samples whose fractions keep kPouMirrorMargin from 0 and 1.
constexpr float kPouMirrorMargin = 1.f / 65536.f;

__device__ __forceinline__ bool pou_mirror_cell(const TabCell& c, int P) {
  const unsigned lim = static_cast<unsigned>(P - 3);  // cell i = e - 1 in 1 .. P-2
  return static_cast<unsigned>(c.ex - 2) <= lim && static_cast<unsigned>(c.ey - 2) <= lim &&
         static_cast<unsigned>(c.ez - 2) <= lim;
}

__device__ __forceinline__ bool pou_mirror_cell_deriv(const TabCell& c, int P) {
  constexpr float lo = kPouMirrorMargin, hi = 1.f - kPouMirrorMargin;
  return pou_mirror_cell(c, P) && c.tx >= lo && c.tx <= hi && c.ty >= lo && c.ty <= hi && c.tz >= lo && c.tz <= hi;
}

// Gathers slice row `i` (table order) at the natural-order columns lane + 32 m
// into x.
template <int DT, int M>
__device__ __forceinline__ void pou_gather_row(const Stencil& st, const AxisTables& tab, int i, int lane,
                                               Cx<float> (&x)[M]) {
  constexpr int P = 32 * M, H = P / 2;
  const int4 ia = tab.idx[P + i];
  const float4 fa = tab.frac[P + i];
  Raw<DT> raw[M];
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const int c = lane + 32 * m;
    const int jj = c + H < P ? c + H : c - H;
    tab_load<DT>(st, tab_cell(st, ia, fa, tab.idx[jj], tab.frac[jj]), raw[m]);
  }
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const int c = lane + 32 * m;
    const int jj = c + H < P ? c + H : c - H;
    Interp o;
    pou_table_sample<DT, false>(st, raw[m], fa, tab.frac[jj], o);
    x[m] = Cx<float>{o.sr, o.si};
  }
}

// Value at natural column (P - c) mod P of a row held as lane + 32 m: lane
// 32 - lane, register M - 1 - m; lane 0 keeps its own register (M - m) mod M.
template <int M>
__device__ __forceinline__ Cx<float> pou_row_mirror(const Cx<float> (&x)[M], int m, int lane) {
  const int from = (32 - lane) & 31;
  const float vx = __shfl_sync(0xffffffffu, x[M - 1 - m].x, from);
  const float vy = __shfl_sync(0xffffffffu, x[M - 1 - m].y, from);
  return lane == 0 ? x[(M - m) % M] : Cx<float>{vx, vy};
}

// Hermitian part (x[c] + conj x[-c]) / 2 of a row that is its own mirror (the
// DC row and the Nyquist row, whose negated frequency is the row itself).
template <int M>
__device__ __forceinline__ void pou_row_hermitian(Cx<float> (&x)[M], int lane) {
  Cx<float> v[M];
#pragma unroll
  for (int m = 0; m < M; ++m) v[m] = pou_row_mirror<M>(x, m, lane);
#pragma unroll
  for (int m = 0; m < M; ++m) x[m] = Cx<float>{0.5f * (x[m].x + v[m].x), 0.5f * (x[m].y - v[m].y)};
}

// Hermitian part of natural row u (1 <= u < P/2): h[c] = (S(u, c) +
// conj S(P - u, P - c)) / 2.  Where the sample's cell has a Hermitian mirror
// this is S(u, c) itself; the partner sample is gathered only elsewhere (the
// Nyquist column, cells on the spectrum's border).  The first partner a lane
// needs is loaded together with the row; further ones (rare) in more rounds.
template <int DT, int M>
__device__ __forceinline__ void pou_gather_row_hermitian(const Stencil& st, const AxisTables& tab, int u, int lane,
                                                         Cx<float> (&h)[M]) {
  constexpr int P = 32 * M, H = P / 2;
  const int ti = u + H, tp = H - u;  // table rows of natural rows u and P - u
  const int4 ia = tab.idx[P + ti], iap = tab.idx[P + tp];
  const float4 fa = tab.frac[P + ti], fap = tab.frac[P + tp];
  Raw<DT> raw[M];
  unsigned pend = 0;
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const int c = lane + 32 * m;
    const int jj = c + H < P ? c + H : c - H;
    const TabCell cell = tab_cell(st, ia, fa, tab.idx[jj], tab.frac[jj]);
    if (c == H || !pou_mirror_cell(cell, P)) pend |= 1u << m;
    tab_load<DT>(st, cell, raw[m]);
  }
  // partner of the first pending column, in the same round
  int mp = pend ? __ffs(pend) - 1 : 0;
  int jp = (P - ((lane + 32 * mp + H) % P)) % P;  // table column of natural column P - c
  Raw<DT> rawp;
  {
    TabCell pc = tab_cell(st, iap, fap, tab.idx[jp], tab.frac[jp]);
    if (!pend) pc.e = -1;
    tab_load<DT>(st, pc, rawp);
  }
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const int c = lane + 32 * m;
    const int jj = c + H < P ? c + H : c - H;
    Interp o;
    pou_table_sample<DT, false>(st, raw[m], fa, tab.frac[jj], o);
    h[m] = Cx<float>{o.sr, o.si};
  }
  for (;;) {
    if (pend) {
      Interp o;
      pou_table_sample<DT, false>(st, rawp, fap, tab.frac[jp], o);
#pragma unroll
      for (int m = 0; m < M; ++m)
        if (m == mp) h[m] = Cx<float>{0.5f * (h[m].x + o.sr), 0.5f * (h[m].y - o.si)};
      pend &= pend - 1;
    }
    if (!__any_sync(0xffffffffu, pend != 0)) break;
    mp = pend ? __ffs(pend) - 1 : 0;
    jp = (P - ((lane + 32 * mp + H) % P)) % P;
    TabCell pc = tab_cell(st, iap, fap, tab.idx[jp], tab.frac[jp]);
    if (!pend) pc.e = -1;
    tab_load<DT>(st, pc, rawp);
  }
}

// imgs[b][n] = Re fftshift(ifft2(ifftshift(S))) for the slice S of block b at
// pose n (the reference's _slice_and_ifft, cone_beam_fvr.py:480-505).
//
// Re ifft2(S) = ifft2(Herm S) with Herm S(k) = (S(k) + conj S(-k)) / 2 (index
// -k mod P), and the slice of a real block is Hermitian wherever the mirror
// relation above holds, so Herm S needs about half of the slice's stencil
// entries.  Herm S is Hermitian by construction, so the row pass transforms
// natural rows 0 .. P/2 only (rows P - u are the conjugates of rows u; rows 0
// and P/2 are real after the transform and share one FFT as real and
// imaginary part), and the column pass transforms two real-output columns per
// complex FFT.  That is P/2 + P/2 FFTs instead of 2P.
template <int DT, int M>
__global__ void __launch_bounds__(kPouImgThreads, 1) pou_slice_ifft_kernel(PouSliceArgs a, float* __restrict__ imgs) {
  constexpr int P = 32 * M, PITCH = P + 1, H = P / 2, NW = kPouImgThreads / 32;
  extern __shared__ __align__(16) unsigned char smem[];
  Cx<float>* buf = reinterpret_cast<Cx<float>*>(smem);
  const AxisTables tab = axis_tables(smem + ((static_cast<int64_t>(P) * PITCH * 8 + 15) / 16) * 16, 2 * P);
  const int n = blockIdx.x, b = blockIdx.y;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const Stencil st = pou_block_stencil(a, b);
  pou_image_tables(tab, a, a.geo + n * kGeo);
  WarpFft<M, true> fft;
  fft.init(lane);
  __syncthreads();
  // rows: unit 0 = natural rows 0 and H (table rows H and 0), unit u = row u
  for (int u = wid; u < H; u += NW) {
    Cx<float> h[M];
    if (u == 0) {
      Cx<float> x[M];
      pou_gather_row<DT, M>(st, tab, H, lane, x);
      pou_row_hermitian<M>(x, lane);
      pou_gather_row<DT, M>(st, tab, 0, lane, h);
      pou_row_hermitian<M>(h, lane);
#pragma unroll
      for (int m = 0; m < M; ++m) h[m] = Cx<float>{x[m].x - h[m].y, x[m].y + h[m].x};
    } else {
      pou_gather_row_hermitian<DT, M>(st, tab, u, lane, h);
    }
    fft.run(h, lane);
    if (u == 0) {
#pragma unroll
      for (int k = 0; k < M; ++k) {
        buf[lane + 32 * k] = Cx<float>{h[k].x, 0.f};
        buf[H * PITCH + lane + 32 * k] = Cx<float>{h[k].y, 0.f};
      }
    } else {
#pragma unroll
      for (int k = 0; k < M; ++k) buf[u * PITCH + lane + 32 * k] = h[k];
    }
  }
  __syncthreads();
  // columns: buffer columns 2t and 2t + 1 as real and imaginary part of one
  // transform (rows r > H read as the conjugate of row P - r); the real
  // results of both land in column 2t
  for (int t = wid; t < H; t += NW) {
    const int c1 = 2 * t;
    Cx<float> z[M];
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const int r = lane + 32 * m;
      const int rr = r <= H ? r : P - r;
      const float sg = r <= H ? 1.f : -1.f;
      const Cx<float> p = buf[rr * PITCH + c1], q = buf[rr * PITCH + c1 + 1];
      z[m] = Cx<float>{p.x - sg * q.y, sg * p.y + q.x};
    }
    fft.run(z, lane);
#pragma unroll
    for (int k = 0; k < M; ++k) buf[(lane + 32 * k) * PITCH + c1] = z[k];
  }
  __syncthreads();
  // fftshift-ordered image, coalesced rows
  const float scale = 1.f / static_cast<float>(P * P);
  float* out = imgs + (static_cast<int64_t>(b) * a.N + n) * P * P;
  for (int q = threadIdx.x; q < P * P; q += kPouImgThreads) {
    const int y = q / P, xq = q - y * P;
    const int ky = y + H < P ? y + H : y - H, kx = xq + H < P ? xq + H : xq - H;
    const int px = wfft_pos<M>(kx);
    const Cx<float> v = buf[wfft_pos<M>(ky) * PITCH + (px & ~1)];
    out[q] = ((px & 1) ? v.y : v.x) * scale;
  }
}

// Shared memory of the adjoint: the row-pair spectra [P/2][P + 1], the half
// spectrum G [P][P/2 + 1], the axis tables, one partner queue per warp.
constexpr int kPouQueue = 256;

__host__ __device__ constexpr int64_t pou_adjoint_tables_at(int P) {
  return ((static_cast<int64_t>(P / 2) * (P + 1) + static_cast<int64_t>(P) * (P / 2 + 1)) * 8 + 15) / 16 * 16;
}

__host__ __device__ constexpr int64_t pou_adjoint_smem(int P) {
  return pou_adjoint_tables_at(P) + 40 * 2 * static_cast<int64_t>(P) + (kPouImgThreads / 32) * kPouQueue * 2;
}

// G at natural frequency indices (ki, kj) from the stored half kj <= P/2
// (rows in transform order): G(-k) = conj G(k) for the transform of a real image.
template <int M>
__device__ __forceinline__ Cx<float> pou_half_spectrum(const Cx<float>* gb, int ki, int kj) {
  constexpr int P = 32 * M, H = P / 2, GP = H + 1;
  if (kj <= H) return gb[wfft_pos<M>(ki) * GP + kj];
  const Cx<float> v = gb[wfft_pos<M>(ki == 0 ? 0 : P - ki) * GP + (P - kj)];
  return Cx<float>{v.x, -v.y};
}

// acc += w (fx, fy) x <G, dS/dp> for the sample at table position (i, j).
template <int DT, int M>
__device__ __forceinline__ void pou_adjoint_sample(const Stencil& st, const AxisTables& tab, const Cx<float>* gb,
                                                   const Raw<DT>& raw, int i, int j, float w, float (&acc)[6]) {
  constexpr int P = 32 * M, H = P / 2;
  const float4 fa = tab.frac[P + i], fb = tab.frac[j];
  Interp o;
  pou_table_sample<DT, true>(st, raw, fa, fb, o);
  const Cx<float> G = pou_half_spectrum<M>(gb, i + H < P ? i + H : i - H, j + H < P ? j + H : j - H);
  const float gx = G.x * w, gy = G.y * w;
  const float e0 = gx * o.dxr + gy * o.dxi, e1 = gx * o.dyr + gy * o.dyi, e2 = gx * o.dzr + gy * o.dzi;
  const float fx = fb.w, fy = fa.w;
  acc[0] = fmaf(fx, e0, acc[0]);
  acc[1] = fmaf(fx, e1, acc[1]);
  acc[2] = fmaf(fx, e2, acc[2]);
  acc[3] = fmaf(fy, e0, acc[3]);
  acc[4] = fmaf(fy, e1, acc[4]);
  acc[5] = fmaf(fy, e2, acc[5]);
}

// One warp's pass over `cnt` (<= 32 GROUP) queued samples from `head`.
template <int DT, int M, int GROUP>
__device__ __forceinline__ void pou_adjoint_queue(const Stencil& st, const AxisTables& tab, const Cx<float>* gb,
                                                  const unsigned short* queue, int head, int cnt, int lane,
                                                  float wscale, float (&acc)[6]) {
  constexpr int P = 32 * M;
  Raw<DT> raw[GROUP];
  int qq[GROUP];
#pragma unroll
  for (int u = 0; u < GROUP; ++u) {
    const bool ok = lane + 32 * u < cnt;
    const int q = ok ? queue[(head + lane + 32 * u) & (kPouQueue - 1)] : 0;
    qq[u] = ok ? q : -1;
    const int i = q / P, j = q - (q / P) * P;
    TabCell cell = tab_cell(st, tab.idx[P + i], tab.frac[P + i], tab.idx[j], tab.frac[j]);
    if (!ok) cell.e = -1;
    tab_load<DT>(st, cell, raw[u]);
  }
#pragma unroll
  for (int u = 0; u < GROUP; ++u)
    if (qq[u] >= 0) pou_adjoint_sample<DT, M>(st, tab, gb, raw[u], qq[u] / P, qq[u] % P, wscale, acc);
  __syncwarp();
}

// Detector side of the fused warp + block-image adjoint, for a separable
// pinhole lattice: every detector column shares one ray coordinate rx and
// every detector row one ry (the invariant lattice's rays agree per column and
// per row up to float rounding; rxc / ryr hold the midpoints).  Block b of pose
// n then samples image column ix + tx = (d_b rx - cu) / ds + c of every pixel
// in a column and image row iy + ty = (d_b ry - cv) / ds + c of every pixel in
// a row, so the warp's adjoint separates: per detector row r, a gather along x
// (no atomics) gives T_r[x] = sum_c g[r][c] wx(c, x) and its x-slope versions;
// image row iy(r) receives (1 - ty) T_r and row iy(r) + 1 receives ty T_r.
struct PouWarpSep {
  const float* imgs;   // [B][N][P][P] forward block images
  const double* offs;  // [B][N][3]: d_b, cu, cv
  const float* rxc;    // [W] column ray coordinate
  const float* ryr;    // [Hd] row ray coordinate
  const float* ic;     // [Hd W]
  const float* gout;   // [N][Hd W]
  double* goffs;       // [3][B][N]: dL/d(d_b, cu, cv)
  int Hd, W;
  double inv_ds, c_idx;
};

// Shared memory of the fused adjoint beyond the block-image adjoint's: one
// detector-row buffer per warp [16][W + 4], column map (ix, tx) [W], row map
// (iy, ty) [Hd], per image index -1 .. P-1 the first and last detector column
// and row with that index [4][P + 1], the largest tap count [4].
constexpr int kPouFusedMaxW = 256;

__host__ __device__ constexpr int64_t pou_fused_extra(int P, int Hd, int W) {
  return 4LL * (kPouImgThreads / 32) * (W + 4) + 8LL * W + 8LL * Hd + 16LL * (P + 1) + 16;
}

__host__ __device__ constexpr int64_t pou_fused_smem(int P, int Hd, int W) {
  return (pou_adjoint_smem(P) + 15) / 16 * 16 + pou_fused_extra(P, Hd, W);
}

// Detector-row pass of the fused adjoint for one layout: warp = (row band,
// column part); the image rows that receive contributions, [Y0, Y1], split in
// 16 / NCP equal bands, and the image columns [h P/NCP, (h + 1) P/NCP); each
// lane keeps up to TCR/2 taps of each class of each of its columns in
// registers (more, or detector columns out of order, take column loops).
template <int M, int NCP, int TCR>
__device__ void pou_gather_rows(const PouWarpSep& w, int n, float* wbuf, const int2* cmap, const int2* rmap,
                                const int* clo, const int* chi, const int* rlo, const int* rhi, const float* img,
                                float* gimg, double (&sums)[4]) {
  constexpr int P = 32 * M, PART = P / NCP, MW = (PART + 31) / 32, RG = kPouImgThreads / 32 / NCP;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int W = w.W, Hd = w.Hd;
  const int rg = wid / NCP, h = wid % NCP, xa = h * PART;
  int ylo = 0x7fffffff, yhi = -1;  // valid iy + 1 range
  for (int k = lane; k <= P; k += 32)
    if (rlo[k] <= rhi[k]) {
      ylo = min(ylo, k);
      yhi = max(yhi, k);
    }
  ylo = __reduce_min_sync(0xffffffffu, ylo);
  yhi = __reduce_max_sync(0xffffffffu, yhi);
  if (ylo > yhi) return;
  const int Y0 = max(ylo - 1, 0), Y1 = min(yhi, P - 1);  // rows iy and iy + 1 of the valid detector rows
  const int y_lo = Y0 + (rg * (Y1 - Y0 + 1)) / RG, y_hi = Y0 + ((rg + 1) * (Y1 - Y0 + 1)) / RG;
  if (y_lo >= y_hi) return;
  int ra = 0x7fffffff, rb = -1;  // detector rows with iy + 1 in [y_lo, y_hi]
  for (int k = y_lo + lane; k <= y_hi; k += 32) {
    ra = min(ra, rlo[k]);
    rb = max(rb, rhi[k]);
  }
  int ca = 0x7fffffff, cb = -1;  // detector columns with ix + 1 in [xa, xa + PART]
  for (int k = xa + lane; k <= xa + PART; k += 32) {
    ca = min(ca, clo[k]);
    cb = max(cb, chi[k]);
  }
  ra = __reduce_min_sync(0xffffffffu, ra);
  rb = __reduce_max_sync(0xffffffffu, rb);
  ca = __reduce_min_sync(0xffffffffu, ca);
  cb = __reduce_max_sync(0xffffffffu, cb);
  if (ra > rb || ca > cb) return;
  ca &= ~3;  // float4 staging from a 16-byte boundary (W is a multiple of 4)
  const int nq = (cb - ca + 4) / 4, ncw = 4 * nq;  // staged float4 chunks, columns
  float* mybuf = wbuf + static_cast<int64_t>(wid) * (W + 4);  // the row's columns [ca, ca + ncw), then a zero
  // taps of image column x: slots [0, TCR/2) hold the detector columns with
  // ix == x (weight 1 - tx, slope -1), slots [TCR/2, TCR) those with
  // ix == x - 1 (weight tx, slope +1); unused slots read the zero
  constexpr int HT = TCR / 2;
  int toff[MW][TCR];  // mybuf index
  float tt[MW][TCR], trx[MW][TCR];
  bool over = false;
#pragma unroll
  for (int m = 0; m < MW; ++m) {
#pragma unroll
    for (int k = 0; k < TCR; ++k) {
      toff[m][k] = ncw;
      tt[m][k] = 0.f;
      trx[m][k] = 0.f;
    }
    const int x = xa + lane + 32 * m;
    if (lane + 32 * m >= PART) continue;
    // the columns of one index form the range [clo, chi] when px is monotone
    // in the column (checked per tap; otherwise the column loops below)
    const int a0 = clo[x + 1], a1 = clo[x];
    const int n0 = max(chi[x + 1] - a0 + 1, 0), n1 = max(chi[x] - a1 + 1, 0);
    over |= n0 > HT || n1 > HT;
#pragma unroll
    for (int q = 0; q < TCR; ++q) {
      const bool cls = q >= HT;  // false: ix == x, true: ix == x - 1
      const int qq = cls ? q - HT : q;
      if (qq >= (cls ? n1 : n0)) continue;
      const int c = (cls ? a1 : a0) + qq;
      const int2 e = cmap[c];
      over |= e.x != (cls ? x - 1 : x);
      toff[m][q] = c - ca;
      tt[m][q] = __int_as_float(e.y);
      trx[m][q] = __ldg(w.rxc + c);
    }
  }
  const bool regs = !__any_sync(0xffffffffu, over);  // else the column loops below
  const float4* gp = reinterpret_cast<const float4*>(w.gout + static_cast<int64_t>(n) * Hd * W);
  const float4* ip = reinterpret_cast<const float4*>(w.ic);
  constexpr int NJ = kPouFusedMaxW / 128;  // float4 chunks per lane
  float4 gv[NJ], iv[NJ];
  auto load = [&](int r) {
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
      const int q = lane + 32 * j;
      const int64_t e = (static_cast<int64_t>(r) * W + ca) / 4 + q;
      const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
      gv[j] = q < nq ? __ldg(gp + e) : z;
      iv[j] = q < nq ? __ldg(ip + e) : z;
    }
  };
  if (lane == 0) mybuf[ncw] = 0.f;
  load(ra);
  for (int r = ra; r <= rb; ++r) {
#pragma unroll
    for (int j = 0; j < NJ; ++j)
      if (lane + 32 * j < nq)
        reinterpret_cast<float4*>(mybuf)[lane + 32 * j] =
            make_float4(gv[j].x * iv[j].x, gv[j].y * iv[j].y, gv[j].z * iv[j].z, gv[j].w * iv[j].w);
    if (r < rb) load(r + 1);
    __syncwarp();
    const int iy = rmap[r].x;
    if (iy >= y_lo - 1 && iy < y_hi && iy >= -1) {
      const float ty = __int_as_float(rmap[r].y), uy = 1.f - ty;
      float fs[3] = {0.f, 0.f, 0.f};
#pragma unroll
      for (int m = 0; m < MW; ++m) {
        const int xl = lane + 32 * m;
        if (xl >= PART) continue;
        const int x = xa + xl;
        float T = 0.f, Td = 0.f, Tr = 0.f;
        if (regs) {  // per class: sum g, sum tx g, sum rx g
          float s0 = 0.f, u0 = 0.f, r0 = 0.f, s1 = 0.f, u1 = 0.f, r1 = 0.f;
#pragma unroll
          for (int k = 0; k < HT; ++k) {
            const int i0 = toff[m][k], i1 = toff[m][HT + k];
            const float g0 = fvr_checked(i0, ncw + 1, kSiteWarpFused) ? mybuf[i0] : 0.f;
            const float g1 = fvr_checked(i1, ncw + 1, kSiteWarpFused) ? mybuf[i1] : 0.f;
            s0 += g0;
            u0 = fmaf(tt[m][k], g0, u0);
            r0 = fmaf(trx[m][k], g0, r0);
            s1 += g1;
            u1 = fmaf(tt[m][HT + k], g1, u1);
            r1 = fmaf(trx[m][HT + k], g1, r1);
          }
          T = (s0 - u0) + u1;
          Td = s1 - s0;
          Tr = r1 - r0;
        } else {
          for (int c = clo[x + 1]; c <= chi[x + 1]; ++c) {  // ix == x: weight 1 - tx, slope -1
            const int2 e = cmap[c];
            if (e.x != x || !fvr_checked(c - ca, ncw, kSiteWarpFused)) continue;
            const float g = mybuf[c - ca];
            T = fmaf(g, 1.f - __int_as_float(e.y), T);
            Td -= g;
            Tr = fmaf(-g, __ldg(w.rxc + c), Tr);
          }
          for (int c = clo[x]; c <= chi[x]; ++c) {  // ix == x - 1: weight tx, slope +1
            const int2 e = cmap[c];
            if (e.x != x - 1 || !fvr_checked(c - ca, ncw, kSiteWarpFused)) continue;
            const float g = mybuf[c - ca];
            T = fmaf(g, __int_as_float(e.y), T);
            Td += g;
            Tr = fmaf(g, __ldg(w.rxc + c), Tr);
          }
        }
        const float iu = iy >= 0 ? img[iy * P + x] : 0.f, il = iy + 1 < P ? img[(iy + 1) * P + x] : 0.f;
        const float it = uy * iu + ty * il, di = il - iu;
        fs[0] = fmaf(Td, it, fs[0]);
        fs[1] = fmaf(Tr, it, fs[1]);
        fs[2] = fmaf(T, di, fs[2]);
        if (iy >= y_lo) gimg[iy * P + x] += uy * T;
        if (iy + 1 < y_hi) gimg[(iy + 1) * P + x] += ty * T;
      }
      if (max(iy, 0) >= y_lo) {
        const double ryv = static_cast<double>(__ldg(w.ryr + r));
        sums[0] += static_cast<double>(fs[0]);
        sums[1] += static_cast<double>(fs[1]);
        sums[2] += static_cast<double>(fs[2]);
        sums[3] += ryv * static_cast<double>(fs[2]);
      }
    }
    __syncwarp();
  }
}

// dL/dimgs of block b at pose n into `gimg` [P][P] (shared memory, zeroed
// here) and the pose-offset sums (sum g dv/dpx, sum g rx dv/dpx, sum g dv/dpy,
// sum g ry dv/dpy) of this (pose, block), with the forward image staged in
// `img` [P][P].  The x gather of a detector row is T[x] = sum of the row's
// values over image column x's taps (every row has the same taps).  Each warp
// owns a band of image rows at a part of the image columns, whose taps its
// lanes hold in registers: it runs over the detector rows whose iy lies in
// [band start - 1, band end - 1] and adds only into its own rows and columns,
// so no two warps write one element; a detector row's sums are counted by the
// warps owning image row max(iy, 0), each over its own columns.  Two column
// parts with up to 3 detector columns per image index (6 taps per column),
// or (larger detector-to-image magnification) four parts with up to 6 (12).
template <int M>
__device__ void pou_warp_gather_adjoint(const PouWarpSep& w, int n, int b, int N, unsigned char* sep, float* img,
                                        float* gimg, double (&sums)[4]) {
  constexpr int P = 32 * M, NW = kPouImgThreads / 32;
  const int W = w.W, Hd = w.Hd;
  float* wbuf = reinterpret_cast<float*>(sep);
  int2* cmap = reinterpret_cast<int2*>(wbuf + NW * (W + 4));
  int2* rmap = cmap + W;
  int* clo = reinterpret_cast<int*>(rmap + Hd);
  int* chi = clo + (P + 1);
  int* rlo = chi + (P + 1);
  int* rhi = rlo + (P + 1);
  int* tmax = rhi + (P + 1);
  const double* o = w.offs + 3 * (static_cast<int64_t>(b) * N + n);
  const double db = o[0], cu = o[1], cv = o[2];
  for (int k = threadIdx.x; k < 4 * (P + 1); k += kPouImgThreads) clo[k] = ((k / (P + 1)) & 1) ? -1 : 0x7fffffff;
  if (threadIdx.x == 0) *tmax = 0;
  for (int c = threadIdx.x; c < W; c += kPouImgThreads) {
    const double px = (db * static_cast<double>(__ldg(w.rxc + c)) - cu) * w.inv_ds + w.c_idx;
    const bool ok = px > -1.0 && px < static_cast<double>(P);
    const double f = floor(px);
    cmap[c] = make_int2(ok ? static_cast<int>(f) : -2, __float_as_int(static_cast<float>(px - f)));
  }
  for (int r = threadIdx.x; r < Hd; r += kPouImgThreads) {
    const double py = (db * static_cast<double>(__ldg(w.ryr + r)) - cv) * w.inv_ds + w.c_idx;
    const bool ok = py > -1.0 && py < static_cast<double>(P);
    const double f = floor(py);
    rmap[r] = make_int2(ok ? static_cast<int>(f) : -2, __float_as_int(static_cast<float>(py - f)));
  }
  const float4* src = reinterpret_cast<const float4*>(w.imgs + (static_cast<int64_t>(b) * N + n) * P * P);
  for (int q = threadIdx.x; q < P * P / 4; q += kPouImgThreads) {
    reinterpret_cast<float4*>(img)[q] = __ldg(src + q);
    reinterpret_cast<float4*>(gimg)[q] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < W; c += kPouImgThreads) {
    const int ix = cmap[c].x;
    if (ix >= -1) {
      atomicMin(clo + ix + 1, c);
      atomicMax(chi + ix + 1, c);
    }
  }
  for (int r = threadIdx.x; r < Hd; r += kPouImgThreads) {
    const int iy = rmap[r].x;
    if (iy >= -1) {
      atomicMin(rlo + iy + 1, r);
      atomicMax(rhi + iy + 1, r);
    }
  }
  __syncthreads();
  // the most detector columns on one image index picks the register layout
  for (int k = threadIdx.x; k <= P; k += kPouImgThreads) atomicMax(tmax, max(chi[k] - clo[k] + 1, 0));
  __syncthreads();
  if (*tmax <= 3)
    pou_gather_rows<M, 2, 6>(w, n, wbuf, cmap, rmap, clo, chi, rlo, rhi, img, gimg, sums);
  else
    pou_gather_rows<M, 4, 12>(w, n, wbuf, cmap, rmap, clo, chi, rlo, rhi, img, gimg, sums);
}

// Adjoint of pou_slice_ifft_kernel for one (pose, block): G = fftshift(fft2(
// ifftshift(g))) / P^2, then per slice sample the products of G with the
// spectrum's spatial derivatives, weighted by fx and fy:
// partial[n][b][6] = sum (fx <G, dS/dp_k>, fy <G, dS/dp_k>), k = x, y, z.
//
// G of a real image is Hermitian, so it is formed for kx <= P/2 only: the row
// pass transforms image rows two at a time (real and imaginary part of one
// FFT), the column pass separates them and transforms the P/2 + 1 columns
// needed.  A slice sample and its mirror (fx, fy, dS/dp change sign, G and
// dS/dp are conjugated) contribute the same products, so one stencil gather
// serves both wherever the mirror relation holds: the loop runs over the
// samples of positive row frequency (plus the Nyquist column), counts those
// with a mirror twice, and queues the partners of the others; the Nyquist row
// has no partner and goes through the queue once.
//
// FUSED: dL/dimgs is not read from memory but formed in shared memory from
// the detector gradient (pou_warp_gather_adjoint), which also gives this
// (pose, block)'s pose-offset gradients; the warp adjoint kernel and the
// block-image gradient buffer drop out.
template <int DT, int M, bool FUSED>
__global__ void __launch_bounds__(kPouImgThreads, 1) pou_fft_slice_adjoint_kernel(PouSliceArgs a,
                                                                                  const float* __restrict__ gimg,
                                                                                  PouWarpSep wsep,
                                                                                  double* __restrict__ partial) {
  constexpr int P = 32 * M, PITCH = P + 1, H = P / 2, GP = H + 1, NW = kPouImgThreads / 32, GROUP = 4;
  constexpr int BATCH = 32 * GROUP, NQ = P / NW;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double red[6 * NW];
  Cx<float>* zr = reinterpret_cast<Cx<float>*>(smem);
  Cx<float>* gb = zr + H * PITCH;
  const AxisTables tab = axis_tables(smem + pou_adjoint_tables_at(P), 2 * P);
  const int n = blockIdx.x, b = blockIdx.y;
  const int64_t nblk = gridDim.y;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned short* queue =
      reinterpret_cast<unsigned short*>(smem + pou_adjoint_tables_at(P) + 80 * P) + wid * kPouQueue;
  const Stencil st = pou_block_stencil(a, b);
  pou_image_tables(tab, a, a.geo + n * kGeo);
  WarpFft<M, false> fft;
  fft.init(lane);
  const float* g = FUSED ? reinterpret_cast<const float*>(gb)
                         : gimg + (static_cast<int64_t>(b) * a.N + n) * P * P;
  if constexpr (FUSED) {
    double sums[4] = {0.0, 0.0, 0.0, 0.0};
    pou_warp_gather_adjoint<M>(wsep, n, b, a.N, smem + (pou_adjoint_smem(P) + 15) / 16 * 16,
                               reinterpret_cast<float*>(zr), reinterpret_cast<float*>(gb), sums);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double v = warp_sum(sums[k]);
      if (lane == 0) red[k * NW + wid] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double t[4] = {0.0, 0.0, 0.0, 0.0};
      for (int k = 0; k < 4; ++k)
        for (int v = 0; v < NW; ++v) t[k] += red[k * NW + v];
      const int64_t B = nblk, e = static_cast<int64_t>(b) * a.N + n;
      wsep.goffs[e] = wsep.inv_ds * (t[1] + t[3]);
      wsep.goffs[B * a.N + e] = -wsep.inv_ds * t[0];
      wsep.goffs[2 * B * a.N + e] = -wsep.inv_ds * t[2];
    }
  }
  // rows: transform input rows 2s, 2s + 1 (image rows y0, y0 + 1 after ifftshift) together
  for (int s = wid; s < H; s += NW) {
    const int y0 = 2 * s + H < P ? 2 * s + H : 2 * s - H;
    Cx<float> z[M];
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const int c = lane + 32 * m;
      const int xc = c + H < P ? c + H : c - H;
      if constexpr (FUSED)
        z[m] = Cx<float>{g[y0 * P + xc], g[(y0 + 1) * P + xc]};
      else
        z[m] = Cx<float>{__ldg(g + y0 * P + xc), __ldg(g + (y0 + 1) * P + xc)};
    }
    fft.run(z, lane);
#pragma unroll
    for (int k = 0; k < M; ++k) zr[s * PITCH + lane + 32 * k] = z[k];
  }
  __syncthreads();
  // columns kx = 0 .. P/2: split the pair spectra (Z(k) + conj Z(-k)) / 2 and
  // (Z(k) - conj Z(-k)) / 2i, then transform over the rows
  for (int kx = wid; kx <= H; kx += NW) {
    const int p0 = wfft_pos<M>(kx), p1 = wfft_pos<M>(kx == 0 ? 0 : P - kx);
    Cx<float> x[M];
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const int y = lane + 32 * m, sr = (y >> 1) * PITCH;
      const Cx<float> A = zr[sr + p0], B = zr[sr + p1];
      x[m] = (y & 1) ? Cx<float>{0.5f * (A.y + B.y), 0.5f * (B.x - A.x)}
                     : Cx<float>{0.5f * (A.x + B.x), 0.5f * (A.y - B.y)};
    }
    fft.run(x, lane);
#pragma unroll
    for (int k = 0; k < M; ++k) gb[(lane + 32 * k) * GP + kx] = x[k];
  }
  // the Nyquist row (table row 0) starts the queue
  if (lane < NQ) queue[lane] = static_cast<unsigned short>(wid * NQ + lane);
  int head = 0, tail = NQ;
  __syncthreads();
  const float scale = 1.f / static_cast<float>(P * P);
  float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  const unsigned below = (1u << lane) - 1u;
  // own samples t < H P: table rows H+1 .. P-1 (all columns), row H (columns
  // 0 and H .. P-1), rows 1 .. H-1 (column 0); H P is a multiple of the
  // thread count, so every warp runs the same iterations
  for (int t0 = threadIdx.x; t0 < H * P; t0 += kPouImgThreads * GROUP) {
    Raw<DT> raw[GROUP];
    int qi[GROUP], qj[GROUP];
    float wt[GROUP];
#pragma unroll
    for (int u = 0; u < GROUP; ++u) {
      const int t = t0 + u * kPouImgThreads;
      int i, j;
      if (t < (H - 1) * P) {
        i = H + 1 + t / P;
        j = t - (t / P) * P;
      } else if (t < (H - 1) * P + H + 1) {
        i = H;
        j = t == (H - 1) * P ? 0 : H + t - (H - 1) * P - 1;
      } else if (t < H * P) {
        i = t - (H - 1) * P - H;
        j = 0;
      } else {
        i = 0;
        j = 0;
      }
      TabCell cell = tab_cell(st, tab.idx[P + i], tab.frac[P + i], tab.idx[j], tab.frac[j]);
      float w = t < H * P ? scale : 0.f;
      bool need = false;
      if (j >= 1 && (i > H || (i == H && j > H)) && w != 0.f) {
        if (pou_mirror_cell_deriv(cell, P)) {
          w *= 2.f;
        } else {
          const TabCell pc = tab_cell(st, tab.idx[2 * P - i], tab.frac[2 * P - i], tab.idx[P - j], tab.frac[P - j]);
          need = pc.e >= 0;
        }
      }
      const unsigned mask = __ballot_sync(0xffffffffu, need);
      if (need) queue[(tail + __popc(mask & below)) & (kPouQueue - 1)] = static_cast<unsigned short>((P - i) * P + P - j);
      tail += __popc(mask);
      if (w == 0.f) cell.e = -1;
      qi[u] = i;
      qj[u] = j;
      wt[u] = w;
      tab_load<DT>(st, cell, raw[u]);
    }
#pragma unroll
    for (int u = 0; u < GROUP; ++u)
      if (wt[u] != 0.f) pou_adjoint_sample<DT, M>(st, tab, gb, raw[u], qi[u], qj[u], wt[u], acc);
    __syncwarp();
    if (tail - head >= BATCH) {
      pou_adjoint_queue<DT, M, GROUP>(st, tab, gb, queue, head, BATCH, lane, scale, acc);
      head += BATCH;
    }
  }
  while (tail > head) {
    const int cnt = tail - head < BATCH ? tail - head : BATCH;
    pou_adjoint_queue<DT, M, GROUP>(st, tab, gb, queue, head, cnt, lane, scale, acc);
    head += cnt;
  }
#pragma unroll
  for (int m = 0; m < 6; ++m) {
    const double v = warp_sum(static_cast<double>(acc[m]));
    if (lane == 0) red[m * NW + wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double sum = 0.0;
    for (int w = 0; w < NW; ++w) sum += red[threadIdx.x * NW + w];
    partial[(static_cast<int64_t>(n) * nblk + b) * 6 + threadIdx.x] = sum;
  }
}


// ----------------------------------------------------------------------------
// pinhole warp + sum  (triton_slice.py:348-407 / 409-496)
// ----------------------------------------------------------------------------

template <typename OT>
struct WarpArgs {
  const float* imgs;  // [B][N][P][P]
  const OT* db;       // d_b[b][n] at db[(b*N + n) * ostride]
  const OT* cu;
  const OT* cv;
  int ostride;
  const float *rx, *ry, *ic;  // [K], or [N][K] with ray_stride = K
  double inv_ds, c_idx;
  int B, N, P, K;
  int64_t ray_stride;
  int chunk;  // blocks per row-strip round (0: every CTA takes the per-pixel path)
};

// Row strips.  The pinhole lattice's detector rows share one ray coordinate
// ry up to the float rounding of the lattice (about 1e-7 relative), so for a
// CTA whose pixels lie on one row every block is sampled on one image row
// pair (iy, iy + 1) with one fraction ty.  Such a CTA blends that row pair
// once per block into a shared-memory strip and interpolates it along x per
// pixel; the adjoint gathers each pixel's contributions into strips and
// spreads them onto the two image rows once per block.  A CTA takes this path
// when its ry spread moves py by at most kWarpRowTolPx image pixels on every
// block it touches (the row is sampled at the midpoint of its ry range); that
// shift is far below the fp32 rounding of py in the reference's own kernel.
constexpr int kWarpStripMax = 16;
constexpr double kWarpRowTolPx = 1e-4;

struct WarpCull {
  int nt;      // blocks the CTA samples: tl[0..nt), in increasing order
  bool rows;   // the row-strip path applies
  double ry0;  // the row's ray coordinate for that path
};

// Block culling for a CTA of detector pixels: the box of its live pixels'
// ray coordinates (rx, ry), then per block whether any of those pixels can
// sample inside the block image.  The image coordinate is the same monotone
// fp64 expression of rx (or ry) that the sampling uses, evaluated at the box
// corners, so a block is skipped only if no pixel would have sampled it.
// Surviving blocks are listed in increasing order (touch: per-block flags).
template <typename OT>
__device__ __forceinline__ WarpCull warp_cull(const WarpArgs<OT>& a, int n, bool live, double rx, double ry,
                                              unsigned char* touch, short* tl) {
  __shared__ double s_box[4][8];
  __shared__ double box[4];
  __shared__ unsigned s_dbmax;  // max |d_b| over the touched blocks (float bits; non-negative floats order as ints)
  __shared__ int s_nt;
  const double inf = 1e300;
  double v[4] = {live ? rx : inf, live ? -rx : inf, live ? ry : inf, live ? -ry : inf};  // mins of +-r
#pragma unroll
  for (int k = 0; k < 4; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] = fmin(v[k], __shfl_xor_sync(0xffffffffu, v[k], o));
    if ((threadIdx.x & 31) == 0) s_box[k][threadIdx.x >> 5] = v[k];
  }
  if (threadIdx.x == 0) s_dbmax = 0u;
  __syncthreads();
  if (threadIdx.x < 4) {
    double m = inf;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) m = fmin(m, s_box[threadIdx.x][w]);
    box[threadIdx.x] = m;
  }
  __syncthreads();
  const bool any = box[0] < inf;
  for (int b = threadIdx.x; b < a.B; b += blockDim.x) {
    const int64_t bn = static_cast<int64_t>(b) * a.N + n;
    const double db = static_cast<double>(a.db[bn * a.ostride]);
    const double cu = static_cast<double>(a.cu[bn * a.ostride]), cv = static_cast<double>(a.cv[bn * a.ostride]);
    const double x0 = (db * box[0] - cu) * a.inv_ds + a.c_idx, x1 = (db * -box[1] - cu) * a.inv_ds + a.c_idx;
    const double y0 = (db * box[2] - cv) * a.inv_ds + a.c_idx, y1 = (db * -box[3] - cv) * a.inv_ds + a.c_idx;
    const double P = static_cast<double>(a.P);
    const bool t = any && fmax(x0, x1) > -1.0 && fmin(x0, x1) < P && fmax(y0, y1) > -1.0 && fmin(y0, y1) < P;
    touch[b] = t;
    if (t) atomicMax(&s_dbmax, __float_as_uint(static_cast<float>(fabs(db)) * 1.001f));
  }
  __syncthreads();
  if (threadIdx.x < 32) {  // ordered compaction by warp 0
    const int lane = threadIdx.x;
    int base = 0;
    for (int c0 = 0; c0 < a.B; c0 += 32) {
      const int b = c0 + lane;
      const bool f = b < a.B && touch[b];
      const unsigned m = __ballot_sync(0xffffffffu, f);
      if (f) tl[base + __popc(m & ((1u << lane) - 1u))] = static_cast<short>(b);
      base += __popc(m);
    }
    if (lane == 0) s_nt = base;
  }
  __syncthreads();
  WarpCull wc;
  wc.nt = s_nt;
  const double lo = box[2], hi = -box[3];
  wc.ry0 = any ? 0.5 * (lo + hi) : 0.0;
  wc.rows = a.chunk > 0 && any &&
            0.5 * (hi - lo) * static_cast<double>(__uint_as_float(s_dbmax)) * fabs(a.inv_ds) <= kWarpRowTolPx;
  return wc;
}

// Per block of a row-strip round: the affine map from a pixel's rx to its
// image column, (d_b / ds) rx + (c - cu / ds) (one fp64 FMA per pixel), the
// image row iy (-2: the row misses the image) and fraction ty.
struct WarpRow {
  double sx, ox;  // the pixel's image column is sx * rx + ox
  int iy;
  float ty;
};

template <typename OT>
__device__ __forceinline__ WarpRow warp_row(const WarpArgs<OT>& a, int64_t bn, double ry0) {
  WarpRow r;
  const double db = static_cast<double>(a.db[bn * a.ostride]);
  const double cu = static_cast<double>(a.cu[bn * a.ostride]);
  const double cv = static_cast<double>(a.cv[bn * a.ostride]);
  r.sx = db * a.inv_ds;
  r.ox = a.c_idx - cu * a.inv_ds;
  const double py = (db * ry0 - cv) * a.inv_ds + a.c_idx;
  r.iy = -2;
  r.ty = 0.f;
  if (py > -1.0 && py < static_cast<double>(a.P)) {
    const double fy = floor(py);
    r.iy = static_cast<int>(fy);
    r.ty = static_cast<float>(py - fy);
  }
  return r;
}

// Image rows iy and iy + 1 of a block image at columns 4 xq .. 4 xq + 3 (P a
// multiple of 4, so each row starts on a 16-byte boundary); zero outside.
__device__ __forceinline__ void warp_row_quads(const float* img, int P, int iy, int xq, float4& r0, float4& r1) {
  const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
  const bool q_in = fvr_checked(4 * xq + 3, P, kSiteWarpStripRow);
  r0 = q_in && iy >= 0 && iy < P ? __ldg(reinterpret_cast<const float4*>(img + static_cast<int64_t>(iy) * P) + xq) : z;
  r1 = q_in && iy + 1 >= 0 && iy + 1 < P
           ? __ldg(reinterpret_cast<const float4*>(img + static_cast<int64_t>(iy + 1) * P) + xq)
           : z;
}

// Image rows iy and iy + 1 of block image bn at column x (zero outside).
__device__ __forceinline__ void warp_row_pair(const float* img, int P, int iy, int x, float& r0, float& r1) {
  const bool xin = x >= 0 && x < P;
  r0 = xin && iy >= 0 && iy < P ? ldg_in(img, static_cast<int64_t>(iy) * P + x, P * P, kSiteWarpStripRow) : 0.f;
  r1 = xin && iy + 1 >= 0 && iy + 1 < P ? ldg_in(img, static_cast<int64_t>(iy + 1) * P + x, P * P, kSiteWarpStripRow)
                                        : 0.f;
}

// Row-strip forward of one CTA: the pixel's sum over the listed blocks in
// list order.  Strip k holds the blend rb[x] = (1 - ty) img[iy][x] + ty
// img[iy + 1][x] at index x + 1 for x in [-1, P] (zero outside the image).
template <typename OT>
__device__ float warp_rows_forward(const WarpArgs<OT>& a, int n, bool live, double rx, const WarpCull& wc,
                                   const short* tl, float* strip) {
  __shared__ WarpRow s_row[kWarpStripMax];
  const int P = a.P, W2 = P + 2;
  float acc = 0.f;
  for (int c0 = 0; c0 < wc.nt; c0 += a.chunk) {
    const int cn = min(a.chunk, wc.nt - c0);
    __syncthreads();  // the previous round's strips are no longer read
    if (threadIdx.x < cn) s_row[threadIdx.x] = warp_row(a, static_cast<int64_t>(tl[c0 + threadIdx.x]) * a.N + n, wc.ry0);
    __syncthreads();
    // element e = k * W2 + xr of the strips, walked without a division per element
    if ((P & 3) == 0) {  // four columns per thread, 16-byte loads
      const int Q = P >> 2;
      for (int k = threadIdx.x / Q, xq = threadIdx.x % Q; k < cn;) {
        float4 r0, r1;
        warp_row_quads(a.imgs + (static_cast<int64_t>(tl[c0 + k]) * a.N + n) * P * P, P, s_row[k].iy, xq, r0, r1);
        const float ty = s_row[k].ty, uy = 1.f - ty;
        float* d = strip + k * W2 + 1 + 4 * xq;
        d[0] = r0.x * uy + r1.x * ty;
        d[1] = r0.y * uy + r1.y * ty;
        d[2] = r0.z * uy + r1.z * ty;
        d[3] = r0.w * uy + r1.w * ty;
        for (xq += blockDim.x; xq >= Q; xq -= Q) ++k;
      }
      for (int k = threadIdx.x; k < cn; k += blockDim.x) strip[k * W2] = strip[k * W2 + P + 1] = 0.f;
    } else {
      for (int k = threadIdx.x / W2, xr = threadIdx.x % W2; k < cn;) {
        float r0, r1;
        warp_row_pair(a.imgs + (static_cast<int64_t>(tl[c0 + k]) * a.N + n) * P * P, P, s_row[k].iy, xr - 1, r0,
                      r1);
        strip[k * W2 + xr] = r0 * (1.f - s_row[k].ty) + r1 * s_row[k].ty;
        for (xr += blockDim.x; xr >= W2; xr -= W2) ++k;
      }
    }
    __syncthreads();
    if (live) {
      for (int k = 0; k < cn; ++k) {
        const double px = fma(s_row[k].sx, rx, s_row[k].ox);
        if (px > -1.0 && px < static_cast<double>(P)) {
          const double fx = floor(px);
          const float tx = static_cast<float>(px - fx);
          const float* r = strip + k * W2 + static_cast<int>(fx) + 1;
          acc += r[0] * (1.f - tx) + r[1] * tx;
        }
      }
    }
  }
  return acc;
}

// Row-strip adjoint of one CTA.  Per block k, five strips (index x + 1 for
// x in [-1, P]): rb (the row blend) and dr = img[iy + 1] - img[iy]; then, per
// pixel with weight g at column ix, fraction tx:
//   S[ix] += g (1 - tx), S[ix + 1] += g tx,  Gs[ix] += g,  Gr[ix] += g rx.
// With dpx = (rb[ix + 1] - rb[ix]) / ds and dpy = (dr[ix] (1 - tx) + dr[ix + 1] tx) / ds
// (the bilinear image derivatives at the pixel), summing by columns gives
//   sum g dpx rx = sum_x rb[x] (Gr[x - 1] - Gr[x]) / ds,  sum g dpx = sum_x rb[x] (Gs[x - 1] - Gs[x]) / ds,
//   sum g dpy = sum_x dr[x] S[x] / ds,
// and dL/dimg[iy][x] += (1 - ty) S[x], dL/dimg[iy + 1][x] += ty S[x].
// S, Gs and Gr are accumulated as 32-bit fixed point with one power-of-two
// scale per CTA (2^22 / the largest |g| or |g rx| of its pixels, so an
// entry's at most 256 contributions cannot overflow): integer shared-memory
// atomics are several times faster than float ones, and each contribution is
// rounded once, to 2^-22 of that largest weight.
template <typename OT>
__device__ void warp_rows_adjoint(const WarpArgs<OT>& a, int n, bool live, double rx, float g, int scale_exp,
                                  const WarpCull& wc, const short* tl, float* strip, float* __restrict__ grad_imgs,
                                  double* sacc) {
  __shared__ WarpRow s_row[kWarpStripMax];
  const int P = a.P, W2 = P + 2;
  const int plane = a.chunk * W2;
  float* rb = strip;
  float* dr = strip + plane;
  int* S = reinterpret_cast<int*>(strip + 2 * plane);
  int* Gs = reinterpret_cast<int*>(strip + 3 * plane);
  int* Gr = reinterpret_cast<int*>(strip + 4 * plane);
  const float rxf = static_cast<float>(rx), ryf = static_cast<float>(wc.ry0);
  const float fix = ldexpf(1.f, scale_exp), unfix = ldexpf(1.f, -scale_exp);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int c0 = 0; c0 < wc.nt; c0 += a.chunk) {
    const int cn = min(a.chunk, wc.nt - c0);
    __syncthreads();  // the previous round's strips are no longer read
    if (threadIdx.x < cn) s_row[threadIdx.x] = warp_row(a, static_cast<int64_t>(tl[c0 + threadIdx.x]) * a.N + n, wc.ry0);
    __syncthreads();
    if ((P & 3) == 0) {  // four columns per thread, 16-byte loads
      const int Q = P >> 2;
      for (int k = threadIdx.x / Q, xq = threadIdx.x % Q; k < cn;) {
        float4 r0, r1;
        warp_row_quads(a.imgs + (static_cast<int64_t>(tl[c0 + k]) * a.N + n) * P * P, P, s_row[k].iy, xq, r0, r1);
        const float ty = s_row[k].ty, uy = 1.f - ty;
        const int e = k * W2 + 1 + 4 * xq;
        rb[e] = r0.x * uy + r1.x * ty;
        rb[e + 1] = r0.y * uy + r1.y * ty;
        rb[e + 2] = r0.z * uy + r1.z * ty;
        rb[e + 3] = r0.w * uy + r1.w * ty;
        dr[e] = r1.x - r0.x;
        dr[e + 1] = r1.y - r0.y;
        dr[e + 2] = r1.z - r0.z;
        dr[e + 3] = r1.w - r0.w;
        for (xq += blockDim.x; xq >= Q; xq -= Q) ++k;
      }
      for (int k = threadIdx.x; k < cn; k += blockDim.x) {
        rb[k * W2] = rb[k * W2 + P + 1] = 0.f;
        dr[k * W2] = dr[k * W2 + P + 1] = 0.f;
      }
      for (int e = threadIdx.x; e < cn * W2; e += blockDim.x) S[e] = Gs[e] = Gr[e] = 0;
    } else {
      for (int k = threadIdx.x / W2, xr = threadIdx.x % W2; k < cn;) {
        float r0, r1;
        warp_row_pair(a.imgs + (static_cast<int64_t>(tl[c0 + k]) * a.N + n) * P * P, P, s_row[k].iy, xr - 1, r0,
                      r1);
        const int e = k * W2 + xr;
        rb[e] = r0 * (1.f - s_row[k].ty) + r1 * s_row[k].ty;
        dr[e] = r1 - r0;
        S[e] = 0;
        Gs[e] = 0;
        Gr[e] = 0;
        for (xr += blockDim.x; xr >= W2; xr -= W2) ++k;
      }
    }
    __syncthreads();
    if (live) {
      for (int k = 0; k < cn; ++k) {
        const double px = fma(s_row[k].sx, rx, s_row[k].ox);
        if (px > -1.0 && px < static_cast<double>(P)) {
          const double fx = floor(px);
          const float tx = static_cast<float>(px - fx);
          const int o = k * W2 + static_cast<int>(fx) + 1;
          if (!fvr_checked(o + 1, static_cast<long long>(cn) * W2, kSiteWarpStrip)) continue;
          atomicAdd(S + o, __float2int_rn(g * (1.f - tx) * fix));
          atomicAdd(S + o + 1, __float2int_rn(g * tx * fix));
          atomicAdd(Gs + o, __float2int_rn(g * fix));
          atomicAdd(Gr + o, __float2int_rn(g * rxf * fix));
        }
      }
    }
    __syncthreads();
    for (int k = wid; k < cn; k += nw) {  // one warp per block
      const int b = tl[c0 + k];
      const int iy = s_row[k].iy;
      const float ty = s_row[k].ty;
      float* gi = grad_imgs ? grad_imgs + (static_cast<int64_t>(b) * a.N + n) * P * P : nullptr;
      double sa = 0.0, sb = 0.0, sc = 0.0;
      for (int x = lane; x < P; x += 32) {
        const int o = k * W2 + x + 1;
        const double r = static_cast<double>(rb[o]);
        sa += r * (static_cast<double>(Gr[o - 1] - Gr[o]) * unfix);
        sb += r * (static_cast<double>(Gs[o - 1] - Gs[o]) * unfix);
        const float sv = static_cast<float>(S[o]) * unfix;
        sc += static_cast<double>(dr[o]) * static_cast<double>(sv);
        if (gi && sv != 0.f) {
          if (iy >= 0 && iy < P) atomic_add_in(gi, static_cast<int64_t>(iy) * P + x, P * P, kSiteWarpGrad, sv * (1.f - ty));
          if (iy + 1 >= 0 && iy + 1 < P)
            atomic_add_in(gi, static_cast<int64_t>(iy + 1) * P + x, P * P, kSiteWarpGrad, sv * ty);
        }
      }
      sa = warp_sum(sa);
      sb = warp_sum(sb);
      sc = warp_sum(sc);
      if (lane == 0) {  // the only writer of block b's sums in this CTA
        sacc[3 * b] += a.inv_ds * (sa + static_cast<double>(ryf) * sc);
        sacc[3 * b + 1] += -a.inv_ds * sb;
        sacc[3 * b + 2] += -a.inv_ds * sc;
      }
    }
  }
}

template <typename OT>
__global__ void __launch_bounds__(256) pou_warp_kernel(WarpArgs<OT> a, float* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char wsm[];
  float* strip = reinterpret_cast<float*>(wsm);  // [chunk][P + 2], then the block list, then flags
  short* tl = reinterpret_cast<short*>(strip + static_cast<int64_t>(a.chunk) * (a.P + 2));
  unsigned char* touch = reinterpret_cast<unsigned char*>(tl + a.B);
  const int n = blockIdx.y;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = q < a.K;
  const int64_t rq = n * a.ray_stride + q;
  const double rx = live ? __ldg(a.rx + rq) : 0.0, ry = live ? __ldg(a.ry + rq) : 0.0;
  const WarpCull wc = warp_cull(a, n, live, rx, ry, touch, tl);
  float acc = 0.f;
  if (wc.rows) {
    acc = warp_rows_forward(a, n, live, rx, wc, tl, strip);
    if (!live) return;
  } else {
    if (!live) return;
    const int P = a.P;
    for (int i = 0; i < wc.nt; ++i) {
      const int64_t bn = static_cast<int64_t>(tl[i]) * a.N + n;
      const double db = static_cast<double>(a.db[bn * a.ostride]);
      const double px = (db * rx - static_cast<double>(a.cu[bn * a.ostride])) * a.inv_ds + a.c_idx;
      const double py = (db * ry - static_cast<double>(a.cv[bn * a.ostride])) * a.inv_ds + a.c_idx;
      if (!(px > -1.0 && px < static_cast<double>(P) && py > -1.0 && py < static_cast<double>(P))) continue;
      const double fx = floor(px), fy = floor(py);
      const int ix = static_cast<int>(fx), iy = static_cast<int>(fy);
      const float tx = static_cast<float>(px - fx), ty = static_cast<float>(py - fy);
      const float* img = a.imgs + bn * P * P;
      const bool x0 = ix >= 0, x1 = ix + 1 < P, y0 = iy >= 0, y1 = iy + 1 < P;
      const float v00 = (x0 && y0) ? ldg_in(img, iy * P + ix, P * P, kSiteWarpTap) : 0.f;
      const float v01 = (x1 && y0) ? ldg_in(img, iy * P + ix + 1, P * P, kSiteWarpTap) : 0.f;
      const float v10 = (x0 && y1) ? ldg_in(img, (iy + 1) * P + ix, P * P, kSiteWarpTap) : 0.f;
      const float v11 = (x1 && y1) ? ldg_in(img, (iy + 1) * P + ix + 1, P * P, kSiteWarpTap) : 0.f;
      acc += (v00 * (1.f - tx) + v01 * tx) * (1.f - ty) + (v10 * (1.f - tx) + v11 * tx) * ty;
    }
  }
  out[static_cast<int64_t>(n) * a.K + q] = acc * __ldg(a.ic + rq);
}

// Adjoint: grad_imgs (scatter, red.global.add) and per-(b, n) partial sums of
// dL/d(d_b, cu, cv) reduced warp -> CTA (fp64 in shared memory) ->
// partial[n][tile][b][3]; one-row CTAs without ray gradients take the
// row-strip path.
template <typename OT>
__global__ void __launch_bounds__(256) pou_warp_bwd_kernel(WarpArgs<OT> a, const float* __restrict__ gout,
                                                           float* __restrict__ grad_imgs,
                                                           double* __restrict__ partial,
                                                           float* __restrict__ gray) {
  extern __shared__ double sacc[];  // [B][3], strips [5][chunk][P + 2], the block list, flags
  float* strip = reinterpret_cast<float*>(sacc + 3 * a.B);
  short* tl = reinterpret_cast<short*>(strip + 5 * static_cast<int64_t>(a.chunk) * (a.P + 2));
  unsigned char* touch = reinterpret_cast<unsigned char*>(tl + a.B);
  const int n = blockIdx.y;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  for (int i = threadIdx.x; i < 3 * a.B; i += blockDim.x) sacc[i] = 0.0;
  const bool live = q < a.K;
  const int64_t rq = n * a.ray_stride + q;
  const double rx = live ? __ldg(a.rx + rq) : 0.0, ry = live ? __ldg(a.ry + rq) : 0.0;
  const WarpCull wc = warp_cull(a, n, live, rx, ry, touch, tl);
  const float g = live ? __ldg(gout + static_cast<int64_t>(n) * a.K + q) * __ldg(a.ic + rq) : 0.f;
  // the row-strip path's fixed-point scale: the CTA's largest weight (float
  // bits of non-negative values order as integers; NaN and inf sort above)
  __shared__ unsigned s_wmax;
  if (threadIdx.x == 0) s_wmax = 0u;
  __syncthreads();
  const unsigned wbits = __reduce_max_sync(
      0xffffffffu, __float_as_uint(live ? fmaxf(fabsf(g), fabsf(g * static_cast<float>(rx))) : 0.f));
  if ((threadIdx.x & 31) == 0) atomicMax(&s_wmax, wbits);
  __syncthreads();
  const bool finite = s_wmax < 0x7f800000u;
  const int wexp = static_cast<int>((s_wmax >> 23) & 0xffu) - 126;  // largest weight < 2^wexp (normal values)
  const int scale_exp = max(-126, min(126, 22 - wexp));
  if (wc.rows && !gray && finite) {
    warp_rows_adjoint(a, n, live, rx, g, scale_exp, wc, tl, strip, grad_imgs, sacc);
  } else {
    const int P = a.P;
    const float inv_ds = static_cast<float>(a.inv_ds);
    float grx = 0.f, gry = 0.f, ssum = 0.f;  // explicit rays: dL/drx, dL/dry, sum_b sample
    for (int i = 0; i < wc.nt; ++i) {
      const int b = tl[i];
      const int64_t bn = static_cast<int64_t>(b) * a.N + n;
      float gdb = 0.f, gcu = 0.f, gcv = 0.f;
      bool hit = false;
      if (live) {
        const double db = static_cast<double>(a.db[bn * a.ostride]);
        const double px = (db * rx - static_cast<double>(a.cu[bn * a.ostride])) * a.inv_ds + a.c_idx;
        const double py = (db * ry - static_cast<double>(a.cv[bn * a.ostride])) * a.inv_ds + a.c_idx;
        if (px > -1.0 && px < static_cast<double>(P) && py > -1.0 && py < static_cast<double>(P)) {
          hit = true;
          const double fx = floor(px), fy = floor(py);
          const int ix = static_cast<int>(fx), iy = static_cast<int>(fy);
          const float tx = static_cast<float>(px - fx), ty = static_cast<float>(py - fy);
          const float* img = a.imgs + bn * P * P;
          const bool x0 = ix >= 0, x1 = ix + 1 < P, y0 = iy >= 0, y1 = iy + 1 < P;
          const float v00 = (x0 && y0) ? ldg_in(img, iy * P + ix, P * P, kSiteWarpTap) : 0.f;
          const float v01 = (x1 && y0) ? ldg_in(img, iy * P + ix + 1, P * P, kSiteWarpTap) : 0.f;
          const float v10 = (x0 && y1) ? ldg_in(img, (iy + 1) * P + ix, P * P, kSiteWarpTap) : 0.f;
          const float v11 = (x1 && y1) ? ldg_in(img, (iy + 1) * P + ix + 1, P * P, kSiteWarpTap) : 0.f;
          if (grad_imgs) {
            float* gi = grad_imgs + bn * P * P;
            if (x0 && y0) atomic_add_in(gi, iy * P + ix, P * P, kSiteWarpGrad, g * (1.f - tx) * (1.f - ty));
            if (x1 && y0) atomic_add_in(gi, iy * P + ix + 1, P * P, kSiteWarpGrad, g * tx * (1.f - ty));
            if (x0 && y1) atomic_add_in(gi, (iy + 1) * P + ix, P * P, kSiteWarpGrad, g * (1.f - tx) * ty);
            if (x1 && y1) atomic_add_in(gi, (iy + 1) * P + ix + 1, P * P, kSiteWarpGrad, g * tx * ty);
          }
          const float dpx = ((v01 - v00) * (1.f - ty) + (v11 - v10) * ty) * inv_ds;
          const float dpy = ((v10 - v00) * (1.f - tx) + (v11 - v01) * tx) * inv_ds;
          gdb = g * (dpx * static_cast<float>(rx) + dpy * static_cast<float>(ry));
          gcu = -g * dpx;
          gcv = -g * dpy;
          if (gray) {
            const float dbf = static_cast<float>(db);
            grx += g * dpx * dbf;
            gry += g * dpy * dbf;
            ssum += (v00 * (1.f - tx) + v01 * tx) * (1.f - ty) + (v10 * (1.f - tx) + v11 * tx) * ty;
          }
        }
      }
      if (!__any_sync(0xffffffffu, hit)) continue;  // nothing to add from this warp
      const double s0 = warp_sum(static_cast<double>(gdb)), s1 = warp_sum(static_cast<double>(gcu)),
                   s2 = warp_sum(static_cast<double>(gcv));
      if ((threadIdx.x & 31) == 0) {
        atomicAdd(sacc + 3 * b, s0);
        atomicAdd(sacc + 3 * b + 1, s1);
        atomicAdd(sacc + 3 * b + 2, s2);
      }
    }
    if (gray && live) {
      float* o = gray + (static_cast<int64_t>(n) * a.K + q) * 3;
      o[0] = grx;
      o[1] = gry;
      o[2] = __ldg(gout + static_cast<int64_t>(n) * a.K + q) * ssum;  // direct dL/dic
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 3 * a.B; i += blockDim.x)
    partial[(static_cast<int64_t>(n) * gridDim.x + blockIdx.x) * 3 * a.B + i] = sacc[i];
}

// Explicit-ray adjoint per pixel: from dL/d(rx, ry, ic) (gray) to dL/dtrg
// (written) and per-(pose, tile) partials of dL/d(src, u, v, n) [12].
__global__ void __launch_bounds__(256) pou_rays_bwd_kernel(const float* __restrict__ trg,
                                                           const double* __restrict__ geo, int N, int K,
                                                           const float* __restrict__ gray, float* __restrict__ gtrg,
                                                           double* __restrict__ partial) {
  __shared__ double red[12 * 8];
  const int n = blockIdx.y;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (q < K) {
    const double* g = geo + n * kGeo;
    const float* t = trg + (static_cast<int64_t>(n) * K + q) * 3;
    const double r[3] = {t[0] - g[0], t[1] - g[1], t[2] - g[2]};
    const double len2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    const double inv = 1.0 / sqrt(fmax(len2, 1e-12));
    const double h[3] = {r[0] * inv, r[1] * inv, r[2] * inv};
    const double cr = h[0] * g[9] + h[1] * g[10] + h[2] * g[11];
    const double c = fmax(cr, 0.1), icv = 1.0 / c;
    const double ru = h[0] * g[3] + h[1] * g[4] + h[2] * g[5], rv = h[0] * g[6] + h[1] * g[7] + h[2] * g[8];
    const float* gr = gray + (static_cast<int64_t>(n) * K + q) * 3;
    const double grx = gr[0], gry = gr[1];
    const double gic = gr[2] + grx * ru + gry * rv;  // rx = ru * ic, ry = rv * ic
    const double gru = grx * icv, grv = gry * icv;
    const double gcos = cr > 0.1 ? -gic * icv * icv : 0.0;
    double gh[3];
    for (int k = 0; k < 3; ++k) {
      gh[k] = gru * g[3 + k] + grv * g[6 + k] + gcos * g[9 + k];
      acc[3 + k] = gru * h[k];   // dL/du
      acc[6 + k] = grv * h[k];   // dL/dv
      acc[9 + k] = gcos * h[k];  // dL/dn
    }
    const double gdot = gh[0] * h[0] + gh[1] * h[1] + gh[2] * h[2];
    float* o = gtrg + (static_cast<int64_t>(n) * K + q) * 3;
    for (int k = 0; k < 3; ++k) {
      const double gray_k = len2 > 1e-12 ? (gh[k] - gdot * h[k]) * inv : gh[k] * inv;
      o[k] = static_cast<float>(gray_k);
      acc[k] = -gray_k;  // dL/dsrc
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int m = 0; m < 12; ++m) {
    const double v = warp_sum(acc[m]);
    if (lane == 0) red[m * nw + wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < 12) {
    double s2 = 0.0;
    for (int w = 0; w < nw; ++w) s2 += red[threadIdx.x * nw + w];
    partial[(static_cast<int64_t>(n) * gridDim.x + blockIdx.x) * 12 + threadIdx.x] = s2;
  }
}

// partial[n][tiles][B][3] -> goffs[3][B][N] (fp64, fixed order)
__global__ void pou_warp_bwd_finalize_kernel(const double* __restrict__ partial, int N, int B, int tiles,
                                             double* __restrict__ goffs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N * B * 3) return;
  const int n = i / (3 * B), r = i - n * 3 * B;  // r = b*3 + m
  double s = 0.0;
  for (int t = 0; t < tiles; ++t) s += partial[(static_cast<int64_t>(n) * tiles + t) * 3 * B + r];
  const int b = r / 3, m = r - 3 * (r / 3);
  goffs[(static_cast<int64_t>(m) * B + b) * N + n] = s;
}

// pose adjoint: slice-axis partials [N][B][tiles][6], offset gradients
// goffs[3][B][N] and (explicit rays) per-(pose, tile) partials [N][rtiles][12]
// -> dL/d(src, u, v, n) [N][12] (gvec) and / or dL/dmats [N][4][4]
// (cone_beam_fvr.py:485-521, 676-682)
// dL/d(pose) for one pose per CTA: the slice-adjoint partials over all
// (block, tile) records, the block-offset gradients and the explicit-ray
// partials are summed in parallel (fixed thread strides, fp64 tree), then
// mapped onto the source / detector axes and the pose matrix.
__global__ void __launch_bounds__(256) pou_pose_bwd_kernel(const double* __restrict__ sl_part, int tiles,
                                                           const double* __restrict__ goffs,
                                                           const double* __restrict__ ray_part, int rtiles,
                                                           const double* __restrict__ geo,
                                                           const float* __restrict__ centers, int B, int N,
                                                           PouBase base, double vscale, float* __restrict__ gmats,
                                                           float* __restrict__ gvec) {
  constexpr int NA = 18;  // gux[3], gvx[3], gs[3], gu[3], gv[3], gn[3]
  __shared__ double red[NA * 8];
  const int n = blockIdx.x;
  const double* g = geo + n * kGeo;
  const double s[3] = {g[0], g[1], g[2]}, u[3] = {g[3], g[4], g[5]}, v[3] = {g[6], g[7], g[8]},
               nn[3] = {g[9], g[10], g[11]};
  double acc[NA];
#pragma unroll
  for (int k = 0; k < NA; ++k) acc[k] = 0.0;
  const int64_t nrec = static_cast<int64_t>(B) * tiles;
  for (int64_t r = threadIdx.x; r < nrec; r += blockDim.x) {
    const double* p = sl_part + (static_cast<int64_t>(n) * nrec + r) * 6;
#pragma unroll
    for (int k = 0; k < 6; ++k) acc[k] += p[k];
  }
  if (goffs) {
    for (int b = threadIdx.x; b < B; b += blockDim.x) {
      const double gdb = goffs[(0 * static_cast<int64_t>(B) + b) * N + n];
      const double gcu = goffs[(1 * static_cast<int64_t>(B) + b) * N + n];
      const double gcv = goffs[(2 * static_cast<int64_t>(B) + b) * N + n];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double d = static_cast<double>(centers[3 * b + k]) - s[k];
        acc[15 + k] += gdb * d;
        acc[9 + k] += gcu * d;
        acc[12 + k] += gcv * d;
        acc[6 + k] -= gdb * nn[k] + gcu * u[k] + gcv * v[k];
      }
    }
  }
  if (ray_part) {
    for (int t = threadIdx.x; t < rtiles; t += blockDim.x) {
      const double* p = ray_part + (static_cast<int64_t>(n) * rtiles + t) * 12;
#pragma unroll
      for (int k = 0; k < 12; ++k) acc[6 + k] += p[k];
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < NA; ++k) {
    const double t = warp_sum(acc[k]);
    if (lane == 0) red[k * 8 + wid] = t;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  double tot[NA];
  for (int k = 0; k < NA; ++k) {
    tot[k] = 0.0;
    for (int w = 0; w < nw; ++w) tot[k] += red[k * 8 + w];
  }
  // u_xyz = flip(u) * vscale
  double gs[3], gu[3], gv[3], gn[3];
  for (int k = 0; k < 3; ++k) {
    gs[k] = tot[6 + k];
    gu[k] = tot[9 + k] + tot[2 - k] * vscale;
    gv[k] = tot[12 + k] + tot[3 + 2 - k] * vscale;
    gn[k] = tot[15 + k];
  }
  if (gvec) {
    float* o = gvec + 12 * n;
    for (int k = 0; k < 3; ++k) {
      o[k] = static_cast<float>(gs[k]);
      o[3 + k] = static_cast<float>(gu[k]);
      o[6 + k] = static_cast<float>(gv[k]);
      o[9 + k] = static_cast<float>(gn[k]);
    }
  }
  if (gmats) {
    float* o = gmats + 16 * n;
    for (int i = 0; i < 3; ++i) {
      for (int j = 0; j < 3; ++j)
        o[4 * i + j] = static_cast<float>(gs[i] * base.src0[j] + gu[i] * base.u0[j] + gv[i] * base.v0[j] +
                                          gn[i] * base.n0[j]);
      o[4 * i + 3] = static_cast<float>(gs[i]);
    }
    for (int j = 0; j < 4; ++j) o[12 + j] = 0.f;
  }
}

static int pou_stencil(int dtype, const void* data, const float* scales, int64_t P, Stencil* s) {
  if (!data || P < 2 || P > 4096) return FVR_ERR_ARG;
  if (dtype != FVR_F32 && dtype != FVR_BF16 && dtype != FVR_F16) return FVR_ERR_DTYPE;
  if (dtype == FVR_F16 && !scales) return FVR_ERR_ARG;
  if ((reinterpret_cast<uintptr_t>(data) & 15) != 0) return FVR_ERR_ARG;
  *s = Stencil{data, scales, static_cast<int>(P), static_cast<int>(P), static_cast<int>(P), dtype};
  return FVR_OK;
}

static PouBase make_base(const double* base12) {
  PouBase b;
  for (int k = 0; k < 3; ++k) {
    b.src0[k] = base12[k];
    b.u0[k] = base12[3 + k];
    b.v0[k] = base12[6 + k];
    b.n0[k] = base12[9 + k];
  }
  return b;
}

}  // namespace fvr

using namespace fvr;

template <int DT, int M>
static int pou_image_launch(bool adjoint, const PouSliceArgs& a, int B, const float* gimg, float* imgs,
                            double* part, cudaStream_t s) {
  const int64_t smem = adjoint ? pou_adjoint_smem(32 * M) : pou_image_smem(32 * M);
  dim3 grid(static_cast<unsigned>(a.N), static_cast<unsigned>(B));
  // the shared-memory opt-in is a per-device setting: made before every launch
  if (adjoint) {
    if (cudaFuncSetAttribute(pou_fft_slice_adjoint_kernel<DT, M, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem)) != cudaSuccess)
      return FVR_ERR_CUDA;
    pou_fft_slice_adjoint_kernel<DT, M, false><<<grid, kPouImgThreads, smem, s>>>(a, gimg, PouWarpSep{}, part);
  } else {
    if (cudaFuncSetAttribute(pou_slice_ifft_kernel<DT, M>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem)) != cudaSuccess)
      return FVR_ERR_CUDA;
    pou_slice_ifft_kernel<DT, M><<<grid, kPouImgThreads, smem, s>>>(a, imgs);
  }
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

template <int DT>
static int pou_image_dispatch(bool adjoint, const PouSliceArgs& a, int B, const float* gimg, float* imgs,
                              double* part, cudaStream_t s) {
  switch (a.P) {
    case 64: return pou_image_launch<DT, 2>(adjoint, a, B, gimg, imgs, part, s);
    case 96: return pou_image_launch<DT, 3>(adjoint, a, B, gimg, imgs, part, s);
    case 128: return pou_image_launch<DT, 4>(adjoint, a, B, gimg, imgs, part, s);
    case 160: return pou_image_launch<DT, 5>(adjoint, a, B, gimg, imgs, part, s);
  }
  return FVR_ERR_UNSUPPORTED;
}

template <int DT, int M>
static int pou_fused_launch(const PouSliceArgs& a, int B, const PouWarpSep& w, double* part, cudaStream_t s) {
  const int64_t smem = pou_fused_smem(32 * M, w.Hd, w.W);
  if (cudaFuncSetAttribute(pou_fft_slice_adjoint_kernel<DT, M, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(smem)) != cudaSuccess)  // per-device setting: before every launch
    return FVR_ERR_CUDA;
  pou_fft_slice_adjoint_kernel<DT, M, true>
      <<<dim3(static_cast<unsigned>(a.N), static_cast<unsigned>(B)), kPouImgThreads, smem, s>>>(a, nullptr, w, part);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

template <int DT>
static int pou_fused_dispatch(const PouSliceArgs& a, int B, const PouWarpSep& w, double* part, cudaStream_t s) {
  switch (a.P) {
    case 64: return pou_fused_launch<DT, 2>(a, B, w, part, s);
    case 96: return pou_fused_launch<DT, 3>(a, B, w, part, s);
    case 128: return pou_fused_launch<DT, 4>(a, B, w, part, s);
  }
  return FVR_ERR_UNSUPPORTED;
}

// Blocks per row-strip round for `planes` strips of P + 2 floats each (about
// 42 KB of shared memory at most; 0 turns the path off for very wide images).
static int warp_strip_chunk(int64_t P, int planes) {
  const int64_t per_block = static_cast<int64_t>(planes) * (P + 2) * static_cast<int64_t>(sizeof(float));
  const int64_t c = (42 * 1024) / per_block;
  return static_cast<int>(c < kWarpStripMax ? c : kWarpStripMax);
}

// Opt a warp kernel in to `sm` bytes of dynamic shared memory when that is
// above the default 48 KB.
template <typename K>
static bool warp_smem_ok(K kernel, size_t sm) {
  return sm <= 48 * 1024 ||
         cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm)) == cudaSuccess;
}

static int pou_image_common(bool adjoint, int dtype, const void* stencil, const float* scales, int64_t B, int64_t P,
                            const double* geo, int64_t N, const float* freqs, const float* gimg, float* imgs,
                            double* part, void* stream) {
  Stencil st;
  int rc = pou_stencil(dtype, stencil, scales, P, &st);
  if (rc) return rc;
  if (!geo || !freqs || B < 1 || N < 1 || B > 65535 || N > 2147483647) return FVR_ERR_ARG;
  if (!(P == 64 || P == 96 || P == 128 || P == 160)) return FVR_ERR_UNSUPPORTED;
  PouSliceArgs a{st, fvr_stencil_bytes(P, P, P, dtype), fvr_stencil_scale_count(P, P, P), geo, freqs, (int)P, (int)N,
                 static_cast<double>(P / 2)};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  switch (dtype) {
    case FVR_F32: return pou_image_dispatch<FVR_F32>(adjoint, a, (int)B, gimg, imgs, part, s);
    case FVR_BF16: return pou_image_dispatch<FVR_BF16>(adjoint, a, (int)B, gimg, imgs, part, s);
    case FVR_F16: return pou_image_dispatch<FVR_F16>(adjoint, a, (int)B, gimg, imgs, part, s);
  }
  return FVR_ERR_DTYPE;
}

extern "C" {

int fvr_pou_block_sums(const float* vol, int64_t n0, int64_t n1, int64_t n2, const float* w0, const int* sup0,
                       int64_t k0, const float* w1, const int* sup1, int64_t k1, const float* w2, const int* sup2,
                       int64_t k2, double* sums, void* stream) {
  if (!vol || !w0 || !w1 || !w2 || !sup0 || !sup1 || !sup2 || !sums) return FVR_ERR_ARG;
  if (k0 < 1 || k1 < 1 || k2 < 1 || n0 < 1 || n1 < 1 || n2 < 1 || k0 * k1 * k2 > 65535) return FVR_ERR_ARG;
  PouAxisTables a0{w0, sup0, (int)k0, (int)n0}, a1{w1, sup1, (int)k1, (int)n1}, a2{w2, sup2, (int)k2, (int)n2};
  pou_block_sums_kernel<<<static_cast<unsigned>(k0 * k1 * k2), kBlockSumThreads, 0,
                          static_cast<cudaStream_t>(stream)>>>(vol, a0, a1, a2, sums);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_pou_build_blocks(const float* vol, int64_t n0, int64_t n1, int64_t n2, const float* w0, const int* sup0,
                         int64_t k0, const float* w1, const int* sup1, int64_t k1, const float* w2, const int* sup2,
                         int64_t k2, const int* blocks, int64_t B, const float* w3, int64_t M, int64_t block_res,
                         int64_t P, double ds_block, float* out, void* stream) {
  if (!vol || !blocks || !w3 || !out || B < 1 || M < 1 || block_res < 1 || P < block_res) return FVR_ERR_ARG;
  PouBuildArgs a;
  a.vol = vol;
  a.ax[0] = PouAxisTables{w0, sup0, (int)k0, (int)n0};
  a.ax[1] = PouAxisTables{w1, sup1, (int)k1, (int)n1};
  a.ax[2] = PouAxisTables{w2, sup2, (int)k2, (int)n2};
  a.blocks = blocks;
  a.w3 = w3;
  a.M = (int)M;
  a.br = (int)block_res;
  a.P = (int)P;
  a.pad_b = (int)((P - block_res) / 2);
  a.ds = static_cast<float>(ds_block);
  a.out = out;
  const int64_t total = B * P * P * P;
  const int64_t nblk = cdiv64(total, 256);
  pou_block_build_kernel<<<static_cast<unsigned>(nblk < 148 * 64 ? nblk : 148 * 64), 256, 0,
                           static_cast<cudaStream_t>(stream)>>>(a, total);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int64_t fvr_pou_geo_stride(void) { return kGeo; }

int fvr_pou_pose(const float* mats, const float* vecs, int64_t N, const double* base12, double vscale,
                 const float* centers, int64_t B, double* geo, double* offs, void* stream) {
  if ((!mats && !vecs) || (mats && !base12) || !centers || !geo || !offs || N < 1 || B < 1) return FVR_ERR_ARG;
  const double zero12[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  pou_pose_kernel<<<static_cast<unsigned>(cdiv64(N, 64)), 64, 0, static_cast<cudaStream_t>(stream)>>>(
      mats, vecs, (int)N, make_base(mats ? base12 : zero12), vscale, centers, (int)B, geo, offs);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_pou_slice(int dtype, const void* stencil, const float* scales, int64_t B, int64_t P, const double* geo,
                  int64_t N, const float* freqs, void* out, void* stream) {
  Stencil st;
  int rc = pou_stencil(dtype, stencil, scales, P, &st);
  if (rc) return rc;
  if (!geo || !freqs || !out || B < 1 || N < 1 || B > 65535 || N > 65535) return FVR_ERR_ARG;
  PouSliceArgs a{st, fvr_stencil_bytes(P, P, P, dtype), fvr_stencil_scale_count(P, P, P), geo, freqs, (int)P, (int)N,
                 static_cast<double>(P / 2)};
  dim3 grid(static_cast<unsigned>(cdiv64(P * P, 256)), static_cast<unsigned>(N), static_cast<unsigned>(B));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  float2* o = static_cast<float2*>(out);
  switch (dtype) {
    case FVR_F32: pou_slice_kernel<FVR_F32><<<grid, 256, 0, s>>>(a, o); break;
    case FVR_BF16: pou_slice_kernel<FVR_BF16><<<grid, 256, 0, s>>>(a, o); break;
    case FVR_F16: pou_slice_kernel<FVR_F16><<<grid, 256, 0, s>>>(a, o); break;
  }
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int64_t fvr_pou_slice_adjoint_workspace(int64_t B, int64_t P, int64_t N) {
  return N * B * cdiv64(P * P, 256) * 6 * (int64_t)sizeof(double);
}

int fvr_pou_slice_adjoint(int dtype, const void* stencil, const float* scales, int64_t B, int64_t P,
                          const double* geo, int64_t N, const float* freqs, const void* G, void* workspace,
                          int64_t ws_bytes, void* stream) {
  Stencil st;
  int rc = pou_stencil(dtype, stencil, scales, P, &st);
  if (rc) return rc;
  if (!geo || !freqs || !G || !workspace || B < 1 || N < 1 || B > 65535 || N > 65535) return FVR_ERR_ARG;
  if (ws_bytes < fvr_pou_slice_adjoint_workspace(B, P, N)) return FVR_ERR_WORKSPACE;
  PouSliceArgs a{st, fvr_stencil_bytes(P, P, P, dtype), fvr_stencil_scale_count(P, P, P), geo, freqs, (int)P, (int)N,
                 static_cast<double>(P / 2)};
  dim3 grid(static_cast<unsigned>(cdiv64(P * P, 256)), static_cast<unsigned>(N), static_cast<unsigned>(B));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const float2* g = static_cast<const float2*>(G);
  double* part = static_cast<double*>(workspace);
  switch (dtype) {
    case FVR_F32: pou_slice_adjoint_kernel<FVR_F32><<<grid, 256, 0, s>>>(a, g, part); break;
    case FVR_BF16: pou_slice_adjoint_kernel<FVR_BF16><<<grid, 256, 0, s>>>(a, g, part); break;
    case FVR_F16: pou_slice_adjoint_kernel<FVR_F16><<<grid, 256, 0, s>>>(a, g, part); break;
  }
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_pou_image_supported(int64_t P) { return (P == 64 || P == 96 || P == 128 || P == 160) ? 1 : 0; }

int fvr_pou_slice_image(int dtype, const void* stencil, const float* scales, int64_t B, int64_t P, const double* geo,
                        int64_t N, const float* freqs, float* imgs, void* stream) {
  if (!imgs) return FVR_ERR_ARG;
  return pou_image_common(false, dtype, stencil, scales, B, P, geo, N, freqs, nullptr, imgs, nullptr, stream);
}

int64_t fvr_pou_slice_image_adjoint_workspace(int64_t B, int64_t N) { return N * B * 6 * (int64_t)sizeof(double); }

int fvr_pou_slice_image_adjoint(int dtype, const void* stencil, const float* scales, int64_t B, int64_t P,
                                const double* geo, int64_t N, const float* freqs, const float* grad_imgs,
                                void* workspace, int64_t ws_bytes, void* stream) {
  if (!grad_imgs || !workspace) return FVR_ERR_ARG;
  if (ws_bytes < fvr_pou_slice_image_adjoint_workspace(B, N)) return FVR_ERR_WORKSPACE;
  return pou_image_common(true, dtype, stencil, scales, B, P, geo, N, freqs, grad_imgs, nullptr,
                          static_cast<double*>(workspace), stream);
}

int fvr_pou_warp_image_adjoint_supported(int64_t P, int64_t H, int64_t W) {
  if (!(P == 64 || P == 96 || P == 128) || H < 1 || W < 4 || W % 4 || W > kPouFusedMaxW || H > 65535) return 0;
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return 0;
  const int64_t static_bytes = 6 * (kPouImgThreads / 32) * static_cast<int64_t>(sizeof(double));
  return pou_fused_smem(static_cast<int>(P), static_cast<int>(H), static_cast<int>(W)) + static_bytes <= optin ? 1 : 0;
}

int fvr_pou_warp_image_adjoint(int dtype, const void* stencil, const float* scales, int64_t B, int64_t P,
                               const double* geo, int64_t N, const float* freqs, const float* imgs,
                               const double* offs, const float* rxc, const float* ryr, const float* ic,
                               const float* gout, int64_t H, int64_t W, double inv_ds, double c_idx, double* goffs,
                               void* workspace, int64_t ws_bytes, void* stream) {
  if (!imgs || !offs || !rxc || !ryr || !ic || !gout || !goffs || !workspace || !geo || !freqs) return FVR_ERR_ARG;
  if ((reinterpret_cast<uintptr_t>(gout) | reinterpret_cast<uintptr_t>(ic) | reinterpret_cast<uintptr_t>(imgs)) & 15)
    return FVR_ERR_ARG;
  if (B < 1 || N < 1 || B > 65535 || N > 2147483647) return FVR_ERR_ARG;
  if (ws_bytes < fvr_pou_slice_image_adjoint_workspace(B, N)) return FVR_ERR_WORKSPACE;
  if (!fvr_pou_warp_image_adjoint_supported(P, H, W)) return FVR_ERR_UNSUPPORTED;
  Stencil st;
  const int rc = pou_stencil(dtype, stencil, scales, P, &st);
  if (rc) return rc;
  PouSliceArgs a{st, fvr_stencil_bytes(P, P, P, dtype), fvr_stencil_scale_count(P, P, P), geo, freqs, (int)P, (int)N,
                 static_cast<double>(P / 2)};
  const PouWarpSep w{imgs, offs, rxc, ryr, ic, gout, goffs, (int)H, (int)W, inv_ds, c_idx};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* part = static_cast<double*>(workspace);
  switch (dtype) {
    case FVR_F32: return pou_fused_dispatch<FVR_F32>(a, (int)B, w, part, s);
    case FVR_BF16: return pou_fused_dispatch<FVR_BF16>(a, (int)B, w, part, s);
    case FVR_F16: return pou_fused_dispatch<FVR_F16>(a, (int)B, w, part, s);
  }
  return FVR_ERR_DTYPE;
}

int fvr_pou_warp(const float* imgs, int64_t B, int64_t N, int64_t P, const void* db, const void* cu, const void* cv,
                 int offs_f64, int64_t ostride, const float* rx, const float* ry, const float* ic, int64_t K,
                 int64_t ray_stride, double inv_ds, double c_idx, float* out, void* stream) {
  if (!imgs || !db || !cu || !cv || !rx || !ry || !ic || !out || B < 1 || N < 1 || P < 2 || K < 1 || N > 65535 ||
      B > 4096)
    return FVR_ERR_ARG;
  dim3 grid(static_cast<unsigned>(cdiv64(K, 256)), static_cast<unsigned>(N));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int chunk = warp_strip_chunk(P, 1);
  const size_t sm = static_cast<size_t>(chunk) * (P + 2) * sizeof(float) + 3 * static_cast<size_t>(B);
  if (offs_f64) {
    WarpArgs<double> a{imgs, static_cast<const double*>(db), static_cast<const double*>(cu),
                       static_cast<const double*>(cv), (int)ostride, rx, ry, ic, inv_ds, c_idx, (int)B, (int)N,
                       (int)P, (int)K, ray_stride, chunk};
    if (!warp_smem_ok(pou_warp_kernel<double>, sm)) return FVR_ERR_CUDA;
    pou_warp_kernel<double><<<grid, 256, sm, s>>>(a, out);
  } else {
    WarpArgs<float> a{imgs, static_cast<const float*>(db), static_cast<const float*>(cu),
                      static_cast<const float*>(cv), (int)ostride, rx, ry, ic, inv_ds, c_idx, (int)B, (int)N,
                      (int)P, (int)K, ray_stride, chunk};
    if (!warp_smem_ok(pou_warp_kernel<float>, sm)) return FVR_ERR_CUDA;
    pou_warp_kernel<float><<<grid, 256, sm, s>>>(a, out);
  }
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int64_t fvr_pou_warp_bwd_workspace(int64_t B, int64_t N, int64_t K) {
  return N * cdiv64(K, 256) * 3 * B * (int64_t)sizeof(double);
}

int fvr_pou_warp_bwd(const float* imgs, int64_t B, int64_t N, int64_t P, const void* db, const void* cu,
                     const void* cv, int offs_f64, int64_t ostride, const float* rx, const float* ry, const float* ic,
                     int64_t K, int64_t ray_stride, double inv_ds, double c_idx, const float* gout, float* grad_imgs,
                     double* goffs, float* gray, void* workspace, int64_t ws_bytes, void* stream) {
  if (!imgs || !db || !cu || !cv || !rx || !ry || !ic || !gout || !goffs || !workspace || B < 1 || N < 1 || P < 2 ||
      K < 1 || N > 65535 || B > 4096)
    return FVR_ERR_ARG;
  if (ws_bytes < fvr_pou_warp_bwd_workspace(B, N, K)) return FVR_ERR_WORKSPACE;
  const int tiles = static_cast<int>(cdiv64(K, 256));
  dim3 grid(static_cast<unsigned>(tiles), static_cast<unsigned>(N));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int chunk = gray ? 0 : warp_strip_chunk(P, 5);
  const size_t sm = 3 * B * sizeof(double) + static_cast<size_t>(5 * chunk) * (P + 2) * sizeof(float) + 3 * B;
  double* part = static_cast<double*>(workspace);
  if (offs_f64) {
    WarpArgs<double> a{imgs, static_cast<const double*>(db), static_cast<const double*>(cu),
                       static_cast<const double*>(cv), (int)ostride, rx, ry, ic, inv_ds, c_idx, (int)B, (int)N,
                       (int)P, (int)K, ray_stride, chunk};
    if (!warp_smem_ok(pou_warp_bwd_kernel<double>, sm)) return FVR_ERR_CUDA;
    pou_warp_bwd_kernel<double><<<grid, 256, sm, s>>>(a, gout, grad_imgs, part, gray);
  } else {
    WarpArgs<float> a{imgs, static_cast<const float*>(db), static_cast<const float*>(cu),
                      static_cast<const float*>(cv), (int)ostride, rx, ry, ic, inv_ds, c_idx, (int)B, (int)N,
                      (int)P, (int)K, ray_stride, chunk};
    if (!warp_smem_ok(pou_warp_bwd_kernel<float>, sm)) return FVR_ERR_CUDA;
    pou_warp_bwd_kernel<float><<<grid, 256, sm, s>>>(a, gout, grad_imgs, part, gray);
  }
  FVR_LAUNCH_CHECK();
  pou_warp_bwd_finalize_kernel<<<static_cast<unsigned>(cdiv64(N * B * 3, 256)), 256, 0, s>>>(part, (int)N, (int)B,
                                                                                             tiles, goffs);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_pou_pose_backward(const double* sl_part, int64_t tiles, const double* goffs, const double* ray_part,
                          int64_t rtiles, const double* geo, const float* centers, int64_t B, int64_t N,
                          const double* base12, double vscale, float* gmats, float* gvec, void* stream) {
  if (!sl_part || !geo || !centers || (!gmats && !gvec) || (gmats && !base12) || B < 1 || N < 1 || tiles < 1)
    return FVR_ERR_ARG;
  const double zero12[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (N > 2147483647) return FVR_ERR_ARG;
  pou_pose_bwd_kernel<<<static_cast<unsigned>(N), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      sl_part, (int)tiles, goffs, ray_part, (int)rtiles, geo, centers, (int)B, (int)N,
      make_base(base12 ? base12 : zero12), vscale, gmats, gvec);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_pou_rays_prep(const float* trg, const double* geo, int64_t N, int64_t K, float* rx, float* ry, float* ic,
                      void* stream) {
  if (!trg || !geo || !rx || !ry || !ic || N < 1 || K < 1 || N > 65535) return FVR_ERR_ARG;
  pou_rays_prep_kernel<<<dim3((unsigned)cdiv64(K, 256), (unsigned)N), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      trg, geo, (int)N, (int)K, rx, ry, ic);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int64_t fvr_pou_rays_bwd_workspace(int64_t N, int64_t K) { return N * cdiv64(K, 256) * 12 * (int64_t)sizeof(double); }

int fvr_pou_rays_bwd(const float* trg, const double* geo, int64_t N, int64_t K, const float* gray, float* gtrg,
                     void* workspace, int64_t ws_bytes, void* stream) {
  if (!trg || !geo || !gray || !gtrg || !workspace || N < 1 || K < 1 || N > 65535) return FVR_ERR_ARG;
  if (ws_bytes < fvr_pou_rays_bwd_workspace(N, K)) return FVR_ERR_WORKSPACE;
  pou_rays_bwd_kernel<<<dim3((unsigned)cdiv64(K, 256), (unsigned)N), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      trg, geo, (int)N, (int)K, gray, gtrg, static_cast<double*>(workspace));
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

}  // extern "C"

FVR_CHECK_ACCESSOR(check_word_pou)
