// Batched mixed-radix FFTs in shared memory (Stockham autosort), sm_100a.
//
// One CTA transforms `L` lines of length n entirely in shared memory
// (ping-pong buffers, radix 4/2/3/5 butterflies plus direct-DFT passes for
// the other prime factors up to 127).  Multi-dimensional transforms are sequences of line passes; the
// fftshift / ifftshift permutations, zero-padding of real volumes, sinc^2
// pre-compensation, 1/n scaling and real-part / ReLU extraction are folded
// into the first pass's loads and the last pass's stores, so every pass moves
// each element through HBM exactly once.
//
// Replaces the reference's library calls torch.fft.fftn / ifft2 / fft2
// (src/fvr/torch_engine.py:80-81, 239, 263, 322-323;
//  src/fvr/cone_beam_fvr.py:291-294, 502-505) and scipy.fft in
// src/fvr/diff_fvr.py:54, 168.
#include "fvr_dft.cuh"

namespace fvr {

constexpr int kMaxPass = 24;
// Largest prime factor of a transform length (direct DFT pass, O(n * p) work).
constexpr int kMaxPrime = 127;

struct FftPlan {
  int n;
  int npass;
  int radix[kMaxPass];
};

static bool make_plan(int64_t n, FftPlan* plan) {
  if (n < 1 || n > 16384) return false;
  plan->n = static_cast<int>(n);
  plan->npass = 0;
  int64_t m = n;
  const int order[] = {4, 2, 3, 5, 7, 11, 13};
  for (int r : order) {
    while (m % r == 0) {
      if (plan->npass >= kMaxPass) return false;
      plan->radix[plan->npass++] = r;
      m /= r;
    }
  }
  // remaining odd prime factors up to kMaxPrime run as direct DFT passes
  for (int r = 17; r <= kMaxPrime && m > 1; r += 2) {
    while (m % r == 0) {
      if (plan->npass >= kMaxPass) return false;
      plan->radix[plan->npass++] = r;
      m /= r;
    }
  }
  return m == 1;
}

template <typename T, int R>
__device__ __forceinline__ void bfly(const Cx<T>* __restrict__ src, Cx<T>* __restrict__ dst, int j, int Ns, int n,
                                     const Cx<T>* __restrict__ tw, bool inv) {
  const int nb = n / R;
  const int k = j % Ns;
  Cx<T> v[R];
#pragma unroll
  for (int t = 0; t < R; ++t) v[t] = src[j + t * nb];
  if (Ns > 1) {
    const int step = n / (Ns * R);
#pragma unroll
    for (int t = 1; t < R; ++t) {
      Cx<T> w = tw[k * t * step];
      if (inv) w.y = -w.y;
      v[t] = cmul(v[t], w);
    }
  }
  Dft<T, R>::run(v, inv);
  const int idx = (j / Ns) * Ns * R + k;
#pragma unroll
  for (int t = 0; t < R; ++t) dst[idx + t * Ns] = v[t];
}

// Generic prime radix (7, 11, 13): direct DFT with table twiddles.
template <typename T>
__device__ __forceinline__ void bfly_generic(const Cx<T>* __restrict__ src, Cx<T>* __restrict__ dst, int j, int Ns,
                                             int n, int R, const Cx<T>* __restrict__ tw, bool inv) {
  const int nb = n / R;
  const int k = j % Ns;
  Cx<T> v[13];
  for (int t = 0; t < R; ++t) {
    Cx<T> x = src[j + t * nb];
    if (Ns > 1 && t > 0) {
      Cx<T> w = tw[k * t * (n / (Ns * R))];
      if (inv) w.y = -w.y;
      x = cmul(x, w);
    }
    v[t] = x;
  }
  const int idx = (j / Ns) * Ns * R + k;
  for (int m = 0; m < R; ++m) {
    Cx<T> acc = v[0];
    for (int t = 1; t < R; ++t) {
      Cx<T> w = tw[((t * m) % R) * nb];
      if (inv) w.y = -w.y;
      Cx<T> p = cmul(v[t], w);
      acc.x += p.x;
      acc.y += p.y;
    }
    dst[idx + m * Ns] = acc;
  }
}

// Prime radix 17..kMaxPrime: direct DFT, inputs re-read from shared memory
// for every output (no per-thread array of R values).
template <typename T>
__device__ __noinline__ void bfly_generic_wide(const Cx<T>* __restrict__ src, Cx<T>* __restrict__ dst, int j, int Ns,
                                               int n, int R, const Cx<T>* __restrict__ tw, bool inv) {
  const int nb = n / R;
  const int k = j % Ns;
  const int ts = n / (Ns * R);
  const int idx = (j / Ns) * Ns * R + k;
  for (int m = 0; m < R; ++m) {
    Cx<T> acc = src[j];
    for (int t = 1; t < R; ++t) {
      Cx<T> x = src[j + t * nb];
      if (Ns > 1) {
        Cx<T> w = tw[k * t * ts];
        if (inv) w.y = -w.y;
        x = cmul(x, w);
      }
      Cx<T> w = tw[((t * m) % R) * nb];
      if (inv) w.y = -w.y;
      const Cx<T> p = cmul(x, w);
      acc.x += p.x;
      acc.y += p.y;
    }
    dst[idx + m * Ns] = acc;
  }
}

// ----------------------------------------------------------------------------
// loaders / storers.  A line l of a pass is (o, i) = (l / inner, l % inner);
// element k of the line sits at o*so + i*si + k*sk.  `kc` selects the element
// order used for global accesses (contiguous along k, or across lines).
// ----------------------------------------------------------------------------

__device__ __forceinline__ void map_elem(bool kc, int e, int Lc, int n, int& l, int& k) {
  if (kc) {
    l = e / n;
    k = e - l * n;
  } else {
    k = e / Lc;
    l = e - k * Lc;
  }
}

__device__ __forceinline__ int rot(int k, int s, int n) {
  int r = k + s;
  return r >= n ? r - n : r;
}

template <typename T, typename IT>
struct LdStrided {  // complex (IT = Cx<T>) or real (IT = float/double) strided input
  const IT* p;
  int64_t inner, so, si, sk;
  int shift, n;
  bool kc;
  __device__ __forceinline__ Cx<T> load(int64_t line, int k) const {
    const int64_t o = line / inner, i = line - o * inner;
    const IT* q = p + o * so + i * si + static_cast<int64_t>(rot(k, shift, n)) * sk;
    return conv(*q);
  }
  __device__ __forceinline__ static Cx<T> conv(const Cx<T>& v) { return v; }
  __device__ __forceinline__ static Cx<T> conv(const float& v) { return Cx<T>{static_cast<T>(v), T(0)}; }
  __device__ __forceinline__ static Cx<T> conv(const double& v) { return Cx<T>{static_cast<T>(v), T(0)}; }
};

// First (x-axis) pass of a 3D transform of a zero-padded real volume batch:
// padded[b][z][y][x] = vol[b][z-oz][y-oy][x-ox] * wz[.]*wy[.]*wx[.] (0 outside),
// read through per-axis index rotations (the ifftshift of the padded array).
template <typename T, typename VT>
struct LdRealPad3 {
  const VT* vol;
  int d, h, w, Dp, Hp, Wp, oz, oy, ox, sz, sy, sx;
  const double *wz, *wy, *wx;
  __device__ __forceinline__ Cx<T> load(int64_t line, int k) const {
    const int64_t b = line / (static_cast<int64_t>(Dp) * Hp);
    const int64_t zy = line - b * Dp * Hp;
    const int z = static_cast<int>(zy / Hp), y = static_cast<int>(zy - static_cast<int64_t>(z) * Hp);
    const int iz = rot(z, sz, Dp) - oz, iy = rot(y, sy, Hp) - oy, ix = rot(k, sx, Wp) - ox;
    if (iz < 0 || iz >= d || iy < 0 || iy >= h || ix < 0 || ix >= w) return Cx<T>{T(0), T(0)};
    T v = static_cast<T>(vol[((b * d + iz) * h + iy) * static_cast<int64_t>(w) + ix]);
    if (wz) v = static_cast<T>(static_cast<double>(v) * (wz[iz] * wy[iy] * wx[ix]));
    return Cx<T>{v, T(0)};
  }
};

template <typename T>
struct StCx {
  Cx<T>* p;
  int64_t inner, so, si, sk;
  int shift, n;
  T scale;
  __device__ __forceinline__ void store(int64_t line, int k, Cx<T> v) const {
    const int64_t o = line / inner, i = line - o * inner;
    p[o * so + i * si + static_cast<int64_t>(rot(k, shift, n)) * sk] = Cx<T>{v.x * scale, v.y * scale};
  }
};

// scale * Re(v), optional ReLU, optional crop window (k in [k0, k0+kn), line
// index i in [i0, i0+in_)) written to out[o*so + (i-i0)*si + (k-k0)*sk].
template <typename T, typename OT>
struct StReal {
  OT* p;
  int64_t inner, so, si, sk;
  int shift, n;
  T scale;
  int relu;
  int k0, kn;
  int64_t i0, in_;
  __device__ __forceinline__ void store(int64_t line, int k, Cx<T> v) const {
    const int64_t o = line / inner, i = line - o * inner;
    const int kk = rot(k, shift, n) - k0;
    const int64_t ii = i - i0;
    if (kk < 0 || kk >= kn || ii < 0 || ii >= in_) return;
    T r = v.x * scale;
    if (relu && !(r > T(0))) r = T(0);
    p[o * so + ii * si + static_cast<int64_t>(kk) * sk] = static_cast<OT>(r);
  }
};

template <typename T, class LD, class ST>
__global__ void __launch_bounds__(256) fft_lines_kernel(LD ld, bool ld_kc, ST st, bool st_kc, FftPlan plan,
                                                        const Cx<T>* __restrict__ tw, int64_t n_lines, int L,
                                                        int inv) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<T>* b0 = reinterpret_cast<Cx<T>*>(smem_raw);
  const int n = plan.n;
  const int pitch = n + 1;
  Cx<T>* b1 = b0 + static_cast<int64_t>(L) * pitch;
  const int64_t l0 = static_cast<int64_t>(blockIdx.x) * L;
  const int Lc = static_cast<int>(min(static_cast<int64_t>(L), n_lines - l0));
  const int tot = Lc * n;
  for (int e = threadIdx.x; e < tot; e += blockDim.x) {
    int l, k;
    map_elem(ld_kc, e, Lc, n, l, k);
    b0[l * pitch + k] = ld.load(l0 + l, k);
  }
  __syncthreads();
  Cx<T>* src = b0;
  Cx<T>* dst = b1;
  int Ns = 1;
  const bool binv = inv != 0;
  for (int p = 0; p < plan.npass; ++p) {
    const int r = plan.radix[p];
    const int nb = n / r;
    const int totb = Lc * nb;
    for (int b = threadIdx.x; b < totb; b += blockDim.x) {
      const int l = b / nb;
      const int j = b - l * nb;
      const Cx<T>* s = src + l * pitch;
      Cx<T>* d = dst + l * pitch;
      switch (r) {
        case 4: bfly<T, 4>(s, d, j, Ns, n, tw, binv); break;
        case 2: bfly<T, 2>(s, d, j, Ns, n, tw, binv); break;
        case 3: bfly<T, 3>(s, d, j, Ns, n, tw, binv); break;
        case 5: bfly<T, 5>(s, d, j, Ns, n, tw, binv); break;
        default:
          if (r <= 13)
            bfly_generic<T>(s, d, j, Ns, n, r, tw, binv);
          else
            bfly_generic_wide<T>(s, d, j, Ns, n, r, tw, binv);
          break;
      }
    }
    __syncthreads();
    Cx<T>* t = src;
    src = dst;
    dst = t;
    Ns *= r;
  }
  for (int e = threadIdx.x; e < tot; e += blockDim.x) {
    int l, k;
    map_elem(st_kc, e, Lc, n, l, k);
    st.store(l0 + l, k, src[l * pitch + k]);
  }
}

template <typename T>
__global__ void twiddle_kernel(Cx<T>* tw, int n) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  double s, c;
  sincospi(2.0 * static_cast<double>(m) / static_cast<double>(n), &s, &c);
  tw[m] = Cx<T>{static_cast<T>(c), static_cast<T>(-s)};
}

// Lines per CTA: about 4096 complex elements per CTA (two ping-pong buffers).
template <typename T>
static int lines_per_cta(int n, int64_t n_lines) {
  int L = 4096 / n;
  if (L < 1) L = 1;
  if (L > 64) L = 64;
  if (L > n_lines) L = static_cast<int>(n_lines);
  return L;
}

template <typename T>
static size_t smem_bytes(int n, int L) {
  return 2 * static_cast<size_t>(L) * (n + 1) * sizeof(Cx<T>);
}

template <typename T, class LD, class ST>
static int launch_pass(const LD& ld, bool ld_kc, const ST& st, bool st_kc, const FftPlan& plan, const void* tw,
                       int64_t n_lines, int inv, cudaStream_t stream) {
  if (n_lines <= 0) return FVR_OK;
  const int L = lines_per_cta<T>(plan.n, n_lines);
  const size_t sm = smem_bytes<T>(plan.n, L);
  if (sm > 227 * 1024) return FVR_ERR_UNSUPPORTED;
  auto kern = fft_lines_kernel<T, LD, ST>;
  if (sm > 48 * 1024) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm)) != cudaSuccess)
      return FVR_ERR_CUDA;
  }
  const int64_t grid = cdiv64(n_lines, L);
  if (grid > 0x7fffffff) return FVR_ERR_ARG;
  kern<<<static_cast<unsigned>(grid), 256, sm, stream>>>(ld, ld_kc, st, st_kc, plan,
                                                           static_cast<const Cx<T>*>(tw), n_lines, L, inv);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

static int shift_amount(int mode, int n) {
  // mode 0: none; 1: ifftshift (y[k] = x[k + n/2]); 2: fftshift (y[k] = x[k - n/2])
  if (mode == 1) return n / 2;
  if (mode == 2) return n - n / 2;
  return 0;
}
static int store_shift(int mode, int n) {
  // storing y[k] at position k + s realises out = shift(y)
  if (mode == 2) return n / 2;      // fftshift
  if (mode == 1) return n - n / 2;  // ifftshift
  return 0;
}

// 3D transform of a batch of zero-padded real volumes -> complex spectrum.
template <typename T, typename VT>
static int spectrum3d_impl(const VT* vol, int64_t nb, int d, int h, int w, int Dp, int Hp, int Wp, int conv,
                           const double* wz, const double* wy, const double* wx, Cx<T>* out, const void* twx,
                           const void* twy, const void* twz, cudaStream_t stream) {
  FftPlan px, py, pz;
  if (!make_plan(Wp, &px) || !make_plan(Hp, &py) || !make_plan(Dp, &pz)) return FVR_ERR_UNSUPPORTED;
  // conv 0 (torch_engine.py:61-81): pad low side (P-n)//2, fftn, fftshift.
  // conv 1 (diff_fvr.py:47-54): pad low side (P-n)//2, ifftshift, fftn, fftshift.
  // conv 2 (cone_beam_fvr.py:291-294): input already padded; ifftshift, fftn, fftshift.
  const int oz = (Dp - d) / 2, oy = (Hp - h) / 2, ox = (Wp - w) / 2;
  const bool pre = conv != 0;
  LdRealPad3<T, VT> ld{vol, d, h, w, Dp, Hp, Wp, oz, oy, ox,
                       pre ? shift_amount(1, Dp) : 0, pre ? shift_amount(1, Hp) : 0, pre ? shift_amount(1, Wp) : 0,
                       wz, wy, wx};
  const int64_t plane = static_cast<int64_t>(Hp) * Wp;
  const int64_t vol3 = static_cast<int64_t>(Dp) * plane;
  // x pass: lines (b, z, y), contiguous along x
  StCx<T> sx{out, 1, Wp, 0, 1, store_shift(2, Wp), Wp, T(1)};
  int st = launch_pass<T>(ld, true, sx, true, px, twx, nb * Dp * Hp, 0, stream);
  if (st) return st;
  // y pass: lines (b*z, x); elements strided by Wp
  LdStrided<T, Cx<T>> ly{out, Wp, plane, 1, Wp, 0, Hp, false};
  StCx<T> sy{out, Wp, plane, 1, Wp, store_shift(2, Hp), Hp, T(1)};
  st = launch_pass<T>(ly, false, sy, false, py, twy, nb * Dp * Wp, 0, stream);
  if (st) return st;
  // z pass: lines (b, y*x); elements strided by the plane
  LdStrided<T, Cx<T>> lz{out, plane, vol3, 1, plane, 0, Dp, false};
  StCx<T> sz{out, plane, vol3, 1, plane, store_shift(2, Dp), Dp, T(1)};
  return launch_pass<T>(lz, false, sz, false, pz, twz, nb * plane, 0, stream);
}

// Batched 2D transform [batch][n0][n1]: pass along n1, then along n0.
template <typename T, typename IT>
static int fft2d_impl(const IT* in, int64_t batch, int n0, int n1, int inverse, int in_shift, int out_shift,
                      double scale, int out_mode, void* out, int out_f64, int crop_r0, int crop_nr, int crop_c0,
                      int crop_nc, const void* tw0, const void* tw1, Cx<T>* work, cudaStream_t stream) {
  FftPlan p0, p1;
  if (!make_plan(n0, &p0) || !make_plan(n1, &p1)) return FVR_ERR_UNSUPPORTED;
  const int64_t img = static_cast<int64_t>(n0) * n1;
  // pass 1: rows (lines (b, r), contiguous along columns)
  LdStrided<T, IT> l1{in, 1, n1, 0, 1, shift_amount(in_shift, n1), n1, true};
  StCx<T> s1{work, 1, n1, 0, 1, store_shift(out_shift, n1), n1, T(1)};
  int st = launch_pass<T>(l1, true, s1, true, p1, tw1, batch * n0, inverse, stream);
  if (st) return st;
  // pass 2: columns (lines (b, c), strided by n1)
  LdStrided<T, Cx<T>> l2{work, n1, img, 1, n1, shift_amount(in_shift, n0), n0, false};
  if (out_mode == 0) {
    StCx<T> s2{static_cast<Cx<T>*>(out), n1, img, 1, n1, store_shift(out_shift, n0), n0, static_cast<T>(scale)};
    return launch_pass<T>(l2, false, s2, false, p0, tw0, batch * n1, inverse, stream);
  }
  const int relu = out_mode == 2;
  const int64_t oimg = static_cast<int64_t>(crop_nr) * crop_nc;
  if (out_f64) {
    StReal<T, double> s2{static_cast<double*>(out), n1, oimg, 1, crop_nc, store_shift(out_shift, n0), n0,
                         static_cast<T>(scale), relu, crop_r0, crop_nr, crop_c0, crop_nc};
    return launch_pass<T>(l2, false, s2, false, p0, tw0, batch * n1, inverse, stream);
  }
  StReal<T, float> s2{static_cast<float*>(out), n1, oimg, 1, crop_nc, store_shift(out_shift, n0), n0,
                      static_cast<T>(scale), relu, crop_r0, crop_nr, crop_c0, crop_nc};
  return launch_pass<T>(l2, false, s2, false, p0, tw0, batch * n1, inverse, stream);
}

}  // namespace fvr

using namespace fvr;

extern "C" {

int fvr_fft_supported(int64_t n) {
  FftPlan p;
  return make_plan(n, &p) ? 1 : 0;
}

int fvr_fft_twiddles(int64_t n, int prec, void* tw_out, void* stream) {
  FftPlan p;
  if (!make_plan(n, &p)) return FVR_ERR_UNSUPPORTED;
  if (!tw_out) return FVR_ERR_ARG;
  const unsigned grid = static_cast<unsigned>(cdiv64(n, 256));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (prec == FVR_F64)
    twiddle_kernel<double><<<grid, 256, 0, s>>>(static_cast<Cx<double>*>(tw_out), static_cast<int>(n));
  else if (prec == FVR_F32)
    twiddle_kernel<float><<<grid, 256, 0, s>>>(static_cast<Cx<float>*>(tw_out), static_cast<int>(n));
  else
    return FVR_ERR_DTYPE;
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_spectrum3d(const void* vol, int vol_dtype, int64_t batch, int64_t d, int64_t h, int64_t w, int64_t Dp,
                   int64_t Hp, int64_t Wp, int convention, const double* wz, const double* wy, const double* wx,
                   int prec, void* out, const void* tw_x, const void* tw_y, const void* tw_z, void* stream) {
  if (!vol || !out || !tw_x || !tw_y || !tw_z) return FVR_ERR_ARG;
  if (batch < 1 || d < 1 || h < 1 || w < 1 || Dp < d || Hp < h || Wp < w) return FVR_ERR_ARG;
  if (Dp > 16384 || Hp > 16384 || Wp > 16384) return FVR_ERR_UNSUPPORTED;
  if (convention < 0 || convention > 2) return FVR_ERR_ARG;
  if ((wz != nullptr) != (wy != nullptr) || (wy != nullptr) != (wx != nullptr)) return FVR_ERR_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int D = (int)Dp, H = (int)Hp, W = (int)Wp;
  if (prec == FVR_F32) {
    if (vol_dtype != FVR_F32) return FVR_ERR_DTYPE;
    return spectrum3d_impl<float, float>(static_cast<const float*>(vol), batch, (int)d, (int)h, (int)w, D, H, W,
                                         convention, wz, wy, wx, static_cast<Cx<float>*>(out), tw_x, tw_y, tw_z, s);
  }
  if (prec == FVR_F64) {
    if (vol_dtype == FVR_F64)
      return spectrum3d_impl<double, double>(static_cast<const double*>(vol), batch, (int)d, (int)h, (int)w, D, H,
                                             W, convention, wz, wy, wx, static_cast<Cx<double>*>(out), tw_x, tw_y,
                                             tw_z, s);
    if (vol_dtype == FVR_F32)
      return spectrum3d_impl<double, float>(static_cast<const float*>(vol), batch, (int)d, (int)h, (int)w, D, H, W,
                                            convention, wz, wy, wx, static_cast<Cx<double>*>(out), tw_x, tw_y, tw_z,
                                            s);
    return FVR_ERR_DTYPE;
  }
  return FVR_ERR_DTYPE;
}

int fvr_fft2d(const void* in, int in_real, int64_t batch, int64_t n0, int64_t n1, int prec, int inverse,
              int in_shift, int out_shift, double scale, int out_mode, void* out, int64_t crop_r0, int64_t crop_nr,
              int64_t crop_c0, int64_t crop_nc, const void* tw0, const void* tw1, void* work, void* stream) {
  if (!in || !out || !tw0 || !tw1 || !work) return FVR_ERR_ARG;
  if (batch < 1 || n0 < 1 || n1 < 1 || n0 > 16384 || n1 > 16384) return FVR_ERR_ARG;
  if (in_shift < 0 || in_shift > 2 || out_shift < 0 || out_shift > 2 || out_mode < 0 || out_mode > 2)
    return FVR_ERR_ARG;
  if (out_mode == 0) {
    crop_r0 = 0;
    crop_nr = n0;
    crop_c0 = 0;
    crop_nc = n1;
  }
  if (crop_r0 < 0 || crop_c0 < 0 || crop_nr < 1 || crop_nc < 1 || crop_r0 + crop_nr > n0 || crop_c0 + crop_nc > n1)
    return FVR_ERR_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (prec == FVR_F32) {
    Cx<float>* wk = static_cast<Cx<float>*>(work);
    if (in_real)
      return fft2d_impl<float, float>(static_cast<const float*>(in), batch, (int)n0, (int)n1, inverse, in_shift,
                                      out_shift, scale, out_mode, out, 0, (int)crop_r0, (int)crop_nr, (int)crop_c0,
                                      (int)crop_nc, tw0, tw1, wk, s);
    return fft2d_impl<float, Cx<float>>(static_cast<const Cx<float>*>(in), batch, (int)n0, (int)n1, inverse,
                                        in_shift, out_shift, scale, out_mode, out, 0, (int)crop_r0, (int)crop_nr,
                                        (int)crop_c0, (int)crop_nc, tw0, tw1, wk, s);
  }
  if (prec == FVR_F64) {
    Cx<double>* wk = static_cast<Cx<double>*>(work);
    if (in_real)
      return fft2d_impl<double, double>(static_cast<const double*>(in), batch, (int)n0, (int)n1, inverse, in_shift,
                                        out_shift, scale, out_mode, out, 1, (int)crop_r0, (int)crop_nr, (int)crop_c0,
                                        (int)crop_nc, tw0, tw1, wk, s);
    return fft2d_impl<double, Cx<double>>(static_cast<const Cx<double>*>(in), batch, (int)n0, (int)n1, inverse,
                                          in_shift, out_shift, scale, out_mode, out, 1, (int)crop_r0, (int)crop_nr,
                                          (int)crop_c0, (int)crop_nc, tw0, tw1, wk, s);
  }
  return FVR_ERR_DTYPE;
}

}  // extern "C"
