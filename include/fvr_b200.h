/*
 * fvr_b200.h -- C ABI of the B200 (sm_100a) Diff-FVR hot-path library
 * (libfvr_b200.so).
 *
 * Conventions shared by every entry point:
 *   - All array arguments are DEVICE pointers owned by the caller; the library
 *     never allocates per call.  Temporary space comes from a caller-provided
 *     `workspace` whose minimum size is returned by the matching
 *     fvr_*_workspace() query.
 *   - `stream` is a cudaStream_t passed as void*; work is stream-ordered and
 *     no call synchronises the device.
 *   - Every entry point returns an fvr_status; nothing throws across the ABI.
 *   - Complex arrays are interleaved (re, im) pairs.
 *   - Sizes are int64_t element counts.
 *
 * The comment above each function names the reference interface it replaces
 * (paths inside the pareelamre/diff-fvr project).
 */
#ifndef FVR_B200_H
#define FVR_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  FVR_OK = 0,
  FVR_ERR_ARG = 1,         /* null pointer, bad size, stride or alignment   */
  FVR_ERR_DTYPE = 2,       /* unsupported storage dtype for this entry      */
  FVR_ERR_UNSUPPORTED = 3, /* e.g. FFT length with a prime factor above 127 */
  FVR_ERR_WORKSPACE = 4,   /* caller workspace smaller than the query says  */
  FVR_ERR_CUDA = 5         /* launch or driver error (cudaGetLastError)     */
} fvr_status;

/* FVR_BF16_PAIR / FVR_F16_PAIR / FVR_F32_PAIR name the x-pair spectrum
 * storage (below), accepted by the spectral-NCC moments entry points only. */
typedef enum {
  FVR_F32 = 0,
  FVR_BF16 = 1,
  FVR_F16 = 2,
  FVR_F64 = 3,
  FVR_BF16_PAIR = 4,
  FVR_F16_PAIR = 5,
  FVR_F32_PAIR = 6
} fvr_dtype;

const char* fvr_status_string(int status);
int fvr_version(void);
/* Check words of the bounds-checked debug build (libfvr_b200_check.so, built
 * with -DFVR_CHECK; no reference counterpart): out[0..4) receive one word per
 * kernel family (parallel-beam, PoU, planar drop-in gather, NumPy
 * convention), 0 when every checked access stayed in bounds, else the first
 * out-of-bounds access (site code << 40 | low 40 bits of its index), which
 * the kernel skipped; clear != 0 resets them.  n >= 4.  The normal build
 * returns FVR_ERR_UNSUPPORTED. */
int fvr_check_words(unsigned long long* out, int n, int clear);
/* 1 if the device (ordinal) is sm_100 (B200 family), 0 otherwise. */
int fvr_device_supported(int device);

/* ---------------------------------------------------------------- FFT ---- */
/* Replaces torch.fft.fftn/ifft2/fft2 + fftshift/ifftshift at
 * src/fvr/torch_engine.py:80-81, 238-239, 263, 322-323,
 * src/fvr/cone_beam_fvr.py:291-294, 502-505 and scipy.fft at
 * src/fvr/diff_fvr.py:54, 168.  Lengths <= 16384 whose prime factors are all <= 127. */
int fvr_fft_supported(int64_t n);
/* tw_out: n complex (prec FVR_F32: float2, FVR_F64: double2) = exp(-2 pi i m/n) */
int fvr_fft_twiddles(int64_t n, int prec, void* tw_out, void* stream);
/* Batch of zero-padded real volumes [batch][d][h][w] -> centred spectra
 * [batch][Dp][Hp][Wp] complex.  convention 0: torch engine (pad, fftn,
 * fftshift; torch_engine.py:56-86); 1: NumPy renderer (optional sinc^2
 * premultiplication tables wz/wy/wx, pad, ifftshift, fftn, fftshift;
 * diff_fvr.py:34-54); 2: PoU blocks (already padded; ifftshift, fftn,
 * fftshift; cone_beam_fvr.py:291-294). */
int fvr_spectrum3d(const void* vol, int vol_dtype, int64_t batch, int64_t d, int64_t h, int64_t w, int64_t Dp,
                   int64_t Hp, int64_t Wp, int convention, const double* wz, const double* wy, const double* wx,
                   int prec, void* out, const void* tw_x, const void* tw_y, const void* tw_z, void* stream);
/* Batched 2D FFT of [batch][n0][n1] (complex, or real if in_real).
 * in_shift / out_shift: 0 none, 1 ifftshift, 2 fftshift (applied before /
 * after the transform).  out_mode 0: complex (scaled); 1: real part; 2: real
 * part + ReLU, written into the crop window [r0, r0+nr) x [c0, c0+nc).
 * `work` holds batch*n0*n1 complex and may alias `in` for complex input. */
int fvr_fft2d(const void* in, int in_real, int64_t batch, int64_t n0, int64_t n1, int prec, int inverse,
              int in_shift, int out_shift, double scale, int out_mode, void* out, int64_t crop_r0, int64_t crop_nr,
              int64_t crop_c0, int64_t crop_nc, const void* tw0, const void* tw1, void* work, void* stream);

/* ------------------------------------------------- stencil spectrum ---- */
/* Stencil layout of a D x H x W centred complex spectrum: (D+1)(H+1)(W+1)
 * entries, each the 8 complex corners of one trilinear cell (corners outside
 * the volume are zero).  f32: 64 B per entry; bf16 / f16: 32 B per entry, f16
 * with a power-of-two scale per 16^3-entry brick.  Built from a "master"
 * spectrum in f32, bf16 or f16, planar [2][D][H][W] (master_planar = 1, the
 * reference's f_vol_5d[0]) or interleaved [D][H][W][2] (master_planar = 0).  Storage for the
 * spectrum buffer f_vol_5d of src/fvr/torch_engine.py:83-88 and its
 * to_precision cast (:90-95). */
int64_t fvr_stencil_bytes(int64_t D, int64_t H, int64_t W, int dtype);
int64_t fvr_stencil_scale_count(int64_t D, int64_t H, int64_t W);
/* `items` spectra back to back (master item stride 2*D*H*W; out item stride
 * fvr_stencil_bytes(); scales item stride fvr_stencil_scale_count()).
 * scratch_max: items * fvr_stencil_scale_count() uint32 (f16 only, else NULL). */
int fvr_stencil_build(const void* master, int master_dtype, int master_planar, int64_t items, int64_t D, int64_t H,
                      int64_t W, int out_dtype, void* out, float* scales, unsigned int* scratch_max, void* stream);
/* x-pair layout of the same spectrum (out_dtype FVR_BF16_PAIR, FVR_F16_PAIR
 * or FVR_F32_PAIR): (D+1)(H+1)(W+2) entries of 16 B (16-bit) or 32 B (f32);
 * entry (ez, ey, ex) holds the 4 complex values of voxel column x = ex-1 at
 * (y, z) = (ey-1+dy, ez-1+dz), ordered dz*2 + dy (zero outside the volume).
 * A trilinear sample in the stencil cell (ez, ey, ex) reads entries ex and
 * ex+1: 32 (64) contiguous bytes, half the storage of the stencil, so the
 * samples of many slices meet in fewer sectors.  f16: a power-of-two scale
 * per slab of 16 x 16 (z, y) entry rows over the whole x extent, so a
 * sample's two entries share it (fvr_stencil_pair_scale_count floats).
 * Same master formats and `items` batching as fvr_stencil_build (out item
 * stride fvr_stencil_pair_bytes(); scales item stride
 * fvr_stencil_pair_scale_count()); scratch_max as there (f16 only). */
int64_t fvr_stencil_pair_bytes(int64_t D, int64_t H, int64_t W, int dtype);
int64_t fvr_stencil_pair_scale_count(int64_t D, int64_t H, int64_t W);
int fvr_stencil_pair_build(const void* master, int master_dtype, int master_planar, int64_t items, int64_t D,
                           int64_t H, int64_t W, int out_dtype, void* out, float* scales, unsigned int* scratch_max,
                           void* stream);

/* --------------------------------------- drop-in trilinear slice gather -- */
/* fourier_slice_3d on the reference layout vol[B][2][D][H][W] (dtype f32 /
 * bf16 / f16), p = c + fx[q] u[n] + fy[q] v[n], zero-padding partial
 * interpolation; out[B][N][2][K] in the volume dtype.
 * Replaces _TritonFourierSlice3DFn.forward, src/fvr/triton_slice.py:274-303. */
int fvr_slice3d_fwd(const void* vol, int dtype, int64_t B, int64_t D, int64_t H, int64_t W, const float* u,
                    const float* v, int64_t N, const float* fx, const float* fy, int64_t K, float cx, float cy,
                    float cz, void* out, void* stream);
int64_t fvr_slice3d_bwd_workspace(int64_t N, int64_t K);
/* dL/du, dL/dv [N][3] (fp64 accumulation, deterministic).
 * Replaces _TritonFourierSlice3DFn.backward, src/fvr/triton_slice.py:305-339. */
int fvr_slice3d_bwd(const void* vol, int dtype, int64_t B, int64_t D, int64_t H, int64_t W, const void* grad_out,
                    const float* u, const float* v, int64_t N, const float* fx, const float* fy, int64_t K, float cx,
                    float cy, float cz, float* gu, float* gv, void* workspace, int64_t ws_bytes, void* stream);

/* -------------------------------------- parallel-beam (torch engine) ---- */
/* Slice axes for poses[C][6] (yaw, pitch, roll deg; tx, ty, tz): axes[C][8]
 * (fp64) = (u_xyz, v_xyz, tx, ty), u = R[0,:]*((W-1)/2,(H-1)/2,(D-1)/2),
 * v = R[1,:]*(..), R = Rz(yaw) Ry(pitch) Rx(roll) in fp64, lateral view
 * R . Rz(90 deg).  view 0 = 'ap', 1 = 'lateral'.  src/fvr/torch_engine.py:139-211. */
int fvr_tc_axes(const float* poses, int64_t C, int view, int64_t D, int64_t H, int64_t W, double* axes,
                void* stream);
int64_t fvr_tc_sncc_workspace(int64_t C, int64_t R, int64_t nviews);
/* Per-(view, candidate) record length of `mom` (17 moments + ncc). */
int64_t fvr_tc_sncc_mom_stride(void);
/* Fused zero-IFFT spectral NCC, pass 1: for every candidate and each of
 * nviews (<= 4) views (views[v] = 0 'ap' / 1 'lateral', ftargs[v] the
 * complex [R][R] target spectrum of that view, host arrays of device
 * pointers) one pass forms the slice axes from the pose in fp64, gathers the
 * slice at positions assembled from fp64 per-row and per-column parts
 * (within 2^-24 of a cell of the fp64 position), applies the phase ramp
 * kappa*(ku tx + kv ty) (per-row x per-column factors from fp64 sincospi) and
 * the high-pass table hp (NULL = none), and reduces the NCC moments; with
 * with_grad also the 14 pose-gradient moments.  Partial sums (one record per
 * CTA and (candidate, view) it covers) go to `workspace`.
 * lin = torch.linspace(-1, 1, R).  `variant` in [0, fvr_tc_sncc_variants())
 * selects the launch shape (rows in flight per thread, resident CTAs per SM);
 * results do not depend on it beyond float summation order.  dtype: the
 * stencil storage (FVR_F32 / FVR_BF16 / FVR_F16) or the x-pair storage
 * (FVR_*_PAIR; stencil = its data, scales = its slab scales), in this and
 * the two value-and-gradient entry points below.
 * Replaces TorchDiffFVREngine._spectral_ncc_core / forward_spectral_ncc,
 * src/fvr/torch_engine.py:269-307 (the gather of :176-234 included). */
int fvr_tc_sncc_variants(void);
int fvr_tc_sncc_moments(int dtype, const void* stencil, const float* scales, int64_t D, int64_t H, int64_t W,
                        const float* poses, int64_t C, int nviews, const int* views, const void* const* ftargs,
                        const float* hp, const float* lin, int64_t R, double kappa, int with_grad, int variant,
                        void* workspace, int64_t ws_bytes, void* stream);
/* Pass 2 (same variant): record sums in fp64 -> mom[nviews][C][stride] (kept
 * for the backward); loss[v] = 1 - mean_c ncc (f32), loss[nviews] = sum of the
 * view losses; ncc_out[nviews][C] optional. */
int fvr_tc_sncc_finalize(const void* workspace, int64_t C, int64_t R, int nviews, int with_grad, int variant,
                         double* mom, float* loss, float* ncc_out, void* stream);
/* dL/dposes[C][6] from the saved moments and the device scalars
 * g[v * g_stride] = dL/dloss_v (tz column is zero: the reference never reads
 * poses[:, 5]); accumulate != 0 adds into grad_poses.
 * Autograd backward of torch_engine.py:269-307. */
int fvr_tc_sncc_backward(const double* mom, int nviews, const int* views, const float* g, int64_t g_stride,
                         const float* poses, int64_t C, int64_t D, int64_t H, int64_t W, double kappa,
                         float* grad_poses, int accumulate, void* stream);
/* Loss + pose gradient in two stream-ordered launches (moments, finalize and
 * backward fused): the moments kernel, then one epilogue kernel launched as
 * its programmatic dependent, which forms the slice-axes Jacobians while the
 * moments run and then writes every candidate's fp64 moments, ncc_out[v][c]
 * (optional) and grad_poses[c][6] (g = dL/dloss_v at g[v * g_stride], NULL =
 * all ones; accumulate != 0 adds), and loss[nviews + 1] as
 * fvr_tc_sncc_finalize does.  `workspace` (>= fvr_tc_sncc_fused_workspace
 * bytes, 256-byte aligned) needs no initialisation.  Calls sharing one
 * workspace must be stream-ordered.  loss, ncc_out and grad_poses may be
 * device memory or page-locked host memory mapped into the device address
 * space (the epilogue kernel writes them directly).
 * Replaces the forward + autograd backward of TorchDiffFVREngine.
 * forward_spectral_ncc over several views, src/fvr/torch_engine.py:269-307. */
int64_t fvr_tc_sncc_fused_workspace(int64_t C, int64_t R, int64_t nviews);
int fvr_tc_sncc_value_and_grad(int dtype, const void* stencil, const float* scales, int64_t D, int64_t H, int64_t W,
                               const float* poses, int64_t C, int nviews, const int* views,
                               const void* const* ftargs, const float* hp, const float* lin, int64_t R,
                               double kappa, int variant, const float* g, int64_t g_stride, void* workspace,
                               int64_t ws_bytes, float* loss, float* ncc_out, float* grad_poses, int accumulate,
                               void* stream);
/* Allocation-free form of fvr_tc_sncc_value_and_grad (no counterpart in the
 * reference): same arguments and results, but the workspace is a fixed
 * per-device scratch array inside the library (about 352 KB), so the call
 * allocates nothing.  For callers that cannot allocate device memory where
 * they call (a host linking only this C ABI, with no device allocator; a
 * loop that must not enter an allocator between steps).
 * Limits: C * nviews <= 512 and at most 2048 partial records (partial
 * records = C * nviews * tiles, tiles chosen by the launch variant; on a
 * 148-SM B200 every variant stays within the limit when C * nviews <= 512);
 * larger calls return FVR_ERR_WORKSPACE without launching.
 * The first call on a device (that device current) resolves the scratch
 * address once; make it before any stream capture begins.  The cached address
 * is tied to that device's context: after cudaDeviceReset on a device, do not
 * call this entry point on it again in the same process.  Nothing has to be
 * zeroed by the caller: every call writes the scratch before reading it.
 * All callers in the process share one
 * scratch per device, so calls on one device must not overlap in time (use
 * one stream or synchronise between them). */
int fvr_tc_sncc_value_and_grad_static(int dtype, const void* stencil, const float* scales, int64_t D, int64_t H,
                                      int64_t W, const float* poses, int64_t C, int nviews, const int* views,
                                      const void* const* ftargs, const float* hp, const float* lin, int64_t R,
                                      double kappa, int variant, const float* g, int64_t g_stride, float* loss,
                                      float* ncc_out, float* grad_poses, int accumulate, void* stream);
/* Modulated slice S*exp(i phase) -> out[C][R][R] complex from fp64 axes;
 * shift != 0 writes it in ifftshift order (input of the image IFFT).
 * Replaces TorchDiffFVREngine._extract_slice_spectrum, torch_engine.py:176-234. */
int fvr_tc_slice(int dtype, const void* stencil, const float* scales, int64_t D, int64_t H, int64_t W,
                 const double* axes, int64_t C, const float* lin, int64_t R, double kappa, int shift, void* out,
                 void* stream);
int64_t fvr_tc_slice_adjoint_workspace(int64_t C, int64_t R);
/* Pose gradient for an upstream gradient G[C][R][R] (complex) with respect to
 * the modulated slice (same order as fvr_tc_slice with the same shift).
 * Autograd backward of torch_engine.py:176-241. */
int fvr_tc_slice_adjoint(int dtype, const void* stencil, const float* scales, int64_t D, int64_t H, int64_t W,
                         const double* axes, const float* poses, int64_t C, int view, const float* lin, int64_t R,
                         double kappa, int shift, const void* G, void* workspace, int64_t ws_bytes,
                         float* grad_poses, int accumulate, void* stream);
/* out = (img > 0) ? g : 0  (ReLU adjoint of torch_engine.py:240) */
int fvr_relu_mask(const float* img, const float* g, float* out, int64_t n, void* stream);
/* x[i] *= table[i % per] for complex x (high-pass of prepare_spectral_target,
 * torch_engine.py:264-266) */
int fvr_cmul_table(void* x, const float* table, int64_t per, int64_t n, void* stream);
/* 1 - exp(-r^2 / (2 sigma^2)), torch_engine.py:123-136 */
int fvr_hp_filter(float* out, int64_t H, int64_t W, double sigma, void* stream);
/* torch.linspace(start, end, n) in float32 */
int fvr_linspace(float* out, float start, float end, int64_t n, void* stream);

/* ------------------------------------------------ PoU-FVR cone beam ---- */
/* Per-candidate-block windowed mass sum(vol * w0 * w1 * w2) over the block's
 * support (fp64), k0*k1*k2 blocks in (i0, i1, i2) row-major order.  w_d are the
 * 1D partition-of-unity windows [k_d][n_d] (float32), sup_d [k_d][2] = (first
 * index, length) of each window's support.  The energy pruning input of
 * PerspectiveSlabFVR.__init__, src/fvr/cone_beam_fvr.py:231-245. */
int fvr_pou_block_sums(const float* vol, int64_t n0, int64_t n1, int64_t n2, const float* w0, const int* sup0,
                       int64_t k0, const float* w1, const int* sup1, int64_t k1, const float* w2, const int* sup2,
                       int64_t k2, double* sums, void* stream);
/* Padded real blocks out[B][P][P][P] for the active candidate indices
 * blocks[B]: windowed sub-volume centred in an M^3 cube, trilinear resize to
 * block_res^3 (align_corners=False) times ds_block, times the sinc^2 table
 * w3[block_res] per axis, zero pad to P^3.  cone_beam_fvr.py:241-283. */
int fvr_pou_build_blocks(const float* vol, int64_t n0, int64_t n1, int64_t n2, const float* w0, const int* sup0,
                         int64_t k0, const float* w1, const int* sup1, int64_t k1, const float* w2, const int* sup2,
                         int64_t k2, const int* blocks, int64_t B, const float* w3, int64_t M, int64_t block_res,
                         int64_t P, double ds_block, float* out, void* stream);
/* Per pose: geo[N][18] (fp64) = source, u, v, n (the lattice basis base12 =
 * src0, u0, v0, n0 moved by mats[N][4][4], or given directly as
 * vecs[N][12] = (s, u, v, n) when mats is NULL), slice axes flip(u)*vscale,
 * flip(v)*vscale; offs[B][N][3] (fp64) = (d_b, cu, cv) = (c_b - s).(n, u, v)
 * for the block centres [B][3].  cone_beam_fvr.py:485-488, 507-521, 676-682. */
/* Pinhole lattice of an H x W detector from k_inv[9] (row-major K^-1, host
 * memory) and the source-to-detector distance, all in FP64: per pixel the
 * detector point trg0[H][W][3] = d sdd / max(d_z, 1e-6) with
 * d = K^-1 (c + 1/2, r + 1/2, 1), the ray numbers rx, ry, ic [H][W]
 * (ic = 1 / max(r.n0, 0.1), rx = (r.u0) ic, ry = (r.v0) ic for the unit ray r
 * to the point), and basis[9] (device) = u0, v0, n0: unit vectors along the
 * first row and first column and the unit normal facing the lattice.
 * Replaces PerspectiveSlabFVR.make_pinhole_lattice with _make_ray_cache and
 * _extract_detector_basis, src/fvr/cone_beam_fvr.py:523-545, 575-596, 705-728. */
int fvr_pou_pinhole_lattice(const double* k_inv, double sdd_mm, int64_t H, int64_t W, float* trg0, float* rx,
                            float* ry, float* ic, double* basis, void* stream);
int64_t fvr_pou_geo_stride(void);
int fvr_pou_pose(const float* mats, const float* vecs, int64_t N, const double* base12, double vscale,
                 const float* centers, int64_t B, double* geo, double* offs, void* stream);
/* Explicit rays (cone_beam_fvr.py:451-457): per pose and pixel of
 * trg[N][K][3], rx = (r.u)/cos, ry = (r.v)/cos, ic = 1/cos, cos = max(r.n, 0.1). */
int fvr_pou_rays_prep(const float* trg, const double* geo, int64_t N, int64_t K, float* rx, float* ry, float* ic,
                      void* stream);
int64_t fvr_pou_rays_bwd_workspace(int64_t N, int64_t K);
/* Explicit-ray adjoint: gray[N][K][3] = dL/d(rx, ry, ic) -> gtrg[N][K][3] and
 * per-(pose, tile) partials of dL/d(src, u, v, n) in `workspace`. */
int fvr_pou_rays_bwd(const float* trg, const double* geo, int64_t N, int64_t K, const float* gray, float* gtrg,
                     void* workspace, int64_t ws_bytes, void* stream);
/* Block slices out[B][N][P][P] (complex, ifftshift order for the image IFFT)
 * from the stacked per-block stencil spectra (B items), at
 * p = P//2 + freqs[j] u_xyz + freqs[i] v_xyz.  cone_beam_fvr.py:480-501. */
int fvr_pou_slice(int dtype, const void* stencil, const float* scales, int64_t B, int64_t P, const double* geo,
                  int64_t N, const float* freqs, void* out, void* stream);
int64_t fvr_pou_slice_adjoint_workspace(int64_t B, int64_t P, int64_t N);
/* Slice adjoint for G[B][N][P][P] (complex, natural order): per-(pose, block,
 * tile) partials of dL/du_xyz, dL/dv_xyz in `workspace` (consumed by
 * fvr_pou_pose_backward). */
int fvr_pou_slice_adjoint(int dtype, const void* stencil, const float* scales, int64_t B, int64_t P,
                          const double* geo, int64_t N, const float* freqs, const void* G, void* workspace,
                          int64_t ws_bytes, void* stream);
/* Fused block images for P in {64, 96, 128, 160} (fvr_pou_image_supported):
 * one CTA per (pose, block) gathers the slice, runs the 2D inverse FFT in
 * shared memory and writes imgs[B][N][P][P] = Re fftshift(ifft2(ifftshift(S)))
 * (f32), i.e. fvr_pou_slice + fvr_fft2d without the complex intermediate.
 * Replaces PerspectiveSlabFVR._slice_and_ifft, src/fvr/cone_beam_fvr.py:480-505. */
int fvr_pou_image_supported(int64_t P);
int fvr_pou_slice_image(int dtype, const void* stencil, const float* scales, int64_t B, int64_t P, const double* geo,
                        int64_t N, const float* freqs, float* imgs, void* stream);
/* Its adjoint: from dL/dimgs [B][N][P][P] (f32), G = fftshift(fft2(ifftshift(
 * g))) / P^2 in shared memory and the slice adjoint in the same CTA;
 * workspace[N][B][6] fp64 (one tile per (pose, block)) feeds
 * fvr_pou_pose_backward with tiles = 1.  Autograd backward of
 * cone_beam_fvr.py:480-505. */
int64_t fvr_pou_slice_image_adjoint_workspace(int64_t B, int64_t N);
int fvr_pou_slice_image_adjoint(int dtype, const void* stencil, const float* scales, int64_t B, int64_t P,
                                const double* geo, int64_t N, const float* freqs, const float* grad_imgs,
                                void* workspace, int64_t ws_bytes, void* stream);
/* Fused warp + block-image adjoint for a separable pinhole lattice (every
 * detector column shares one ray coordinate rxc[c], every row one ryr[r]):
 * from the detector gradient gout[N][H][W] (times ic[H][W]) and the forward
 * block images imgs[B][N][P][P], one CTA per (pose, block) forms dL/dimgs in
 * shared memory by a gather along detector rows (no atomics, no image-gradient
 * buffer), writes goffs[3][B][N] = dL/d(d_b, cu, cv) (offs[B][N][3] fp64) and
 * the slice partials workspace[N][B][6] that fvr_pou_pose_backward takes with
 * tiles = 1, i.e. fvr_pou_warp_bwd + fvr_pou_slice_image_adjoint in one
 * launch.  Supported (fvr_pou_warp_image_adjoint_supported) for P in
 * {64, 96, 128}, W a multiple of 4 up to 256 and the shared memory that
 * takes; gout, ic and imgs start on 16-byte boundaries.  Autograd of
 * src/fvr/triton_slice.py:409-496 with cone_beam_fvr.py:480-505. */
int fvr_pou_warp_image_adjoint_supported(int64_t P, int64_t H, int64_t W);
int fvr_pou_warp_image_adjoint(int dtype, const void* stencil, const float* scales, int64_t B, int64_t P,
                               const double* geo, int64_t N, const float* freqs, const float* imgs,
                               const double* offs, const float* rxc, const float* ryr, const float* ic,
                               const float* gout, int64_t H, int64_t W, double inv_ds, double c_idx, double* goffs,
                               void* workspace, int64_t ws_bytes, void* stream);
/* out[N][K] = ic[q] * sum_b bilinear(imgs[b][n], (d_b rx - cu)/ds + c, (d_b ry - cv)/ds + c),
 * zero padding; offsets float (offs_f64 = 0) or double, element (b, n) at
 * index (b*N + n) * ostride; ray tables shared (ray_stride 0) or per pose
 * (ray_stride K).  Replaces pou_pinhole_warp_sum and
 * _PouPinholeWarpSumFn.forward, src/fvr/triton_slice.py:341-407, 498-545, 787-808. */
int fvr_pou_warp(const float* imgs, int64_t B, int64_t N, int64_t P, const void* db, const void* cu, const void* cv,
                 int offs_f64, int64_t ostride, const float* rx, const float* ry, const float* ic, int64_t K,
                 int64_t ray_stride, double inv_ds, double c_idx, float* out, void* stream);
int64_t fvr_pou_warp_bwd_workspace(int64_t B, int64_t N, int64_t K);
/* Adjoint: grad_imgs[B][N][P][P] += (scatter; NULL to skip; caller zeroes it),
 * goffs[3][B][N] (fp64) = dL/d(d_b, cu, cv), and with gray != NULL the
 * per-pixel dL/d(rx, ry, ic) [N][K][3] of the explicit-ray path.
 * _PouPinholeWarpSumFn.backward, src/fvr/triton_slice.py:409-496, 547-591. */
int fvr_pou_warp_bwd(const float* imgs, int64_t B, int64_t N, int64_t P, const void* db, const void* cu,
                     const void* cv, int offs_f64, int64_t ostride, const float* rx, const float* ry, const float* ic,
                     int64_t K, int64_t ray_stride, double inv_ds, double c_idx, const float* gout, float* grad_imgs,
                     double* goffs, float* gray, void* workspace, int64_t ws_bytes, void* stream);
/* d loss / d(src, u, v, n) gvec[N][12] and / or d loss / d mats[N][4][4]
 * from the slice-adjoint partials (tiles per (pose, block)), the offset
 * gradients goffs[3][B][N] and the explicit-ray partials (rtiles per pose);
 * goffs and ray_part may be NULL.  Autograd of cone_beam_fvr.py:423-521, 676-682. */
int fvr_pou_pose_backward(const double* sl_part, int64_t tiles, const double* goffs, const double* ray_part,
                          int64_t rtiles, const double* geo, const float* centers, int64_t B, int64_t N,
                          const double* base12, double vscale, float* gmats, float* gvec, void* stream);

/* ----------------------------------------------- NumPy-convention path -- */
/* Items are packed host-side as the struct
 *   { double yaw, pitch, roll, tx, ty; int view, sh, sw, pad; int64 off; }
 * (fvr_np_item_bytes() bytes; view 0 lateral, 1 ap, 2 axial; sh x sw slice
 * rows x columns; off = element offset of the item's slice / target).  The
 * spectrum f3d[D][H][W] is complex fp64 (fftshift(fftn(ifftshift(...)))). */
int64_t fvr_np_item_bytes(void);
/* Articulated multi-segment spectra: out[o] = sum over s < n_seg (in order) of
 * the phase-ramped slice of segment spectrum f3ds[s] (host array of device
 * pointers to complex128 [D][H][W] spectra of one common padded shape) at
 * item (o, s) of items[n_out][n_seg] (fvr_np_item_bytes each); output o is
 * written at the offset of item (o, 0); max_n = largest sh * sw; n_seg <= 16.
 * Replaces ArticulatedSpineModel.render_articulated_spectrum,
 * src/fvr/articulated_spine.py:39-71 (one launch for all segments). */
int fvr_np_segment_slices(const void* const* f3ds, int64_t n_seg, int64_t D, int64_t H, int64_t W, const void* items,
                          int64_t n_out, int64_t max_n, void* out, void* stream);
/* Phase-ramped frequency slices (complex fp64) with map_coordinates
 * (order 1, mode 'constant') sampling and the basis rz(yaw).ry(roll).rx(pitch)
 * on (Z, Y, X).  Replaces DifferentiableFourierVolumeRenderer._euler_to_basis /
 * extract_frequency_slice, src/fvr/diff_fvr.py:56-150; max_n >= sh*sw of every item. */
int fvr_np_slices(const void* f3d, int64_t D, int64_t H, int64_t W, const void* items, int64_t n_items,
                  int64_t max_n, void* out, void* stream);
int64_t fvr_np_ncc_workspace(int64_t n_items);
/* Per item, against targets (complex fp64, item's offset): mom[item][5] =
 * (Re sum S conj T, sum |S|^2, sum |T|^2, sum u Im(S conj T), sum v Im(S conj T))
 * in fp64 -> spectral NCC and its closed-form translation gradient
 * (diff_fvr.py:184-195, gradients.py:27-74). */
int fvr_np_ncc_moments(const void* f3d, int64_t D, int64_t H, int64_t W, const void* items, int64_t n_items,
                       const void* targets, void* workspace, int64_t ws_bytes, double* mom, void* stream);
int64_t fvr_np_pair_workspace(void);
/* mom[5] of two complex fp64 [sh][sw] arrays, with u = j - sw/2, v = i - sh/2:
 * (Re sum a conj b, sum |a|^2, sum |b|^2, sum u Im(a conj b), sum v Im(a conj b))
 * (compute_spectral_ncc, diff_fvr.py:184-195; closed-form translation
 * gradient, gradients.py:27-74). */
int fvr_np_pair_moments(const void* a, const void* b, int64_t sh, int64_t sw, void* workspace, int64_t ws_bytes,
                        double* mom, void* stream);

/* ------------------------------------------------------- volume ingest -- */
/* CT (HU, float32 [Z][Y][X], spacing sz, sy, sx mm) -> isotropic cube
 * out[target_res]^3 keeping the whole physical field of view centred:
 * voxel_mm = max(n_k * s_k) / target_res; input coordinate
 * c_k = (voxel_mm / s_k) * o_k + (n_k - 1) / 2 - (voxel_mm / s_k) (target_res - 1) / 2,
 * linear interpolation, -1000 HU unless 0 <= c_k <= n_k - 1 on every axis;
 * with to_mu the float32 attenuation max(0, (HU + 1000) / 1000) instead of HU.
 * *voxel_mm (optional, host) receives the cube's voxel size.  Replaces
 * resample_isotropic_cube + hu_to_attenuation, src/fvr/dicom_loader.py:11-30,
 * 179-188 (scipy affine_transform, order 1, mode 'constant', cval -1000). */
int fvr_ingest_resample(const float* hu, int64_t Z, int64_t Y, int64_t X, double sz, double sy, double sx,
                        int64_t target_res, int to_mu, float* out, double* voxel_mm, void* stream);
/* out[i] = max(0, (hu[i] + 1000) / 1000) in float32 (hu_to_attenuation,
 * src/fvr/dicom_loader.py:179-188). */
int fvr_hu_to_attenuation(const float* hu, int64_t n, float* out, void* stream);
/* Spine phantom out[n][n][n] (Z, Y, X) in HU: air, a soft-tissue torso and
 * five vertebrae (cortical and trabecular body, canal, spinous and transverse
 * processes), evaluated in float32 exactly as the NumPy construction of
 * create_spine_phantom, src/fvr/dicom_loader.py:114-176.  n <= 2048. */
int fvr_spine_phantom(int64_t n, float* out, void* stream);

/* ----------------------------------------------------------- timing ---- */
/* cudaEventRecordWithFlags(event, stream, external ? cudaEventRecordExternal
 * : 0): lets a caller time one kernel inside a captured CUDA graph (no
 * reference counterpart; measurement utility). */
int fvr_event_record(void* event, void* stream, int external);
/* dst[0..n) = src[0..n) by a kernel (no reference counterpart): both
 * pointers may be device memory or pinned host memory (unified addressing),
 * so a captured step can move its small inputs and outputs between host and
 * device in kernel nodes instead of copy-engine memcpy nodes. */
int fvr_copy_bytes(void* dst, const void* src, int64_t n, void* stream);

/* ------------------------------------------- image-domain spectral NCC -- */
/* Between centred spectra Fp[B][n] and Ft[Bt][n] (Bt = 1 or B, complex), both
 * multiplied by hp[n] (NULL = none): mom[B][3] = (cross, Ep, Et) in fp64,
 * loss = 1 - mean_b ncc_b.  Replaces TorchDiffFVREngine.spectral_ncc_loss,
 * src/fvr/torch_engine.py:309-337 (after the fft2 + fftshift of both images). */
int64_t fvr_cncc_workspace(int64_t B, int64_t n);
int fvr_cncc_forward(const void* Fp, const void* Ft, int64_t B, int64_t Bt, int64_t n, const float* hp,
                     void* workspace, int64_t ws_bytes, double* mom, float* loss, void* stream);
/* X[B][n] = dL/dFp (complex) for the device scalar g = dL/dloss. */
int fvr_cncc_backward(const void* Fp, const void* Ft, int64_t B, int64_t Bt, int64_t n, const float* hp,
                      const double* mom, const float* g, void* X, void* stream);

/* ------------------------------------------------------ SE(3) exp map -- */
/* theta[N][6] = (w_x, w_y, w_z, t_x, t_y, t_z) (rad, mm) -> mats[N][4][4]
 * = [[exp([w]x), t], [0, 1]] (Rodrigues, fp64 inside).  The map the
 * reference builds with torch.matrix_exp of the skew matrix:
 * experiments/exp30_gpu_multistart_registration.py:42-55,
 * tests/test_cone_beam_fvr.py:221-229. */
int fvr_se3_exp(const float* theta, int64_t N, float* mats, void* stream);
/* grad_theta[N][6] from grad_mats[N][4][4] (dR/dw in closed form). */
int fvr_se3_exp_backward(const float* theta, const float* grad_mats, int64_t N, float* grad_theta, void* stream);

/* ------------------------------------------ edge-dominant gradient NCC -- */
/* pred a[B][C][H][W], target b[Bt][C][H][W] (Bt = 1 broadcast, or B), f32.
 * Sobel-x / Sobel-y responses (zero padding) on the interior [crop, H-crop) x
 * [crop, W-crop), NCC per direction (denominator sqrt(max(Suu Svv, 1e-12))),
 * 0.5 (x + y) averaged over channels; when ms_weight > 0 and W >= 96 mixed
 * (1 - w) fine + w (same on 3x3 box-blurred images, zero padding, divisor 9).
 * out[0] = batch mean (reduction_mean) or out[B].  stats[B*C][20] (fp64
 * moments) is kept for the backward.
 * Replaces edge_dominant_ncc, src/fvr/cone_beam_fvr.py:71-112. */
int64_t fvr_edge_ncc_workspace(int64_t B, int64_t C, int64_t H, int64_t W, int64_t crop);
int64_t fvr_edge_ncc_stats_count(void);
int fvr_edge_ncc_forward(const float* a, const float* b, int64_t B, int64_t Bt, int64_t C, int64_t H, int64_t W,
                         int64_t crop, float ms_weight, int reduction_mean, void* workspace, int64_t ws_bytes,
                         double* stats, float* out, void* stream);
/* d out / d a (wrt_b = 0) or d out / d b per batch item (wrt_b = 1; the
 * caller sums over the batch for a broadcast target) into grad[B][C][H][W],
 * scaled by the upstream g[b * g_stride] (g_stride 0 for the mean). */
int fvr_edge_ncc_backward(const float* a, const float* b, int64_t B, int64_t Bt, int64_t C, int64_t H, int64_t W,
                          int64_t crop, float ms_weight, int reduction_mean, const double* stats, const float* g,
                          int64_t g_stride, int wrt_b, float* grad, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FVR_B200_H */
