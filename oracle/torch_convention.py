"""Oracle (test infrastructure only): float64 NumPy restatement of the
parallel-beam ``TorchDiffFVREngine`` path and of ``fourier_slice_3d``.

Reference files restated here:

* ``src/fvr/torch_engine.py``  -- spectrum precompute, Euler angles, slice axes,
  phase ramp, high-pass filter, zero-IFFT spectral NCC, image forward.
* ``src/fvr/triton_slice.py`` -- the trilinear complex gather with
  zero-padding partial interpolation (``grid_sample`` ``padding_mode='zeros'``,
  ``align_corners=True``) and its adjoint to the slice axes u, v.

Gradients are written out by hand (per-sample chain rule), independent of the
moment-based formulation the CUDA kernels use.
"""
from __future__ import annotations

import math

import numpy as np

# ----------------------------------------------------------------------------
# spectrum precompute  (torch_engine.py:56-88)
# ----------------------------------------------------------------------------


def padded_shape(shape, pad_factor=2.0):
    """``int(round(n * pad_factor))`` per axis (torch_engine.py:57-59)."""
    return tuple(int(round(n * pad_factor)) for n in shape)


def spectrum(volume, pad_factor=2.0):
    """Centred zero-pad -> fftn -> fftshift, returned as ``[2, Dp, Hp, Wp]``.

    torch_engine.py:56-86: the low-side pad is ``(P - n) // 2``; there is no
    ifftshift before the transform and no sinc^2 pre-compensation.
    """
    vol = np.asarray(volume, dtype=np.float64)
    pshape = padded_shape(vol.shape, pad_factor)
    padded = np.zeros(pshape, dtype=np.float64)
    lo = [(p - n) // 2 for p, n in zip(pshape, vol.shape)]
    padded[lo[0]:lo[0] + vol.shape[0], lo[1]:lo[1] + vol.shape[1], lo[2]:lo[2] + vol.shape[2]] = vol
    f = np.fft.fftshift(np.fft.fftn(padded))
    return np.stack([f.real, f.imag], axis=0)


# ----------------------------------------------------------------------------
# pose -> rotation  (torch_engine.py:139-174, 193-211)
# ----------------------------------------------------------------------------


def _rz(a):
    c, s = np.cos(a), np.sin(a)
    z, o = np.zeros_like(a), np.ones_like(a)
    return np.stack([np.stack([c, -s, z], -1), np.stack([s, c, z], -1), np.stack([z, z, o], -1)], -2)


def _ry(a):
    c, s = np.cos(a), np.sin(a)
    z, o = np.zeros_like(a), np.ones_like(a)
    return np.stack([np.stack([c, z, s], -1), np.stack([z, o, z], -1), np.stack([-s, z, c], -1)], -2)


def _rx(a):
    c, s = np.cos(a), np.sin(a)
    z, o = np.zeros_like(a), np.ones_like(a)
    return np.stack([np.stack([o, z, z], -1), np.stack([z, c, -s], -1), np.stack([z, s, c], -1)], -2)


def _drz(a):
    c, s = np.cos(a), np.sin(a)
    z = np.zeros_like(a)
    return np.stack([np.stack([-s, -c, z], -1), np.stack([c, -s, z], -1), np.stack([z, z, z], -1)], -2)


def _dry(a):
    c, s = np.cos(a), np.sin(a)
    z = np.zeros_like(a)
    return np.stack([np.stack([-s, z, c], -1), np.stack([z, z, z], -1), np.stack([-c, z, -s], -1)], -2)


def _drx(a):
    c, s = np.cos(a), np.sin(a)
    z = np.zeros_like(a)
    return np.stack([np.stack([z, z, z], -1), np.stack([z, -s, -c], -1), np.stack([z, c, -s], -1)], -2)


DEG = math.pi / 180.0


def euler_rotation(yaw_deg, pitch_deg, roll_deg):
    """R = Rz(yaw) . Ry(pitch) . Rx(roll) on (x, y, z) (torch_engine.py:139-174)."""
    rz, ry, rx = (np.asarray(a, np.float64) * DEG for a in (yaw_deg, pitch_deg, roll_deg))
    return _rz(rz) @ _ry(ry) @ _rx(rx)


def euler_rotation_grad(yaw_deg, pitch_deg, roll_deg, g_r):
    """d<g_r, R>/d(yaw, pitch, roll) in 1/deg; ``g_r`` is ``[C,3,3]``."""
    rz, ry, rx = (np.asarray(a, np.float64) * DEG for a in (yaw_deg, pitch_deg, roll_deg))
    Z, Y, X = _rz(rz), _ry(ry), _rx(rx)
    dz = (_drz(rz) @ Y @ X * g_r).sum((-2, -1)) * DEG
    dy = (Z @ _dry(ry) @ X * g_r).sum((-2, -1)) * DEG
    dx = (Z @ Y @ _drx(rx) * g_r).sum((-2, -1)) * DEG
    return np.stack([dz, dy, dx], -1)


def lateral_rotation():
    """``Rz(90 deg)`` exactly as the reference evaluates it: the angle is formed
    and its cos/sin taken in float32, so the zero entries are -4.37e-8
    (torch_engine.py:194-198)."""
    a = np.float32(90.0) * np.float32(math.pi / 180.0)
    c, s = float(np.cos(a, dtype=np.float32)), float(np.sin(a, dtype=np.float32))
    return np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]], dtype=np.float64)


def slice_axes(poses, view, pad_shape):
    """u_xyz, v_xyz ``[C,3]`` and the volume centre (torch_engine.py:190-211).

    ``u = R[0,:] * ((W-1)/2, (H-1)/2, (D-1)/2)``, ``v = R[1,:] * (same)``;
    the lateral view uses ``R_pose . Rz(90 deg)``.
    """
    poses = np.asarray(poses, np.float64)
    R = euler_rotation(poses[:, 0], poses[:, 1], poses[:, 2])
    if view.lower() == "lateral":
        R = R @ lateral_rotation()
    D, H, W = pad_shape
    c = np.array([0.5 * max(W - 1, 1), 0.5 * max(H - 1, 1), 0.5 * max(D - 1, 1)])
    return R[:, 0, :] * c, R[:, 1, :] * c, c, R


def linspace_f32(start, end, n):
    """The float32 values of ``torch.linspace(start, end, n)``: a float32 step,
    then each value start + step * i (lower half) or end - step * (n - 1 - i)
    (upper half) rounded once to float32; returned as float64."""
    if n == 1:
        return np.array([float(np.float32(start))])
    s32, e32 = np.float32(start), np.float32(end)
    step = np.float64(np.float32((e32 - s32) / np.float32(n - 1)))
    i = np.arange(n, dtype=np.float64)
    lo = (np.float64(s32) + step * i).astype(np.float32)
    hi = (np.float64(e32) - step * (n - 1 - i)).astype(np.float32)
    return np.where(np.arange(n) < n // 2, lo, hi).astype(np.float64)


def freq_grid(out_res):
    """``ku, kv = meshgrid(linspace(-1,1,R), linspace(-1,1,R), 'ij')`` with the
    float32 grid values the reference samples at (torch_engine.py:115-121)."""
    lin = linspace_f32(-1.0, 1.0, out_res)
    ku, kv = np.meshgrid(lin, lin, indexing="ij")
    return ku, kv


def hp_filter(H, W, sigma=4.0):
    """``1 - exp(-r^2 / (2 sigma^2))`` on ``linspace(-H/2, H/2, H)`` grids (torch_engine.py:123-136)."""
    y = np.linspace(-H / 2, H / 2, H)
    x = np.linspace(-W / 2, W / 2, W)
    yy, xx = np.meshgrid(y, x, indexing="ij")
    return 1.0 - np.exp(-(xx * xx + yy * yy) / (2.0 * sigma ** 2))


# ----------------------------------------------------------------------------
# trilinear complex gather  (triton_slice.py:37-143, 594-715)
# ----------------------------------------------------------------------------


def trilinear(vol, px, py, pz, deriv=False):
    """Zero-padding partial trilinear interpolation of ``vol[..., D, H, W]``.

    Corners outside the volume contribute zero (``grid_sample``
    ``padding_mode='zeros'``, ``align_corners=True``; triton_slice.py:38-44,
    664-715).  Returns the value ``[..., *px.shape]`` and, with ``deriv``, the
    three spatial derivatives of the piecewise-linear interpolant (floor
    convention at integer positions, triton_slice.py:246-252).
    """
    D, H, W = vol.shape[-3:]
    x0, y0, z0 = np.floor(px), np.floor(py), np.floor(pz)
    tx, ty, tz = px - x0, py - y0, pz - z0
    ix0, iy0, iz0 = x0.astype(np.int64), y0.astype(np.int64), z0.astype(np.int64)
    lead = vol.shape[:-3]
    out = np.zeros(lead + px.shape)
    if deriv:
        gx, gy, gz = np.zeros_like(out), np.zeros_like(out), np.zeros_like(out)
    for dz in (0, 1):
        iz = iz0 + dz
        wz, sz = (tz, 1.0) if dz else (1.0 - tz, -1.0)
        for dy in (0, 1):
            iy = iy0 + dy
            wy, sy = (ty, 1.0) if dy else (1.0 - ty, -1.0)
            for dx in (0, 1):
                ix = ix0 + dx
                wx, sx = (tx, 1.0) if dx else (1.0 - tx, -1.0)
                inb = (ix >= 0) & (ix < W) & (iy >= 0) & (iy < H) & (iz >= 0) & (iz < D)
                val = vol[..., np.clip(iz, 0, D - 1), np.clip(iy, 0, H - 1), np.clip(ix, 0, W - 1)] * inb
                out += val * (wx * wy * wz)
                if deriv:
                    gx += val * (sx * wy * wz)
                    gy += val * (wx * sy * wz)
                    gz += val * (wx * wy * sz)
    if deriv:
        return out, gx, gy, gz
    return out


def _sample_points(u_xyz, v_xyz, fx, fy, center):
    fx = np.asarray(fx, np.float64).reshape(1, -1)
    fy = np.asarray(fy, np.float64).reshape(1, -1)
    u = np.asarray(u_xyz, np.float64)
    v = np.asarray(v_xyz, np.float64)
    px = center[0] + fx * u[:, 0:1] + fy * v[:, 0:1]
    py = center[1] + fx * u[:, 1:2] + fy * v[:, 1:2]
    pz = center[2] + fx * u[:, 2:3] + fy * v[:, 2:3]
    return px, py, pz


def fourier_slice_3d(vol_ri, u_xyz, v_xyz, fx, fy, center):
    """``slice[b, n, 2, K]`` at ``p = c + fx*u_n + fy*v_n`` (triton_slice.py:594-645)."""
    vol_ri = np.asarray(vol_ri, np.float64)
    px, py, pz = _sample_points(u_xyz, v_xyz, fx, fy, center)
    out = trilinear(vol_ri, px, py, pz)  # [B, 2, N, K]
    return np.transpose(out, (0, 2, 1, 3))


def fourier_slice_3d_adjoint(vol_ri, u_xyz, v_xyz, fx, fy, center, grad_out):
    """dL/du, dL/dv ``[N,3]`` for upstream ``grad_out[B, N, 2, K]`` (triton_slice.py:145-271, 305-339)."""
    vol_ri = np.asarray(vol_ri, np.float64)
    px, py, pz = _sample_points(u_xyz, v_xyz, fx, fy, center)
    _, gx, gy, gz = trilinear(vol_ri, px, py, pz, deriv=True)  # [B, 2, N, K]
    g = np.transpose(np.asarray(grad_out, np.float64), (0, 2, 1, 3))
    dp = [(g * d).sum(axis=(0, 1)) for d in (gx, gy, gz)]  # [N, K] each
    fxr = np.asarray(fx, np.float64).reshape(1, -1)
    fyr = np.asarray(fy, np.float64).reshape(1, -1)
    gu = np.stack([(d * fxr).sum(-1) for d in dp], -1)
    gv = np.stack([(d * fyr).sum(-1) for d in dp], -1)
    return gu, gv


# ----------------------------------------------------------------------------
# slice spectrum, phase ramp, losses  (torch_engine.py:176-337)
# ----------------------------------------------------------------------------


def phase_scale(out_res, spacing0):
    """kappa in ``phase = kappa * (ku*tx + kv*ty)`` (torch_engine.py:227-232)."""
    return -2.0 * math.pi / (out_res * spacing0 + 1e-6)


def _slice_parts(spec, poses, view, out_res, deriv=False):
    poses = np.asarray(poses, np.float64)
    u, v, c, R = slice_axes(poses, view, spec.shape[-3:])
    ku, kv = freq_grid(out_res)
    px, py, pz = _sample_points(u, v, ku.reshape(-1), kv.reshape(-1), c)
    res = trilinear(spec, px, py, pz, deriv=deriv)
    return res, (u, v, c, R, ku, kv)


def extract_slice_spectrum(spec, poses, view="ap", out_res=128, spacing0=1.0):
    """Phase-modulated complex slice ``[C, R, R]`` (torch_engine.py:176-234).

    ``poses[:, 5]`` (tz) is never read, as in the reference (torch_engine.py:190-191).
    """
    poses = np.asarray(poses, np.float64)
    C = poses.shape[0]
    s, (u, v, c, R, ku, kv) = _slice_parts(spec, poses, view, out_res)
    S = (s[0] + 1j * s[1]).reshape(C, out_res, out_res)
    phase = phase_scale(out_res, spacing0) * (ku[None] * poses[:, 3, None, None] + kv[None] * poses[:, 4, None, None])
    return S * np.exp(1j * phase)


def forward_image(spec, poses, view="ap", out_res=128, spacing0=1.0):
    """``relu(real(ifft2(ifftshift(S))))`` -> ``[C,1,R,R]`` (torch_engine.py:236-241)."""
    Sm = extract_slice_spectrum(spec, poses, view, out_res, spacing0)
    img = np.fft.ifft2(np.fft.ifftshift(Sm, axes=(-2, -1)), axes=(-2, -1)).real
    return np.maximum(img, 0.0)[:, None]


def prepare_spectral_target(target, high_pass=True, sigma=4.0):
    """``fftshift(fft2(target)) * HP`` (torch_engine.py:255-267)."""
    t = np.asarray(target, np.float64)
    H, W = t.shape[-2:]
    f = np.fft.fftshift(np.fft.fft2(t, axes=(-2, -1)), axes=(-2, -1))
    if high_pass:
        f = f * hp_filter(H, W, sigma)
    return f


def _ncc_terms(Sh, T):
    cross = (Sh * np.conj(T)).real.sum((-2, -1))
    ep = (np.abs(Sh) ** 2).sum((-2, -1))
    et = (np.abs(T) ** 2).sum((-2, -1))
    return cross, ep, et


def spectral_ncc(spec, poses, f_targ, view="ap", high_pass=True, sigma=4.0, spacing0=1.0):
    """Zero-IFFT spectral NCC loss and per-candidate NCC (torch_engine.py:269-307)."""
    f_targ = np.asarray(f_targ).reshape(np.asarray(f_targ).shape[-2:])
    R = f_targ.shape[-1]
    Sh = extract_slice_spectrum(spec, poses, view, R, spacing0)
    if high_pass:
        Sh = Sh * hp_filter(R, R, sigma)
    cross, ep, et = _ncc_terms(Sh, f_targ[None])
    ncc = cross / (np.sqrt(ep * et) + 1e-8)
    return 1.0 - ncc.mean(), ncc


def spectral_ncc_grad(spec, poses, f_targ, view="ap", high_pass=True, sigma=4.0, spacing0=1.0, g=1.0):
    """dL/dposes ``[C,6]`` of :func:`spectral_ncc` by the per-sample chain rule.

    ``G = dL/dS_hat = gc (a T + 2 b S_hat)``; ``dL/dS = HP e^{-i phi} G``;
    ``dL/dphi = Re(conj(G) i S_hat)``; then through the trilinear derivative
    to u, v, through ``u = R[0]*scale`` to R and the Euler angles.  Column 5
    (tz) is always zero.
    """
    poses = np.asarray(poses, np.float64)
    C = poses.shape[0]
    f_targ = np.asarray(f_targ).reshape(np.asarray(f_targ).shape[-2:])
    R_ = f_targ.shape[-1]
    (s, sx, sy, sz), (u, v, c, Rt, ku, kv) = _slice_parts(spec, poses, view, R_, deriv=True)
    S = (s[0] + 1j * s[1]).reshape(C, R_, R_)
    dS = [(d[0] + 1j * d[1]).reshape(C, R_, R_) for d in (sx, sy, sz)]
    kap = phase_scale(R_, spacing0)
    phase = kap * (ku[None] * poses[:, 3, None, None] + kv[None] * poses[:, 4, None, None])
    hp = hp_filter(R_, R_, sigma) if high_pass else np.ones((R_, R_))
    M = hp[None] * np.exp(1j * phase)
    Sh = M * S
    cross, ep, et = _ncc_terms(Sh, f_targ[None])
    s_ = np.sqrt(ep * et)
    a = 1.0 / (s_ + 1e-8)
    b = -cross * et / (2.0 * s_ * (s_ + 1e-8) ** 2)
    gc = -g / C
    G = gc * (a[:, None, None] * f_targ[None] + 2.0 * b[:, None, None] * Sh)
    dLdS = np.conj(M) * G
    dphi = (np.conj(G) * 1j * Sh).real
    dtx = (dphi * kap * ku[None]).sum((-2, -1))
    dty = (dphi * kap * kv[None]).sum((-2, -1))
    dp = [(np.conj(dLdS) * d).real for d in dS]
    du = np.stack([(d * ku[None]).sum((-2, -1)) for d in dp], -1)
    dv = np.stack([(d * kv[None]).sum((-2, -1)) for d in dp], -1)
    gR = np.zeros((C, 3, 3))
    gR[:, 0, :] = du * c
    gR[:, 1, :] = dv * c
    if view.lower() == "lateral":
        gR = gR @ lateral_rotation().T
    gang = euler_rotation_grad(poses[:, 0], poses[:, 1], poses[:, 2], gR)
    out = np.zeros((C, 6))
    out[:, 0:3] = gang
    out[:, 3] = dtx
    out[:, 4] = dty
    return out


def forward_image_grad(spec, poses, grad_img, view="ap", out_res=128, spacing0=1.0):
    """dL/dposes of :func:`forward_image` for upstream ``grad_img[C,1,R,R]``.

    Adjoint chain: relu mask -> real part -> ifft2 (adjoint = fft2 / n) ->
    ifftshift (adjoint = fftshift) -> phase ramp -> trilinear gather.
    """
    poses = np.asarray(poses, np.float64)
    C = poses.shape[0]
    R_ = out_res
    (s, sx, sy, sz), (u, v, c, Rt, ku, kv) = _slice_parts(spec, poses, view, R_, deriv=True)
    S = (s[0] + 1j * s[1]).reshape(C, R_, R_)
    dS = [(d[0] + 1j * d[1]).reshape(C, R_, R_) for d in (sx, sy, sz)]
    kap = phase_scale(R_, spacing0)
    phase = kap * (ku[None] * poses[:, 3, None, None] + kv[None] * poses[:, 4, None, None])
    M = np.exp(1j * phase)
    Sh = M * S
    img = np.fft.ifft2(np.fft.ifftshift(Sh, axes=(-2, -1)), axes=(-2, -1)).real
    g = np.asarray(grad_img, np.float64).reshape(C, R_, R_) * (img > 0)
    G = np.fft.fftshift(np.fft.fft2(g.astype(np.complex128), axes=(-2, -1)), axes=(-2, -1)) / (R_ * R_)
    dLdS = np.conj(M) * G
    dphi = (np.conj(G) * 1j * Sh).real
    dtx = (dphi * kap * ku[None]).sum((-2, -1))
    dty = (dphi * kap * kv[None]).sum((-2, -1))
    dp = [(np.conj(dLdS) * d).real for d in dS]
    du = np.stack([(d * ku[None]).sum((-2, -1)) for d in dp], -1)
    dv = np.stack([(d * kv[None]).sum((-2, -1)) for d in dp], -1)
    gR = np.zeros((C, 3, 3))
    gR[:, 0, :] = du * c
    gR[:, 1, :] = dv * c
    if view.lower() == "lateral":
        gR = gR @ lateral_rotation().T
    out = np.zeros((C, 6))
    out[:, 0:3] = euler_rotation_grad(poses[:, 0], poses[:, 1], poses[:, 2], gR)
    out[:, 3] = dtx
    out[:, 4] = dty
    return out


def spectral_ncc_loss_images(pred, target, high_pass=True, sigma=4.0):
    """Image-domain spectral NCC via fft2 of both images (torch_engine.py:309-337)."""
    p = np.asarray(pred, np.float64)
    t = np.asarray(target, np.float64)
    H, W = p.shape[-2:]
    Fp = np.fft.fftshift(np.fft.fft2(p, axes=(-2, -1)), axes=(-2, -1))
    Ft = np.fft.fftshift(np.fft.fft2(t, axes=(-2, -1)), axes=(-2, -1))
    if high_pass:
        hp = hp_filter(H, W, sigma)
        Fp, Ft = Fp * hp, Ft * hp
    cross, ep, et = _ncc_terms(Fp, Ft)
    ncc = cross / (np.sqrt(ep * et) + 1e-8)
    return 1.0 - ncc.mean()


def spectral_ncc_loss_images_grad(pred, target, high_pass=True, sigma=4.0, g=1.0):
    """dL/dpred of :func:`spectral_ncc_loss_images` (pred is ``[B,1,H,W]``)."""
    p = np.asarray(pred, np.float64)
    t = np.asarray(target, np.float64)
    H, W = p.shape[-2:]
    Fp = np.fft.fftshift(np.fft.fft2(p, axes=(-2, -1)), axes=(-2, -1))
    Ft = np.fft.fftshift(np.fft.fft2(t, axes=(-2, -1)), axes=(-2, -1))
    hp = hp_filter(H, W, sigma) if high_pass else np.ones((H, W))
    Fp, Ft = Fp * hp, Ft * hp
    cross, ep, et = _ncc_terms(Fp, Ft)
    s_ = np.sqrt(ep * et)
    n = cross.size
    a = 1.0 / (s_ + 1e-8)
    b = -cross * et / (2.0 * s_ * (s_ + 1e-8) ** 2)
    G = (-g / n) * (a[..., None, None] * Ft + 2.0 * b[..., None, None] * Fp)
    # adjoint of x -> hp * fftshift(fft2(x)): real part of ifft2(ifftshift(hp G)) * (H W)
    Gx = np.fft.ifft2(np.fft.ifftshift(hp * G, axes=(-2, -1)), axes=(-2, -1)) * (H * W)
    return Gx.real


def make_ellipsoid_volume(n, seed, n_ellipsoids=12, shape=None):
    """Seeded synthetic volume of additive ellipsoids (attenuation U(0, 0.05)/mm).

    Centres ~U(0.3N, 0.7N), semi-axes ~U(0.05N, 0.2N), per axis.  Used by the
    benchmark and the parity tests as the stand-in for CT data.
    """
    shape = tuple(shape) if shape is not None else (n, n, n)
    rng = np.random.default_rng(seed)
    vol = np.zeros(shape, np.float32)
    grids = np.meshgrid(*[np.arange(s, dtype=np.float32) for s in shape], indexing="ij")
    for _ in range(n_ellipsoids):
        c = [rng.uniform(0.3 * s, 0.7 * s) for s in shape]
        r = [rng.uniform(0.05 * s, 0.2 * s) for s in shape]
        mu = rng.uniform(0.0, 0.05)
        q = sum(((g - ci) / ri) ** 2 for g, ci, ri in zip(grids, c, r))
        vol += np.float32(mu) * (q <= 1.0)
    return vol


def make_poses(n, seed, rot_deg=10.0, trans_mm=5.0):
    """Seeded poses ``[n,6]``: rotations U(+-rot_deg) deg, translations U(+-trans_mm) mm."""
    rng = np.random.default_rng(seed)
    p = np.zeros((n, 6), np.float32)
    p[:, :3] = rng.uniform(-rot_deg, rot_deg, (n, 3))
    p[:, 3:] = rng.uniform(-trans_mm, trans_mm, (n, 3))
    return p
