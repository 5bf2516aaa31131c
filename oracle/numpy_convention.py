"""Oracle (test infrastructure only): restatement of the reference's NumPy
renderer ``DifferentiableFourierVolumeRenderer`` (src/fvr/diff_fvr.py) and
``SpectralGradientEngine`` (src/fvr/gradients.py) in float64 NumPy, with its
own order-1 ``map_coordinates(mode='constant')`` (zero unless every
coordinate lies in [0, n-1]).
"""
from __future__ import annotations

import numpy as np


def spectrum(volume, pad_factor=2.0, premult=True):
    """sinc^2 pre-compensation, centred pad, fftshift(fftn(ifftshift(.))) (diff_fvr.py:22-54)."""
    vol = np.asarray(volume, np.float64)
    nz, ny, nx = vol.shape
    pz, py, px = (int(round(n * pad_factor)) for n in vol.shape)
    if premult:
        def corr(n, p):
            return 1.0 / np.maximum(np.sinc((np.arange(n) - n / 2.0) / p) ** 2, 0.05)

        vol = vol * (corr(nz, pz)[:, None, None] * corr(ny, py)[None, :, None] * corr(nx, px)[None, None, :])
    padded = np.zeros((pz, py, px))
    sz, sy, sx = (pz - nz) // 2, (py - ny) // 2, (px - nx) // 2
    padded[sz:sz + nz, sy:sy + ny, sx:sx + nx] = vol
    return np.fft.fftshift(np.fft.fftn(np.fft.ifftshift(padded)))


def basis(yaw, pitch, roll, view):
    """rot = rz(yaw on Y,X) . ry(roll on Z,X) . rx(pitch on Z,Y); u, v per view (diff_fvr.py:56-104)."""
    y, p, r = np.radians(yaw), np.radians(pitch), np.radians(roll)
    rz = np.array([[1.0, 0, 0], [0, np.cos(y), -np.sin(y)], [0, np.sin(y), np.cos(y)]])
    ry = np.array([[np.cos(r), 0, np.sin(r)], [0, 1.0, 0], [-np.sin(r), 0, np.cos(r)]])
    rx = np.array([[np.cos(p), -np.sin(p), 0], [np.sin(p), np.cos(p), 0], [0, 0, 1.0]])
    rot = rz @ ry @ rx
    ub, vb = {"lateral": ([0.0, 1, 0], [1.0, 0, 0]), "ap": ([0.0, 0, 1], [1.0, 0, 0])}.get(
        view, ([0.0, 0, 1], [0.0, 1, 0]))
    return rot @ np.array(ub), rot @ np.array(vb)


def map_coordinates_linear(vol, z, y, x):
    """Order-1 interpolation with mode='constant' (scipy.ndimage semantics)."""
    D, H, W = vol.shape
    ok = (z >= 0) & (z <= D - 1) & (y >= 0) & (y <= H - 1) & (x >= 0) & (x <= W - 1)
    z, y, x = np.where(ok, z, 0), np.where(ok, y, 0), np.where(ok, x, 0)
    z0, y0, x0 = np.floor(z).astype(int), np.floor(y).astype(int), np.floor(x).astype(int)
    tz, ty, tx = z - z0, y - y0, x - x0
    z1, y1, x1 = np.minimum(z0 + 1, D - 1), np.minimum(y0 + 1, H - 1), np.minimum(x0 + 1, W - 1)
    out = 0.0
    for zz, wz in ((z0, 1 - tz), (z1, tz)):
        for yy, wy in ((y0, 1 - ty), (y1, ty)):
            for xx, wx in ((x0, 1 - tx), (x1, tx)):
                out = out + vol[zz, yy, xx] * (wz * wy * wx)
    return np.where(ok, out, 0.0)


def dims(shape_pad, view):
    pz, py, px = shape_pad
    return {"lateral": (pz, py), "ap": (pz, px)}.get(view, (py, px))


def extract_frequency_slice(f3d, yaw=0.0, pitch=0.0, roll=0.0, tx=0.0, ty=0.0, view="lateral"):
    """diff_fvr.py:106-150."""
    sh, sw = dims(f3d.shape, view)
    u, v = basis(yaw, pitch, roll, view)
    uu, vv = np.meshgrid(np.arange(sw) - sw / 2.0, np.arange(sh) - sh / 2.0)
    c = np.array(f3d.shape) / 2.0
    z, y, x = (uu * u[k] + vv * v[k] + c[k] for k in range(3))
    s = map_coordinates_linear(f3d.real, z, y, x) + 1j * map_coordinates_linear(f3d.imag, z, y, x)
    if tx != 0.0 or ty != 0.0:
        s = s * np.exp(-2j * np.pi * (uu * tx / sw + vv * ty / sh))
    return s


def render_drr(f3d, orig_shape, yaw=0.0, pitch=0.0, roll=0.0, tx=0.0, ty=0.0, view="lateral", crop_to_roi=True):
    """diff_fvr.py:152-182."""
    s = extract_frequency_slice(f3d, yaw, pitch, roll, tx, ty, view)
    sh, sw = s.shape
    drr = np.fft.fftshift(np.fft.ifft2(np.fft.ifftshift(s))).real
    drr = np.maximum(drr * (np.prod(f3d.shape) / (sh * sw)), 0.0)
    if crop_to_roi:
        nz, ny, nx = orig_shape
        th = nz if view in ("lateral", "ap") else ny
        tw = ny if view == "lateral" else nx
        a, b = (sh - th) // 2, (sw - tw) // 2
        drr = drr[a:a + th, b:b + tw]
    return drr


def spectral_ncc(a, b):
    """diff_fvr.py:184-195."""
    na, nb = np.linalg.norm(a), np.linalg.norm(b)
    return 0.0 if na * nb == 0 else float(np.real(np.sum(a * np.conj(b))) / (na * nb))


def ncc_and_grad_translation(f_cand, f_target):
    """gradients.py:27-74 (residual form)."""
    sh, sw = f_cand.shape
    ns, nt = np.linalg.norm(f_cand), np.linalg.norm(f_target)
    if ns * nt == 0:
        return 0.0, 0.0, 0.0
    ncc = float(np.real(np.sum(f_cand * np.conj(f_target))) / (ns * nt))
    r = (f_target - ncc * (nt / ns) * f_cand) / (ns * nt)
    uu, vv = np.meshgrid(np.arange(sw) - sw / 2.0, np.arange(sh) - sh / 2.0)
    du = float(np.real(np.sum(-2j * np.pi * (uu / sw) * f_cand * np.conj(r))))
    dv = float(np.real(np.sum(-2j * np.pi * (vv / sh) * f_cand * np.conj(r))))
    return ncc, du, dv


def biplanar_loss_and_gradients(f3d, pose, t_ap, t_lat, delta=0.2):
    """gradients.py:76-135."""
    yaw, pitch, roll, tx, ty, tz = pose
    n_ap, d_ap_x, d_ap_z = ncc_and_grad_translation(extract_frequency_slice(f3d, yaw, pitch, roll, tx, tz, "ap"), t_ap)
    n_lat, d_lat_y, d_lat_z = ncc_and_grad_translation(
        extract_frequency_slice(f3d, yaw, pitch, roll, ty, tz, "lateral"), t_lat)
    loss = 0.5 * (1 - n_ap) + 0.5 * (1 - n_lat)
    g = np.zeros(6)
    for i in range(3):
        pp, pm = np.array(pose[:3], float), np.array(pose[:3], float)
        pp[i] += delta
        pm[i] -= delta
        d_ap = (spectral_ncc(extract_frequency_slice(f3d, *pp, tx, tz, "ap"), t_ap) -
                spectral_ncc(extract_frequency_slice(f3d, *pm, tx, tz, "ap"), t_ap)) / (2 * delta)
        d_lat = (spectral_ncc(extract_frequency_slice(f3d, *pp, ty, tz, "lateral"), t_lat) -
                 spectral_ncc(extract_frequency_slice(f3d, *pm, ty, tz, "lateral"), t_lat)) / (2 * delta)
        g[i] = -0.5 * (d_ap + d_lat)
    g[3], g[4], g[5] = -0.5 * d_ap_x, -0.5 * d_lat_y, -0.5 * (d_ap_z + d_lat_z)
    return float(loss), g


def articulated_spectrum(f3ds, base_pose, arts, view):
    """Sum over segments of their phase-ramped slices, each at the base pose
    plus the accumulated joint articulations below it; lateral slices take
    (ty, tz), ap (tx, tz), anything else the axial slice with (tx, ty)
    (articulated_spine.py:39-71)."""
    curr = np.array(base_pose, np.float64)
    total = None
    for i, f3d in enumerate(f3ds):
        if i > 0 and len(arts) >= i:
            curr = curr + np.asarray(arts[i - 1], np.float64)
        yaw, pitch, roll, tx, ty, tz = curr
        if view == "lateral":
            s = extract_frequency_slice(f3d, yaw, pitch, roll, ty, tz, "lateral")
        elif view == "ap":
            s = extract_frequency_slice(f3d, yaw, pitch, roll, tx, tz, "ap")
        else:
            s = extract_frequency_slice(f3d, yaw, pitch, roll, tx, ty, "axial")
        total = s if total is None else total + s
    return total


def articulated_drr(f3ds, base_pose, arts, view):
    """max(real(fftshift(ifft2(ifftshift(F)))), 0) (articulated_spine.py:73-85)."""
    f = articulated_spectrum(f3ds, base_pose, arts, view)
    return np.maximum(np.real(np.fft.fftshift(np.fft.ifft2(np.fft.ifftshift(f)))), 0.0)


def resample_isotropic_cube(volume_hu, spacing, target_res):
    """Isotropic cube keeping the CT's physical field of view centred
    (dicom_loader.py:11-30): input coordinate ratio * index + offset per axis,
    linear interpolation, -1000 HU unless every coordinate lies in [0, n-1]."""
    vol = np.asarray(volume_hu, np.float32).astype(np.float64)
    sp = np.asarray(spacing, np.float64)
    shape = np.array(vol.shape)
    vmm = float(np.max(shape * sp) / target_res)
    ratio = vmm / sp
    off = (shape - 1) / 2 - ratio * (target_res - 1) / 2
    o = np.arange(target_res, dtype=np.float64)
    cz, cy, cx = (off[k] + ratio[k] * o for k in range(3))
    Z, Y, X = np.meshgrid(cz, cy, cx, indexing="ij")
    inside = (Z >= 0) & (Z <= vol.shape[0] - 1) & (Y >= 0) & (Y <= vol.shape[1] - 1) & (X >= 0) & \
        (X <= vol.shape[2] - 1)
    fz, fy, fx = np.floor(Z), np.floor(Y), np.floor(X)
    tz, ty, tx = Z - fz, Y - fy, X - fx
    iz, iy, ix = (np.clip(a, 0, n - 1).astype(int) for a, n in ((fz, vol.shape[0]), (fy, vol.shape[1]),
                                                                 (fx, vol.shape[2])))
    iz1, iy1, ix1 = (np.minimum(a + 1, n - 1) for a, n in ((iz, vol.shape[0]), (iy, vol.shape[1]),
                                                           (ix, vol.shape[2])))
    out = np.zeros(Z.shape)
    for zi, wz in ((iz, 1 - tz), (iz1, tz)):
        for yi, wy in ((iy, 1 - ty), (iy1, ty)):
            for xi, wx in ((ix, 1 - tx), (ix1, tx)):
                out += wz * wy * wx * vol[zi, yi, xi]
    out = np.where(inside, out, -1000.0).astype(np.float32)
    return out, (vmm,) * 3


def hu_to_attenuation(volume_hu):
    """mu = max(0, (HU + 1000) / 1000) in float32 (dicom_loader.py:179-188)."""
    h = np.asarray(volume_hu, np.float32)
    return np.maximum(np.float32(0.0), (h + np.float32(1000.0)) / np.float32(1000.0)).astype(np.float32)


def prepare_spectrum(shape_pad, img, view):
    """Target image zero-padded into the view's slice frame (low side
    (S - n) // 2) and fftshift(fft2(ifftshift(.))) (core_engine.py:71-85)."""
    sh, sw = dims(shape_pad, view)
    img = np.asarray(img, np.float64)
    th, tw = img.shape
    padded = np.zeros((sh, sw))
    r0, c0 = (sh - th) // 2, (sw - tw) // 2
    padded[r0:r0 + th, c0:c0 + tw] = img
    return np.fft.fftshift(np.fft.fft2(np.fft.ifftshift(padded)))
