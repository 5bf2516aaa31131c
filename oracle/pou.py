"""Oracle (test infrastructure only): float64 NumPy restatement of the PoU-FVR
cone-beam renderer (src/fvr/cone_beam_fvr.py) and of the pinhole warp-sum
(src/fvr/triton_slice.py:718-808), with hand-derived adjoints.
"""
from __future__ import annotations

import math

import numpy as np

from .torch_convention import trilinear

# ----------------------------------------------------------------------------
# partition of unity and block spectra  (cone_beam_fvr.py:42-68, 172-303)
# ----------------------------------------------------------------------------


def make_pou_1d(length, n_blocks, overlap):
    """Raised-cosine windows summing to one (cone_beam_fvr.py:42-61)."""
    if n_blocks <= 1:
        return [np.ones(length)], float(length)
    step = length / float(n_blocks)
    ov = max(2.0, step * overlap)
    coords = np.arange(length) + 0.5
    ws = []
    for i in range(n_blocks):
        w = np.ones(length)
        if i > 0:
            x0, x1 = i * step - ov, i * step + ov
            t = np.clip((coords - x0) / (x1 - x0), 0.0, 1.0)
            w = w * 0.5 * (1.0 - np.cos(np.pi * t))
        if i < n_blocks - 1:
            x0, x1 = (i + 1) * step - ov, (i + 1) * step + ov
            t = np.clip((coords - x0) / (x1 - x0), 0.0, 1.0)
            w = w * 0.5 * (1.0 + np.cos(np.pi * t))
        ws.append(w)
    return ws, step


def sinc2_precomp_1d(n, p):
    """1 / max(sinc^2(c), 0.05), c = (i - (n-1)/2)/p (cone_beam_fvr.py:64-68)."""
    c = (np.arange(n) - (n - 1) / 2.0) / float(p)
    s = np.where(c == 0, 1.0, np.sin(np.pi * np.where(c == 0, 1.0, c)) / (np.pi * np.where(c == 0, 1.0, c)))
    return 1.0 / np.maximum(s ** 2, 0.05)


def resize_trilinear(cube, out):
    """``F.interpolate(mode='trilinear', align_corners=False)`` of a cube to out^3."""
    res = np.asarray(cube, np.float64)
    for ax in range(3):
        n_in = res.shape[ax]
        scale = n_in / out
        src = np.maximum((np.arange(out) + 0.5) * scale - 0.5, 0.0)
        i0 = np.floor(src).astype(np.int64)
        i0 = np.minimum(i0, n_in - 1)
        i1 = np.minimum(i0 + 1, n_in - 1)
        lam = src - i0
        a = np.take(res, i0, axis=ax)
        b = np.take(res, i1, axis=ax)
        shp = [1, 1, 1]
        shp[ax] = out
        lam = lam.reshape(shp)
        res = a * (1.0 - lam) + b * lam
    return res


class PoUModel:
    """Block decomposition + spectra of ``PerspectiveSlabFVR.__init__``
    (cone_beam_fvr.py:172-303) and ``from_volume`` (:331-376)."""

    def __init__(self, vol, vox_mm=1.0, grid_blocks=(2, 2, 2), block_res=80, pad_mult=2, overlap=0.25,
                 energy_thresh=1e-4, center_mode="pixel_center", origin=None):
        vol = np.asarray(vol, np.float64)
        n0, n1, n2 = vol.shape
        v = float(vox_mm)
        if origin is None:
            if center_mode == "pixel_center":
                origin = (-0.5 * (n0 - 1) * v, -0.5 * (n1 - 1) * v, -0.5 * (n2 - 1) * v)
            elif center_mode == "grid_center":
                origin = (-0.5 * n0 * v, -0.5 * n1 * v, -0.5 * n2 * v)
            else:
                raise ValueError(center_mode)
        self.vox_mm = v
        self.block_res = int(block_res)
        self.P = self.block_res * int(pad_mult)
        k = grid_blocks
        wl, st = [], []
        for n, kk in zip(vol.shape, k):
            w, s = make_pou_1d(n, kk, overlap)
            wl.append(w)
            st.append(s)
        ov = [max(2, int(round(s * overlap))) if kk > 1 else 0 for s, kk in zip(st, k)]
        m = [int(np.ceil(s + 2 * o)) for s, o in zip(st, ov)]
        M = max(m) + (1 if max(k) > 1 else 0)
        self.M = M
        self.ds_block = (M * v) / float(self.block_res)
        ws = sinc2_precomp_1d(self.block_res, self.P)
        w3 = ws[:, None, None] * ws[None, :, None] * ws[None, None, :]
        pad_b = (self.P - self.block_res) // 2
        half = ((self.P // 2) - (pad_b + (self.block_res - 1) * 0.5)) * self.ds_block
        blocks, centers, meta = [], [], []
        for i0, w0 in enumerate(wl[0]):
            nz0 = np.nonzero(w0 > 1e-6)[0]
            a0, b0 = int(nz0[0]), int(nz0[-1]) + 1
            for i1, w1 in enumerate(wl[1]):
                nz1 = np.nonzero(w1 > 1e-6)[0]
                a1, b1 = int(nz1[0]), int(nz1[-1]) + 1
                for i2, w2 in enumerate(wl[2]):
                    nz2 = np.nonzero(w2 > 1e-6)[0]
                    a2, b2 = int(nz2[0]), int(nz2[-1]) + 1
                    sub = vol[a0:b0, a1:b1, a2:b2] * (w0[a0:b0, None, None] * w1[None, a1:b1, None] *
                                                      w2[None, None, a2:b2])
                    if float(sub.sum()) <= energy_thresh:
                        continue
                    l0, l1, l2 = sub.shape
                    m0, m1, m2 = (M - l0) // 2, (M - l1) // 2, (M - l2) // 2
                    cube = np.zeros((M, M, M))
                    cube[m0:m0 + l0, m1:m1 + l1, m2:m2 + l2] = sub
                    c = [a0 + (M - 1) * 0.5 - m0, a1 + (M - 1) * 0.5 - m1, a2 + (M - 1) * 0.5 - m2]
                    centers.append([origin[i] + c[i] * v + half for i in range(3)])
                    cr = resize_trilinear(cube, self.block_res) * self.ds_block if M != self.block_res else \
                        cube * self.ds_block
                    pad = np.zeros((self.P,) * 3)
                    br = self.block_res
                    pad[pad_b:pad_b + br, pad_b:pad_b + br, pad_b:pad_b + br] = cr * w3
                    blocks.append(pad)
                    meta.append((i0, i1, i2))
        if not blocks:
            raise ValueError("Input volume contains no non-zero attenuation mass above threshold.")
        self.B = len(blocks)
        self.blocks = np.stack(blocks)
        self.centers = np.asarray(centers)
        self.block_ids = meta
        F = np.fft.fftshift(np.fft.fftn(np.fft.ifftshift(self.blocks, axes=(-3, -2, -1)), axes=(-3, -2, -1)),
                            axes=(-3, -2, -1))
        self.F_blk_ri = np.stack([F.real, F.imag], axis=1)
        freqs = np.fft.fftshift(np.fft.fftfreq(self.P, d=self.ds_block))
        fy, fx = np.meshgrid(freqs, freqs, indexing="ij")
        self.FX_flat = fx.reshape(-1)
        self.FY_flat = fy.reshape(-1)


# ----------------------------------------------------------------------------
# geometry  (cone_beam_fvr.py:523-545, 575-596, 670-688, 705-728)
# ----------------------------------------------------------------------------


def extract_detector_basis(srcs, trg_pts, u_det=None, v_det=None, n_0=None):
    c_det = trg_pts.mean(axis=(1, 2))
    if u_det is None:
        ur = trg_pts[:, 0, -1] - trg_pts[:, 0, 0]
        u_det = ur / (np.linalg.norm(ur, axis=-1, keepdims=True) + 1e-12)
    if v_det is None:
        vr = trg_pts[:, -1, 0] - trg_pts[:, 0, 0]
        v_det = vr / (np.linalg.norm(vr, axis=-1, keepdims=True) + 1e-12)
    if n_0 is None:
        nr = np.cross(v_det, u_det)
        n_0 = nr / (np.linalg.norm(nr, axis=-1, keepdims=True) + 1e-12)
        flip = ((c_det - srcs) * n_0).sum(-1, keepdims=True) < 0
        n_0 = np.where(flip, -n_0, n_0)
    return u_det, v_det, n_0


def ray_cache(src0, trg0, u0, v0, n0):
    rays = trg0 - src0.reshape(1, 1, 3)
    r = rays / np.sqrt(np.maximum((rays * rays).sum(-1, keepdims=True), 1e-12))
    cos0 = np.maximum((r * n0).sum(-1), 0.1)
    ic = 1.0 / cos0
    return (r * u0).sum(-1) * ic, (r * v0).sum(-1) * ic, ic


def make_pinhole_lattice(k_inv, sdd_mm, height, width):
    k0 = np.asarray(k_inv, np.float64).reshape(3, 3)
    cols = np.arange(width) + 0.5
    rows = np.arange(height) + 0.5
    rr, cc = np.meshgrid(rows, cols, indexing="ij")
    pix = np.stack([cc, rr, np.ones_like(cc)], -1)
    cam = np.einsum("ij,hwj->hwi", k0, pix)
    trg0 = cam * (float(sdd_mm) / np.maximum(cam[..., 2:3], 1e-6))
    src0 = np.zeros(3)
    u0, v0, n0 = extract_detector_basis(src0[None], trg0[None])
    u0, v0, n0 = u0[0], v0[0], n0[0]
    rx, ry, ic = ray_cache(src0, trg0, u0, v0, n0)
    return src0, trg0, u0, v0, n0, rx, ry, ic


def slice_and_ifft(model, u_det, v_det):
    """imgs [B, N, P, P] (cone_beam_fvr.py:480-505)."""
    P = model.P
    vs = float(P) * model.ds_block
    u_xyz = u_det[:, ::-1] * vs
    v_xyz = v_det[:, ::-1] * vs
    c = float(P // 2)
    fx = model.FX_flat.reshape(1, -1)
    fy = model.FY_flat.reshape(1, -1)
    px = c + fx * u_xyz[:, 0:1] + fy * v_xyz[:, 0:1]
    py = c + fx * u_xyz[:, 1:2] + fy * v_xyz[:, 1:2]
    pz = c + fx * u_xyz[:, 2:3] + fy * v_xyz[:, 2:3]
    s = trilinear(model.F_blk_ri, px, py, pz)  # [B, 2, N, K]
    N = u_det.shape[0]
    S = (s[:, 0] + 1j * s[:, 1]).reshape(model.B, N, P, P)
    return np.fft.fftshift(np.fft.ifft2(np.fft.ifftshift(S, axes=(-2, -1)), axes=(-2, -1)), axes=(-2, -1)).real


def block_offsets(centers, srcs, u_det, v_det, n_0):
    diff = centers[:, None, :] - srcs[None, :, :]
    return (diff * n_0[None]).sum(-1), (diff * u_det[None]).sum(-1), (diff * v_det[None]).sum(-1)


def bilinear_zeros(img, px, py):
    """Zero-padding bilinear of img[..., P, P] at (x=px, y=py) (grid_sample align_corners=True)."""
    P0, P1 = img.shape[-2:]
    x0, y0 = np.floor(px), np.floor(py)
    tx, ty = px - x0, py - y0
    ix, iy = x0.astype(np.int64), y0.astype(np.int64)
    out = 0.0
    gx = 0.0
    gy = 0.0
    for dy in (0, 1):
        for dx in (0, 1):
            xx, yy = ix + dx, iy + dy
            inb = (xx >= 0) & (xx < P1) & (yy >= 0) & (yy < P0)
            val = np.take_along_axis(img.reshape(img.shape[:-2] + (-1,)),
                                     (np.clip(yy, 0, P0 - 1) * P1 + np.clip(xx, 0, P1 - 1)), axis=-1) * inb
            wx = tx if dx else 1 - tx
            wy = ty if dy else 1 - ty
            out = out + val * wx * wy
            gx = gx + val * (1.0 if dx else -1.0) * wy
            gy = gy + val * wx * (1.0 if dy else -1.0)
    return out, gx, gy


def warp_sum(imgs, d_b, cu, cv, rx, ry, ic, inv_ds, c_idx):
    """out[n, q] = ic[q] sum_b bilinear(imgs[b, n], (d_b rx - cu)/ds + c, (d_b ry - cv)/ds + c)
    (triton_slice.py:718-784)."""
    B, N, P, _ = imgs.shape
    H, W = rx.shape
    rxf, ryf = rx.reshape(1, 1, -1), ry.reshape(1, 1, -1)
    px = (d_b[..., None] * rxf - cu[..., None]) * inv_ds + c_idx
    py = (d_b[..., None] * ryf - cv[..., None]) * inv_ds + c_idx
    val, _, _ = bilinear_zeros(imgs, px, py)
    return (val.sum(0) * ic.reshape(1, -1)).reshape(N, H, W)


def warp_sum_adjoint(imgs, d_b, cu, cv, rx, ry, ic, inv_ds, c_idx, g_out):
    """(grad_imgs, g_db, g_cu, g_cv) of :func:`warp_sum` (triton_slice.py:409-496)."""
    B, N, P, _ = imgs.shape
    rxf, ryf = rx.reshape(1, 1, -1), ry.reshape(1, 1, -1)
    px = (d_b[..., None] * rxf - cu[..., None]) * inv_ds + c_idx
    py = (d_b[..., None] * ryf - cv[..., None]) * inv_ds + c_idx
    _, gx, gy = bilinear_zeros(imgs, px, py)
    g = (np.asarray(g_out).reshape(1, N, -1) * ic.reshape(1, 1, -1))
    g = np.broadcast_to(g, (B, N, g.shape[-1]))
    dpx = g * gx * inv_ds
    dpy = g * gy * inv_ds
    g_db = (dpx * rxf + dpy * ryf).sum(-1)
    g_cu = -dpx.sum(-1)
    g_cv = -dpy.sum(-1)
    grad = np.zeros((B, N, P * P))
    x0, y0 = np.floor(px), np.floor(py)
    tx, ty = px - x0, py - y0
    ix, iy = x0.astype(np.int64), y0.astype(np.int64)
    bi = np.arange(B)[:, None, None]
    ni = np.arange(N)[None, :, None]
    for dy in (0, 1):
        for dx in (0, 1):
            xx, yy = ix + dx, iy + dy
            inb = (xx >= 0) & (xx < P) & (yy >= 0) & (yy < P)
            w = (tx if dx else 1 - tx) * (ty if dy else 1 - ty)
            idx = np.clip(yy, 0, P - 1) * P + np.clip(xx, 0, P - 1)
            np.add.at(grad, (np.broadcast_to(bi, idx.shape)[inb], np.broadcast_to(ni, idx.shape)[inb], idx[inb]),
                      (g * w)[inb])
    return grad.reshape(B, N, P, P), g_db, g_cu, g_cv


def pose_geometry(mats, lattice):
    src0, trg0, u0, v0, n0 = lattice[:5]
    R = mats[:, :3, :3]
    t = mats[:, :3, 3]
    return R @ src0 + t, R @ u0, R @ v0, R @ n0


def forward_pinhole(model, mats, lattice):
    """[N, 1, H, W] via the SE(3)-invariant ray cache (cone_beam_fvr.py:670-686, 547-573)."""
    mats = np.asarray(mats, np.float64)
    srcs, u, v, n = pose_geometry(mats, lattice)
    imgs = slice_and_ifft(model, u, v)
    d_b, cu, cv = block_offsets(model.centers, srcs, u, v, n)
    rx, ry, ic = lattice[5:8]
    return warp_sum(imgs, d_b, cu, cv, rx, ry, ic, 1.0 / model.ds_block, float(model.P // 2))[:, None]


def project_core(model, srcs, trg_pts, u_det, v_det, n_0):
    """Explicit-ray renderer (cone_beam_fvr.py:423-478) -> [N, H, W]."""
    N, H, W, _ = trg_pts.shape
    imgs = slice_and_ifft(model, u_det, v_det)
    d_b, cu, cv = block_offsets(model.centers, srcs, u_det, v_det, n_0)
    rays = trg_pts - srcs[:, None, None, :]
    r = rays / np.sqrt(np.maximum((rays * rays).sum(-1, keepdims=True), 1e-12))
    cos = np.maximum((r * n_0[:, None, None, :]).sum(-1), 0.1)
    ic = 1.0 / cos
    ru = (r * u_det[:, None, None, :]).sum(-1)
    rv = (r * v_det[:, None, None, :]).sum(-1)
    tau = d_b[:, :, None, None] * ic[None]
    xi = tau * ru[None] - cu[:, :, None, None]
    eta = tau * rv[None] - cv[:, :, None, None]
    c = float(model.P // 2)
    px = (xi / model.ds_block + c).reshape(model.B, N, -1)
    py = (eta / model.ds_block + c).reshape(model.B, N, -1)
    val, _, _ = bilinear_zeros(imgs, px, py)
    return val.sum(0).reshape(N, H, W) * ic


def forward_explicit(model, mats, lattice):
    """5-tuple lattice path (cone_beam_fvr.py:686-688)."""
    mats = np.asarray(mats, np.float64)
    srcs, u, v, n = pose_geometry(mats, lattice)
    trg = np.einsum("nij,hwj->nhwi", mats[:, :3, :3], lattice[1]) + mats[:, None, None, :3, 3]
    return project_core(model, srcs, trg, u, v, n)[:, None]


def carm_geometry(yaw, pitch, roll, tx, ty, tz, vox_mm, sad_mm, sdd_mm, det_px, det_fov_mm, view):
    """forward_carm_view geometry (cone_beam_fvr.py:761-832)."""
    yr, pr, rr = (math.radians(a) for a in (yaw, pitch, roll))
    cy, sy, cp, sp, cr, sr = math.cos(yr), math.sin(yr), math.cos(pr), math.sin(pr), math.cos(rr), math.sin(rr)
    rz = np.array([[1, 0, 0], [0, cy, -sy], [0, sy, cy]])
    ry = np.array([[cr, 0, sr], [0, 1, 0], [-sr, 0, cr]])
    rx = np.array([[cp, -sp, 0], [sp, cp, 0], [0, 0, 1]])
    rot = rz @ ry @ rx
    lin = np.linspace(-0.5, 0.5, det_px) * float(det_fov_mm)
    vv, uu = np.meshgrid(lin, lin, indexing="ij")
    det_d = float(sdd_mm - sad_mm)
    if view == "ap":
        src0 = np.array([0.0, -float(sad_mm), 0.0])
        trg0 = np.stack([vv, np.full_like(uu, det_d), uu], -1)
        u0, v0, n0 = np.array([0.0, 0, 1]), np.array([1.0, 0, 0]), np.array([0.0, 1, 0])
    else:
        src0 = np.array([0.0, 0.0, -float(sad_mm)])
        trg0 = np.stack([vv, uu, np.full_like(uu, det_d)], -1)
        u0, v0, n0 = np.array([0.0, 1, 0]), np.array([1.0, 0, 0]), np.array([0.0, 0, 1])
    t_shift = np.array([tz, ty, tx]) * vox_mm
    src = rot @ src0 - t_shift
    trg = np.einsum("ij,hwj->hwi", rot, trg0) - t_shift
    return src, trg, rot @ u0, rot @ v0, rot @ n0


def forward_carm_view(model, yaw, pitch, roll, tx, ty, tz, sad_mm, sdd_mm, det_px, det_fov_mm, view="ap"):
    src, trg, u, v, n = carm_geometry(yaw, pitch, roll, tx, ty, tz, model.vox_mm, sad_mm, sdd_mm, det_px,
                                      det_fov_mm, view)
    return project_core(model, src[None], trg[None], u[None], v[None], n[None])[0]


# ----------------------------------------------------------------------------
# adjoint of the lattice (SE(3)-invariant) path
# ----------------------------------------------------------------------------


def forward_pinhole_grad(model, mats, lattice, w):
    """d<w, forward_pinhole>/dmats [N, 4, 4] by the chain
    warp adjoint -> IFFT adjoint -> slice adjoint -> offsets -> pose matrices."""
    mats = np.asarray(mats, np.float64)
    N = mats.shape[0]
    P = model.P
    srcs, u, v, n = pose_geometry(mats, lattice)
    imgs = slice_and_ifft(model, u, v)
    d_b, cu, cv = block_offsets(model.centers, srcs, u, v, n)
    rx, ry, ic = lattice[5:8]
    inv_ds, c_idx = 1.0 / model.ds_block, float(P // 2)
    g_imgs, g_db, g_cu, g_cv = warp_sum_adjoint(imgs, d_b, cu, cv, rx, ry, ic, inv_ds, c_idx,
                                                np.asarray(w, np.float64).reshape(N, -1))
    # imgs = Re fftshift(ifft2(ifftshift(S)))  ->  G = fftshift(fft2(ifftshift(g))) / P^2
    G = np.fft.fftshift(np.fft.fft2(np.fft.ifftshift(g_imgs, axes=(-2, -1)), axes=(-2, -1)), axes=(-2, -1)) / (P * P)
    vs = float(P) * model.ds_block
    u_xyz, v_xyz = u[:, ::-1] * vs, v[:, ::-1] * vs
    fx, fy = model.FX_flat.reshape(1, -1), model.FY_flat.reshape(1, -1)
    c = float(P // 2)
    px = c + fx * u_xyz[:, 0:1] + fy * v_xyz[:, 0:1]
    py = c + fx * u_xyz[:, 1:2] + fy * v_xyz[:, 1:2]
    pz = c + fx * u_xyz[:, 2:3] + fy * v_xyz[:, 2:3]
    _, sx, sy, sz = trilinear(model.F_blk_ri, px, py, pz, deriv=True)  # [B, 2, N, K]
    Gr = G.real.reshape(model.B, N, -1)
    Gi = G.imag.reshape(model.B, N, -1)
    dp = [(Gr * d[:, 0] + Gi * d[:, 1]).sum(0) for d in (sx, sy, sz)]  # [N, K]
    g_uxyz = np.stack([(d * fx).sum(-1) for d in dp], -1)
    g_vxyz = np.stack([(d * fy).sum(-1) for d in dp], -1)
    g_u = g_uxyz[:, ::-1] * vs
    g_v = g_vxyz[:, ::-1] * vs
    diff = model.centers[:, None, :] - srcs[None]  # [B, N, 3]
    g_n = (g_db[..., None] * diff).sum(0)
    g_u = g_u + (g_cu[..., None] * diff).sum(0)
    g_v = g_v + (g_cv[..., None] * diff).sum(0)
    g_s = -(g_db[..., None] * n[None] + g_cu[..., None] * u[None] + g_cv[..., None] * v[None]).sum(0)
    src0, _, u0, v0, n0 = lattice[:5]
    gm = np.zeros((N, 4, 4))
    gm[:, :3, :3] = (np.einsum("ni,j->nij", g_s, src0) + np.einsum("ni,j->nij", g_u, u0) +
                     np.einsum("ni,j->nij", g_v, v0) + np.einsum("ni,j->nij", g_n, n0))
    gm[:, :3, 3] = g_s
    return gm


def edge_dominant_ncc(pred, target, border_crop=None, multiscale_weight=0.25, reduction="mean"):
    """Sobel gradient NCC with border crop and 3x3-blurred second scale (cone_beam_fvr.py:71-112)."""
    pred = np.asarray(pred, np.float64)
    target = np.asarray(target, np.float64)
    H = pred.shape[-1]
    crop = max(4, H // 8) if border_crop is None else int(border_crop)
    kx = np.array([[-1.0, 0, 1], [-2, 0, 2], [-1, 0, 1]])
    ky = kx.T.copy()

    def conv(a, k):
        p = np.pad(a, [(0, 0)] * (a.ndim - 2) + [(1, 1), (1, 1)])
        out = np.zeros_like(a)
        for i in range(3):
            for j in range(3):
                out += k[i, j] * p[..., i:i + a.shape[-2], j:j + a.shape[-1]]
        return out

    def grad_ncc(a, b):
        sl = slice(crop, -crop if crop > 0 else None)
        ax, ay = conv(a, kx)[..., sl, sl], conv(a, ky)[..., sl, sl]
        bx, by = conv(b, kx)[..., sl, sl], conv(b, ky)[..., sl, sl]

        def ncc(u, v):
            u0 = u - u.mean((-2, -1), keepdims=True)
            v0 = v - v.mean((-2, -1), keepdims=True)
            num = (u0 * v0).sum((-2, -1))
            den = np.sqrt(np.maximum((u0 ** 2).sum((-2, -1)) * (v0 ** 2).sum((-2, -1)), 1e-12))
            val = (num / den).mean(1)
            return val.mean() if reduction == "mean" else val

        return 0.5 * (ncc(ax, bx) + ncc(ay, by))

    g_fine = grad_ncc(pred, target)
    if multiscale_weight <= 0.0 or H < 96:
        return g_fine

    def blur(a):
        p = np.pad(a, [(0, 0)] * (a.ndim - 2) + [(1, 1), (1, 1)])
        out = np.zeros_like(a)
        for i in range(3):
            for j in range(3):
                out += p[..., i:i + a.shape[-2], j:j + a.shape[-1]]
        return out / 9.0

    return (1.0 - multiscale_weight) * g_fine + multiscale_weight * grad_ncc(blur(pred), blur(target))
