"""Partition-of-unity cone-beam Fourier volume renderer on B200 (drop-in for
``PerspectiveSlabFVR`` and the helpers of src/fvr/cone_beam_fvr.py).

The volume is split into overlapping raised-cosine (cos^2) blocks; each
block's zero-padded spectrum is sliced along the pose's detector plane,
inverse-transformed and pinhole-warped onto the detector, and the blocks are
summed with the 1/cos obliquity factor.  Block extraction, the block spectra
(batched shared-memory FFT), the per-pose slices (stencil layout), the
batched 2D IFFT, the warp-sum and the whole adjoint chain back to the pose
matrices run in ``libfvr_b200.so``, and so does the FP64 pinhole lattice.
The one-time block layout (1D windows and their supports, block centres) is
small host arithmetic.  Inputs on the CPU are moved to the model's CUDA
device and results come back on the device of the pose inputs; there is no
CPU compute path.
"""
from __future__ import annotations

import ctypes as _ct
import math
from typing import Dict, Optional, Tuple, Union

import numpy as np
import torch
import torch.nn as nn

from . import _lib as L
from . import _runtime as RT
from . import profiling

SLAB_PRESETS: Dict[str, Dict[str, object]] = {
    "fast_coarse": {"grid_blocks": (2, 2, 2), "block_res": 64, "dtype": torch.bfloat16},
    "balanced": {"grid_blocks": (2, 4, 2), "block_res": 80, "dtype": torch.bfloat16},
    "isotropic": {"grid_blocks": (4, 4, 4), "block_res": 64, "dtype": torch.bfloat16},
}


def _pou_windows(length: int, n_blocks: int, overlap: float):
    """Partition-of-unity weights along one axis as an fp64 array
    ``[n_blocks, length]`` and the block pitch (cone_beam_fvr.py:42-61).

    The axis is cut at the ``n_blocks - 1`` interior boundaries ``j * step``.
    Around each boundary the two neighbouring blocks cross-fade over a band of
    half-width ``h = max(2, step * overlap)`` voxels: with ``s`` the voxel
    centre's progress through the band (0 before it, 1 after it), the block
    above takes ``sin^2(pi s / 2)`` and the block below ``cos^2(pi s / 2)``,
    so the weights at every voxel sum to one."""
    if n_blocks <= 1:
        return np.ones((1, length)), float(length)
    step = length / float(n_blocks)
    h = max(2.0, step * overlap)
    centres = np.arange(length) + 0.5
    bounds = step * np.arange(1, n_blocks)
    s = np.clip((centres[None, :] - (bounds[:, None] - h)) / (2.0 * h), 0.0, 1.0)
    fade_in = np.sin(0.5 * np.pi * s) ** 2
    fade_out = np.cos(0.5 * np.pi * s) ** 2
    w = np.ones((n_blocks, length))
    w[1:] *= fade_in
    w[:-1] *= fade_out
    return w, step


def _make_pou_1d(length: int, n_blocks: int, overlap: float):
    """Raised-cosine partition-of-unity windows summing to 1, as a list of
    float32 tensors (cone_beam_fvr.py:42-61)."""
    w, step = _pou_windows(length, n_blocks, overlap)
    return [torch.from_numpy(row.astype(np.float32)) for row in w], float(step)


def _sinc2_precomp_1d(n: int, p: int) -> torch.Tensor:
    """1 / max(sinc^2, 0.05) trilinear pre-compensation window (cone_beam_fvr.py:64-68)."""
    c = (np.arange(n) - (n - 1) / 2.0) / float(p)
    s = np.sinc(c)
    return torch.from_numpy((1.0 / np.maximum(s ** 2, 0.05)).astype(np.float32))


def sample_isocenter_parity_offsets(vox_spacing) -> torch.Tensor:
    """27-point {-0.5, 0, 0.5}^3 voxel parity offsets scaled by the spacing (cone_beam_fvr.py:122-135)."""
    sp = torch.as_tensor(vox_spacing, dtype=torch.float32)
    if sp.ndim == 0:
        sp = sp.repeat(3)
    sp = sp.flatten()[:3]
    vals = (-0.5, 0.0, 0.5)
    grid = torch.tensor([[ix, iy, iz] for ix in vals for iy in vals for iz in vals], dtype=torch.float32,
                        device=sp.device)
    return grid * sp.unsqueeze(0)


class _EdgeNCCFn(torch.autograd.Function):
    """Edge-dominant gradient NCC on ``libfvr_b200.so``: one tiled Sobel +
    moment pass and a finalize forward; backward applies the transposed Sobel
    and box filters to the closed-form NCC gradient fields."""

    @staticmethod
    def forward(ctx, pred, target, crop, weight, mean):
        dev = L.require_cuda(pred)
        a = pred.detach().to(torch.float32).contiguous()
        b = target.detach().to(device=dev, dtype=torch.float32).contiguous()
        if a.dim() != 4 or b.dim() != 4 or b.shape[1:] != a.shape[1:] or b.shape[0] not in (1, a.shape[0]):
            raise ValueError(f"edge_dominant_ncc expects [B, C, H, W] inputs (target batch 1 or B), got "
                             f"{tuple(a.shape)} and {tuple(b.shape)}")
        B, C, H, W = (int(x) for x in a.shape)
        Bt = int(b.shape[0])
        ws_bytes = int(L.query("fvr_edge_ncc_workspace", B, C, H, W, crop))
        ws = torch.empty(max(ws_bytes, 8), dtype=torch.uint8, device=dev)
        stats = torch.empty((B * C, int(L.query("fvr_edge_ncc_stats_count"))), dtype=torch.float64, device=dev)
        out = torch.empty(1 if mean else B, dtype=torch.float32, device=dev)
        L.call("fvr_edge_ncc_forward", L.ptr(a), L.ptr(b), B, Bt, C, H, W, int(crop), float(weight), int(mean),
               L.ptr(ws), ws_bytes, L.ptr(stats), L.ptr(out), L.stream_ptr(dev))
        ctx.save_for_backward(a, b, stats)
        ctx.meta = (B, Bt, C, H, W, int(crop), float(weight), int(mean), pred.dtype, target.dtype)
        return out[0] if mean else out

    @staticmethod
    def backward(ctx, g):
        a, b, stats = ctx.saved_tensors
        B, Bt, C, H, W, crop, weight, mean, pdt, tdt = ctx.meta
        dev = a.device
        g = g.detach().to(device=dev, dtype=torch.float32).contiguous().reshape(-1)
        g_stride = 0 if mean else 1
        s = L.stream_ptr(dev)
        ga = gb = None
        if ctx.needs_input_grad[0]:
            ga = torch.empty_like(a)
            L.call("fvr_edge_ncc_backward", L.ptr(a), L.ptr(b), B, Bt, C, H, W, crop, weight, mean, L.ptr(stats),
                   L.ptr(g), g_stride, 0, L.ptr(ga), s)
            ga = ga.to(pdt)
        if ctx.needs_input_grad[1]:
            gb = torch.empty_like(a)
            L.call("fvr_edge_ncc_backward", L.ptr(a), L.ptr(b), B, Bt, C, H, W, crop, weight, mean, L.ptr(stats),
                   L.ptr(g), g_stride, 1, L.ptr(gb), s)
            gb = (gb.sum(0, keepdim=True) if Bt == 1 else gb).to(tdt)
        return ga, gb, None, None, None


def edge_dominant_ncc(pred, target, border_crop=None, multiscale_weight=0.25, reduction="mean"):
    """Edge-dominant gradient NCC of ``pred`` [B, C, H, W] against ``target``
    ([B or 1, C, H, W]): Sobel-x / Sobel-y NCC on the interior after a border
    crop of ``max(4, W // 8)`` pixels (W the last dim), averaged over
    directions and channels, plus ``multiscale_weight`` x the same on 3x3
    box-blurred images when the last dim is at least 96
    (cone_beam_fvr.py:71-112).  ``reduction`` 'mean' gives a scalar, anything
    else the per-item values [B]."""
    W = int(pred.shape[-1])
    crop = max(4, W // 8) if border_crop is None else int(border_crop)
    home = pred.device
    dev = RT.compute_device(pred, target)
    out = _EdgeNCCFn.apply(pred.to(dev), target.to(dev), crop, float(multiscale_weight), reduction == "mean")
    return out if out.device == home else out.to(home)


_LATTICE_CACHE: Dict[Tuple, Tuple] = {}


# A lattice is taken as separable (one ray coordinate per detector column and
# one per row) when its per-column rx and per-row ry spreads are within this
# fraction of the largest |rx| / |ry|: float rounding of rays that agree
# exactly, so a pixel's sampling position moves by about the rounding of the
# position arithmetic itself.
_SEPARABLE_REL = 2.0 ** -20


def _separable_rays(rx, ry):
    """(rxc [W], ryr [H]) midpoints of the per-column rx and per-row ry ranges
    of a lattice, or None when the rays do not separate (see _SEPARABLE_REL)."""
    if rx.ndim != 2 or rx.shape != ry.shape:
        return None
    cmax, cmin = rx.amax(0), rx.amin(0)
    rmax, rmin = ry.amax(1), ry.amin(1)
    sx = float((cmax - cmin).max()) / max(float(rx.abs().max()), 1e-30)
    sy = float((rmax - rmin).max()) / max(float(ry.abs().max()), 1e-30)
    if not (sx <= _SEPARABLE_REL and sy <= _SEPARABLE_REL):
        return None
    rxc = (0.5 * (cmax.double() + cmin.double())).float().contiguous()
    ryr = (0.5 * (rmax.double() + rmin.double())).float().contiguous()
    return rxc, ryr


def _prepared_lattice(lattice, device):
    """Device copies of an 11-tuple lattice's ray tables and its basis
    (src0, u0, v0, n0) as 12 host doubles, and its separable ray tables when
    it has them, cached per (storage, device): the lattice is a per-geometry
    constant, moved once.  The entry holds the lattice's own tensors, so their
    storage cannot be freed and reused by another lattice while the entry
    exists."""
    key = tuple(int(t.data_ptr()) for t in lattice[:8]) + (str(device),)
    hit = _LATTICE_CACHE.get(key)
    if hit is None:
        if len(_LATTICE_CACHE) > 64:
            _LATTICE_CACHE.clear()
        basis = torch.cat([lattice[i].reshape(3) for i in (0, 2, 3, 4)]).detach().double().cpu()
        base = (_ct.c_double * 12)(*[float(x) for x in basis])
        rays = tuple(t.detach().to(device=device, dtype=torch.float32).contiguous() for t in lattice[5:8])
        hit = (key, base, rays, tuple(lattice[:8]), _separable_rays(rays[0], rays[1]))
        _LATTICE_CACHE[key] = hit
    return hit


def _block_images(model, geo, N, s):
    """imgs [B, N, P, P] = Re fftshift(ifft2(ifftshift(slice))) for every block
    and pose (cone_beam_fvr.py:480-505): fused slice + inverse FFT in shared
    memory where P allows, else slice kernel + batched 2D IFFT."""
    dev = geo.device
    B, P = model.B, model.P
    st = model._stencil
    imgs = torch.empty((B, N, P, P), dtype=torch.float32, device=dev)
    if L.query("fvr_pou_image_supported", P):
        L.call("fvr_pou_slice_image", st.code, L.ptr(st.data), L.ptr(st.scales), B, P, L.ptr(geo), N,
               L.ptr(model._freqs), L.ptr(imgs), s)
        return imgs
    slices = torch.empty((B, N, P, P), dtype=torch.complex64, device=dev)
    L.call("fvr_pou_slice", st.code, L.ptr(st.data), L.ptr(st.scales), B, P, L.ptr(geo), N, L.ptr(model._freqs),
           L.ptr(slices), s)
    RT.fft2d(slices, inverse=True, out_shift=RT.SHIFT_FFT, scale=1.0 / (P * P), out_mode=RT.OUT_REAL, out=imgs,
             work=slices)
    return imgs


def _block_images_adjoint(model, geo, N, grad_imgs, s):
    """Slice-adjoint partials (workspace, tiles per (pose, block)) from dL/dimgs:
    fused FFT + slice adjoint where P allows, else batched 2D FFT + adjoint kernel."""
    dev = geo.device
    B, P = model.B, model.P
    st = model._stencil
    if L.query("fvr_pou_image_supported", P):
        wsb = L.query("fvr_pou_slice_image_adjoint_workspace", B, N)
        ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
        with profiling.section("pou_slice_adjoint"):
            L.call("fvr_pou_slice_image_adjoint", st.code, L.ptr(st.data), L.ptr(st.scales), B, P, L.ptr(geo), N,
                   L.ptr(model._freqs), L.ptr(grad_imgs), L.ptr(ws), wsb, s)
        return ws, 1
    # adjoint of S -> Re fftshift(ifft2(ifftshift(S))): fftshift(fft2(ifftshift(g))) / P^2
    G = RT.fft2d(grad_imgs, inverse=False, in_shift=RT.SHIFT_IFFT, out_shift=RT.SHIFT_FFT, scale=1.0 / (P * P))
    wsb = L.query("fvr_pou_slice_adjoint_workspace", B, P, N)
    ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
    L.call("fvr_pou_slice_adjoint", st.code, L.ptr(st.data), L.ptr(st.scales), B, P, L.ptr(geo), N,
           L.ptr(model._freqs), L.ptr(G), L.ptr(ws), wsb, s)
    return ws, (P * P + 255) // 256


class _PinholeFn(torch.autograd.Function):
    """SE(3)-invariant pinhole path (cone_beam_fvr.py:547-573, 670-686):
    mats -> pose geometry -> block slices -> batched IFFT -> warp-sum."""

    @staticmethod
    def forward(ctx, mats, model, rx, ry, ic, base_key):
        dev = model._dev
        m = mats.detach().to(device=dev, dtype=torch.float32).contiguous()
        N = int(m.shape[0])
        B, P = model.B, model.P
        base = _LATTICE_CACHE[base_key][1]
        geo = torch.empty((N, int(L.query("fvr_pou_geo_stride"))), dtype=torch.float64, device=dev)
        offs = torch.empty((B, N, 3), dtype=torch.float64, device=dev)
        s = L.stream_ptr(dev)
        vscale = float(P) * model.ds_block
        L.call("fvr_pou_pose", L.ptr(m), None, N, base, vscale, L.ptr(model.centers), B, L.ptr(geo), L.ptr(offs), s)
        with profiling.section("pou_slice"):
            imgs = _block_images(model, geo, N, s)
        H, W = int(rx.shape[0]), int(rx.shape[1])
        out = torch.empty((N, 1, H, W), dtype=torch.float32, device=dev)
        with profiling.section("pou_warp"):
            L.call("fvr_pou_warp", L.ptr(imgs), B, N, P, L.ptr(offs), _ct.c_void_p(offs.data_ptr() + 8),
                   _ct.c_void_p(offs.data_ptr() + 16), 1, 3, L.ptr(rx), L.ptr(ry), L.ptr(ic), H * W, 0,
                   1.0 / model.ds_block, float(P // 2), L.ptr(out), s)
        ctx.save_for_backward(geo, offs, imgs, rx, ry, ic)
        ctx.meta = (model, base, mats.dtype, _LATTICE_CACHE[base_key][4])
        return out

    @staticmethod
    def backward(ctx, g_out):
        geo, offs, imgs, rx, ry, ic = ctx.saved_tensors
        model, base, mdt, sep = ctx.meta
        dev = geo.device
        B, N, P = model.B, int(geo.shape[0]), model.P
        H, W = int(rx.shape[0]), int(rx.shape[1])
        s = L.stream_ptr(dev)
        g = g_out.detach().to(device=dev, dtype=torch.float32).contiguous()
        goffs = torch.empty((3, B, N), dtype=torch.float64, device=dev)
        if (sep is not None and model.fused_warp_adjoint and g.data_ptr() % 16 == 0 and ic.data_ptr() % 16 == 0
                and L.query("fvr_pou_warp_image_adjoint_supported", P, H, W)):
            # warp adjoint + block-image adjoint in one launch: dL/dimgs stays in shared memory
            st = model._stencil
            wsb = L.query("fvr_pou_slice_image_adjoint_workspace", B, N)
            ws2 = torch.empty(wsb, dtype=torch.uint8, device=dev)
            with profiling.section("pou_slice_adjoint"):
                L.call("fvr_pou_warp_image_adjoint", st.code, L.ptr(st.data), L.ptr(st.scales), B, P, L.ptr(geo), N,
                       L.ptr(model._freqs), L.ptr(imgs), L.ptr(offs), L.ptr(sep[0]), L.ptr(sep[1]), L.ptr(ic), L.ptr(g),
                       H, W, 1.0 / model.ds_block, float(P // 2), L.ptr(goffs), L.ptr(ws2), wsb, s)
            tiles = 1
        else:
            grad_imgs = torch.zeros((B, N, P, P), dtype=torch.float32, device=dev)
            wsb = L.query("fvr_pou_warp_bwd_workspace", B, N, H * W)
            ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
            with profiling.section("pou_warp_bwd"):
                L.call("fvr_pou_warp_bwd", L.ptr(imgs), B, N, P, L.ptr(offs), _ct.c_void_p(offs.data_ptr() + 8),
                       _ct.c_void_p(offs.data_ptr() + 16), 1, 3, L.ptr(rx), L.ptr(ry), L.ptr(ic), H * W, 0,
                       1.0 / model.ds_block, float(P // 2), L.ptr(g), L.ptr(grad_imgs), L.ptr(goffs), None,
                       L.ptr(ws), wsb, s)
            ws2, tiles = _block_images_adjoint(model, geo, N, grad_imgs, s)
            del grad_imgs
        gm = torch.empty((N, 4, 4), dtype=torch.float32, device=dev)
        L.call("fvr_pou_pose_backward", L.ptr(ws2), tiles, L.ptr(goffs), None, 0, L.ptr(geo), L.ptr(model.centers), B,
               N, base, float(P) * model.ds_block, L.ptr(gm), None, s)
        return gm.to(mdt), None, None, None, None, None


class PerspectiveSlabFVR(nn.Module):
    """Differentiable partition-of-unity cone-beam Fourier volume renderer
    (src/fvr/cone_beam_fvr.py:138-832).  ``use_triton`` is accepted and ignored;
    ``device`` defaults to the current CUDA device."""

    SLAB_PRESETS = SLAB_PRESETS

    @classmethod
    def resolve_slab_preset(cls, preset, grid_blocks=None, block_res=None, dtype=None):
        if preset is not None:
            if preset not in cls.SLAB_PRESETS:
                raise ValueError(f"Unknown slab preset {preset!r}; expected one of {tuple(cls.SLAB_PRESETS)}")
            cfg = cls.SLAB_PRESETS[preset]
            gb = grid_blocks if grid_blocks is not None else tuple(cfg["grid_blocks"])
            br = int(block_res if block_res is not None else cfg["block_res"])
            dt = dtype if dtype is not None else cfg["dtype"]
            return gb, br, dt
        return (grid_blocks if grid_blocks is not None else (2, 2, 2), int(block_res if block_res is not None else 64),
                dtype if dtype is not None else torch.float32)

    def __init__(self, vol_3d, vox_mm=1.0, origin_world_mm=(0.0, 0.0, 0.0), axis_signs=(1.0, 1.0, 1.0),
                 grid_blocks=(2, 2, 2), block_res=80, pad_mult=2, overlap=0.25, energy_thresh=1e-4,
                 dtype=torch.float32, use_triton=True, device=None):
        super().__init__()
        self.use_triton = bool(use_triton)
        # pinhole adjoint: warp + block-image adjoint in one launch on separable lattices
        self.fused_warp_adjoint = True
        self._compiled_project_core = None
        self._compiled_project_invariant = None
        vol = torch.as_tensor(vol_3d).detach().float()
        if vol.ndim != 3:
            raise ValueError(f"Expected 3D volume tensor, got shape {tuple(vol.shape)}")
        if device is None and vol.is_cuda:
            device = vol.device
        self._dev = RT.device_of(device)
        n0, n1, n2 = (int(s) for s in vol.shape)
        if isinstance(vox_mm, (tuple, list)):
            sp = tuple(float(x) for x in vox_mm)
            if not (abs(sp[0] - sp[1]) < 1e-3 and abs(sp[1] - sp[2]) < 1e-3):
                raise ValueError(f"Volume spacing must be isotropic (got {sp})")
            self.vox_mm = sp[0]
        else:
            self.vox_mm = float(vox_mm)
        self.block_res = int(block_res)
        self.pad_mult = int(pad_mult)
        self.P = self.block_res * self.pad_mult
        ks = tuple(int(k) for k in grid_blocks)
        wl, steps = zip(*[_pou_windows(n, k, overlap) for n, k in zip((n0, n1, n2), ks)])
        ov = [max(2, int(round(s * overlap))) if k > 1 else 0 for s, k in zip(steps, ks)]
        M = max(int(np.ceil(s + 2 * o)) for s, o in zip(steps, ov)) + (1 if max(ks) > 1 else 0)
        self.M = M
        self.ds_block = (M * self.vox_mm) / float(self.block_res)
        pad_b = (self.P - self.block_res) // 2
        half_vox_mm = ((self.P // 2) - (pad_b + (self.block_res - 1) * 0.5)) * self.ds_block
        dev = self._dev
        # 1D windows (float32, as the reference builds them) and their supports
        wt, st = [], []
        for ws in wl:
            w32 = np.stack([w.astype(np.float32) for w in ws])
            sup = []
            for w in ws:
                nz = np.nonzero(w.astype(np.float32) > 1e-6)[0]
                sup.append([int(nz[0]), int(nz[-1]) + 1 - int(nz[0])])
            wt.append(torch.from_numpy(w32).to(dev))
            st.append(torch.tensor(sup, dtype=torch.int32, device=dev))
        v = vol.to(dev).contiguous()
        s = L.stream_ptr(dev)
        kk = ks[0] * ks[1] * ks[2]
        sums = torch.empty(kk, dtype=torch.float64, device=dev)
        axes_args = []
        for d in range(3):
            axes_args += [L.ptr(wt[d]), L.ptr(st[d]), ks[d]]
        L.call("fvr_pou_block_sums", L.ptr(v), n0, n1, n2, *axes_args, L.ptr(sums), s)
        sums_h = sums.cpu().numpy()
        active = [i for i in range(kk) if float(sums_h[i]) > energy_thresh]
        if not active:
            raise ValueError("Input volume contains no non-zero attenuation mass above threshold.")
        self.B = len(active)
        sup_h = [t.cpu().numpy() for t in st]
        centers = []
        for kb in active:
            ib = (kb // (ks[1] * ks[2]), (kb // ks[2]) % ks[1], kb % ks[2])
            c = []
            for d in range(3):
                a, ln = int(sup_h[d][ib[d]][0]), int(sup_h[d][ib[d]][1])
                m = (M - ln) // 2
                cidx = a + (M - 1) * 0.5 - m
                c.append(origin_world_mm[d] + axis_signs[d] * cidx * self.vox_mm + axis_signs[d] * half_vox_mm)
            centers.append(c)
        blocks_t = torch.tensor(active, dtype=torch.int32, device=dev)
        w3 = _sinc2_precomp_1d(self.block_res, self.P).to(dev)
        real = torch.empty((self.B, self.P, self.P, self.P), dtype=torch.float32, device=dev)
        L.call("fvr_pou_build_blocks", L.ptr(v), n0, n1, n2, *axes_args, L.ptr(blocks_t), self.B, L.ptr(w3), M,
               self.block_res, self.P, float(self.ds_block), L.ptr(real), s)
        spec = RT.spectrum3d(real, (self.P,) * 3, 2, batch_first=True)
        del real
        F_ri = torch.view_as_real(spec).permute(0, 4, 1, 2, 3).contiguous()
        del spec
        # the stencil comes from the float32 spectra (f16 storage takes its brick scales from them)
        self._stencil = RT.Stencil(F_ri, True, (self.P,) * 3, self._stencil_dtype(dtype), items=self.B)
        self.register_buffer("F_blk_ri", F_ri.to(dtype=dtype))
        del F_ri
        self.register_buffer("centers", torch.tensor(centers, dtype=torch.float32, device=dev))
        freqs = torch.from_numpy(np.fft.fftshift(np.fft.fftfreq(self.P, d=self.ds_block)).astype(np.float32)).to(dev)
        fy, fx = torch.meshgrid(freqs, freqs, indexing="ij")
        self.register_buffer("FX", fx)
        self.register_buffer("FY", fy)
        self.register_buffer("FX_flat", fx.reshape(-1).contiguous())
        self.register_buffer("FY_flat", fy.reshape(-1).contiguous())
        self._freqs = freqs.contiguous()

    @staticmethod
    def _stencil_dtype(dtype):
        if dtype in (torch.float32, torch.bfloat16, torch.float16):
            return dtype
        if dtype == torch.float64:
            return torch.float32
        raise L.FvrError(f"unsupported spectrum dtype {dtype}")

    def to_precision(self, dtype):
        """Cast the block spectra (cone_beam_fvr.py:305-313); f16 storage is brick-scaled."""
        self._stencil = RT.Stencil(self.F_blk_ri, True, (self.P,) * 3, self._stencil_dtype(dtype), items=self.B)
        self.F_blk_ri = self.F_blk_ri.to(dtype=dtype)
        return self

    def compile_renderer(self, mode="reduce-overhead", fullgraph=False):
        """Accepted for compatibility (cone_beam_fvr.py:315-329); use fvr.graphs for graph capture."""
        return self

    @classmethod
    def from_volume(cls, vol_zyx, vox_mm=1.0, grid_blocks=None, block_res=None, pad_mult=2, overlap=0.25,
                    center_mode="pixel_center", preset=None, dtype=None, **kwargs):
        """Isotropic (Z, Y, X) volume constructor (cone_beam_fvr.py:331-376)."""
        gb, br, dt = cls.resolve_slab_preset(preset, grid_blocks, block_res, dtype)
        vt = torch.as_tensor(np.asarray(vol_zyx) if not isinstance(vol_zyx, torch.Tensor) else vol_zyx,
                             dtype=torch.float32)
        nz, ny, nx = vt.shape
        v = float(vox_mm)
        if center_mode == "pixel_center":
            origin = (-0.5 * (nz - 1) * v, -0.5 * (ny - 1) * v, -0.5 * (nx - 1) * v)
        elif center_mode == "grid_center":
            origin = (-0.5 * nz * v, -0.5 * ny * v, -0.5 * nx * v)
        else:
            raise ValueError(f"Unknown center_mode={center_mode!r}; expected 'pixel_center' or 'grid_center'")
        return cls(vt, vox_mm=v, origin_world_mm=origin, axis_signs=(1.0, 1.0, 1.0), grid_blocks=gb, block_res=br,
                   pad_mult=pad_mult, overlap=overlap, dtype=dt, **kwargs)

    @classmethod
    def from_diffdrr_subject(cls, subject, grid_blocks=None, block_res=None, pad_mult=2, overlap=0.25, preset=None,
                             dtype=None, **kwargs):
        """DiffDRR-subject constructor (cone_beam_fvr.py:378-421): world RAS geometry from
        ``subject.density.data`` / ``.affine``."""
        gb, br, dt = cls.resolve_slab_preset(preset, grid_blocks if grid_blocks is not None or preset is not None
                                             else (2, 2, 2),
                                             block_res if block_res is not None or preset is not None else 80, dtype)
        vol_world = subject.density.data.squeeze(0).float().flip(0, 1)
        nx, ny, nz = vol_world.shape
        aff = subject.density.affine
        sx, sy, sz = abs(float(aff[0, 0])), abs(float(aff[1, 1])), abs(float(aff[2, 2]))
        origin = (-(nx - 1) * sx + float(aff[0, 3]), -(ny - 1) * sy + float(aff[1, 3]), float(aff[2, 3]))
        return cls(vol_world, vox_mm=(sx, sy, sz), origin_world_mm=origin, axis_signs=(1.0, 1.0, 1.0),
                   grid_blocks=gb, block_res=br, pad_mult=pad_mult, overlap=overlap, energy_thresh=1e-3, dtype=dt,
                   **kwargs)

    # ----------------------------------------------------------------- geometry

    @staticmethod
    def _extract_detector_basis(srcs, trg_pts, u_det=None, v_det=None, n_0=None):
        """Unit detector axes ``(N, 3)`` of explicit lattices ``trg_pts (N, H, W, 3)``
        (cone_beam_fvr.py:575-596): u along each lattice's first row, v along its
        first column, n the unit ``v x u`` turned to face away from the source
        (towards the lattice's centroid).  Axes that are given are kept;
        differentiable in the lattice and the sources."""
        first = trg_pts[:, 0, 0]
        edges = torch.stack([trg_pts[:, 0, -1] - first, trg_pts[:, -1, 0] - first], dim=1)
        edges = edges / (edges.norm(dim=-1, keepdim=True) + 1e-12)
        u = edges[:, 0] if u_det is None else u_det
        v = edges[:, 1] if v_det is None else v_det
        if n_0 is None:
            normal = torch.linalg.cross(v, u, dim=-1)
            normal = normal / (normal.norm(dim=-1, keepdim=True) + 1e-12)
            facing = ((trg_pts.mean(dim=(1, 2)) - srcs) * normal).sum(dim=-1, keepdim=True)
            n_0 = torch.where(facing < 0, -normal, normal)
        return u, v, n_0

    @staticmethod
    def make_pinhole_lattice(k_inv, sdd_mm, height, width):
        """Camera-frame pinhole lattice and SE(3)-invariant ray cache as the
        reference's 11-tuple ``(src0, trg0, u0, v0, n0, rx_hw, ry_hw, ic_hw,
        rx_flat, ry_flat, ic_flat)`` (cone_beam_fvr.py:705-728), formed in FP64
        by ``fvr_pou_pinhole_lattice`` and stored as float32 on ``k_inv``'s
        device (pixel centres at +1/2, source at the camera origin)."""
        k0 = k_inv.squeeze(0) if k_inv.ndim == 3 else k_inv
        home = k0.device
        dev = RT.device_of(home if home.type == "cuda" else None)
        H, W = int(height), int(width)
        kk = (_ct.c_double * 9)(*[float(x) for x in k0.detach().double().cpu().reshape(9)])
        trg0 = torch.empty((H, W, 3), dtype=torch.float32, device=dev)
        rays = torch.empty((3, H, W), dtype=torch.float32, device=dev)
        basis = torch.empty(9, dtype=torch.float64, device=dev)
        L.call("fvr_pou_pinhole_lattice", kk, float(sdd_mm), H, W, L.ptr(trg0), L.ptr(rays[0]), L.ptr(rays[1]),
               L.ptr(rays[2]), L.ptr(basis), L.stream_ptr(dev))
        trg0, rays, basis = trg0.to(home), rays.to(home), basis.float().to(home)
        rx, ry, ic = rays[0], rays[1], rays[2]
        src0 = torch.zeros(3, dtype=torch.float32, device=home)
        return (src0, trg0, basis[0:3], basis[3:6], basis[6:9], rx, ry, ic, rx.reshape(-1), ry.reshape(-1),
                ic.reshape(-1))

    # ---------------------------------------------------------------- rendering

    def _forward_from_lattice(self, pose_mats, lattice):
        """Camera-frame lattice moved by pose matrices (cone_beam_fvr.py:670-688)."""
        home = pose_mats.device
        if pose_mats.shape[0] == 0:  # no poses: an empty batch of images
            H, W = int(lattice[1].shape[0]), int(lattice[1].shape[1])
            return torch.zeros((0, 1, H, W), dtype=torch.float32, device=home) + 0.0 * pose_mats.sum()
        if len(lattice) >= 11:
            key, _, (rx, ry, ic), _, _ = _prepared_lattice(lattice, self._dev)
            mats = pose_mats if home == self._dev else pose_mats.to(self._dev)
            out = _PinholeFn.apply(mats, self, rx, ry, ic, key)
        else:
            out = self._forward_explicit(pose_mats, lattice)
        return out if out.device == home else out.to(home)

    def _forward_explicit(self, pose_mats, lattice):
        from .cone_beam_rays import forward_explicit

        return forward_explicit(self, pose_mats, lattice)

    def forward_pinhole(self, rt_inv, lattice):
        """Batched pinhole projection ``(N, 1, H, W)`` from pose matrices ``(N, 4, 4)``
        (cone_beam_fvr.py:730-740)."""
        return self._forward_from_lattice(rt_inv, lattice)

    def warmup_pinhole(self, lattice, batch_size=1, backward=True):
        """Run one forward (and backward) so later calls are free of first-use costs
        (cone_beam_fvr.py:742-759)."""
        eye = torch.eye(4, device=self._dev, dtype=torch.float32).unsqueeze(0).repeat(max(1, int(batch_size)), 1, 1)
        if backward:
            eye = eye.requires_grad_(True)
            self.forward_pinhole(eye, lattice).sum().backward()
        else:
            with torch.no_grad():
                self.forward_pinhole(eye, lattice)
        torch.cuda.synchronize(self._dev)

    def project_rays_batched(self, srcs, trg_pts, u_det=None, v_det=None, n_0=None):
        """Cone-beam line integrals for explicit sources ``(N, 3)`` and detector
        lattices ``(N, H, W, 3)`` (cone_beam_fvr.py:598-612)."""
        from .cone_beam_rays import project_rays_batched

        home, dev = trg_pts.device, self._dev
        srcs, trg_pts = srcs.to(dev), trg_pts.to(dev)
        u_det, v_det, n_0 = (None if a is None else a.to(dev) for a in (u_det, v_det, n_0))
        u_det, v_det, n_0 = self._extract_detector_basis(srcs, trg_pts, u_det, v_det, n_0)
        out = project_rays_batched(self, srcs, trg_pts, u_det, v_det, n_0)
        return out if out.device == home else out.to(home)

    def project_rays(self, src, trg_pts, u_det=None, v_det=None, n_0=None):
        """Single-pose form of :meth:`project_rays_batched` (cone_beam_fvr.py:614-632)."""
        return self.project_rays_batched(
            src.unsqueeze(0), trg_pts.unsqueeze(0), None if u_det is None else u_det.unsqueeze(0),
            None if v_det is None else v_det.unsqueeze(0), None if n_0 is None else n_0.unsqueeze(0)).squeeze(0)

    # Detector frames of the two C-arm views in the volume's (z, y, x) axes:
    # (u0, v0, n0) = detector columns, detector rows, beam direction.  The
    # source sits at -SAD along n0 and the detector plane at SDD - SAD.
    _CARM_AXES = {"ap": ((0.0, 0.0, 1.0), (1.0, 0.0, 0.0), (0.0, 1.0, 0.0)),
                  "lateral": ((0.0, 1.0, 0.0), (1.0, 0.0, 0.0), (0.0, 0.0, 1.0))}

    @staticmethod
    def _axis_rotation(angle_rad, axis):
        """Rotation by ``angle_rad`` (0-d tensor) about coordinate axis ``axis``
        (differentiable): the plane of the two following axes turns."""
        i, j = (axis + 1) % 3, (axis + 2) % 3
        c, s = torch.cos(angle_rad), torch.sin(angle_rad)
        one, zero = torch.ones_like(c), torch.zeros_like(c)
        rows = [[one if r == k else zero for k in range(3)] for r in range(3)]
        rows[i][i], rows[i][j], rows[j][i], rows[j][j] = c, -s, s, c
        return torch.stack([torch.stack(r) for r in rows])

    def forward_carm_view(self, yaw_deg, pitch_deg, roll_deg, tx_vox, ty_vox, tz_vox, sad_mm, sdd_mm, det_px,
                          det_fov_mm, view="ap"):
        """C-arm AP / lateral projection ``(det_px, det_px)`` (cone_beam_fvr.py:761-832).

        The pose turns the C-arm about the volume's z axis by yaw, then its y
        axis by roll, then its x axis by pitch (``R = R_z R_y R_x`` on (z, y, x)
        coordinates, degrees) and shifts it by ``-(tz, ty, tx)`` voxels.
        Detector pixels span ``det_fov_mm`` on a ``det_px``-point grid from
        edge to edge.  Rendered by the explicit-ray path; differentiable in
        the six pose scalars, returned on their device."""
        home = torch.as_tensor(yaw_deg).device
        dev = self._dev
        ang = [torch.deg2rad(torch.as_tensor(a, dtype=torch.float32).to(dev)) for a in (yaw_deg, roll_deg, pitch_deg)]
        rot = (self._axis_rotation(ang[0], 0) @ self._axis_rotation(ang[1], 1)) @ self._axis_rotation(ang[2], 2)
        shift = torch.stack([torch.as_tensor(t, dtype=torch.float32).to(dev) for t in (tz_vox, ty_vox, tx_vox)])
        shift = shift * self.vox_mm
        axes = self._CARM_AXES["ap" if view == "ap" else "lateral"]
        u0, v0, n0 = (torch.tensor(a, dtype=torch.float32, device=dev) for a in axes)
        grid = torch.linspace(-0.5, 0.5, int(det_px), device=dev) * float(det_fov_mm)
        plane = float(sdd_mm - sad_mm) * n0
        trg0 = grid[:, None, None] * v0 + grid[None, :, None] * u0 + plane
        src = rot @ (-float(sad_mm) * n0) - shift
        trg_pts = trg0 @ rot.T - shift
        img = self.project_rays(src, trg_pts, u_det=rot @ u0, v_det=rot @ v0, n_0=rot @ n0)
        return img if img.device == home else img.to(home)

    def cache_diffdrr_geometry(self, drr_mod, out_res):
        raise ImportError("cache_diffdrr_geometry needs the third-party diffdrr package, which this build does "
                          "not depend on; build the lattice with make_pinhole_lattice instead")

    def forward_diffdrr_batched(self, drr_mod, pose_mats, out_res):
        return self._forward_from_lattice(pose_mats, self.cache_diffdrr_geometry(drr_mod, out_res))

    def forward_diffdrr(self, drr_mod, pose, out_res):
        mat = pose.matrix
        if mat.ndim == 2:
            mat = mat.unsqueeze(0)
        return self.forward_diffdrr_batched(drr_mod, mat, out_res)
