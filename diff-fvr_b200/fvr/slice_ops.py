"""Trilinear Fourier-slice gather and PoU pinhole warp-sum (drop-in for the
public functions of src/fvr/triton_slice.py), computed by libfvr_b200.so.

``fourier_slice_3d(vol_ri, u_xyz, v_xyz, fx, fy, center_xyz)`` returns
``(B_vol, N_pose, 2, K)`` in the volume dtype with zero-padding partial
interpolation on the volume's device (CPU inputs are computed on the current
CUDA device and copied back), differentiable in ``u_xyz`` and ``v_xyz`` (the reference never
returns a volume gradient from its fused path, triton_slice.py:339; a volume
that requires grad raises here instead of silently routing elsewhere).

The reference also exports ``fourier_slice_3d_torch`` (grid_sample) and
``trilinear_slice_analytical_ref`` (explicit stencil) as CPU references.  The
names are kept for API compatibility and run the same CUDA gather; the
independent CPU checker of this project lives in ``oracle/`` and is never
imported by the product.
"""
from __future__ import annotations

from typing import Tuple

import torch

from . import _lib as L
from . import _runtime as RT


class _Slice3DFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vol_ri, u_xyz, v_xyz, fx, fy, cx, cy, cz):
        dev = L.require_cuda(vol_ri)
        vol = vol_ri.detach().contiguous()
        B, _, D, H, W = (int(s) for s in vol.shape)
        u = u_xyz.detach().to(dev, torch.float32).contiguous()
        v = v_xyz.detach().to(dev, torch.float32).contiguous()
        fxc = fx.detach().to(dev, torch.float32).contiguous()
        fyc = fy.detach().to(dev, torch.float32).contiguous()
        N, K = int(u.shape[0]), int(fxc.numel())
        out = torch.empty((B, N, 2, K), dtype=vol.dtype, device=dev)
        L.call("fvr_slice3d_fwd", L.ptr(vol), L.dtype_code(vol.dtype), B, D, H, W, L.ptr(u), L.ptr(v), N, L.ptr(fxc),
               L.ptr(fyc), K, float(cx), float(cy), float(cz), L.ptr(out), L.stream_ptr(dev))
        ctx.save_for_backward(vol, u, v, fxc, fyc)
        ctx.meta = (float(cx), float(cy), float(cz), u_xyz.dtype, v_xyz.dtype)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        vol, u, v, fxc, fyc = ctx.saved_tensors
        cx, cy, cz, udt, vdt = ctx.meta
        dev = vol.device
        B, _, D, H, W = (int(s) for s in vol.shape)
        N, K = int(u.shape[0]), int(fxc.numel())
        go = grad_out.detach().to(dtype=vol.dtype).contiguous()
        gu = torch.empty((N, 3), dtype=torch.float32, device=dev)
        gv = torch.empty((N, 3), dtype=torch.float32, device=dev)
        ws_bytes = L.query("fvr_slice3d_bwd_workspace", N, K)
        ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
        L.call("fvr_slice3d_bwd", L.ptr(vol), L.dtype_code(vol.dtype), B, D, H, W, L.ptr(go), L.ptr(u), L.ptr(v), N,
               L.ptr(fxc), L.ptr(fyc), K, cx, cy, cz, L.ptr(gu), L.ptr(gv), L.ptr(ws), ws_bytes, L.stream_ptr(dev))
        return None, gu.to(udt), gv.to(vdt), None, None, None, None, None


def fourier_slice_3d(
    vol_ri: torch.Tensor,
    u_xyz: torch.Tensor,
    v_xyz: torch.Tensor,
    fx: torch.Tensor,
    fy: torch.Tensor,
    center_xyz: Tuple[float, float, float],
    use_triton: bool = True,
) -> torch.Tensor:
    """3D Fourier slice ``(B_vol, N_pose, 2, K)`` at ``p = c + fx*u + fy*v``
    (src/fvr/triton_slice.py:648-661).  ``use_triton`` is accepted and ignored."""
    if vol_ri.requires_grad:
        raise L.FvrError("fourier_slice_3d: gradients with respect to the volume are not provided "
                         "(the reference's fused path does not return them either)")
    cx, cy, cz = center_xyz
    home = vol_ri.device
    dev = RT.compute_device(vol_ri, u_xyz, v_xyz)
    out = _Slice3DFn.apply(vol_ri.to(dev), u_xyz.to(dev), v_xyz.to(dev), fx.to(dev), fy.to(dev), cx, cy, cz)
    return out if out.device == home else out.to(home)


def fourier_slice_3d_torch(vol_ri, u_xyz, v_xyz, fx, fy, center_xyz):
    """API-compatible name for triton_slice.py:594-645; runs the CUDA gather."""
    return fourier_slice_3d(vol_ri, u_xyz, v_xyz, fx, fy, center_xyz)


def trilinear_slice_analytical_ref(vol_ri, u_xyz, v_xyz, fx, fy, center_xyz):
    """API-compatible name for triton_slice.py:664-715; runs the CUDA gather."""
    return fourier_slice_3d(vol_ri, u_xyz, v_xyz, fx, fy, center_xyz)


def triton_slice_available(tensor: torch.Tensor) -> bool:
    """Reference name (triton_slice.py:30-32): True when the fused CUDA path can run."""
    try:
        L.load()
    except L.FvrError:
        return False
    return bool(tensor.is_cuda)


HAS_TRITON = False


class _WarpSumFn(torch.autograd.Function):
    """PoU pinhole warp + obliquity sum (triton_slice.py:498-591)."""

    @staticmethod
    def forward(ctx, imgs, d_b, cu, cv, rx, ry, ic, inv_ds, c_idx):
        dev = L.require_cuda(imgs)
        im = imgs.detach().float().contiguous()
        B, N, P, _ = (int(x) for x in im.shape)
        offs = [x.detach().to(dev, torch.float64).contiguous() for x in (d_b, cu, cv)]
        r = [x.detach().to(dev, torch.float32).reshape(-1).contiguous() for x in (rx, ry, ic)]
        K = int(r[0].numel())
        out = torch.empty((N, K), dtype=torch.float32, device=dev)
        L.call("fvr_pou_warp", L.ptr(im), B, N, P, L.ptr(offs[0]), L.ptr(offs[1]), L.ptr(offs[2]), 1, 1, L.ptr(r[0]),
               L.ptr(r[1]), L.ptr(r[2]), K, 0, float(inv_ds), float(c_idx), L.ptr(out), L.stream_ptr(dev))
        ctx.save_for_backward(im, *offs, *r)
        ctx.meta = (float(inv_ds), float(c_idx), imgs.dtype, d_b.dtype)
        return out

    @staticmethod
    def backward(ctx, g_out):
        im, db, cu, cv, rx, ry, ic = ctx.saved_tensors
        inv_ds, c_idx, idt, odt = ctx.meta
        dev = im.device
        B, N, P, _ = (int(x) for x in im.shape)
        K = int(rx.numel())
        g = g_out.detach().to(dev, torch.float32).reshape(N, K).contiguous()
        gi = torch.zeros_like(im) if ctx.needs_input_grad[0] else None
        goffs = torch.empty((3, B, N), dtype=torch.float64, device=dev)
        wsb = L.query("fvr_pou_warp_bwd_workspace", B, N, K)
        ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
        L.call("fvr_pou_warp_bwd", L.ptr(im), B, N, P, L.ptr(db), L.ptr(cu), L.ptr(cv), 1, 1, L.ptr(rx), L.ptr(ry),
               L.ptr(ic), K, 0, inv_ds, c_idx, L.ptr(g), L.ptr(gi), L.ptr(goffs), None, L.ptr(ws), wsb,
               L.stream_ptr(dev))
        return (None if gi is None else gi.to(idt), goffs[0].to(odt), goffs[1].to(odt), goffs[2].to(odt), None, None,
                None, None, None)


def pou_pinhole_warp_sum(imgs, d_b, cu, cv, rx_hw, ry_hw, inv_cos_hw, rx_flat, ry_flat, ic_flat, inv_ds, c_idx,
                         use_triton: bool = True):
    """Batched PoU pinhole bilinear warp + obliquity sum ``(N, H, W)``
    (triton_slice.py:787-808); differentiable in imgs, d_b, cu, cv."""
    H, W = int(rx_hw.shape[0]), int(rx_hw.shape[1])
    home = imgs.device
    dev = RT.compute_device(imgs, d_b, cu, cv)
    out = _WarpSumFn.apply(imgs.to(dev), d_b.to(dev), cu.to(dev), cv.to(dev), rx_flat.to(dev), ry_flat.to(dev),
                           ic_flat.to(dev), inv_ds, c_idx)
    out = out.view(out.shape[0], H, W)
    return out if out.device == home else out.to(home)


def pou_pinhole_warp_sum_torch(imgs, d_b, cu, cv, rx_hw, ry_hw, inv_cos_hw, inv_ds, c_idx):
    """API-compatible name for triton_slice.py:718-745; runs the CUDA warp."""
    return pou_pinhole_warp_sum(imgs, d_b, cu, cv, rx_hw, ry_hw, inv_cos_hw, rx_hw.reshape(-1), ry_hw.reshape(-1),
                                inv_cos_hw.reshape(-1), inv_ds, c_idx)


def pou_pinhole_warp_sum_analytical_ref(imgs, d_b, cu, cv, rx_hw, ry_hw, inv_cos_hw, inv_ds, c_idx):
    """API-compatible name for triton_slice.py:748-784; runs the CUDA warp."""
    return pou_pinhole_warp_sum_torch(imgs, d_b, cu, cv, rx_hw, ry_hw, inv_cos_hw, inv_ds, c_idx)
