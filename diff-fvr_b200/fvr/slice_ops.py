"""Trilinear Fourier-slice gather and PoU pinhole warp-sum (drop-in for the
public functions of src/fvr/triton_slice.py), computed by libfvr_b200.so.

``fourier_slice_3d(vol_ri, u_xyz, v_xyz, fx, fy, center_xyz)`` returns
``(B_vol, N_pose, 2, K)`` in the volume dtype with zero-padding partial
interpolation, differentiable in ``u_xyz`` and ``v_xyz`` (the reference never
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
    return _Slice3DFn.apply(vol_ri, u_xyz, v_xyz, fx, fy, cx, cy, cz)


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
