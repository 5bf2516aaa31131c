"""Explicit-ray PoU-FVR renderer (``_project_core``, src/fvr/cone_beam_fvr.py:423-478):
per-pose detector lattices ``trg_pts (N, H, W, 3)`` with sources ``(N, 3)``
and detector axes, differentiable in all of them.  Used by
``project_rays(_batched)``, ``forward_carm_view`` and 5-tuple lattices."""
from __future__ import annotations

import ctypes as _ct

import torch

from . import _lib as L


class _RaysFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, srcs, trg, u_det, v_det, n_0, model):
        dev = model._dev
        f32 = dict(device=dev, dtype=torch.float32)
        N, H, W, _ = (int(x) for x in trg.shape)
        K = H * W
        B, P = model.B, model.P
        vecs = torch.cat([srcs.detach().to(**f32).reshape(N, 3), u_det.detach().to(**f32).reshape(N, 3),
                          v_det.detach().to(**f32).reshape(N, 3), n_0.detach().to(**f32).reshape(N, 3)], 1)
        vecs = vecs.contiguous()
        t = trg.detach().to(**f32).contiguous()
        s = L.stream_ptr(dev)
        vscale = float(P) * model.ds_block
        geo = torch.empty((N, int(L.query("fvr_pou_geo_stride"))), dtype=torch.float64, device=dev)
        offs = torch.empty((B, N, 3), dtype=torch.float64, device=dev)
        L.call("fvr_pou_pose", None, L.ptr(vecs), N, None, vscale, L.ptr(model.centers), B, L.ptr(geo), L.ptr(offs),
               s)
        rx = torch.empty((N, K), **f32)
        ry = torch.empty((N, K), **f32)
        ic = torch.empty((N, K), **f32)
        L.call("fvr_pou_rays_prep", L.ptr(t), L.ptr(geo), N, K, L.ptr(rx), L.ptr(ry), L.ptr(ic), s)
        from .cone_beam_fvr import _block_images

        imgs = _block_images(model, geo, N, s)
        out = torch.empty((N, H, W), **f32)
        L.call("fvr_pou_warp", L.ptr(imgs), B, N, P, L.ptr(offs), _ct.c_void_p(offs.data_ptr() + 8),
               _ct.c_void_p(offs.data_ptr() + 16), 1, 3, L.ptr(rx), L.ptr(ry), L.ptr(ic), K, K, 1.0 / model.ds_block,
               float(P // 2), L.ptr(out), s)
        ctx.save_for_backward(t, geo, offs, imgs, rx, ry, ic)
        ctx.meta = (model, srcs.dtype, trg.dtype)
        return out

    @staticmethod
    def backward(ctx, g_out):
        t, geo, offs, imgs, rx, ry, ic = ctx.saved_tensors
        model, sdt, tdt = ctx.meta
        dev = geo.device
        N, H, W = int(t.shape[0]), int(t.shape[1]), int(t.shape[2])
        K = H * W
        B, P = model.B, model.P
        s = L.stream_ptr(dev)
        g = g_out.detach().to(device=dev, dtype=torch.float32).contiguous()
        grad_imgs = torch.zeros((B, N, P, P), dtype=torch.float32, device=dev)
        goffs = torch.empty((3, B, N), dtype=torch.float64, device=dev)
        gray = torch.empty((N, K, 3), dtype=torch.float32, device=dev)
        wsb = L.query("fvr_pou_warp_bwd_workspace", B, N, K)
        ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
        L.call("fvr_pou_warp_bwd", L.ptr(imgs), B, N, P, L.ptr(offs), _ct.c_void_p(offs.data_ptr() + 8),
               _ct.c_void_p(offs.data_ptr() + 16), 1, 3, L.ptr(rx), L.ptr(ry), L.ptr(ic), K, K, 1.0 / model.ds_block,
               float(P // 2), L.ptr(g), L.ptr(grad_imgs), L.ptr(goffs), L.ptr(gray), L.ptr(ws), wsb, s)
        from .cone_beam_fvr import _block_images_adjoint

        ws2, tiles = _block_images_adjoint(model, geo, N, grad_imgs, s)
        del grad_imgs
        gtrg = torch.empty((N, K, 3), dtype=torch.float32, device=dev)
        wsb3 = L.query("fvr_pou_rays_bwd_workspace", N, K)
        ws3 = torch.empty(wsb3, dtype=torch.uint8, device=dev)
        L.call("fvr_pou_rays_bwd", L.ptr(t), L.ptr(geo), N, K, L.ptr(gray), L.ptr(gtrg), L.ptr(ws3), wsb3, s)
        gvec = torch.empty((N, 12), dtype=torch.float32, device=dev)
        L.call("fvr_pou_pose_backward", L.ptr(ws2), tiles, L.ptr(goffs), L.ptr(ws3), (K + 255) // 256,
               L.ptr(geo), L.ptr(model.centers), B, N, None, float(P) * model.ds_block, None, L.ptr(gvec), s)
        return (gvec[:, 0:3].to(sdt), gtrg.view(N, H, W, 3).to(tdt), gvec[:, 3:6].to(sdt), gvec[:, 6:9].to(sdt),
                gvec[:, 9:12].to(sdt), None)


def project_rays_batched(model, srcs, trg_pts, u_det, v_det, n_0):
    """(N, H, W) line integrals (cone_beam_fvr.py:423-478)."""
    dev = model._dev
    return _RaysFn.apply(srcs.to(dev), trg_pts.to(dev), u_det.to(dev), v_det.to(dev), n_0.to(dev), model)


def forward_explicit(model, pose_mats, lattice):
    """5-tuple lattice path (cone_beam_fvr.py:676-688) -> (N, 1, H, W)."""
    dev = model._dev
    src0, trg0, u0, v0, n0 = (t.to(dev) for t in lattice[:5])
    mats = pose_mats.to(dev)
    R = mats[:, :3, :3]
    t = mats[:, :3, 3]
    srcs = torch.einsum("nij,j->ni", R, src0) + t
    u_det = torch.einsum("nij,j->ni", R, u0)
    v_det = torch.einsum("nij,j->ni", R, v0)
    n_0 = torch.einsum("nij,j->ni", R, n0)
    trg_pts = torch.einsum("nij,hwj->nhwi", R, trg0) + t[:, None, None, :]
    return model.project_rays_batched(srcs, trg_pts, u_det=u_det, v_det=v_det, n_0=n_0).unsqueeze(1)
