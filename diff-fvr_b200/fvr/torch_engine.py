"""Parallel-beam differentiable Fourier volume renderer on B200 (drop-in for
``TorchDiffFVREngine``, src/fvr/torch_engine.py).

Same constructor, methods, conventions and outputs as the reference (the
quirks included: ``poses[:, 5]`` (tz) is never read, the lateral view is
``R . Rz(90 deg)``, the frequency grid is ``linspace(-1, 1, R)`` scaled by
``(N_pad - 1)/2``, the image is ``relu(real(ifft2(ifftshift(S))))`` with no
fftshift and no scale, and the phase uses ``spacing[0]`` only).  Every
computation runs in ``libfvr_b200.so``:

* spectrum precompute: shared-memory radix FFT (``fvr_spectrum3d``);
* spectrum storage: the stencil layout (one aligned 32/64-byte entry per
  trilinear sample) in f32, bf16 or brick-scaled f16;
* ``forward_spectral_ncc``: one fused gather + phase + high-pass + NCC pass
  per view that also reduces the moments of the pose gradient, so backward is
  a per-candidate fp64 epilogue (no slice is stored or recomputed);
* ``forward``: slice in ifftshift order -> 2D IFFT with ReLU fused into the
  last pass; backward re-gathers the slice (recompute, not store).

Inputs on the CPU are moved to the engine's CUDA device (differentiably);
outputs are returned on the CUDA device.  There is no CPU fallback.
"""
from __future__ import annotations

from typing import Optional, Tuple, Union

import ctypes

import numpy as np
import torch
import torch.nn as nn

from . import _lib as L
from . import _runtime as RT
from . import autotune, profiling

try:  # native autograd binding (csrc/fvr_autograd.cpp, built next to the CUDA library)
    from . import _fvr_autograd as _NATIVE
except ImportError:
    _NATIVE = None

VIEW_AP, VIEW_LATERAL = 0, 1


def _view_code(view: str) -> int:
    return VIEW_LATERAL if str(view).lower() == "lateral" else VIEW_AP


def _sncc_forward(eng, p, views, ftargs, hp, R, with_grad):
    """Launch the fused moments pass + finalize for len(views) views.
    Returns (mom [nv, C, 18] fp64, loss [nv + 1] f32: per view, then the sum)."""
    dev = eng._dev
    C = int(p.shape[0])
    nv = len(views)
    st = eng._sncc_storage()
    ws_bytes = L.query("fvr_tc_sncc_workspace", C, R, nv)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    mom = torch.empty((nv, C, int(L.query("fvr_tc_sncc_mom_stride"))), dtype=torch.float64, device=dev)
    loss = torch.empty(nv + 1, dtype=torch.float32, device=dev)
    fts = [f.detach().to(device=dev, dtype=torch.complex64).contiguous() for f in ftargs]
    for f in fts:
        if f.numel() != R * R:
            raise L.FvrError(f"target spectrum has {f.numel()} elements, expected {R}x{R}")
    vcodes = (ctypes.c_int * nv)(*views)
    fptrs = (ctypes.c_void_p * nv)(*[f.data_ptr() for f in fts])
    kap = RT.kappa(R, eng.spacing[0])
    s = L.stream_ptr(dev)
    lin = RT.linspace(R, dev)

    def run(variant):
        L.call("fvr_tc_sncc_moments", *st.args(), L.ptr(p), C, nv, vcodes, fptrs, L.ptr(hp), L.ptr(lin), R, kap,
               int(with_grad), int(variant), L.ptr(ws), ws_bytes, s)

    def finalize(variant):  # the record count (and so this kernel's work) depends on the variant's grid
        L.call("fvr_tc_sncc_finalize", L.ptr(ws), C, R, nv, int(with_grad), int(variant), L.ptr(mom), L.ptr(loss),
               None, s)

    def both(variant):
        run(variant)
        finalize(variant)

    variant = autotune.choose("sncc", (st.code, C, R, nv, int(with_grad), st.dims), both,
                              L.load().fvr_tc_sncc_variants())
    with profiling.section("tc_sncc_moments"):
        run(variant)
    finalize(variant)
    return mom, loss


# Launch variants the value-and-gradient path chooses from: those whose
# gradient kernel keeps every value in registers (the 3- and 4-CTA-per-SM
# register budgets spill the 17 moment pairs); the variant table is in
# csrc/fvr_tc.cu (kSnccVariantTable).
_FUSED_VARIANTS = (0, 3, 6, 7)


class _FusedCall:
    """A prepared launch of fvr_tc_sncc_value_and_grad: every argument except
    the poses, the two outputs and the stream converted to its C type once
    (engine storage, shape, views, target spectra, high-pass table, chosen
    launch variant, cached workspace), so a call costs one foreign call.
    ``native`` is the same launch prepared for the native autograd binding
    (None without it)."""

    __slots__ = ("fn", "head", "mid", "keep", "native")

    def launch(self, p, loss, grad, stream):
        L.launch_count[0] += 2
        rc = self.fn(*self.head, _ct_ptr(p), *self.mid, _ct_ptr(loss), None, _ct_ptr(grad), 0, stream)
        if rc != 0:
            raise L.FvrError(f"fvr_tc_sncc_value_and_grad failed with status {rc}: "
                             f"{L.load().fvr_status_string(rc).decode()}")


def _ct_ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _fused_call(eng, C, R, views, ftargs, hp, p):
    """The prepared launch for this engine storage and call shape, built (and
    the launch variant autotuned on the poses ``p``) on first use.  Target spectra already in
    complex64 on the engine's device are used in place and the preparation
    is cached by their addresses; others are converted for this call only."""
    dev = eng._dev
    st = eng._sncc_storage()
    nv = len(views)
    direct = all(f.is_cuda and f.device == dev and f.dtype == torch.complex64 and f.is_contiguous() for f in ftargs)
    key = (C, R, tuple(views), tuple(int(f.data_ptr()) for f in ftargs), 0 if hp is None else int(hp.data_ptr()),
           id(st))
    hit = eng._fused_calls.get(key) if direct else None
    if hit is not None:
        return hit
    ws_bytes = int(L.query("fvr_tc_sncc_fused_workspace", C, R, nv))
    wkey = (C, R, nv, dev)
    ws = eng._fused_ws.get(wkey)
    if ws is None:
        ws = torch.zeros(ws_bytes, dtype=torch.uint8, device=dev)  # zeroed once: the record flags start clear
        eng._fused_ws[wkey] = ws
    fts = [f.detach().to(device=dev, dtype=torch.complex64).contiguous() for f in ftargs]
    for f in fts:
        if f.numel() != R * R:
            raise L.FvrError(f"target spectrum has {f.numel()} elements, expected {R}x{R}")
    vcodes = (ctypes.c_int * nv)(*views)
    fptrs = (ctypes.c_void_p * nv)(*[f.data_ptr() for f in fts])
    lin = RT.linspace(R, dev)
    call = _FusedCall()
    call.fn = getattr(L.load(), "fvr_tc_sncc_value_and_grad")
    call.head = st.args()
    call.keep = (st, fts, hp, lin, ws, vcodes, fptrs)

    def mid(variant):
        return (ctypes.c_int64(C), ctypes.c_int(nv), vcodes, fptrs, L.ptr(hp), L.ptr(lin), ctypes.c_int64(R),
                ctypes.c_double(RT.kappa(R, eng.spacing[0])), ctypes.c_int(int(variant)), None, ctypes.c_int64(0),
                L.ptr(ws), ctypes.c_int64(ws_bytes))

    p32 = []

    def run(variant):
        if not p32:
            p32.append(p.detach().to(device=dev, dtype=torch.float32).contiguous())
        call.mid = mid(variant)
        loss = torch.empty(nv + 1, dtype=torch.float32, device=dev)
        grad = torch.empty((C, 6), dtype=torch.float32, device=dev)
        call.launch(p32[0], loss, grad, L.stream_ptr(dev))

    variant = autotune.choose("sncc_fused", (st.code, C, R, nv, st.dims), run, L.load().fvr_tc_sncc_variants(),
                              candidates=_FUSED_VARIANTS)
    call.mid = mid(variant)
    call.native = None
    if _NATIVE is not None:
        lib = L.load()
        addr = lambda f: ctypes.cast(f, ctypes.c_void_p).value  # noqa: E731
        sp = 0 if st.scales is None else int(st.scales.data_ptr())
        call.native = _NATIVE.SnccCall(
            fn=addr(lib.fvr_tc_sncc_value_and_grad), status=addr(lib.fvr_status_string), dtype=st.code,
            stencil=int(st.data.data_ptr()), scales=sp, D=st.dims[0], H=st.dims[1], W=st.dims[2], C=C,
            views=list(views), ftargs=[int(f.data_ptr()) for f in fts], hp=0 if hp is None else int(hp.data_ptr()),
            lin=int(lin.data_ptr()), R=R, kappa=RT.kappa(R, eng.spacing[0]), variant=int(variant),
            ws=int(ws.data_ptr()), ws_bytes=ws_bytes, device=dev.index,
            keep=[t for t in (st.data, st.scales, hp, lin, ws) if t is not None] + fts)
    if direct:
        if len(eng._fused_calls) > 64:
            eng._fused_calls.clear()
        eng._fused_calls[key] = call
    return call


def _current_stream(dev):
    getter = getattr(torch._C, "_cuda_getCurrentRawStream", None)
    return ctypes.c_void_p(getter(dev.index)) if getter is not None else L.stream_ptr(dev)


def _sncc_fused(eng, p, views, ftargs, hp, R, out=None, loss_out=None):
    """Moments kernel + its dependent epilogue: per-candidate finalize and pose
    gradient, view losses.  Returns (loss [nv + 1] f32, grad [C, 6] f32).  The
    workspace is cached per shape on the engine, so captured graphs keep a
    stable pointer; launches sharing it are ordered on the engine's stream."""
    dev = eng._dev
    C = int(p.shape[0])
    nv = len(views)
    call = _fused_call(eng, C, int(R), tuple(views), ftargs, hp, p)
    loss = torch.empty(nv + 1, dtype=torch.float32, device=dev) if loss_out is None else loss_out
    grad = torch.empty((C, 6), dtype=torch.float32, device=dev) if out is None else out
    if out is not None or loss_out is not None:
        for t, shape in ((loss, (nv + 1,)), (grad, (C, 6))):
            if tuple(t.shape) != shape or t.dtype != torch.float32 or not t.is_contiguous():
                raise L.FvrError(f"output buffer must be a contiguous float32 tensor of shape {shape}")
            if not (t.is_cuda or t.is_pinned()):
                raise L.FvrError("output buffers must be device memory or pinned host memory")
    if profiling.timing("tc_sncc_moments"):
        with profiling.section("tc_sncc_moments"):
            call.launch(p, loss, grad, _current_stream(dev))
    else:
        call.launch(p, loss, grad, _current_stream(dev))
    return loss, grad


def _sncc_loss(eng, p, views, hp, R, ftargs):
    """sum_v forward_spectral_ncc(p, ftargs[v], views[v]) as one autograd node.
    With a pose gradient to compute, the native binding runs the fused launch
    (moments kernel + dependent epilogue) and keeps dL/dposes; otherwise (or
    without the binding, or while launches are being timed) the Python node
    below does the same."""
    if (_NATIVE is not None and p.requires_grad and torch.is_grad_enabled()
            and not profiling.timing("tc_sncc_moments")):
        call = _fused_call(eng, int(p.shape[0]), R, views, ftargs, hp, p)
        L.launch_count[0] += 2
        try:
            return _NATIVE.sncc_loss(p, call.native)
        except RuntimeError as e:
            raise L.FvrError(str(e)) from None
    return _SpectralNCCFn.apply(p, eng, views, hp, R, *ftargs)


class _SpectralNCCFn(torch.autograd.Function):
    """Zero-IFFT spectral NCC (torch_engine.py:269-307), summed over the given
    views.  When the poses need a gradient, the forward pass already runs the
    fused loss-and-gradient launch (moments kernel + its dependent epilogue)
    and keeps dL/dposes; backward only scales it by the upstream gradient (the
    loss is a scalar, so its pose gradient is linear in that factor).
    Without a gradient the cheaper value-only moments (3 instead of 17) run."""

    @staticmethod
    def forward(ctx, poses, eng, views, hp, R, *ftargs):
        p = poses.detach().to(device=eng._dev, dtype=torch.float32).contiguous()
        nv = len(views)
        ctx.meta = (views, poses.dtype)
        if ctx.needs_input_grad[0]:
            grad = torch.empty((int(p.shape[0]), 6), dtype=torch.float32, device=eng._dev)
            loss = torch.empty(nv + 1, dtype=torch.float32, device=eng._dev)
            _sncc_fused(eng, p, views, ftargs, hp, R, out=grad, loss_out=loss)
            ctx.save_for_backward(grad)
            return loss[nv]
        _, loss = _sncc_forward(eng, p, views, ftargs, hp, R, False)
        return loss[nv]

    @staticmethod
    def backward(ctx, g):
        (grad,) = ctx.saved_tensors
        views, pdt = ctx.meta
        return ((grad * g.to(grad.dtype)).to(pdt), None, None, None, None) + (None,) * len(views)


class _SliceFn(torch.autograd.Function):
    """Modulated slice spectrum (torch_engine.py:176-234); shift=1 returns it in
    ifftshift order for the image IFFT."""

    @staticmethod
    def forward(ctx, poses, eng, view, R, shift):
        dev = eng._dev
        p = poses.detach().to(device=dev, dtype=torch.float32).contiguous()
        C = int(p.shape[0])
        st = eng._stencil
        D, H, W = st.dims
        axes = torch.empty((C, 8), dtype=torch.float64, device=dev)
        s = L.stream_ptr(dev)
        L.call("fvr_tc_axes", L.ptr(p), C, view, D, H, W, L.ptr(axes), s)
        out = torch.empty((C, R, R), dtype=torch.complex64, device=dev)
        kap = RT.kappa(R, eng.spacing[0])
        L.call("fvr_tc_slice", *st.args(), L.ptr(axes), C, L.ptr(RT.linspace(R, dev)), R, kap, int(shift),
               L.ptr(out), s)
        ctx.save_for_backward(p, axes)
        ctx.meta = (eng, view, R, kap, shift, poses.dtype)
        return out

    @staticmethod
    def backward(ctx, G):
        p, axes = ctx.saved_tensors
        eng, view, R, kap, shift, pdt = ctx.meta
        grad = _slice_adjoint(eng, p, axes, view, R, kap, shift, G.to(torch.complex64).contiguous())
        return grad.to(pdt), None, None, None, None


def _slice_adjoint(eng, p, axes, view, R, kap, shift, G):
    dev = p.device
    C = int(p.shape[0])
    st = eng._stencil
    D, H, W = st.dims
    ws_bytes = L.query("fvr_tc_slice_adjoint_workspace", C, R)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    grad = torch.empty((C, 6), dtype=torch.float32, device=dev)
    L.call("fvr_tc_slice_adjoint", *st.args(), L.ptr(axes), L.ptr(p), C, view, L.ptr(RT.linspace(R, dev)), R, kap,
           int(shift), L.ptr(G), L.ptr(ws), ws_bytes, L.ptr(grad), 0, L.stream_ptr(dev))
    return grad


class _ImageFn(torch.autograd.Function):
    """relu(real(ifft2(ifftshift(S)))) (torch_engine.py:236-241); the ReLU and the
    1/R^2 of ifft2 are fused into the last FFT pass."""

    @staticmethod
    def forward(ctx, poses, eng, view, R):
        dev = eng._dev
        p = poses.detach().to(device=dev, dtype=torch.float32).contiguous()
        C = int(p.shape[0])
        st = eng._stencil
        D, H, W = st.dims
        axes = torch.empty((C, 8), dtype=torch.float64, device=dev)
        s = L.stream_ptr(dev)
        L.call("fvr_tc_axes", L.ptr(p), C, view, D, H, W, L.ptr(axes), s)
        buf = torch.empty((C, R, R), dtype=torch.complex64, device=dev)
        kap = RT.kappa(R, eng.spacing[0])
        L.call("fvr_tc_slice", *st.args(), L.ptr(axes), C, L.ptr(RT.linspace(R, dev)), R, kap, 1, L.ptr(buf), s)
        img = torch.empty((C, 1, R, R), dtype=torch.float32, device=dev)
        RT.fft2d(buf, inverse=True, scale=1.0 / (R * R), out_mode=RT.OUT_RELU, out=img, work=buf)
        ctx.save_for_backward(p, axes, img)
        ctx.meta = (eng, view, R, kap, poses.dtype)
        return img

    @staticmethod
    def backward(ctx, g):
        p, axes, img = ctx.saved_tensors
        eng, view, R, kap, pdt = ctx.meta
        dev = p.device
        gm = torch.empty_like(img)
        gc = g.detach().to(device=dev, dtype=torch.float32).contiguous()
        L.call("fvr_relu_mask", L.ptr(img), L.ptr(gc), L.ptr(gm), img.numel(), L.stream_ptr(dev))
        # adjoint of S -> Re(ifft2(ifftshift(S))): fftshift(fft2(g)) / R^2, natural order
        G = RT.fft2d(gm.view(-1, R, R), inverse=False, out_shift=RT.SHIFT_FFT, scale=1.0 / (R * R))
        grad = _slice_adjoint(eng, p, axes, view, R, kap, 0, G)
        return grad.to(pdt), None, None, None


class _ImageSpectralNCCFn(torch.autograd.Function):
    """spectral_ncc_loss (torch_engine.py:309-337): fftshift(fft2(.)) of both
    images, high-pass, NCC; gradient to ``pred``."""

    @staticmethod
    def forward(ctx, pred, target, hp):
        dev = L.require_cuda(pred)
        H, W = int(pred.shape[-2]), int(pred.shape[-1])
        B = pred.numel() // (H * W)
        Bt = target.numel() // (H * W)
        x = pred.detach().float().contiguous()
        t = target.detach().to(device=dev, dtype=torch.float32).contiguous()
        Fp = RT.fft2d(x, inverse=False, out_shift=RT.SHIFT_FFT)
        Ft = RT.fft2d(t, inverse=False, out_shift=RT.SHIFT_FFT)
        ws_bytes = L.query("fvr_cncc_workspace", B, H * W)
        ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
        mom = torch.empty((B, 3), dtype=torch.float64, device=dev)
        loss = torch.empty((), dtype=torch.float32, device=dev)
        L.call("fvr_cncc_forward", L.ptr(Fp), L.ptr(Ft), B, Bt, H * W, L.ptr(hp), L.ptr(ws), ws_bytes, L.ptr(mom),
               L.ptr(loss), L.stream_ptr(dev))
        ctx.save_for_backward(Fp, Ft, mom)
        ctx.meta = (hp, B, Bt, H, W, pred.shape, pred.dtype)
        return loss

    @staticmethod
    def backward(ctx, g):
        Fp, Ft, mom = ctx.saved_tensors
        hp, B, Bt, H, W, shape, dt = ctx.meta
        dev = Fp.device
        X = torch.empty_like(Fp)
        gg = g.detach().to(device=dev, dtype=torch.float32).contiguous()
        L.call("fvr_cncc_backward", L.ptr(Fp), L.ptr(Ft), B, Bt, H * W, L.ptr(hp), L.ptr(mom), L.ptr(gg), L.ptr(X),
               L.stream_ptr(dev))
        # adjoint of x -> fftshift(fft2(x)): Re(N * ifft2(ifftshift(X))) = Re(unnormalised inverse)
        gx = RT.fft2d(X, inverse=True, in_shift=RT.SHIFT_IFFT, out_mode=RT.OUT_REAL)
        return gx.view(shape).to(dt), None, None


class TorchDiffFVREngine(nn.Module):
    """Tensorised differentiable Fourier volume renderer (parallel beam).

    Signature and behaviour of src/fvr/torch_engine.py:17-337.  ``use_triton``
    is accepted for compatibility and ignored: the CUDA path always runs.
    ``device`` defaults to the current CUDA device.

    Attributes
    ----------
    f_vol_5d : torch.Tensor
        Centred 3D spectrum ``(1, 2, D_pad, H_pad, W_pad)`` [real, imag] in the
        storage dtype, exactly as the reference stores it.
    """

    def __init__(
        self,
        volume: Union[torch.Tensor, np.ndarray],
        spacing: Tuple[float, float, float] = (1.0, 1.0, 1.0),
        pad_factor: float = 2.0,
        device: Optional[Union[str, torch.device]] = None,
        dtype: torch.dtype = torch.float32,
        use_triton: bool = True,
    ):
        super().__init__()
        self.use_triton = bool(use_triton)
        if not isinstance(volume, torch.Tensor):
            volume = torch.from_numpy(np.asarray(volume)).float()
        else:
            volume = volume.detach().float()
        if device is None and volume.is_cuda:
            device = volume.device
        self._dev = RT.device_of(device)
        self.device = self._dev
        self._compiled_forward_core = None
        self._compiled_spectral_ncc = None
        self.orig_shape = volume.shape
        self.spacing = spacing
        self.pad_factor = pad_factor
        d, h, w = (int(s) for s in volume.shape)
        self.pad_shape = torch.Size((int(round(d * pad_factor)), int(round(h * pad_factor)),
                                     int(round(w * pad_factor))))
        # the one-time transform runs in fp64 (a 512^3 float32 FFT alone would
        # carry ~1e-5 of relative error into the images); storage is rounded once
        vol = volume.to(device=self._dev, dtype=torch.float64).contiguous()
        spec = RT.spectrum3d(vol, self.pad_shape, 0, prec=L.F64_)  # complex128 [Dp, Hp, Wp]
        del vol
        planar = torch.view_as_real(spec).permute(3, 0, 1, 2).unsqueeze(0).to(torch.float32).contiguous()
        del spec
        self.register_buffer("f_vol_5d", planar.to(dtype=dtype))
        # storage copies come from the float32 spectrum (f16 takes its brick scales from it)
        self._stencil = RT.Stencil(planar[0], True, self.pad_shape, self._stencil_dtype(dtype))
        self._pair = RT.PairStencil(planar[0], True, self.pad_shape, self._stencil_dtype(dtype))
        self.use_pair_storage = True  # the spectral-NCC moments read the x-pair copy
        del planar
        self._fused_ws = {}  # (C, R, views, device) -> workspace of the fused value_and_grad
        self._fused_calls = {}  # prepared launches of the fused value_and_grad

    def _sncc_storage(self):
        """The spectrum copy the spectral-NCC moments kernels read: the x-pair
        copy (unless ``use_pair_storage`` is off), else the stencil."""
        return self._pair if (self._pair is not None and self.use_pair_storage) else self._stencil

    @staticmethod
    def _stencil_dtype(dtype):
        if dtype in (torch.float32, torch.bfloat16, torch.float16):
            return dtype
        if dtype == torch.float64:
            return torch.float32
        raise L.FvrError(f"unsupported spectrum dtype {dtype}")

    def to_precision(self, dtype: torch.dtype) -> "TorchDiffFVREngine":
        """Cast the stored spectrum to ``dtype`` (torch_engine.py:90-95).

        bf16 is a round-to-nearest cast of the stored spectrum, as in the
        reference.  f16 storage is brick-scaled (power-of-two scale per 16^3
        stencil brick) so the spectrum's DC region cannot overflow; the scaled
        copy is built from the current higher-precision spectrum.
        """
        src = self.f_vol_5d[0]
        self._stencil = RT.Stencil(src, True, self.pad_shape, self._stencil_dtype(dtype))
        # the spectral-NCC moments kernels read an x-pair copy (half the
        # stencil's bytes; the image path keeps the stencil)
        self._pair = RT.PairStencil(src, True, self.pad_shape, self._stencil_dtype(dtype))
        self.f_vol_5d = self.f_vol_5d.to(dtype=dtype)
        self._compiled_forward_core = None
        self._compiled_spectral_ncc = None
        return self

    def compile_renderer(self, mode: str = "reduce-overhead", fullgraph: bool = False) -> "TorchDiffFVREngine":
        """Accepted for compatibility (torch_engine.py:97-106); kernels are already
        fused CUDA.  Capture whole optimiser steps with :mod:`fvr.graphs` instead."""
        return self

    def _prep_poses(self, poses):
        if poses.device != self._dev:
            poses = poses.to(self._dev)
        return poses

    def _get_hp_filter(self, H, W, cutoff_sigma, device=None, dtype=torch.float32):
        return RT.hp_filter(H, W, cutoff_sigma, self._dev).view(1, 1, H, W)

    def _extract_slice_spectrum(self, poses: torch.Tensor, view: str = "ap", out_res: int = 128) -> torch.Tensor:
        """Phase-modulated complex slices ``(B, out_res, out_res)`` (torch_engine.py:176-234)."""
        return _SliceFn.apply(self._prep_poses(poses), self, _view_code(view), int(out_res), 0)

    def _forward_core(self, poses: torch.Tensor, view: str = "ap", out_res: int = 128) -> torch.Tensor:
        p = self._prep_poses(poses)
        if p.shape[0] == 0:  # an empty batch renders no image (still connected to the poses)
            R = int(out_res)
            return torch.zeros((0, 1, R, R), dtype=torch.float32, device=self._dev) + 0.0 * p.sum()
        return _ImageFn.apply(p, self, _view_code(view), int(out_res))

    def forward(self, poses: torch.Tensor, view: str = "ap", out_res: int = 128) -> torch.Tensor:
        """Batched differentiable forward pass returning ``(B, 1, out_res, out_res)``."""
        return self._forward_core(poses, view=view, out_res=out_res)

    def prepare_spectral_target(self, target_drr: torch.Tensor, high_pass: bool = True,
                                cutoff_sigma: float = 4.0) -> torch.Tensor:
        """``fftshift(fft2(target)) * HP`` computed once (torch_engine.py:255-267)."""
        t = target_drr.detach().to(device=self._dev, dtype=torch.float32).contiguous()
        H, W = int(t.shape[-2]), int(t.shape[-1])
        f = RT.fft2d(t, inverse=False, out_shift=RT.SHIFT_FFT)
        if high_pass:
            hp = RT.hp_filter(H, W, cutoff_sigma, self._dev)
            L.call("fvr_cmul_table", L.ptr(f), L.ptr(hp), H * W, f.numel(), L.stream_ptr(self._dev))
        return f

    def _spectral_ncc_core(self, poses, f_targ_precomputed, view="ap", high_pass=True, cutoff_sigma=4.0):
        if poses.shape[0] == 0:  # 1 - mean over no candidates, as torch's mean of an empty batch
            return torch.full((), float("nan"), dtype=torch.float32, device=self._dev) + 0.0 * poses.sum().to(self._dev)
        R = int(f_targ_precomputed.shape[-1])
        hp = RT.hp_filter(R, R, cutoff_sigma, self._dev) if high_pass else None
        return _sncc_loss(self, self._prep_poses(poses), (_view_code(view),), hp, R, (f_targ_precomputed,))

    def forward_spectral_ncc(self, poses: torch.Tensor, f_targ_precomputed: torch.Tensor, view: str = "ap",
                             high_pass: bool = True, cutoff_sigma: float = 4.0) -> torch.Tensor:
        """Zero-IFFT Parseval spectral-NCC loss ``1 - mean_B NCC`` (torch_engine.py:292-307)."""
        return self._spectral_ncc_core(poses, f_targ_precomputed, view=view, high_pass=high_pass,
                                       cutoff_sigma=cutoff_sigma)

    def forward_spectral_ncc_multiview(self, poses, f_targs, views=("ap", "lateral"), high_pass=True,
                                       cutoff_sigma=4.0):
        """``sum_v forward_spectral_ncc(poses, f_targs[v], views[v])`` in one fused launch
        (all views of all candidates share the gather pass); differentiable in poses."""
        R = int(f_targs[0].shape[-1])
        hp = RT.hp_filter(R, R, cutoff_sigma, self._dev) if high_pass else None
        codes = tuple(_view_code(v) for v in views)
        return _sncc_loss(self, self._prep_poses(poses), codes, hp, R, tuple(f_targs))

    def spectral_ncc_value_and_grad(self, poses, f_targs, views=("ap", "lateral"), high_pass=True,
                                    cutoff_sigma=4.0, out_grad=None, out_loss=None):
        """``(sum_v loss_v, dloss/dposes [C, 6])`` without autograd: one kernel gathers
        every candidate and view and reduces the NCC and pose moments; its programmatic
        dependent forms every candidate's fp64 pose gradient and the view losses
        (capturable in a CUDA graph).  ``out_grad`` ([C, 6] float32) and ``out_loss``
        ([len(views) + 1] float32: the view losses, then their sum) receive the results
        when given; either may be pinned host memory, which the kernel writes directly.
        Launches through one engine must stay on one stream."""
        p = self._prep_poses(poses).detach().to(torch.float32).contiguous()
        R = int(f_targs[0].shape[-1])
        hp = RT.hp_filter(R, R, cutoff_sigma, self._dev) if high_pass else None
        codes = tuple(_view_code(v) for v in views)
        loss, grad = _sncc_fused(self, p, codes, f_targs, hp, R, out=out_grad, loss_out=out_loss)
        return loss[len(codes)], grad

    def spectral_ncc_loss(self, pred_drr: torch.Tensor, target_drr: torch.Tensor, high_pass: bool = True,
                          cutoff_sigma: float = 4.0) -> torch.Tensor:
        """Image-domain spectral NCC loss (torch_engine.py:309-337); differentiable in ``pred_drr``."""
        pred = pred_drr if pred_drr.is_cuda else pred_drr.to(self._dev)
        H, W = int(pred.shape[-2]), int(pred.shape[-1])
        hp = RT.hp_filter(H, W, cutoff_sigma, pred.device) if high_pass else None
        return _ImageSpectralNCCFn.apply(pred, target_drr, hp)
