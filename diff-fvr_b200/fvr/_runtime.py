"""Device-side constant caches and thin wrappers over the FFT entry points.

Everything here runs through ``libfvr_b200.so``; tensors are allocated by
PyTorch's caching allocator (the library itself never allocates).
"""
from __future__ import annotations

import math

import torch

from . import _lib as L

_tw_cache = {}
_lin_cache = {}
_hp_cache = {}
_one_cache = {}


def device_of(device):
    if not torch.cuda.is_available():
        raise L.FvrError("fvr_b200 computes on a CUDA (B200, sm_100a) device only and none is available; "
                         "there is no CPU fallback")
    d = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    if d.type != "cuda":
        raise L.FvrError(f"fvr_b200 runs on CUDA devices only (requested {d}); there is no CPU path")
    if d.index is None:
        d = torch.device("cuda", torch.cuda.current_device())
    return d


def compute_device(*tensors):
    """The CUDA device a call computes on: that of its first CUDA tensor, else
    the current CUDA device (inputs on the CPU are moved there by the caller)."""
    for t in tensors:
        if isinstance(t, torch.Tensor) and t.is_cuda:
            return t.device
    return device_of(None)


def twiddles(n, prec, device):
    """exp(-2 pi i m / n), m < n, as [n, 2] float32 (prec F32) or float64 (prec F64)."""
    key = (int(n), prec, device.index)
    t = _tw_cache.get(key)
    if t is None:
        if not L.load().fvr_fft_supported(int(n)):
            raise L.FvrError(f"FFT length {n} unsupported (prime factors must be <= 13, n <= 16384)")
        t = torch.empty((int(n), 2), dtype=torch.float64 if prec == L.F64_ else torch.float32, device=device)
        L.call("fvr_fft_twiddles", int(n), prec, L.ptr(t), L.stream_ptr(device))
        _tw_cache[key] = t
    return t


def ones(device):
    """A device-resident float32 1.0 (upstream gradient of a loss that is not
    differentiated further)."""
    t = _one_cache.get(device.index)
    if t is None:
        t = torch.ones(1, dtype=torch.float32, device=device)
        _one_cache[device.index] = t
    return t


def linspace(n, device):
    """torch.linspace(-1, 1, n) in float32, evaluated on the device."""
    key = (int(n), device.index)
    t = _lin_cache.get(key)
    if t is None:
        t = torch.empty(int(n), dtype=torch.float32, device=device)
        L.call("fvr_linspace", L.ptr(t), -1.0, 1.0, int(n), L.stream_ptr(device))
        _lin_cache[key] = t
    return t


def hp_filter(H, W, sigma, device):
    """High-pass 1 - exp(-r^2/(2 sigma^2)) (src/fvr/torch_engine.py:123-136) as [H, W] float32."""
    key = (int(H), int(W), float(sigma), device.index)
    t = _hp_cache.get(key)
    if t is None:
        t = torch.empty((int(H), int(W)), dtype=torch.float32, device=device)
        L.call("fvr_hp_filter", L.ptr(t), int(H), int(W), float(sigma), L.stream_ptr(device))
        _hp_cache[key] = t
    return t


SHIFT_NONE, SHIFT_IFFT, SHIFT_FFT = 0, 1, 2
OUT_COMPLEX, OUT_REAL, OUT_RELU = 0, 1, 2


def fft2d(x, *, inverse, in_shift=SHIFT_NONE, out_shift=SHIFT_NONE, scale=1.0, out_mode=OUT_COMPLEX, out=None,
          crop=None, work=None):
    """Batched 2D FFT over the last two dims of ``x`` (complex64/128 or real float32/64).

    ``inverse`` is unnormalised (pass ``scale=1/(n0*n1)`` for numpy/torch ifft2).
    Returns ``out`` (allocated if None): complex of x's shape, or real of the crop size.
    """
    dev = L.require_cuda(x)
    real_in = not x.is_complex()
    f64 = x.dtype in (torch.float64, torch.complex128)
    prec = L.F64_ if f64 else L.F32_
    x = x.contiguous()
    n0, n1 = int(x.shape[-2]), int(x.shape[-1])
    batch = x.numel() // (n0 * n1)
    cdt = torch.complex128 if f64 else torch.complex64
    rdt = torch.float64 if f64 else torch.float32
    if work is None:
        work = x if (not real_in and x.dtype == cdt) else torch.empty(x.shape, dtype=cdt, device=dev)
    if crop is None:
        crop = (0, n0, 0, n1)
    if out is None:
        if out_mode == OUT_COMPLEX:
            out = torch.empty(x.shape, dtype=cdt, device=dev)
        else:
            out = torch.empty(x.shape[:-2] + (crop[1], crop[3]), dtype=rdt, device=dev)
    L.call("fvr_fft2d", L.ptr(x), int(real_in), batch, n0, n1, prec, int(bool(inverse)), in_shift, out_shift,
           float(scale), out_mode, L.ptr(out), crop[0], crop[1], crop[2], crop[3],
           L.ptr(twiddles(n0, prec, dev)), L.ptr(twiddles(n1, prec, dev)), L.ptr(work), L.stream_ptr(dev))
    return out


def spectrum3d(vol, pad_shape, convention, *, prec=L.F32_, premult=None, batch_first=False):
    """Centred 3D spectrum of a zero-padded real volume (or batch of them).

    convention 0: torch engine, 1: NumPy renderer, 2: PoU blocks (see fvr_spectrum3d).
    Returns complex [.., Dp, Hp, Wp] (complex64 for prec F32, complex128 for F64).
    """
    dev = L.require_cuda(vol)
    v = vol.contiguous()
    if not batch_first:
        v = v.unsqueeze(0)
    nb, d, h, w = (int(s) for s in v.shape)
    Dp, Hp, Wp = (int(s) for s in pad_shape)
    cdt = torch.complex128 if prec == L.F64_ else torch.complex64
    out = torch.empty((nb, Dp, Hp, Wp), dtype=cdt, device=dev)
    wz = wy = wx = None
    if premult is not None:
        wz, wy, wx = (t.to(device=dev, dtype=torch.float64).contiguous() for t in premult)
    L.call("fvr_spectrum3d", L.ptr(v), L.dtype_code(v.dtype), nb, d, h, w, Dp, Hp, Wp, int(convention),
           L.ptr(wz), L.ptr(wy), L.ptr(wx), prec, L.ptr(out), L.ptr(twiddles(Wp, prec, dev)),
           L.ptr(twiddles(Hp, prec, dev)), L.ptr(twiddles(Dp, prec, dev)), L.stream_ptr(dev))
    return out if batch_first else out[0]


class Stencil:
    """Stencil ("corner-cube") copy of a centred spectrum (see include/fvr_b200.h)."""

    def __init__(self, master, planar, dims, dtype, items=1):
        dev = L.require_cuda(master)
        D, H, W = (int(s) for s in dims)
        self.dims = (D, H, W)
        self.items = int(items)
        self.dtype = dtype
        self.code = L.dtype_code(dtype)
        self.item_bytes = L.query("fvr_stencil_bytes", D, H, W, self.code)
        if self.item_bytes <= 0:
            raise L.FvrError(f"unsupported stencil dtype {dtype}")
        self.data = torch.empty(self.item_bytes * self.items, dtype=torch.uint8, device=dev)
        self.scales = None
        self.item_scales = 0
        scratch = None
        if self.code == L.F16_:
            self.item_scales = L.query("fvr_stencil_scale_count", D, H, W)
            self.scales = torch.empty(self.item_scales * self.items, dtype=torch.float32, device=dev)
            scratch = torch.empty(self.item_scales * self.items, dtype=torch.int32, device=dev)
        m = master.contiguous()
        L.call("fvr_stencil_build", L.ptr(m), L.dtype_code(m.dtype), int(planar), self.items, D, H, W, self.code,
               L.ptr(self.data), L.ptr(self.scales), L.ptr(scratch), L.stream_ptr(dev))

    def args(self):
        D, H, W = self.dims
        return (self.code, L.ptr(self.data), L.ptr(self.scales), D, H, W)


class PairStencil:
    """x-pair copy of a centred spectrum (see fvr_stencil_pair_build in
    include/fvr_b200.h), read by the spectral-NCC moments kernels and the
    fused PoU block-image kernels: half the bytes of the stencil, a sample's
    two entries side by side.  ``items`` spectra back to back, as Stencil."""

    def __init__(self, master, planar, dims, dtype, items=1):
        dev = L.require_cuda(master)
        D, H, W = (int(s) for s in dims)
        self.dims = (D, H, W)
        self.items = int(items)
        self.dtype = dtype
        codes = {torch.float16: L.F16_PAIR_, torch.bfloat16: L.BF16_PAIR_, torch.float32: L.F32_PAIR_}
        if dtype not in codes:
            raise L.FvrError(f"unsupported x-pair storage dtype {dtype}")
        self.code = codes[dtype]
        self.item_bytes = L.query("fvr_stencil_pair_bytes", D, H, W, self.code)
        self.data = torch.empty(self.item_bytes * self.items, dtype=torch.uint8, device=dev)
        self.scales = None
        scratch = None
        if self.code == L.F16_PAIR_:
            n = L.query("fvr_stencil_pair_scale_count", D, H, W) * self.items
            self.scales = torch.empty(n, dtype=torch.float32, device=dev)
            scratch = torch.empty(n, dtype=torch.int32, device=dev)
        m = master.contiguous()
        L.call("fvr_stencil_pair_build", L.ptr(m), L.dtype_code(m.dtype), int(planar), self.items, D, H, W,
               self.code, L.ptr(self.data), L.ptr(self.scales), L.ptr(scratch), L.stream_ptr(dev))

    def args(self):
        D, H, W = self.dims
        return (self.code, L.ptr(self.data), L.ptr(self.scales), D, H, W)


def kappa(out_res, spacing0):
    """-2 pi / (R * spacing + 1e-6): phase = kappa * (ku tx + kv ty) (torch_engine.py:227-232)."""
    return -2.0 * math.pi / (out_res * float(spacing0) + 1e-6)
