"""NumPy-convention differentiable Fourier volume renderer on B200 (drop-in for
``DifferentiableFourierVolumeRenderer``, src/fvr/diff_fvr.py).

Same constructor, attributes and NumPy-in / NumPy-out methods as the
reference, computed in fp64 on the GPU by ``libfvr_b200.so``: the sinc^2
pre-compensated, zero-padded ``fftshift(fftn(ifftshift(.)))`` spectrum
(shared-memory radix FFT), frequency slices with ``map_coordinates(order=1,
mode='constant')`` semantics and the phase ramp, the DRR inverse transform,
and the Parseval spectral NCC.  Only the final scalars / arrays are copied
back to the host.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np
import torch

from . import _lib as L
from . import _runtime as RT

_VIEW = {"lateral": 0, "ap": 1}


def _view_code(view):
    return _VIEW.get(view, 2)  # anything else is 'axial' (diff_fvr.py:98)


class _Item(ctypes.Structure):
    _fields_ = [("yaw", ctypes.c_double), ("pitch", ctypes.c_double), ("roll", ctypes.c_double),
                ("tx", ctypes.c_double), ("ty", ctypes.c_double), ("view", ctypes.c_int), ("sh", ctypes.c_int),
                ("sw", ctypes.c_int), ("pad", ctypes.c_int), ("off", ctypes.c_longlong)]


class DifferentiableFourierVolumeRenderer:
    """Differentiable & spectral Fourier volume rendering (diff_fvr.py:7-195)."""

    def __init__(self, volume: np.ndarray, pad_factor: float = 2.0, apply_premultiplication: bool = True,
                 device: Optional[torch.device] = None):
        if ctypes.sizeof(_Item) != L.query("fvr_np_item_bytes"):
            raise L.FvrError("item layout mismatch with libfvr_b200.so")
        self._dev = RT.device_of(device)
        self.orig_shape = volume.shape
        self.pad_factor = pad_factor
        self.apply_premultiplication = apply_premultiplication
        nz, ny, nx = volume.shape
        self.pz = int(round(nz * pad_factor))
        self.py = int(round(ny * pad_factor))
        self.px = int(round(nx * pad_factor))
        premult = None
        if apply_premultiplication:
            def corr(n_orig, n_pad):  # diff_fvr.py:35-39
                c = (np.arange(n_orig) - n_orig / 2.0) / n_pad
                return 1.0 / np.maximum(np.sinc(c) ** 2, 0.05)

            premult = tuple(torch.from_numpy(corr(n, p)) for n, p in ((nz, self.pz), (ny, self.py), (nx, self.px)))
        vol = torch.from_numpy(np.ascontiguousarray(volume, dtype=np.float64)).to(self._dev)
        self._f3d = RT.spectrum3d(vol, (self.pz, self.py, self.px), 1, prec=L.F64_, premult=premult)
        self._f3d_host = None

    @property
    def f_3d(self) -> np.ndarray:
        """Centred complex128 spectrum (copied from the device once)."""
        if self._f3d_host is None:
            self._f3d_host = self._f3d.cpu().numpy()
        return self._f3d_host

    def _dims(self, view):
        if view == "lateral":
            return self.pz, self.py
        if view == "ap":
            return self.pz, self.px
        return self.py, self.px

    def _items(self, specs):
        """specs: (yaw, pitch, roll, tx, ty, view) -> device item array, offsets, sizes."""
        arr = (_Item * len(specs))()
        off = 0
        sizes = []
        for i, (yaw, pitch, roll, tx, ty, view) in enumerate(specs):
            sh, sw = self._dims(view)
            arr[i] = _Item(float(yaw), float(pitch), float(roll), float(tx), float(ty), _view_code(view), sh, sw, 0,
                           off)
            sizes.append((sh, sw, off))
            off += sh * sw
        dev_items = torch.frombuffer(bytearray(arr), dtype=torch.uint8).to(self._dev)
        return dev_items, sizes, off

    def _euler_to_basis(self, yaw_deg, pitch_deg, roll_deg, view="lateral"):
        """Projection-plane basis (diff_fvr.py:56-104)."""
        y, p, r = np.radians(yaw_deg), np.radians(pitch_deg), np.radians(roll_deg)
        rz = np.array([[1.0, 0, 0], [0, np.cos(y), -np.sin(y)], [0, np.sin(y), np.cos(y)]])
        ry = np.array([[np.cos(r), 0, np.sin(r)], [0, 1.0, 0], [-np.sin(r), 0, np.cos(r)]])
        rx = np.array([[np.cos(p), -np.sin(p), 0], [np.sin(p), np.cos(p), 0], [0, 0, 1.0]])
        rot = rz @ ry @ rx
        if view == "lateral":
            ub, vb = np.array([0.0, 1.0, 0.0]), np.array([1.0, 0.0, 0.0])
        elif view == "ap":
            ub, vb = np.array([0.0, 0.0, 1.0]), np.array([1.0, 0.0, 0.0])
        else:
            ub, vb = np.array([0.0, 0.0, 1.0]), np.array([0.0, 1.0, 0.0])
        return rot @ ub, rot @ vb

    def _slices_device(self, specs):
        items, sizes, total = self._items(specs)
        out = torch.empty(total, dtype=torch.complex128, device=self._dev)
        max_n = max(sh * sw for sh, sw, _ in sizes)
        L.call("fvr_np_slices", L.ptr(self._f3d), self.pz, self.py, self.px, L.ptr(items), len(specs), max_n,
               L.ptr(out), L.stream_ptr(self._dev))
        return [out[o:o + sh * sw].view(sh, sw) for sh, sw, o in sizes]

    def extract_frequency_slice(self, yaw_deg=0.0, pitch_deg=0.0, roll_deg=0.0, tx=0.0, ty=0.0, view="lateral",
                                interp_order=1) -> np.ndarray:
        """Phase-ramped parallel-beam frequency slice (diff_fvr.py:106-150); tx, ty in voxels."""
        if interp_order != 1:
            raise L.FvrError("only linear interpolation (interp_order=1) is implemented on the GPU path")
        return self._slices_device([(yaw_deg, pitch_deg, roll_deg, tx, ty, view)])[0].cpu().numpy()

    def render_drr(self, yaw_deg=0.0, pitch_deg=0.0, roll_deg=0.0, tx=0.0, ty=0.0, view="lateral", interp_order=1,
                   crop_to_roi=True) -> np.ndarray:
        """Spatial DRR: fftshift(ifft2(ifftshift(slice))) * scale, ReLU, centre crop (diff_fvr.py:152-182)."""
        if interp_order != 1:
            raise L.FvrError("only linear interpolation (interp_order=1) is implemented on the GPU path")
        return self._drrs_device([(yaw_deg, pitch_deg, roll_deg, tx, ty, view)], crop_to_roi)[0].cpu().numpy()

    def _drrs_device(self, specs, crop_to_roi=True):
        """render_drr for several (yaw, pitch, roll, tx, ty, view) specs: every
        slice in one gather launch, then one inverse FFT per view; device
        float64 images."""
        slices = self._slices_device(specs)
        out = []
        for sl, spec in zip(slices, specs):
            view = spec[5]
            sh, sw = sl.shape
            scale = (self.pz * self.py * self.px) / (sh * sw)
            crop = (0, sh, 0, sw)
            if crop_to_roi:
                nz, ny, nx = self.orig_shape
                th = nz if view in ("lateral", "ap") else ny
                tw = ny if view == "lateral" else nx
                crop = ((sh - th) // 2, th, (sw - tw) // 2, tw)
            out.append(RT.fft2d(sl.contiguous(), inverse=True, in_shift=RT.SHIFT_IFFT, out_shift=RT.SHIFT_FFT,
                                scale=scale / (sh * sw), out_mode=RT.OUT_RELU, crop=crop))
        return out

    def _ncc_moments(self, specs, targets):
        """mom[item][5] for specs against device targets (list of complex128 [sh, sw])."""
        items, sizes, total = self._items(specs)
        tg = torch.empty(total, dtype=torch.complex128, device=self._dev)
        for (sh, sw, o), t in zip(sizes, targets):
            tg[o:o + sh * sw].copy_(t.reshape(-1))
        ws_bytes = L.query("fvr_np_ncc_workspace", len(specs))
        ws = torch.empty(ws_bytes, dtype=torch.uint8, device=self._dev)
        mom = torch.empty((len(specs), 5), dtype=torch.float64, device=self._dev)
        L.call("fvr_np_ncc_moments", L.ptr(self._f3d), self.pz, self.py, self.px, L.ptr(items), len(specs), L.ptr(tg),
               L.ptr(ws), ws_bytes, L.ptr(mom), L.stream_ptr(self._dev))
        return mom.cpu().numpy(), sizes

    def compute_spectral_ncc(self, f_slice_candidate, f_target_precomputed) -> float:
        """Parseval NCC Re<S, T> / (|S| |T|), 0 when a norm vanishes (diff_fvr.py:184-195)."""
        a = torch.as_tensor(np.asarray(f_slice_candidate), dtype=torch.complex128).to(self._dev)
        b = torch.as_tensor(np.asarray(f_target_precomputed), dtype=torch.complex128).to(self._dev)
        if a.shape != b.shape:
            raise ValueError("candidate and target spectra differ in shape")
        m = _pair_moments(a.reshape(a.shape[0], -1) if a.dim() >= 2 else a.reshape(1, -1),
                          b.reshape(b.shape[0], -1) if b.dim() >= 2 else b.reshape(1, -1))
        den = np.sqrt(m[1]) * np.sqrt(m[2])
        return 0.0 if den == 0 else float(m[0] / den)


def _pair_moments(a, b):
    """Five fp64 moments of two device complex128 [sh, sw] arrays (fvr_np_pair_moments)."""
    dev = a.device
    sh, sw = (int(a.shape[0]), int(a.shape[1])) if a.dim() == 2 else (1, int(a.numel()))
    ws_bytes = L.query("fvr_np_pair_workspace")
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    mom = torch.empty(5, dtype=torch.float64, device=dev)
    L.call("fvr_np_pair_moments", L.ptr(a.contiguous()), L.ptr(b.contiguous()), sh, sw, L.ptr(ws), ws_bytes,
           L.ptr(mom), L.stream_ptr(dev))
    return mom.cpu().numpy()


def prepare_target_spectrum(renderer: DifferentiableFourierVolumeRenderer, img: np.ndarray, view: str,
                            keep_on_device: bool = False):
    """Target spectrum for the NumPy-convention spectral NCC
    (RobustDiffFVREngine._prepare_spectrum, core_engine.py:71-85): the image
    zero-padded into the view's slice frame (lateral (pz, py), ap (pz, px),
    else (py, px); low-side offset (S - n) // 2) and
    ``fftshift(fft2(ifftshift(.)))`` in complex128, on the GPU.  Returns a
    NumPy array, or with ``keep_on_device`` the device tensor that
    ``compute_spectral_ncc`` style moments can use without a copy."""
    slice_h, slice_w = renderer._dims(view)
    im = np.asarray(img, dtype=np.float64)
    th, tw = im.shape
    if th > slice_h or tw > slice_w:
        raise ValueError(f"target {th}x{tw} does not fit the {slice_h}x{slice_w} slice frame")
    padded = torch.zeros((slice_h, slice_w), dtype=torch.float64, device=renderer._dev)
    sh, sw = (slice_h - th) // 2, (slice_w - tw) // 2
    padded[sh:sh + th, sw:sw + tw] = torch.from_numpy(np.ascontiguousarray(im)).to(renderer._dev)
    f = RT.fft2d(padded, inverse=False, in_shift=RT.SHIFT_IFFT, out_shift=RT.SHIFT_FFT)
    return f if keep_on_device else f.cpu().numpy()
