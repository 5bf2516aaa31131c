"""Articulated multi-vertebra model on B200 (drop-in for
``src/fvr/articulated_spine.py``).

Each vertebral segment keeps its own fp64 spectrum on the GPU (a
:class:`fvr.diff_fvr.DifferentiableFourierVolumeRenderer`).  By Fourier
linearity the spectrum of the articulated projection is the sum of the
segments' phase-ramped central slices, each at its own accumulated pose
(articulated_spine.py:39-71); here every view's sum is one launch of
``fvr_np_segment_slices`` for all segments at once, and the registration
objective (articulated_spine.py:87-163) keeps the spectra and the targets on
the device, bringing back five fp64 moments per view.
"""
from __future__ import annotations

import ctypes
import time
from typing import Any, Dict, List, Optional

import numpy as np
import torch

from . import _lib as L
from . import _runtime as RT
from .diff_fvr import DifferentiableFourierVolumeRenderer, _Item, _pair_moments, _view_code

_MAX_SEGMENTS = 16


class VertebralSegment:
    """An individually segmented vertebra in 3D Fourier space (articulated_spine.py:20-28)."""

    def __init__(self, name: str, sub_volume: np.ndarray, nominal_offset_z: float, pad_factor: float = 2.0,
                 device: Optional[torch.device] = None):
        self.name = name
        self.nominal_offset_z = nominal_offset_z
        self.renderer = DifferentiableFourierVolumeRenderer(sub_volume, pad_factor=pad_factor, device=device)
        self.shape = sub_volume.shape


def _view_spec(pose, view):
    """(yaw, pitch, roll, in-plane tx, ty, view) of one segment pose for a view
    (articulated_spine.py:60-68: lateral uses (ty, tz), ap (tx, tz), else the
    axial slice with (tx, ty))."""
    yaw, pitch, roll, tx, ty, tz = (float(x) for x in pose)
    if view == "lateral":
        return yaw, pitch, roll, ty, tz, "lateral"
    if view == "ap":
        return yaw, pitch, roll, tx, tz, "ap"
    return yaw, pitch, roll, tx, ty, "axial"


class ArticulatedSpineModel:
    """Hierarchical articulated spine model with physiological joint bounds
    (articulated_spine.py:31-163)."""

    def __init__(self, segments: List[VertebralSegment]):
        self.segments = segments
        self.num_segments = len(segments)
        if not 1 <= self.num_segments <= _MAX_SEGMENTS:
            raise L.FvrError(f"between 1 and {_MAX_SEGMENTS} segments are supported, got {self.num_segments}")
        r0 = segments[0].renderer
        self._shape = (r0.pz, r0.py, r0.px)
        for s in segments[1:]:
            if (s.renderer.pz, s.renderer.py, s.renderer.px) != self._shape:
                raise ValueError("every segment spectrum must have the same padded shape")
            if s.renderer._dev != r0._dev:
                raise ValueError("every segment spectrum must live on the same device")
        self._dev = r0._dev
        self._ptrs = (ctypes.c_void_p * self.num_segments)(*[L.ptr(s.renderer._f3d) for s in segments])

    def _segment_poses(self, base_pose, relative_articulations):
        """Pose of every segment: the base pose plus the accumulated relative
        articulations of the joints below it (articulated_spine.py:55-59)."""
        curr = np.array(base_pose, dtype=np.float64).copy()
        poses = []
        for i in range(self.num_segments):
            if i > 0 and len(relative_articulations) >= i:
                curr = curr + np.asarray(relative_articulations[i - 1], dtype=np.float64)
            poses.append(curr.copy())
        return poses

    def _sum_shape(self, view):
        pz, py, px = self._shape
        return pz, (py if view == "lateral" else px)

    def _spectra_device(self, base_pose, relative_articulations, views):
        """Device complex128 [sh, sw] articulated spectrum per view, all in one launch."""
        poses = self._segment_poses(base_pose, relative_articulations)
        r0 = self.segments[0].renderer
        n_seg = self.num_segments
        arr = (_Item * (len(views) * n_seg))()
        sizes, off = [], 0
        for o, view in enumerate(views):
            sh, sw = self._sum_shape(view)
            for s, pose in enumerate(poses):
                yaw, pitch, roll, tx, ty, v = _view_spec(pose, view)
                ssh, ssw = r0._dims(v)
                if (ssh, ssw) != (sh, sw):  # the reference's += of a differently shaped slice fails the same way
                    raise ValueError(f"operands could not be broadcast together with shapes ({sh},{sw}) ({ssh},{ssw})")
                arr[o * n_seg + s] = _Item(yaw, pitch, roll, tx, ty, _view_code(v), sh, sw, 0, off)
            sizes.append((sh, sw, off))
            off += sh * sw
        items = torch.frombuffer(bytearray(arr), dtype=torch.uint8).to(self._dev)
        out = torch.empty(off, dtype=torch.complex128, device=self._dev)
        pz, py, px = self._shape
        L.call("fvr_np_segment_slices", self._ptrs, n_seg, pz, py, px, L.ptr(items), len(views),
               max(sh * sw for sh, sw, _ in sizes), L.ptr(out), L.stream_ptr(self._dev))
        return [out[o:o + sh * sw].view(sh, sw) for sh, sw, o in sizes]

    def render_articulated_spectrum(self, base_pose: np.ndarray, relative_articulations: List[np.ndarray],
                                    view: str = "lateral") -> np.ndarray:
        """Combined 2D spectrum of the articulated spine by Fourier linearity
        (articulated_spine.py:39-71)."""
        return self._spectra_device(base_pose, relative_articulations, [view])[0].cpu().numpy()

    def render_drr(self, base_pose: np.ndarray, relative_articulations: List[np.ndarray],
                   view: str = "lateral") -> np.ndarray:
        """max(real(fftshift(ifft2(ifftshift(F)))), 0) of the articulated
        spectrum (articulated_spine.py:73-85)."""
        f = self._spectra_device(base_pose, relative_articulations, [view])[0]
        sh, sw = int(f.shape[0]), int(f.shape[1])
        img = RT.fft2d(f.contiguous(), inverse=True, in_shift=RT.SHIFT_IFFT, out_shift=RT.SHIFT_FFT,
                       scale=1.0 / (sh * sw), out_mode=RT.OUT_RELU)
        return img.cpu().numpy()

    def _biplanar_loss(self, pose, arts, t_ap, t_lat):
        f_ap, f_lat = self._spectra_device(pose, arts, ["ap", "lateral"])
        loss = 0.0
        for f, t in ((f_ap, t_ap), (f_lat, t_lat)):
            if f.shape != t.shape:
                raise ValueError("candidate and target spectra differ in shape")
            m = _pair_moments(f, t)
            den = np.sqrt(m[1]) * np.sqrt(m[2])
            ncc = 0.0 if den == 0 else float(m[0] / den)
            loss += 0.5 * (1.0 - ncc)
        return loss

    def register_articulated_biplanar(self, f_target_ap: np.ndarray, f_target_lat: np.ndarray,
                                      init_base_pose: np.ndarray, max_iter_global: int = 40,
                                      max_iter_local: int = 30) -> Dict[str, Any]:
        """Two-stage hierarchical articulated registration (articulated_spine.py:87-163):
        Powell on the rigid base pose with every joint locked, then Powell on
        the joint articulations with a 1e-4 strain prior."""
        from scipy.optimize import minimize

        t0 = time.time()
        num_joints = self.num_segments - 1
        t_ap = torch.as_tensor(np.asarray(f_target_ap), dtype=torch.complex128).to(self._dev)
        t_lat = torch.as_tensor(np.asarray(f_target_lat), dtype=torch.complex128).to(self._dev)
        zero_art = [np.zeros(6) for _ in range(num_joints)]

        def stage1_obj(pose):
            return float(self._biplanar_loss(pose, zero_art, t_ap, t_lat))

        res1 = minimize(stage1_obj, x0=init_base_pose, method="Powell",
                        options={"maxiter": max_iter_global, "ftol": 1e-4})
        base = res1.x
        if num_joints > 0:
            def stage2_obj(art_flat):
                arts = [art_flat[j * 6:(j + 1) * 6] for j in range(num_joints)]
                return float(self._biplanar_loss(base, arts, t_ap, t_lat) + 1e-4 * np.sum(art_flat ** 2))

            res2 = minimize(stage2_obj, x0=np.zeros(num_joints * 6), method="Powell",
                            options={"maxiter": max_iter_local, "ftol": 1e-4})
            arts = [res2.x[j * 6:(j + 1) * 6] for j in range(num_joints)]
            final_loss = float(res2.fun)
        else:
            arts = []
            final_loss = float(res1.fun)
        return {"base_pose": base, "articulations": arts, "final_loss": final_loss, "time_sec": time.time() - t0,
                "stage1_success": res1.success}
