"""Parallel-beam biplanar registration on the NumPy-convention renderer, on
B200 (drop-in for ``RobustDiffFVREngine`` and ``detect_radio_opaque_metal``,
src/fvr/core_engine.py).

Same constructor checks, methods, pose units (degrees; millimetres at this
API, voxels inside the renderer) and result dictionary as the reference.
The optimiser is the same bounded Powell search (``scipy.optimize.minimize``,
a host-side driver of at most a few hundred objective calls); every objective
evaluation runs on the GPU in fp64:

* clean targets: both views' slices gathered and reduced against their
  target spectra in one launch (``fvr_np_ncc_moments``), five moments per
  view copied back;
* targets with radio-opaque metal (more than 3 % saturated pixels): both
  DRRs rendered by one slice launch and two inverse FFTs, and the masked
  normalised cross-correlation reduced on the device.
"""
from __future__ import annotations

import time
from typing import Any, Dict, Optional, Tuple

import numpy as np
import torch

from . import _runtime as RT
from .diff_fvr import DifferentiableFourierVolumeRenderer, prepare_target_spectrum


def _saturated(img, threshold):
    """Pixels whose min-max normalised value reaches ``threshold``, on the device."""
    t = img if isinstance(img, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(img, dtype=np.float64))
    t = t.to(device=RT.device_of(t.device if t.is_cuda else None), dtype=torch.float64)
    lo, hi = t.min(), t.max()
    return (t - lo) / (hi - lo + 1e-8) >= threshold


def detect_radio_opaque_metal(img: np.ndarray, saturation_threshold: float = 0.98) -> np.ndarray:
    """Boolean mask of saturated plateaus (dense surgical hardware): pixels whose
    min-max normalised intensity is at least ``saturation_threshold``
    (core_engine.py:21-27)."""
    return _saturated(img, saturation_threshold).cpu().numpy()


def _masked_zscore_ncc(d, valid, t_norm):
    """mean(z(d[valid]) * t_norm) with z the population z-score (+1e-8 in the
    denominator), on the device."""
    x = d[valid]
    z = (x - x.mean()) / (x.std(unbiased=False) + 1e-8)
    return (z * t_norm).mean()


class RobustDiffFVREngine:
    """Parallel-beam 6-DOF registration on a cubic, isotropic volume
    (core_engine.py:30-224).  Spacing is (Z, Y, X) in mm; poses are (yaw,
    pitch, roll, tx, ty, tz), degrees and mm."""

    def __init__(self, volume: np.ndarray, spacing: Tuple[float, float, float] = (1.0, 1.0, 1.0),
                 pad_factor: float = 2.0, sdd_mm: Optional[float] = None, sad_mm: Optional[float] = None,
                 device: Optional[torch.device] = None):
        if sdd_mm is not None or sad_mm is not None:
            raise ValueError('Only parallel-beam geometry is supported; SDD/SAD calibration is not implemented.')
        spacing = np.asarray(spacing, dtype=float)
        if spacing.shape != (3,) or not np.all(np.isfinite(spacing)) or np.any(spacing <= 0):
            raise ValueError('spacing must contain three finite positive values in mm (Z, Y, X).')
        if not np.allclose(spacing, spacing[0], rtol=1e-6, atol=0):
            raise ValueError('Resample the volume to isotropic spacing before registration.')
        volume = np.asarray(volume)
        if volume.ndim != 3 or len(set(volume.shape)) != 1 or min(volume.shape) < 2:
            raise ValueError('Use a cubic 3D volume with at least two voxels per axis.')
        if not np.all(np.isfinite(volume)):
            raise ValueError('volume must contain only finite values.')
        self.volume = volume.astype(np.float64)
        self.spacing = tuple(float(s) for s in spacing)
        self.renderer = DifferentiableFourierVolumeRenderer(self.volume, pad_factor=pad_factor,
                                                            apply_premultiplication=True, device=device)

    def detect_metal_hardware_mask(self, img: np.ndarray, threshold: float = 0.98) -> np.ndarray:
        """True where the pixel is NOT occluded by metal (core_engine.py:68-70)."""
        return ~detect_radio_opaque_metal(img, saturation_threshold=threshold)

    def _prepare_spectrum(self, img: np.ndarray, view: str) -> np.ndarray:
        """Target spectrum in the view's slice frame (core_engine.py:71-85)."""
        return prepare_target_spectrum(self.renderer, img, view)

    def render_calibrated_drr(self, yaw: float = 0.0, pitch: float = 0.0, roll: float = 0.0, tx: float = 0.0,
                              ty: float = 0.0, view: str = 'lateral', crop_to_roi: bool = True) -> np.ndarray:
        """Parallel-beam DRR; tx, ty are in-view translations in mm (core_engine.py:87-107)."""
        if view not in ('ap', 'lateral', 'axial'):
            raise ValueError('view must be ap, lateral or axial.')
        return self.renderer.render_drr(yaw_deg=yaw, pitch_deg=pitch, roll_deg=roll, tx=tx / self.spacing[0],
                                        ty=ty / self.spacing[0], view=view, crop_to_roi=crop_to_roi)

    def _view_specs(self, p):
        """(AP, lateral) renderer specs of a pose in mm: AP takes (tx, tz), the
        lateral view (ty, tz), both in voxels."""
        yaw, pitch, roll = (float(x) for x in p[:3])
        tx, ty, tz = (float(x) / self.spacing[0] for x in p[3:])
        return [(yaw, pitch, roll, tx, tz, 'ap'), (yaw, pitch, roll, ty, tz, 'lateral')]

    def register_biplanar_robust(self, target_ap: np.ndarray, target_lat: np.ndarray,
                                 initial_pose: Tuple[float, float, float, float, float, float] = (0.0,) * 6,
                                 handle_metal: bool = True, max_iter: int = 50, bounds_trans_mm: float = 25.0,
                                 bounds_rot_deg: float = 20.0) -> Dict[str, Any]:
        """Bounded Powell search over the biplanar loss 0.5 (1 - NCC_AP) +
        0.5 (1 - NCC_LAT) (core_engine.py:109-224): spectral NCC on clean
        targets, masked image NCC on the unoccluded pixels when more than 3 %
        of either target is saturated metal."""
        from scipy.optimize import minimize

        for name, target in (('AP', target_ap), ('lateral', target_lat)):
            if target.shape != self.volume.shape[:2] or not np.all(np.isfinite(target)):
                raise ValueError(f'{name} target must be finite with shape {self.volume.shape[:2]}; '
                                 'match the parallel-beam projection grid before registration.')
            if np.ptp(target) == 0:
                raise ValueError(f'{name} target must contain intensity variation for registration.')
        initial_pose = np.asarray(initial_pose, dtype=float)
        if initial_pose.shape != (6,) or not np.all(np.isfinite(initial_pose)):
            raise ValueError('initial_pose must contain six finite values.')
        if not np.all(np.isfinite([bounds_trans_mm, bounds_rot_deg])) or min(bounds_trans_mm, bounds_rot_deg) <= 0:
            raise ValueError('Translation and rotation bounds must be finite and positive.')
        if max_iter < 1:
            raise ValueError('max_iter must be positive.')
        t0 = time.time()
        evals = [0]
        dev = self.renderer._dev
        if handle_metal:
            m_ap, m_lat = _saturated(target_ap, 0.98), _saturated(target_lat, 0.98)
            metal_present = bool(float(m_ap.double().mean()) > 0.03 or float(m_lat.double().mean()) > 0.03)
        else:
            metal_present = False
        bounds = [(-bounds_rot_deg, bounds_rot_deg)] * 3 + [(-bounds_trans_mm, bounds_trans_mm)] * 3

        if metal_present:
            valid = (~m_ap, ~m_lat)
            t_norm = []
            for tgt, ok in zip((target_ap, target_lat), valid):
                x = torch.from_numpy(np.ascontiguousarray(tgt, dtype=np.float64)).to(dev)[ok]
                t_norm.append((x - x.mean()) / (x.std(unbiased=False) + 1e-8))

            def objective(p):
                evals[0] += 1
                d_ap, d_lat = self.renderer._drrs_device(self._view_specs(p))
                n_ap = _masked_zscore_ncc(d_ap, valid[0], t_norm[0])
                n_lat = _masked_zscore_ncc(d_lat, valid[1], t_norm[1])
                return float(0.5 * (1.0 - n_ap) + 0.5 * (1.0 - n_lat))
        else:
            f_ap = prepare_target_spectrum(self.renderer, target_ap, 'ap', keep_on_device=True)
            f_lat = prepare_target_spectrum(self.renderer, target_lat, 'lateral', keep_on_device=True)

            def objective(p):
                evals[0] += 1
                mom, _ = self.renderer._ncc_moments(self._view_specs(p), [f_ap, f_lat])
                ncc = [0.0 if m[1] * m[2] == 0 else m[0] / (np.sqrt(m[1]) * np.sqrt(m[2])) for m in mom]
                return float(0.5 * (1.0 - ncc[0]) + 0.5 * (1.0 - ncc[1]))

        res = minimize(objective, x0=np.array(initial_pose), method='Powell', bounds=bounds,
                       options={'maxiter': max_iter, 'ftol': 1e-4})
        return {'success': bool(res.success), 'final_pose': res.x, 'final_loss': float(res.fun),
                'evaluations': evals[0], 'metal_detected': metal_present, 'time_sec': time.time() - t0}
