"""Volume ingest on B200: the array side of ``src/fvr/dicom_loader.py``.

``resample_isotropic_cube``, ``hu_to_attenuation`` and ``create_spine_phantom``
keep the reference's signatures, checks and NumPy-in / NumPy-out contract
(dicom_loader.py:11-30, 114-188) and run on the GPU (``fvr_ingest_resample``,
``fvr_hu_to_attenuation``, ``fvr_spine_phantom``).  ``attenuation_cube`` fuses the two into one pass
and returns the device tensor, which a :class:`fvr.TorchDiffFVREngine` or a
:class:`fvr.cone_beam_fvr.PerspectiveSlabFVR` takes directly, so a CT goes
from HU to the spectrum precompute without a host round trip.  Reading DICOM
or NIfTI files (pydicom / SimpleITK) stays on the host and is not part of
this package.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import numpy as np
import torch

from . import _lib as L
from . import _runtime as RT


def _check(volume_hu, spacing, target_res):
    volume_hu = np.asarray(volume_hu)
    spacing = np.asarray(spacing, dtype=float)
    if volume_hu.ndim != 3 or min(volume_hu.shape) < 2 or not np.all(np.isfinite(volume_hu)):
        raise ValueError('CT must be a finite 3D array with at least two voxels per axis.')
    if spacing.shape != (3,) or not np.all(np.isfinite(spacing)) or np.any(spacing <= 0):
        raise ValueError('spacing must contain three finite positive values in mm (Z, Y, X).')
    if not isinstance(target_res, (int, np.integer)) or target_res < 2:
        raise ValueError('target_res must be an integer of at least two.')
    return volume_hu, spacing


def _resample(volume_hu, spacing, target_res, to_mu, device):
    dev = RT.device_of(device)
    hu = torch.as_tensor(np.ascontiguousarray(volume_hu, dtype=np.float32)).to(dev)
    n = int(target_res)
    out = torch.empty((n, n, n), dtype=torch.float32, device=dev)
    vmm = ctypes.c_double(0.0)
    Z, Y, X = (int(s) for s in hu.shape)
    L.call("fvr_ingest_resample", L.ptr(hu), Z, Y, X, float(spacing[0]), float(spacing[1]), float(spacing[2]), n,
           int(to_mu), L.ptr(out), ctypes.byref(vmm), L.stream_ptr(dev))
    return out, float(vmm.value)


def resample_isotropic_cube(volume_hu, spacing, target_res, device: Optional[torch.device] = None):
    """Centre a CT in a cubic grid without cropping its physical field of view
    (dicom_loader.py:11-30): HU data [target_res]^3 (float32) and its
    (Z, Y, X) spacing in mm; outside the acquired CT is air (-1000 HU)."""
    volume_hu, spacing = _check(volume_hu, spacing, target_res)
    out, vmm = _resample(volume_hu, spacing, target_res, False, device)
    return out.cpu().numpy(), (vmm,) * 3


def hu_to_attenuation(volume_hu: np.ndarray, device: Optional[torch.device] = None) -> np.ndarray:
    """mu = max(0, (HU + 1000) / 1000) as float32 (dicom_loader.py:179-188)."""
    dev = RT.device_of(device)
    hu = torch.as_tensor(np.ascontiguousarray(volume_hu, dtype=np.float32)).to(dev)
    out = torch.empty_like(hu)
    L.call("fvr_hu_to_attenuation", L.ptr(hu), int(hu.numel()), L.ptr(out), L.stream_ptr(dev))
    return out.cpu().numpy()


def create_spine_phantom(size: int = 128, device: Optional[torch.device] = None):
    """Synthetic CT of a torso with five vertebrae in HU (dicom_loader.py:114-176):
    ``(volume [size]^3 float32 (Z, Y, X), spacing (1.0, 1.0, 1.0) mm)``.
    Air is -1000 HU, the torso 40, cortical bone 1100, trabecular bone 400,
    the spinal canal 15, spinous processes 900 and transverse processes 850;
    the labels equal the reference's float32 construction voxel for voxel."""
    dev = RT.device_of(device)
    n = int(size)
    out = torch.empty((n, n, n), dtype=torch.float32, device=dev)
    L.call("fvr_spine_phantom", n, L.ptr(out), L.stream_ptr(dev))
    return out.cpu().numpy(), (1.0, 1.0, 1.0)


def attenuation_cube(volume_hu, spacing, target_res,
                     device: Optional[torch.device] = None) -> Tuple[torch.Tensor, Tuple[float, float, float]]:
    """``hu_to_attenuation(resample_isotropic_cube(...))`` in one GPU pass:
    the float32 attenuation cube as a device tensor and its spacing (mm)."""
    volume_hu, spacing = _check(volume_hu, spacing, target_res)
    out, vmm = _resample(volume_hu, spacing, target_res, True, device)
    return out, (vmm,) * 3
