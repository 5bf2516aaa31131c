"""Seeded synthetic inputs standing in for CT data and candidate poses.

The reference benchmarks on clinical volumes (DeepFluoro, not available
offline); its shapes are reproduced with additive ellipsoid phantoms.
"""
from __future__ import annotations

import numpy as np


def make_ellipsoid_volume(n, seed, n_ellipsoids=12, shape=None):
    """Volume of ``n_ellipsoids`` additive ellipsoids, float32 ``(Z, Y, X)``.

    Per ellipsoid and axis: centre ~U(0.3 n, 0.7 n), semi-axis ~U(0.05 n, 0.2 n);
    attenuation ~U(0, 0.05) per mm.  ``numpy.random.default_rng(seed)``.
    """
    shape = tuple(shape) if shape is not None else (n, n, n)
    rng = np.random.default_rng(seed)
    vol = np.zeros(shape, np.float32)
    grids = np.meshgrid(*[np.arange(s, dtype=np.float32) for s in shape], indexing="ij")
    for _ in range(n_ellipsoids):
        c = [rng.uniform(0.3 * s, 0.7 * s) for s in shape]
        r = [rng.uniform(0.05 * s, 0.2 * s) for s in shape]
        mu = rng.uniform(0.0, 0.05)
        q = sum(((g - ci) / ri) ** 2 for g, ci, ri in zip(grids, c, r))
        vol += np.float32(mu) * (q <= 1.0)
    return vol


def make_poses(n, seed, rot_deg=10.0, trans_mm=5.0):
    """Poses ``[n, 6]`` (yaw, pitch, roll deg; tx, ty, tz mm): rotations U(+-rot_deg),
    translations U(+-trans_mm), ``numpy.random.default_rng(seed)``."""
    rng = np.random.default_rng(seed)
    p = np.zeros((n, 6), np.float32)
    p[:, :3] = rng.uniform(-rot_deg, rot_deg, (n, 3))
    p[:, 3:] = rng.uniform(-trans_mm, trans_mm, (n, 3))
    return p


def make_pinhole_mats(n, seed, sad_mm=765.0, rot_deg=10.0, trans_mm=5.0, device=None):
    """Camera-to-world matrices ``[n, 4, 4]`` for ``PerspectiveSlabFVR.forward_pinhole``:
    the camera (source at its origin, looking along +z) sits at distance
    ``sad_mm`` from the isocentre, rotated about it by U(+-rot_deg) per axis
    (rotation vector), then shifted by U(+-trans_mm) per axis."""
    import torch

    rng = np.random.default_rng(seed)
    rv = rng.uniform(-np.radians(rot_deg), np.radians(rot_deg), (n, 3))
    tj = rng.uniform(-trans_mm, trans_mm, (n, 3))
    mats = np.zeros((n, 4, 4), np.float64)
    for i in range(n):
        th = np.linalg.norm(rv[i])
        k = rv[i] / th if th > 0 else np.zeros(3)
        Kx = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
        R = np.eye(3) + np.sin(th) * Kx + (1 - np.cos(th)) * (Kx @ Kx)
        mats[i, :3, :3] = R
        mats[i, :3, 3] = R @ np.array([0.0, 0.0, -sad_mm]) + tj[i]
        mats[i, 3, 3] = 1.0
    return torch.from_numpy(mats.astype(np.float32)).to(device)
