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
