"""Adam registration on the analytical Fourier gradients of the
NumPy-convention renderer, on B200 (drop-in for
``GradientRegistrationOptimizer``, src/fvr/gradient_optimizer.py).

Each iteration is one ``SpectralGradientEngine.compute_biplanar_loss_and_gradients``
call (the 14 slices of the loss and its 6-DOF gradient gathered and reduced in
one fp64 launch); the Adam state is six host doubles.
"""
from __future__ import annotations

import time
from typing import Any, Dict

import numpy as np

from .gradients import SpectralGradientEngine

_BETA1, _BETA2, _EPS = 0.9, 0.999, 1e-8


class GradientRegistrationOptimizer:
    """Biplanar 6-DOF registration with Adam (gradient_optimizer.py:15-90)."""

    def __init__(self, renderer):
        self.renderer = renderer
        self.grad_engine = SpectralGradientEngine(renderer)

    def register_adam(self, f_target_ap: np.ndarray, f_target_lat: np.ndarray, init_pose: np.ndarray,
                      lr_rot: float = 0.25, lr_trans: float = 0.35, max_iter: int = 40,
                      tol: float = 1e-4) -> Dict[str, Any]:
        """Adam with separate step sizes for rotations (degrees) and
        translations (voxels), bias-corrected moments, rotations kept in
        +-20 deg and translations in +-25 after every step; stops when no
        coordinate moves by ``tol`` or more.  Returns the best pose seen and
        the per-iteration trajectory ``(step, loss, pose)``."""
        t0 = time.time()
        pose = np.array(init_pose, dtype=np.float64, copy=True)
        m1 = np.zeros(6)
        m2 = np.zeros(6)
        lr = np.array([lr_rot] * 3 + [lr_trans] * 3, dtype=np.float64)
        trajectory = []
        best_loss, best_pose = float("inf"), pose.copy()
        step = 0
        for step in range(1, int(max_iter) + 1):
            loss, grad = self.grad_engine.compute_biplanar_loss_and_gradients(pose, f_target_ap, f_target_lat)
            trajectory.append((step, loss, pose.copy()))
            if loss < best_loss:
                best_loss, best_pose = loss, pose.copy()
            m1 = _BETA1 * m1 + (1.0 - _BETA1) * grad
            m2 = _BETA2 * m2 + (1.0 - _BETA2) * grad * grad
            move = lr * (m1 / (1.0 - _BETA1 ** step)) / (np.sqrt(m2 / (1.0 - _BETA2 ** step)) + _EPS)
            pose = pose - move
            pose[:3] = np.clip(pose[:3], -20.0, 20.0)
            pose[3:] = np.clip(pose[3:], -25.0, 25.0)
            if np.max(np.abs(move)) < tol:
                break
        return {"success": bool(best_loss < 0.05), "final_pose": best_pose, "final_loss": float(best_loss),
                "iterations": step, "evaluations": step * 7, "time_sec": time.time() - t0,
                "trajectory": trajectory}
