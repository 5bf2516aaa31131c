"""Spectral-NCC loss and 6-DOF gradient of the NumPy-convention renderer on
B200 (drop-in for ``SpectralGradientEngine``, src/fvr/gradients.py).

All 14 slices of one call (AP and lateral at the pose, and at +-delta for
each rotation) are gathered and reduced against their targets in a single
fp64 kernel launch; the closed-form translation gradient comes from the
same moments.  Only the 14 x 5 moments are copied back.
"""
from __future__ import annotations

from typing import Tuple

import numpy as np
import torch


class SpectralGradientEngine:
    """Analytical translation and finite-difference rotation gradients of the
    biplanar spectral NCC (gradients.py:13-135)."""

    def __init__(self, renderer):
        self.renderer = renderer
        self.pz = renderer.pz
        self.py = renderer.py
        self.px = renderer.px
        self.orig_shape = renderer.orig_shape

    @staticmethod
    def _ncc_grad(m, sh, sw):
        """(ncc, d ncc/du, d ncc/dv) from the moments (gradients.py:45-74)."""
        cross, es, et, iu, iv = m
        ns, nt = np.sqrt(es), np.sqrt(et)
        if ns * nt == 0:
            return 0.0, 0.0, 0.0
        # Re sum(-2 pi i (u/W) S conj(r_res)) with r_res = (T - ncc |T|/|S| S)/(|S||T|)
        return float(cross / (ns * nt)), float(2.0 * np.pi / sw * iu / (ns * nt)), \
            float(2.0 * np.pi / sh * iv / (ns * nt))

    def compute_spectral_ncc_and_grad_translation(self, f_cand, f_target, view="lateral") -> Tuple[float, float, float]:
        """NCC of a candidate slice against a target and its exact in-plane
        translation gradient (gradients.py:27-74); view only names the axes."""
        from .diff_fvr import _pair_moments

        dev = self.renderer._dev
        a = torch.as_tensor(np.asarray(f_cand), dtype=torch.complex128).to(dev)
        b = torch.as_tensor(np.asarray(f_target), dtype=torch.complex128).to(dev)
        return self._ncc_grad(_pair_moments(a, b), int(a.shape[0]), int(a.shape[1]))

    def compute_biplanar_loss_and_gradients(self, pose, f_target_ap, f_target_lat,
                                            delta_rot_deg: float = 0.2) -> Tuple[float, np.ndarray]:
        """L = 0.5 (1 - NCC_AP) + 0.5 (1 - NCC_LAT) and [dL/dyaw, dL/dpitch,
        dL/droll, dL/dtx, dL/dty, dL/dtz] (gradients.py:76-135)."""
        r = self.renderer
        yaw, pitch, roll, tx, ty, tz = (float(x) for x in pose)
        base = np.array([yaw, pitch, roll], dtype=np.float64)
        specs = [(yaw, pitch, roll, tx, tz, "ap"), (yaw, pitch, roll, ty, tz, "lateral")]
        for i in range(3):
            pp, pm = base.copy(), base.copy()
            pp[i] += delta_rot_deg
            pm[i] -= delta_rot_deg
            specs += [(*pp, tx, tz, "ap"), (*pm, tx, tz, "ap"), (*pp, ty, tz, "lateral"), (*pm, ty, tz, "lateral")]
        dev = r._dev
        t_ap = torch.as_tensor(np.asarray(f_target_ap), dtype=torch.complex128).to(dev)
        t_lat = torch.as_tensor(np.asarray(f_target_lat), dtype=torch.complex128).to(dev)
        targets = [t_ap if s[5] == "ap" else t_lat for s in specs]
        mom, sizes = r._ncc_moments(specs, targets)
        res = [self._ncc_grad(mom[k], sizes[k][0], sizes[k][1]) for k in range(len(specs))]
        ncc_ap, d_ap_dtx, d_ap_dtz = res[0]
        ncc_lat, d_lat_dty, d_lat_dtz = res[1]
        loss = 0.5 * (1.0 - ncc_ap) + 0.5 * (1.0 - ncc_lat)
        grad_rot = np.zeros(3)
        for i in range(3):
            k = 2 + 4 * i
            d_ap = (res[k][0] - res[k + 1][0]) / (2.0 * delta_rot_deg)
            d_lat = (res[k + 2][0] - res[k + 3][0]) / (2.0 * delta_rot_deg)
            grad_rot[i] = -0.5 * (d_ap + d_lat)
        grad = np.array([grad_rot[0], grad_rot[1], grad_rot[2], -0.5 * d_ap_dtx, -0.5 * d_lat_dty,
                         -0.5 * (d_ap_dtz + d_lat_dtz)], dtype=np.float64)
        return float(loss), grad
