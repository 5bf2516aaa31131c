"""Batched multi-start 6-DoF biplanar registration on the PoU-FVR renderer.

The loop of the reference's GPU multi-start benchmark
(experiments/exp30_gpu_multistart_registration.py:42-55, 108-177): every
candidate pose theta = (w, t) (rad, mm) is mapped through the SE(3)
exponential, both views are rendered with ``forward_pinhole``, the loss per
candidate is 1 - 0.5 (sim_A + sim_B) with sim = 0.75 edge-dominant NCC +
0.25 image NCC, and all candidates run independent Adam steps together
(betas 0.8 / 0.99, gradient clamps 0.25 rad and 2.5 mm, learning rate
0.1 + 0.9 x cosine decay).  Here the SE(3) map and its adjoint, the renderer,
its adjoint and the edge NCC are ``libfvr_b200.so`` kernels, the Adam update
is written on tensors so one whole iteration is captured as a CUDA graph and
replayed.
"""
from __future__ import annotations

import math
from typing import Callable, Tuple

import numpy as np
import torch

from . import _lib as L
from .cone_beam_fvr import edge_dominant_ncc
from .graphs import no_gc_during_capture


class _SE3ExpFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta):
        dev = L.require_cuda(theta)
        th = theta.detach().to(torch.float32).contiguous()
        n = int(th.shape[0])
        mats = torch.empty((n, 4, 4), dtype=torch.float32, device=dev)
        L.call("fvr_se3_exp", L.ptr(th), n, L.ptr(mats), L.stream_ptr(dev))
        ctx.save_for_backward(th)
        ctx.dt = theta.dtype
        return mats

    @staticmethod
    def backward(ctx, g):
        (th,) = ctx.saved_tensors
        dev = th.device
        gm = g.detach().to(torch.float32).contiguous()
        gt = torch.empty_like(th)
        L.call("fvr_se3_exp_backward", L.ptr(th), L.ptr(gm), int(th.shape[0]), L.ptr(gt), L.stream_ptr(dev))
        return gt.to(ctx.dt)


def se3_exp(theta: torch.Tensor) -> torch.Tensor:
    """(N, 6) = [wx, wy, wz, tx, ty, tz] (rad, mm) -> (N, 4, 4) rigid matrices,
    exp of the rotation vector's skew matrix (exp30:42-55); differentiable."""
    return _SE3ExpFn.apply(theta)


def image_ncc(pred: torch.Tensor, target: torch.Tensor) -> torch.Tensor:
    """Per-item zero-mean NCC of [B, 1, H, W] images, denominator clamped at
    1e-12 before the square root (exp30:126-131)."""
    p0 = pred.float() - pred.float().mean(dim=(-2, -1), keepdim=True)
    r0 = target.float() - target.float().mean(dim=(-2, -1), keepdim=True)
    num = (p0 * r0).sum(dim=(-2, -1))
    den = (p0.square().sum(dim=(-2, -1)) * r0.square().sum(dim=(-2, -1))).clamp(min=1e-12).sqrt()
    return (num / den).squeeze(1)


def biplanar_loss_per_candidate(imA, imB, refA, refB) -> torch.Tensor:
    """1 - 0.5 (sim_A + sim_B), sim = 0.75 edge-dominant NCC + 0.25 image NCC
    (exp30:120-134); one value per candidate."""
    def pair(p, r):
        return 0.75 * edge_dominant_ncc(p.float(), r.float(), reduction="none") + 0.25 * image_ncc(p, r)

    return 1.0 - 0.5 * (pair(imA, refA) + pair(imB, refB))


def sample_multistart_theta(B: int, device, seed: int, rot_deg_lim: float = 12.0,
                            trans_mm_lim: float = 15.0) -> torch.Tensor:
    """(B, 6) multi-start seeds (rad, mm), index 0 at the unperturbed start (exp30:108-117)."""
    rng = np.random.default_rng(seed)
    theta = np.zeros((B, 6), dtype=np.float32)
    if B > 1:
        rot_lim = rot_deg_lim * (math.pi / 180.0)
        theta[1:, :3] = rng.uniform(-rot_lim, rot_lim, size=(B - 1, 3)).astype(np.float32)
        theta[1:, 3:] = rng.uniform(-trans_mm_lim, trans_mm_lim, size=(B - 1, 3)).astype(np.float32)
    return torch.from_numpy(theta).to(device=device)


class MultistartRegistration:
    """All candidates' Adam iterations for a biplanar pair rendered by
    ``render_pair(dT) -> (imA, imB)`` ([B, 1, H, W] each) against references
    ``refA``, ``refB`` ([1, 1, H, W]).  ``graph=True`` captures one iteration
    (render, loss, adjoint, Adam update) as a CUDA graph after ``warmup``
    eager iterations; every call of ``step()`` then replays it."""

    def __init__(self, render_pair: Callable[[torch.Tensor], Tuple[torch.Tensor, torch.Tensor]], refA, refB,
                 theta_init: torch.Tensor, steps: int, lr_rot: float = 0.02, lr_trans: float = 2.0,
                 betas=(0.8, 0.99), eps: float = 1e-8, graph: bool = True, warmup: int = 2):
        self.render_pair = render_pair
        self.refA, self.refB = refA, refB
        dev = theta_init.device
        self.theta = theta_init.detach().to(torch.float32).clone().contiguous()
        self.m = torch.zeros_like(self.theta)
        self.v = torch.zeros_like(self.theta)
        self.t = torch.zeros((), dtype=torch.float32, device=dev)  # completed Adam steps
        self.base_lr = torch.tensor([lr_rot] * 3 + [lr_trans] * 3, dtype=torch.float32, device=dev)
        self.clamp = torch.tensor([0.25] * 3 + [2.5] * 3, dtype=torch.float32, device=dev)
        self.t_max = float(max(1, steps))
        self.b1, self.b2, self.eps = float(betas[0]), float(betas[1]), float(eps)
        self._b1t = torch.tensor(self.b1, dtype=torch.float32, device=dev)
        self._b2t = torch.tensor(self.b2, dtype=torch.float32, device=dev)
        self.last_losses = torch.zeros(int(self.theta.shape[0]), dtype=torch.float32, device=dev)
        self._graph = None
        self._start = self.theta.clone()
        if graph:
            side = torch.cuda.Stream(device=dev)
            side.wait_stream(torch.cuda.current_stream(dev))
            with torch.cuda.stream(side):
                for _ in range(warmup):
                    self._iteration()
            torch.cuda.current_stream(dev).wait_stream(side)
            self.reset(self._start)
            self._graph = torch.cuda.CUDAGraph()
            with no_gc_during_capture(), torch.cuda.graph(self._graph, capture_error_mode="thread_local"):
                self._iteration()
            self.reset(self._start)

    def reset(self, theta: torch.Tensor) -> None:
        """Restart every candidate's Adam state from ``theta``."""
        with torch.no_grad():
            self.theta.copy_(theta)
            self.m.zero_()
            self.v.zero_()
            self.t.zero_()

    def _iteration(self) -> None:
        th = self.theta.detach().requires_grad_(True)
        imA, imB = self.render_pair(se3_exp(th))
        losses = biplanar_loss_per_candidate(imA, imB, self.refA, self.refB)
        (g,) = torch.autograd.grad(losses.sum(), th)
        with torch.no_grad():
            self.last_losses.copy_(losses.detach())
            g = torch.maximum(torch.minimum(g, self.clamp), -self.clamp)
            # the learning rate of this step (LambdaLR after `t` completed steps)
            lam = 0.1 + 0.45 * (1.0 + torch.cos(math.pi * torch.clamp(self.t, max=self.t_max) / self.t_max))
            self.t.add_(1.0)
            self.m.mul_(self.b1).add_(g, alpha=1.0 - self.b1)
            self.v.mul_(self.b2).addcmul_(g, g, value=1.0 - self.b2)
            bc1 = 1.0 - torch.pow(self._b1t, self.t)
            bc2 = 1.0 - torch.pow(self._b2t, self.t)
            step = (self.base_lr * lam) * (self.m / bc1) / ((self.v / bc2).sqrt() + self.eps)
            self.theta.sub_(step)

    def step(self) -> None:
        if self._graph is not None:
            self._graph.replay()
        else:
            self._iteration()

    def run(self, steps: int) -> None:
        for _ in range(steps):
            self.step()

    @torch.no_grad()
    def evaluate(self) -> Tuple[torch.Tensor, torch.Tensor]:
        """Per-candidate losses at the current poses, and the best candidate's theta [1, 6]."""
        imA, imB = self.render_pair(se3_exp(self.theta))
        losses = biplanar_loss_per_candidate(imA, imB, self.refA, self.refB)
        best = int(torch.argmin(losses))
        return losses, self.theta[best:best + 1].clone()


class MultiVolumeRegistration:
    """Every volume's multi-start registrations advanced together, one CUDA-graph
    replay per Adam iteration for all of them.

    ``problems`` lists, per volume, ``(model, lattice, initA, initB, refA, refB,
    theta0)``: a :class:`fvr.cone_beam_fvr.PerspectiveSlabFVR`, its pinhole
    lattice, the two views' base camera matrices ([1, 4, 4]), the reference
    images of each of that volume's initialisations ([I, 1, H, W] per view)
    and the starting candidates ([I * C, 6], C per initialisation, grouped by
    initialisation).  One iteration renders each volume's candidates in both
    views with one ``forward_pinhole`` call (views stacked along the pose
    axis), forms every candidate's loss against its own initialisation's
    references and takes the Adam step for all candidates of all volumes
    (the loop of exp30_gpu_multistart_registration.py:140-183, run over the
    uneven volumes and their initialisations at once instead of one after
    another)."""

    def __init__(self, problems, steps: int, **adam):
        self._vols = []
        thetas, refsA, refsB = [], [], []
        start = 0
        for model, lattice, initA, initB, refA, refB, theta0 in problems:
            n_init = int(refA.shape[0])
            n = int(theta0.shape[0])
            if n % n_init:
                raise ValueError("theta0 must hold the same number of candidates for every initialisation")
            per = n // n_init
            self._vols.append((model, lattice, initA, initB, slice(start, start + n), n_init, per))
            start += n
            thetas.append(theta0)
            refsA.append(refA.repeat_interleave(per, dim=0))
            refsB.append(refB.repeat_interleave(per, dim=0))
        self.total = start
        self.reg = MultistartRegistration(self._render_all, torch.cat(refsA).contiguous(),
                                          torch.cat(refsB).contiguous(), torch.cat(thetas), steps, **adam)

    def _render_all(self, dT):
        outA, outB = [], []
        for model, lattice, initA, initB, sl, _, _ in self._vols:
            d = dT[sl]
            n = int(d.shape[0])
            img = model.forward_pinhole(torch.cat([d @ initA, d @ initB]), lattice)
            outA.append(img[:n])
            outB.append(img[n:])
        return torch.cat(outA), torch.cat(outB)

    def run(self, steps: int) -> None:
        self.reg.run(steps)

    @torch.no_grad()
    def evaluate(self):
        """Per volume and initialisation: (best loss, best theta [6]) over its candidates."""
        losses, _ = self.reg.evaluate()
        out = []
        for _, _, _, _, sl, n_init, per in self._vols:
            lv = losses[sl].view(n_init, per)
            tv = self.reg.theta[sl].view(n_init, per, 6)
            best = torch.argmin(lv, dim=1)
            out.append([(float(lv[i, best[i]]), tv[i, best[i]].clone()) for i in range(n_init)])
        return out
