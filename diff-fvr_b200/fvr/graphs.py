"""CUDA-graph capture of whole optimiser / screening steps.

The reference speeds its forward up with ``torch.compile(mode="reduce-overhead")``
and a forward-only CUDA graph (src/fvr/torch_engine.py:97-106,
experiments/exp29_gpu_triton_and_ablation.py:136-151).  Here the fused kernels
need no compiler; a step (forward losses *and* the pose gradient) is captured
once and replayed, which removes every per-kernel launch and Python cost.
"""
from __future__ import annotations

import torch

from . import _lib as L


class GraphedCallable:
    """Capture ``fn(*static_inputs)`` in one CUDA graph; calling copies the new
    inputs into the static buffers and replays.  Outputs are the static output
    tensors of the capture (overwritten by the next call)."""

    def __init__(self, fn, *example_inputs, warmup=3, capture_context=None):
        import contextlib

        for x in example_inputs:
            L.require_cuda(x)
        self.fn = fn
        self.static_in = [x.detach().clone() for x in example_inputs]
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            for _ in range(max(1, int(warmup))):
                fn(*self.static_in)
        torch.cuda.current_stream().wait_stream(side)
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        n0 = L.launch_count[0]
        with capture_context if capture_context is not None else contextlib.nullcontext():
            with torch.cuda.graph(self.graph):
                self.static_out = fn(*self.static_in)
        self.kernels_per_replay = L.launch_count[0] - n0

    def replay(self):
        self.graph.replay()
        return self.static_out

    def __call__(self, *inputs):
        for s, x in zip(self.static_in, inputs):
            s.copy_(x, non_blocking=True)
        return self.replay()


class BiplanarSpectralNCCStep:
    """``loss = forward_spectral_ncc(AP) + forward_spectral_ncc(lateral)`` and
    ``dloss/dposes`` for a batch of candidate poses on a
    :class:`fvr.torch_engine.TorchDiffFVREngine`, as one callable: one fused
    gather pass over both views, an fp64 finalize, an fp64 pose-gradient
    epilogue.

    With ``graph=True`` (default) the whole step is a single CUDA-graph replay
    that uses the engine's spectrum storage of the time of capture (the step
    keeps that storage alive; capture again after ``to_precision``).
    Returns ``(loss, grad)`` device tensors (scalar, ``[C, 6]``).
    """

    def __init__(self, engine, f_targ_ap, f_targ_lat, n_candidates, high_pass=True, cutoff_sigma=4.0, graph=True,
                 warmup=3, capture_context=None):
        self.engine = engine
        self._stencil = engine._stencil
        self.f_ap = f_targ_ap
        self.f_lat = f_targ_lat
        self.hp = bool(high_pass)
        self.sigma = float(cutoff_sigma)
        ex = torch.zeros((int(n_candidates), 6), dtype=torch.float32, device=engine._dev)
        self._g = GraphedCallable(self._step, ex, warmup=warmup, capture_context=capture_context) if graph else None

    def _step(self, poses):
        return self.engine.spectral_ncc_value_and_grad(poses, (self.f_ap, self.f_lat), ("ap", "lateral"),
                                                       high_pass=self.hp, cutoff_sigma=self.sigma)

    def __call__(self, poses):
        if self._g is None:
            return self._step(poses.to(self.engine._dev))
        return self._g(poses)
