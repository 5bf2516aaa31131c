"""CUDA-graph capture of whole optimiser / screening steps.

The reference speeds its forward up with ``torch.compile(mode="reduce-overhead")``
and a forward-only CUDA graph (src/fvr/torch_engine.py:97-106,
experiments/exp29_gpu_triton_and_ablation.py:136-151).  Here the fused kernels
need no compiler; a step (forward losses *and* the pose gradient) is captured
once and replayed, which removes every per-kernel launch and Python cost.
"""
from __future__ import annotations

import contextlib
import functools
import gc

import torch

from . import _lib as L


def _copy_kernel(dst, src):
    """dst <- src (same bytes) by fvr_copy_bytes on the current stream: pinned
    host buffers are read or written by the kernel itself over the bus, which
    costs a small kernel node instead of a copy-engine memcpy node."""
    if dst.numel() * dst.element_size() != src.numel() * src.element_size():
        raise L.FvrError("copy between buffers of different sizes")
    L.call("fvr_copy_bytes", L.ptr(dst), L.ptr(src.contiguous()), int(dst.numel() * dst.element_size()),
           L.stream_ptr())


@contextlib.contextmanager
def no_gc_during_capture():
    """Collect garbage now and keep the cyclic collector off until the block
    ends: collecting an unreachable object that owns a CUDA graph destroys
    that graph, which a capturing stream does not permit (the capture would
    be invalidated)."""
    gc.collect()
    enabled = gc.isenabled()
    gc.disable()
    try:
        yield
    finally:
        if enabled:
            gc.enable()


class GraphedCallable:
    """Capture ``fn(*static_inputs)`` in one CUDA graph; calling copies the new
    inputs into the static buffers and replays.  Outputs are the static output
    tensors of the capture (overwritten by the next call).

    With ``host_io=True`` the graph also holds the transfers: pinned host
    input buffers (``host_in``) are copied to the device, ``fn`` runs, and its
    outputs are copied into pinned host buffers (``host_out``), so one replay
    is the whole host-to-host step; the copies are kernels that read or write
    the pinned buffers directly (``fvr_copy_bytes``).  With
    ``outputs_on_host=True`` as well, ``fn`` itself returns pinned host tensors
    that its kernels write, and no output copy is captured.  Calling then
    takes host tensors (or writes nothing when given ``host_in`` itself),
    replays, and returns ``host_out`` after waiting for the stream
    (``sync=False``: without waiting; ``host_out`` is complete once the
    current stream is)."""

    def __init__(self, fn, *example_inputs, warmup=3, capture_context=None, host_io=False,
                 outputs_on_host=False):
        for x in example_inputs:
            L.require_cuda(x)
        self.fn = fn
        self.host_io = bool(host_io)
        self.static_in = [x.detach().clone() for x in example_inputs]
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            for _ in range(max(1, int(warmup))):
                out = fn(*self.static_in)
        torch.cuda.current_stream().wait_stream(side)
        torch.cuda.synchronize()
        self.outputs_on_host = bool(host_io and outputs_on_host)
        if self.host_io:
            outs = out if isinstance(out, (tuple, list)) else (out,)
            self.host_in = [torch.empty(x.shape, dtype=x.dtype).pin_memory() for x in self.static_in]
            self.host_out = None if self.outputs_on_host else [torch.empty(o.shape, dtype=o.dtype).pin_memory()
                                                                for o in outs]
        self.graph = torch.cuda.CUDAGraph()
        n0 = L.launch_count[0]
        with no_gc_during_capture():
            self._capture(fn, capture_context)
        self.kernels_per_replay = L.launch_count[0] - n0

    def _capture(self, fn, capture_context):
        with capture_context if capture_context is not None else contextlib.nullcontext():
            # thread-local: an unrelated CUDA call from another thread of the
            # process (autograd workers, samplers) cannot invalidate the capture
            with torch.cuda.graph(self.graph, capture_error_mode="thread_local"):
                if self.host_io:
                    for s, h in zip(self.static_in, self.host_in):
                        _copy_kernel(s, h)
                self.static_out = fn(*self.static_in)
                outs = self.static_out if isinstance(self.static_out, (tuple, list)) else (self.static_out,)
                if self.outputs_on_host:  # fn wrote them into pinned host memory itself
                    self.host_out = list(outs)
                elif self.host_io:
                    for h, o in zip(self.host_out, outs):
                        _copy_kernel(h, o)

    def replay(self):
        self.graph.replay()
        return self.static_out

    def __call__(self, *inputs, sync=True):
        if self.host_io:
            for h, x in zip(self.host_in, inputs):
                if x.data_ptr() != h.data_ptr():
                    h.copy_(x)
            self.graph.replay()
            if sync:
                torch.cuda.current_stream().synchronize()
            return tuple(self.host_out) if len(self.host_out) > 1 else self.host_out[0]
        for s, x in zip(self.static_in, inputs):
            s.copy_(x, non_blocking=True)
        return self.replay()


def _biplanar_value_and_grad(engine, f_ap, f_lat, high_pass, sigma, poses, out_grad=None, out_loss=None):
    return engine.spectral_ncc_value_and_grad(poses, (f_ap, f_lat), ("ap", "lateral"), high_pass=high_pass,
                                              cutoff_sigma=sigma, out_grad=out_grad, out_loss=out_loss)


class BiplanarSpectralNCCStep:
    """``loss = forward_spectral_ncc(AP) + forward_spectral_ncc(lateral)`` and
    ``dloss/dposes`` for a batch of candidate poses on a
    :class:`fvr.torch_engine.TorchDiffFVREngine`, as one callable: one fused
    gather pass over both views, an fp64 finalize, an fp64 pose-gradient
    epilogue.

    With ``graph=True`` (default) the whole step is a single CUDA-graph replay
    that uses the engine's spectrum storage of the time of capture (the step
    keeps that storage alive; capture again after ``to_precision``).
    Returns ``(loss, grad)`` device tensors (scalar, ``[C, 6]``).  With
    ``host_io=True`` (graph only) the step takes host poses and returns pinned
    host ``(loss, grad)`` tensors: one graph replay holds a copy kernel that
    reads the pinned poses and the two kernels of the step, whose epilogue
    writes the loss and gradient straight into pinned host memory
    (``host_poses`` is the pinned input buffer; writing poses there directly
    skips one host copy).
    """

    def __init__(self, engine, f_targ_ap, f_targ_lat, n_candidates, high_pass=True, cutoff_sigma=4.0, graph=True,
                 warmup=3, capture_context=None, host_io=False):
        self.engine = engine
        self._stencil = (engine._stencil, engine._pair)  # the storage the captured kernels read
        self.f_ap = f_targ_ap
        self.f_lat = f_targ_lat
        self.hp = bool(high_pass)
        self.sigma = float(cutoff_sigma)
        ex = torch.zeros((int(n_candidates), 6), dtype=torch.float32, device=engine._dev)
        # the captured callable holds no reference back to this object (no
        # reference cycle: the step and its graph are freed as soon as dropped)
        fn = functools.partial(_biplanar_value_and_grad, engine, f_targ_ap, f_targ_lat, self.hp, self.sigma)
        io = graph and host_io
        if io:  # the epilogue kernel writes loss and gradient straight into pinned host buffers
            fn = functools.partial(fn, out_grad=torch.empty((int(n_candidates), 6), dtype=torch.float32).pin_memory(),
                                   out_loss=torch.empty(3, dtype=torch.float32).pin_memory())
        self._g = (GraphedCallable(fn, ex, warmup=warmup, capture_context=capture_context, host_io=host_io,
                                   outputs_on_host=io) if graph else None)
        self.host_poses = self._g.host_in[0] if io else None
        self.host_loss, self.host_grad = self._g.host_out if io else (None, None)

    def _step(self, poses):
        return _biplanar_value_and_grad(self.engine, self.f_ap, self.f_lat, self.hp, self.sigma, poses)

    def __call__(self, poses, sync=True):
        if self._g is None:
            return self._step(poses.to(self.engine._dev))
        return self._g(poses, sync=sync) if self._g.host_io else self._g(poses)
