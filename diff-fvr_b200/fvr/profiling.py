"""Per-launch timing of named kernel sections with CUDA events.

Sections are marked in the library code with ``with profiling.section(name):``
around one kernel launch.  Nothing is recorded unless a :class:`LaunchTimer`
for that name is active.  Inside stream capture the events are recorded as
external event nodes (``fvr_event_record``), so a replayed CUDA graph times
the kernel on every replay.
"""
from __future__ import annotations

import contextlib
import ctypes

import torch

from . import _lib as L

_active = None


class LaunchTimer:
    """Collects (start, end) CUDA event pairs around named sections."""

    def __init__(self, names, capacity=64):
        self.names = set(names)
        self.pairs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                      for _ in range(capacity)]
        for a, b in self.pairs:  # materialise the driver events outside any capture
            a.record()
            b.record()
        torch.cuda.synchronize()
        self.used = []

    def __enter__(self):
        global _active
        self.used = []
        _active = self
        return self

    def __exit__(self, *exc):
        global _active
        _active = None
        return False

    def _take(self):
        if len(self.used) >= len(self.pairs):
            raise L.FvrError("LaunchTimer capacity exceeded")
        return self.pairs[len(self.used)]

    def durations_ms(self, name=None):
        """Elapsed ms of every recorded section (call after synchronising)."""
        return [a.elapsed_time(b) for (n, a, b) in self.used if name is None or n == name]


def _record(ev):
    ext = 1 if torch.cuda.is_current_stream_capturing() else 0
    L.call("fvr_event_record", ctypes.c_void_p(ev.cuda_event), L.stream_ptr(), ext)


@contextlib.contextmanager
def section(name):
    t = _active
    if t is None or name not in t.names:
        yield
        return
    a, b = t._take()
    _record(a)
    yield
    _record(b)
    t.used.append((name, a, b))


def sncc_cell_sequence(engine, poses, views, out_res):
    """The stencil entries a spectral-NCC moments launch reads, in the order
    the CTAs of its tile grid sweep them (all (view, candidate) items advance
    through the slice rows together): int32 entry indices of the cells with
    a corner inside the volume (samples outside read nothing).  Positions
    follow the kernel's tables: p = s + ku u + kv v in FP64 voxel units."""
    from . import _runtime as RT

    dev = engine._dev
    D, H, W = engine._stencil.dims
    p = poses.detach().to(device=dev, dtype=torch.float32).contiguous()
    C = int(p.shape[0])
    R = int(out_res)
    lin = RT.linspace(R, dev).to(torch.float64)
    s = L.stream_ptr(dev)
    half = [0.5 * max(n - 1, 1) for n in (W, H, D)]
    cells = []
    for view in views:
        code = view if isinstance(view, int) else (0 if view == "ap" else 1)
        axes = torch.empty((C, 8), dtype=torch.float64, device=dev)
        L.call("fvr_tc_axes", L.ptr(p), C, code, D, H, W, L.ptr(axes), s)
        ku, kv = lin[None, :, None], lin[None, None, :]
        c = [torch.floor(half[k] + ku * axes[:, k, None, None] + kv * axes[:, 3 + k, None, None]).long() + 1
             for k in range(3)]
        cells.append(torch.stack(c, -1))  # [C, R, R, (x, y, z)]
    cell = torch.stack(cells, 0).permute(2, 0, 1, 3, 4).reshape(-1, 3)  # rows outermost
    lim = torch.tensor([W, H, D], device=dev)
    ok = ((cell >= 0) & (cell <= lim)).all(-1)
    cell = cell[ok]
    e = (cell[:, 2] * (H + 1) + cell[:, 1]) * (W + 1) + cell[:, 0]
    return e.to(torch.int32).contiguous()


def gather_ceiling_ms(engine, cells, flush=None, reps=5, blocks_per_sm=8):
    """Median device time of fvr_bench_gather32 over ``cells`` (16-bit
    stencil), with ``flush`` (a tensor larger than L2) rewritten before each
    timed launch when given."""
    if engine._stencil.code == L.F32_:
        raise L.FvrError("the gather ceiling is measured on 32-byte (16-bit storage) entries")
    dev = engine._dev
    D, H, W = engine._stencil.dims
    n_entries = (D + 1) * (H + 1) * (W + 1)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    blocks = sms * int(blocks_per_sm)
    out = torch.empty(blocks * 256, dtype=torch.int32, device=dev)
    s = L.stream_ptr(dev)
    args = (L.ptr(engine._stencil.data), n_entries, L.ptr(cells), int(cells.numel()), L.ptr(out), int(out.numel()),
            blocks, s)
    L.call("fvr_bench_gather32", *args)
    times = []
    for _ in range(int(reps)):
        if flush is not None:
            flush.add_(1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        L.call("fvr_bench_gather32", *args)
        b.record()
        b.synchronize()
        times.append(a.elapsed_time(b))
    times.sort()
    return times[len(times) // 2]
