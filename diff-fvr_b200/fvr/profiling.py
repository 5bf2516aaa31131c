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


def timing(name):
    """True when a LaunchTimer is collecting ``name`` (a cheap check before
    entering :func:`section` on a hot path)."""
    return _active is not None and name in _active.names


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
