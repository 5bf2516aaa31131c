"""Launch-shape autotuner for the hot kernels.

On the first call for a new shape key, every launch variant the library
offers is timed with CUDA events (after one warm-up launch each, then the
median of several launches that each follow an L2 rewrite: cold-cache
conditions, which is how a step meets the spectrum) and the fastest is
cached for the process (a variant the library refuses for the shape is
skipped).  Inside CUDA-graph capture (where nothing
can be timed) a cached choice or variant 0 is used; ``FVR_SNCC_VARIANT``
pins a variant.
"""
from __future__ import annotations

import os

import torch

from . import _lib as L

_cache = {}
_timings = {}


_flush = {}


def _l2_flush(device):
    """A 192 MiB buffer (more than the 126 MB L2) rewritten before each timed
    launch, so variants are compared on a cold L2 (allocated once per device)."""
    t = _flush.get(device)
    if t is None:
        t = torch.zeros(48 * 1024 * 1024, dtype=torch.float32, device=device)
        _flush[device] = t
    return t


def choose(kind, key, run, n_variants, reps=7, candidates=None):
    """Return the fastest variant of ``run(variant)`` (launches the kernels of
    one call) for ``key``: the median of ``reps`` calls per variant, each after an L2
    rewrite (the flush also keeps the device busy while the launch is
    enqueued, so the events time the launch alone).  ``candidates``
    restricts the variants tried (default: all)."""
    env = os.environ.get(f"FVR_{kind.upper()}_VARIANT")
    if env is not None:
        return int(env)
    k = (kind,) + tuple(key)
    if k in _cache:
        return _cache[k]
    if torch.cuda.is_current_stream_capturing():
        return 0
    flush = _l2_flush(torch.cuda.current_device())
    best, best_ms, times = 0, float("inf"), []
    for v in (range(n_variants) if candidates is None else candidates):
        try:
            run(v)
        except L.FvrError:  # this shape does not fit the variant (e.g. its shared memory)
            times.append(float("inf"))
            continue
        ts = []
        for _ in range(reps):
            flush.add_(1.0)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            run(v)
            b.record()
            b.synchronize()
            ts.append(a.elapsed_time(b))
        ts.sort()
        ms = ts[len(ts) // 2]
        times.append(ms)
        if ms < best_ms:
            best, best_ms = v, ms
    _cache[k] = best
    _timings[k] = times  # per candidate, in the order tried
    return best


def report():
    """{key: (chosen variant, per-variant ms)} of the choices made so far."""
    return {k: (_cache[k], _timings.get(k)) for k in _cache}
