"""Launch-shape autotuner for the hot kernels.

On the first call for a new shape key, every launch variant the library
offers is timed with CUDA events (after one warm-up launch each) and the
fastest is cached for the process (a variant the library refuses for the
shape is skipped).  Inside CUDA-graph capture (where nothing
can be timed) a cached choice or variant 0 is used; ``FVR_SNCC_VARIANT``
pins a variant.
"""
from __future__ import annotations

import os

import torch

from . import _lib as L

_cache = {}
_timings = {}


def choose(kind, key, run, n_variants, reps=3):
    """Return the fastest variant of ``run(variant)`` (launches one kernel) for ``key``."""
    env = os.environ.get(f"FVR_{kind.upper()}_VARIANT")
    if env is not None:
        return int(env)
    k = (kind,) + tuple(key)
    if k in _cache:
        return _cache[k]
    if torch.cuda.is_current_stream_capturing():
        return 0
    best, best_ms, times = 0, float("inf"), []
    for v in range(n_variants):
        try:
            run(v)
        except L.FvrError:  # this shape does not fit the variant (e.g. its shared memory)
            times.append(float("inf"))
            continue
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            run(v)
        b.record()
        b.synchronize()
        ms = a.elapsed_time(b) / reps
        times.append(ms)
        if ms < best_ms:
            best, best_ms = v, ms
    _cache[k] = best
    _timings[k] = times
    return best


def report():
    """{key: (chosen variant, per-variant ms)} of the choices made so far."""
    return {k: (_cache[k], _timings.get(k)) for k in _cache}
