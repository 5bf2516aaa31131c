"""Oracle (test infrastructure only): build and call ``fvr_oracle.c``.

``build()`` compiles it with gcc -O3 -fopenmp into ``oracle/_build/`` (git-ignored;
travels to the GPU box with the rest of the tree).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "fvr_oracle.c"
LIB = HERE / "_build" / "libfvr_oracle.so"

_lib = None


def build(force=False):
    if LIB.exists() and not force and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    LIB.parent.mkdir(parents=True, exist_ok=True)
    subprocess.run(["gcc", "-O3", "-march=x86-64-v2", "-fopenmp", "-fPIC", "-shared", str(SRC), "-o", str(LIB),
                    "-lm"], check=True)
    return LIB


def _load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(str(LIB))
        D = ctypes.POINTER(ctypes.c_double)
        lib.fvr_oracle_sncc.restype = ctypes.c_double
        lib.fvr_oracle_sncc.argtypes = [D, ctypes.c_int, ctypes.c_int, ctypes.c_int, D, ctypes.c_int, ctypes.c_int,
                                        D, D, ctypes.c_int, ctypes.c_double, ctypes.c_double, D, D, ctypes.c_int]
        _lib = lib
    return _lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def sncc(spec, poses, f_targ, view, hp=None, spacing0=1.0, g=1.0, grad=True, threads=None):
    """Loss, per-candidate NCC and (optionally) dL/dposes of the zero-IFFT spectral NCC.

    ``spec`` planar [2, D, H, W]; ``f_targ`` complex [R, R] (already high-passed);
    ``hp`` [R, R] or None; ``view`` 'ap' or 'lateral'.
    """
    lib = _load()
    spec = np.ascontiguousarray(spec, dtype=np.float64)
    poses = np.ascontiguousarray(poses, dtype=np.float64)
    ft = np.asarray(f_targ).reshape(np.asarray(f_targ).shape[-2:])
    R = ft.shape[-1]
    ftr = np.ascontiguousarray(np.stack([ft.real, ft.imag], -1), dtype=np.float64)
    hpa = None if hp is None else np.ascontiguousarray(hp, dtype=np.float64)
    C = poses.shape[0]
    ncc = np.zeros(C)
    gr = np.zeros((C, 6)) if grad else None
    nthr = threads if threads is not None else (os.cpu_count() or 1)
    loss = lib.fvr_oracle_sncc(_dp(spec), spec.shape[1], spec.shape[2], spec.shape[3], _dp(poses), C,
                               1 if view == "lateral" else 0, _dp(ftr), _dp(hpa), R, float(spacing0), float(g),
                               _dp(ncc), _dp(gr), int(nthr))
    return loss, ncc, gr
