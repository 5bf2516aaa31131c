"""Import-path alias of :mod:`fvr.slice_ops` under the reference module name
``fvr.triton_slice`` (src/fvr/triton_slice.py), so code written against the
reference imports unchanged.  Nothing here uses Triton: every function runs
the hand-written CUDA kernels of libfvr_b200.so.
"""
from .slice_ops import *  # noqa: F401,F403
from .slice_ops import (  # noqa: F401
    HAS_TRITON,
    fourier_slice_3d,
    pou_pinhole_warp_sum,
    pou_pinhole_warp_sum_analytical_ref,
    pou_pinhole_warp_sum_torch,
    fourier_slice_3d_torch,
    trilinear_slice_analytical_ref,
    triton_slice_available,
)
