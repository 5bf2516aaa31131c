"""Diff-FVR hot path on NVIDIA B200 (sm_100a): a drop-in for the rendering and
registration-loss entry points of the reference ``fvr`` package
(pareelamre/diff-fvr, src/fvr/), computed by hand-written CUDA kernels in
``libfvr_b200.so`` behind a C ABI (``include/fvr_b200.h``).

Put the directory that contains this package on ``sys.path`` and import it as
``fvr``; the module names mirror the reference (``fvr.torch_engine``,
``fvr.cone_beam_fvr``, ``fvr.triton_slice``, ``fvr.diff_fvr``,
``fvr.gradients``).  :func:`install_src_alias` also registers ``src.fvr``.
"""
from __future__ import annotations

import sys

from ._lib import FvrError  # noqa: F401
from .torch_engine import TorchDiffFVREngine  # noqa: F401

__version__ = "1.2.0+b200"

__all__ = ["TorchDiffFVREngine", "FvrError", "install_src_alias"]

_OPTIONAL = [
    ("cone_beam_fvr", ("PerspectiveSlabFVR", "SLAB_PRESETS", "sample_isocenter_parity_offsets")),
    ("diff_fvr", ("DifferentiableFourierVolumeRenderer",)),
    ("gradients", ("SpectralGradientEngine",)),
    ("core_engine", ("RobustDiffFVREngine", "detect_radio_opaque_metal")),
    ("gradient_optimizer", ("GradientRegistrationOptimizer",)),
    ("dicom_loader", ("create_spine_phantom", "hu_to_attenuation", "resample_isotropic_cube")),
    ("articulated_spine", ("ArticulatedSpineModel", "VertebralSegment")),
]
for _mod, _names in _OPTIONAL:
    try:
        _m = __import__(f"{__name__}.{_mod}", fromlist=list(_names))
    except ImportError:  # module not built yet in this checkout
        continue
    for _n in _names:
        globals()[_n] = getattr(_m, _n)
        __all__.append(_n)


def install_src_alias():
    """Register this package also as ``src.fvr`` (the reference tests import both
    ``fvr.*`` and ``src.fvr.*``)."""
    import types

    pkg = sys.modules[__name__]
    src = sys.modules.get("src") or types.ModuleType("src")
    src.__path__ = []  # namespace-like
    src.fvr = pkg
    sys.modules["src"] = src
    sys.modules["src.fvr"] = pkg
    for name, mod in list(sys.modules.items()):
        if name.startswith(__name__ + "."):
            sys.modules["src." + name] = mod
