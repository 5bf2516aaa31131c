"""ctypes binding of ``libfvr_b200.so`` (the C ABI in ``include/fvr_b200.h``).

There is no fallback: importing works without a GPU (so the C ABI can be
inspected), but every compute call raises ``FvrError`` unless the library is
built and the tensors live on a CUDA device of the B200 family (sm_100).
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import torch

_HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("FVR_B200_LIB", _HERE / "libfvr_b200.so"))

P = ctypes.c_void_p
I64 = ctypes.c_int64
I32 = ctypes.c_int
F32 = ctypes.c_float
F64 = ctypes.c_double

F32_ = 0
BF16_ = 1
F16_ = 2
F64_ = 3
BF16_PAIR_ = 4
F16_PAIR_ = 5
F32_PAIR_ = 6

# name -> (restype, argtypes)
SIGNATURES = {
    "fvr_status_string": (ctypes.c_char_p, [I32]),
    "fvr_version": (I32, []),
    "fvr_check_words": (I32, [P, I32, I32]),
    "fvr_device_supported": (I32, [I32]),
    "fvr_fft_supported": (I32, [I64]),
    "fvr_fft_twiddles": (I32, [I64, I32, P, P]),
    "fvr_spectrum3d": (I32, [P, I32, I64, I64, I64, I64, I64, I64, I64, I32, P, P, P, I32, P, P, P, P, P]),
    "fvr_fft2d": (I32, [P, I32, I64, I64, I64, I32, I32, I32, I32, F64, I32, P, I64, I64, I64, I64, P, P, P, P]),
    "fvr_stencil_bytes": (I64, [I64, I64, I64, I32]),
    "fvr_stencil_scale_count": (I64, [I64, I64, I64]),
    "fvr_stencil_build": (I32, [P, I32, I32, I64, I64, I64, I64, I32, P, P, P, P]),
    "fvr_stencil_pair_bytes": (I64, [I64, I64, I64, I32]),
    "fvr_stencil_pair_scale_count": (I64, [I64, I64, I64]),
    "fvr_stencil_pair_build": (I32, [P, I32, I32, I64, I64, I64, I64, I32, P, P, P, P]),
    "fvr_slice3d_fwd": (I32, [P, I32, I64, I64, I64, I64, P, P, I64, P, P, I64, F32, F32, F32, P, P]),
    "fvr_slice3d_bwd_workspace": (I64, [I64, I64]),
    "fvr_slice3d_bwd": (I32, [P, I32, I64, I64, I64, I64, P, P, P, I64, P, P, I64, F32, F32, F32, P, P, P, I64, P]),
    "fvr_tc_axes": (I32, [P, I64, I32, I64, I64, I64, P, P]),
    "fvr_tc_sncc_workspace": (I64, [I64, I64, I64]),
    "fvr_tc_sncc_mom_stride": (I64, []),
    "fvr_tc_sncc_variants": (I32, []),
    "fvr_tc_sncc_moments": (I32, [I32, P, P, I64, I64, I64, P, I64, I32, P, P, P, P, I64, F64, I32, I32, P, I64,
                                  P]),
    "fvr_tc_sncc_finalize": (I32, [P, I64, I64, I32, I32, I32, P, P, P, P]),
    "fvr_tc_sncc_fused_workspace": (I64, [I64, I64, I64]),
    "fvr_tc_sncc_value_and_grad_static": (I32, [I32, P, P, I64, I64, I64, P, I64, I32, P, P, P, P, I64, F64, I32, P,
                                                I64, P, P, P, I32, P]),
    "fvr_se3_exp": (I32, [P, I64, P, P]),
    "fvr_se3_exp_backward": (I32, [P, P, I64, P, P]),
    "fvr_edge_ncc_workspace": (I64, [I64, I64, I64, I64, I64]),
    "fvr_edge_ncc_stats_count": (I64, []),
    "fvr_edge_ncc_forward": (I32, [P, P, I64, I64, I64, I64, I64, I64, F32, I32, P, I64, P, P, P]),
    "fvr_edge_ncc_backward": (I32, [P, P, I64, I64, I64, I64, I64, I64, F32, I32, P, P, I64, I32, P, P]),
    "fvr_tc_sncc_value_and_grad": (I32, [I32, P, P, I64, I64, I64, P, I64, I32, P, P, P, P, I64, F64, I32, P, I64, P,
                                         I64, P, P, P, I32, P]),
    "fvr_event_record": (I32, [P, P, I32]),
    "fvr_copy_bytes": (I32, [P, P, I64, P]),
    "fvr_tc_sncc_backward": (I32, [P, I32, P, P, I64, P, I64, I64, I64, I64, F64, P, I32, P]),
    "fvr_tc_slice": (I32, [I32, P, P, I64, I64, I64, P, I64, P, I64, F64, I32, P, P]),
    "fvr_tc_slice_adjoint_workspace": (I64, [I64, I64]),
    "fvr_tc_slice_adjoint": (I32, [I32, P, P, I64, I64, I64, P, P, I64, I32, P, I64, F64, I32, P, P, I64, P, I32, P]),
    "fvr_relu_mask": (I32, [P, P, P, I64, P]),
    "fvr_cmul_table": (I32, [P, P, I64, I64, P]),
    "fvr_hp_filter": (I32, [P, I64, I64, F64, P]),
    "fvr_linspace": (I32, [P, F32, F32, I64, P]),
    "fvr_pou_block_sums": (I32, [P, I64, I64, I64, P, P, I64, P, P, I64, P, P, I64, P, P]),
    "fvr_pou_build_blocks": (I32, [P, I64, I64, I64, P, P, I64, P, P, I64, P, P, I64, P, I64, P, I64, I64, I64, F64,
                                   P, P]),
    "fvr_pou_geo_stride": (I64, []),
    "fvr_pou_pinhole_lattice": (I32, [P, F64, I64, I64, P, P, P, P, P, P]),
    "fvr_spine_phantom": (I32, [I64, P, P]),
    "fvr_pou_pose": (I32, [P, P, I64, P, F64, P, I64, P, P, P]),
    "fvr_pou_rays_prep": (I32, [P, P, I64, I64, P, P, P, P]),
    "fvr_pou_rays_bwd_workspace": (I64, [I64, I64]),
    "fvr_pou_rays_bwd": (I32, [P, P, I64, I64, P, P, P, I64, P]),
    "fvr_pou_slice": (I32, [I32, P, P, I64, I64, P, I64, P, P, P]),
    "fvr_pou_slice_adjoint_workspace": (I64, [I64, I64, I64]),
    "fvr_pou_slice_adjoint": (I32, [I32, P, P, I64, I64, P, I64, P, P, P, I64, P]),
    "fvr_pou_image_supported": (I32, [I64]),
    "fvr_pou_slice_image": (I32, [I32, P, P, I64, I64, P, I64, P, P, P]),
    "fvr_pou_slice_image_adjoint_workspace": (I64, [I64, I64]),
    "fvr_pou_slice_image_adjoint": (I32, [I32, P, P, I64, I64, P, I64, P, P, P, I64, P]),
    "fvr_pou_warp_image_adjoint_supported": (I32, [I64, I64, I64]),
    "fvr_pou_warp_image_adjoint": (I32, [I32, P, P, I64, I64, P, I64, P, P, P, P, P, P, P, I64, I64, F64, F64, P, P,
                                         I64, P]),
    "fvr_pou_warp": (I32, [P, I64, I64, I64, P, P, P, I32, I64, P, P, P, I64, I64, F64, F64, P, P]),
    "fvr_pou_warp_bwd_workspace": (I64, [I64, I64, I64]),
    "fvr_pou_warp_bwd": (I32, [P, I64, I64, I64, P, P, P, I32, I64, P, P, P, I64, I64, F64, F64, P, P, P, P, P, I64,
                               P]),
    "fvr_pou_pose_backward": (I32, [P, I64, P, P, I64, P, P, I64, I64, P, F64, P, P, P]),
    "fvr_np_item_bytes": (I64, []),
    "fvr_np_slices": (I32, [P, I64, I64, I64, P, I64, I64, P, P]),
    "fvr_np_ncc_workspace": (I64, [I64]),
    "fvr_np_ncc_moments": (I32, [P, I64, I64, I64, P, I64, P, P, I64, P, P]),
    "fvr_np_pair_workspace": (I64, []),
    "fvr_ingest_resample": (I32, [P, I64, I64, I64, F64, F64, F64, I64, I32, P, P, P]),
    "fvr_hu_to_attenuation": (I32, [P, I64, P, P]),
    "fvr_np_segment_slices": (I32, [P, I64, I64, I64, I64, P, I64, I64, P, P]),
    "fvr_np_pair_moments": (I32, [P, P, I64, I64, P, I64, P, P]),
    "fvr_cncc_workspace": (I64, [I64, I64]),
    "fvr_cncc_forward": (I32, [P, P, I64, I64, I64, P, P, I64, P, P, P]),
    "fvr_cncc_backward": (I32, [P, P, I64, I64, I64, P, P, P, P, P]),
}


class FvrError(RuntimeError):
    """A C-ABI call returned a non-zero fvr_status, or the native path is unavailable."""


_lib = None


def load():
    """Load the shared library (once) and bind every declared symbol."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise FvrError(
            f"libfvr_b200.so not found at {LIB_PATH}; build it with `make -C diff-fvr_b200/csrc` "
            "(or __graft_entry__.build()). There is no CPU fallback."
        )
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols():
    return sorted(SIGNATURES)


# kernels each entry point launches (for launch accounting; default 1)
KERNELS_PER_CALL = {
    "fvr_event_record": 0,
    "fvr_fft2d": 2,
    "fvr_spectrum3d": 3,
    "fvr_slice3d_bwd": 2,
    "fvr_tc_slice_adjoint": 2,
    "fvr_cncc_forward": 2,
    "fvr_pou_warp_bwd": 2,
    "fvr_np_ncc_moments": 2,
    "fvr_np_pair_moments": 2,
    "fvr_edge_ncc_forward": 2,
    "fvr_tc_sncc_value_and_grad": 2,
    "fvr_tc_sncc_value_and_grad_static": 2,
}
launch_count = [0]


def call(name, *args):
    """Invoke an fvr_* entry point that returns fvr_status; raise on failure."""
    lib = load()
    launch_count[0] += KERNELS_PER_CALL.get(name, 1)
    rc = getattr(lib, name)(*args)
    if rc != 0:
        msg = lib.fvr_status_string(rc).decode()
        raise FvrError(f"{name} failed with status {rc}: {msg}")
    return rc


def query(name, *args):
    """Invoke a size-query entry point (returns a non-negative integer)."""
    return getattr(load(), name)(*args)


_checked_devices = set()


def require_cuda(*tensors):
    """Every tensor must be on the same CUDA device, and that device an sm_100 part."""
    dev = None
    for t in tensors:
        if t is None:
            continue
        if not t.is_cuda:
            raise FvrError(
                "fvr_b200 computes on a CUDA (B200, sm_100a) device only; got a tensor on "
                f"{t.device}. There is no CPU fallback."
            )
        if dev is None:
            dev = t.device
        elif t.device != dev:
            raise FvrError(f"tensors on different devices: {dev} and {t.device}")
    if dev is not None and dev.index not in _checked_devices:
        idx = dev.index if dev.index is not None else torch.cuda.current_device()
        if not load().fvr_device_supported(idx):
            cap = torch.cuda.get_device_capability(idx)
            raise FvrError(f"libfvr_b200 is built for sm_100a only; device {idx} is sm_{cap[0]}{cap[1]}")
        _checked_devices.add(dev.index)
    return dev


def ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def stream_ptr(device=None):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def dtype_code(dt):
    if dt == torch.float32:
        return F32_
    if dt == torch.bfloat16:
        return BF16_
    if dt == torch.float16:
        return F16_
    if dt == torch.float64:
        return F64_
    raise FvrError(f"unsupported dtype {dt}")
