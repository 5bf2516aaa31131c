"""The allocation-free entry point fvr_tc_sncc_value_and_grad_static, called
through the C ABI, against the workspace-taking fvr_tc_sncc_value_and_grad on
the same inputs: two calls in a row, then a refused oversize call.  Kept in its
own file, collected last, so it also runs after every other GPU test."""
import ctypes

import numpy as np
import pytest
import torch

from oracle import torch_convention as tc

pytestmark = pytest.mark.gpu

FVR_ERR_WORKSPACE = 4


def _problem(C, R=48, dtype=torch.float32, storage="stencil"):
    from fvr import _lib as L
    from fvr import _runtime as RT
    from fvr.torch_engine import TorchDiffFVREngine

    dev = torch.device("cuda", 0)
    eng = TorchDiffFVREngine(torch.from_numpy(tc.make_ellipsoid_volume(32, 3)), device=dev)
    if dtype != torch.float32:
        eng.to_precision(dtype)
    tp = torch.from_numpy(tc.make_poses(1, 5)).to(dev)
    fts = [eng.prepare_spectral_target(eng(tp, view=v, out_res=R)).reshape(R, R).contiguous()
           for v in ("ap", "lateral")]
    poses = torch.from_numpy(tc.make_poses(C, 4)).to(dev).contiguous()
    views = (ctypes.c_int * 2)(0, 1)
    fptrs = (ctypes.c_void_p * 2)(*[f.data_ptr() for f in fts])
    hp = RT.hp_filter(R, R, 4.0, dev)
    lin = RT.linspace(R, dev)
    st = eng._pair if storage == "pair" else eng._stencil
    head = (*st.args(), L.ptr(poses), C, 2, views, fptrs, L.ptr(hp), L.ptr(lin), R,
            RT.kappa(R, eng.spacing[0]), 0, None, 0)
    return eng, fts, poses, head, dev


def _outputs(C, dev):
    loss = torch.full((3,), float("nan"), dtype=torch.float32, device=dev)
    grad = torch.full((C, 6), float("nan"), dtype=torch.float32, device=dev)
    return loss, grad


@pytest.mark.parametrize("C", [24, 256])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float16, torch.bfloat16])
@pytest.mark.parametrize("storage", ["stencil", "pair"])
def test_static_scratch_matches_workspace_entry(storage, dtype, C):
    """C = 256 with two views is the scratch's limit (512 items: every item
    record row and four 128-item chunks of the epilogue are used); both
    spectrum copies the engine keeps (the stencil, and the x-pair copy its
    own spectral-NCC calls read)."""
    from fvr import _lib as L

    eng, fts, poses, head, dev = _problem(C, dtype=dtype, storage=storage)
    lib = L.load()
    s = L.stream_ptr(dev)
    ws_bytes = int(L.query("fvr_tc_sncc_fused_workspace", C, 48, 2))
    ws = torch.zeros(ws_bytes, dtype=torch.uint8, device=dev)
    loss_ref, grad_ref = _outputs(C, dev)
    assert lib.fvr_tc_sncc_value_and_grad(*head, L.ptr(ws), ws_bytes, L.ptr(loss_ref), None, L.ptr(grad_ref), 0,
                                          s) == 0
    for _ in range(2):  # two calls in a row on the same scratch
        loss, grad = _outputs(C, dev)
        assert lib.fvr_tc_sncc_value_and_grad_static(*head, L.ptr(loss), None, L.ptr(grad), 0, s) == 0
        torch.cuda.synchronize()
        np.testing.assert_allclose(loss.cpu().numpy(), loss_ref.cpu().numpy(), rtol=1e-6, atol=1e-7)
        np.testing.assert_allclose(grad.cpu().numpy(), grad_ref.cpu().numpy(), rtol=1e-5, atol=1e-9)
    # and the result is the reference API's loss
    ref = float(eng.forward_spectral_ncc(poses, fts[0], view="ap") + eng.forward_spectral_ncc(poses, fts[1],
                                                                                             view="lateral"))
    assert abs(float(loss_ref[2]) - ref) < 1e-6


def test_static_scratch_refuses_oversize_without_launching():
    from fvr import _lib as L

    C = 300  # 600 (candidate, view) pairs > 512
    _, _, _, head, dev = _problem(C)
    loss, grad = _outputs(C, dev)
    rc = L.load().fvr_tc_sncc_value_and_grad_static(*head, L.ptr(loss), None, L.ptr(grad), 0, L.stream_ptr(dev))
    torch.cuda.synchronize()
    assert rc == FVR_ERR_WORKSPACE
    assert bool(torch.isnan(loss).all()) and bool(torch.isnan(grad).all())
