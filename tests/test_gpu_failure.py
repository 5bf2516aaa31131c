"""Failure detection without a GPU fault: the bounded wait of the
value-and-gradient epilogue.  The epilogue waits for each partial record's
flag; launched alone (fvr_tc_sncc_finish) on a fresh workspace no flag is
ever set, so its wait runs out after the given limit, the losses come back
NaN and the workspace's status word reads FVR_ERR_TIMEOUT.  The context
stays usable: the next full call on the same workspace gives the results of
a call on a fresh one."""
import ctypes
import time

import numpy as np
import pytest
import torch

from oracle import torch_convention as tc

pytestmark = pytest.mark.gpu

FVR_ERR_TIMEOUT = 6


def test_epilogue_wait_runs_out_and_the_workspace_recovers():
    from fvr import _lib as L
    from fvr import _runtime as RT
    from fvr.torch_engine import TorchDiffFVREngine

    dev = torch.device("cuda", 0)
    C, R, nv = 6, 32, 2
    eng = TorchDiffFVREngine(torch.from_numpy(tc.make_ellipsoid_volume(24, 3)), device=dev)
    tp = torch.from_numpy(tc.make_poses(1, 5)).to(dev)
    fts = [eng.prepare_spectral_target(eng(tp, view=v, out_res=R)).reshape(R, R).contiguous() for v in ("ap", "lateral")]
    poses = torch.from_numpy(tc.make_poses(C, 4)).to(dev).contiguous()
    views = (ctypes.c_int * nv)(0, 1)
    fptrs = (ctypes.c_void_p * nv)(*[f.data_ptr() for f in fts])
    hp, lin = RT.hp_filter(R, R, 4.0, dev), RT.linspace(R, dev)
    kap = RT.kappa(R, eng.spacing[0])
    D, H, W = eng._stencil.dims
    s = L.stream_ptr(dev)
    lib = L.load()
    wsb = int(L.query("fvr_tc_sncc_fused_workspace", C, R, nv))

    def outputs():
        return (torch.full((nv + 1,), 7.0, dtype=torch.float32, device=dev),
                torch.zeros((C, 6), dtype=torch.float32, device=dev))

    def full_call(ws):
        loss, grad = outputs()
        assert lib.fvr_tc_sncc_value_and_grad(*eng._stencil.args(), L.ptr(poses), C, nv, views, fptrs, L.ptr(hp),
                                              L.ptr(lin), R, kap, 0, None, 0, L.ptr(ws), wsb, L.ptr(loss), None,
                                              L.ptr(grad), 0, s) == 0
        torch.cuda.synchronize()
        return loss, grad

    ws = torch.zeros(wsb, dtype=torch.uint8, device=dev)
    loss, grad = outputs()
    t0 = time.perf_counter()
    assert lib.fvr_tc_sncc_finish(L.ptr(poses), C, nv, views, D, H, W, R, kap, 0, None, 0, L.ptr(ws), wsb,
                                  L.ptr(loss), None, L.ptr(grad), 0, 2000, s) == 0
    torch.cuda.synchronize()
    assert time.perf_counter() - t0 < 5.0
    assert bool(torch.isnan(loss).all())
    st = ctypes.c_int(-1)
    assert lib.fvr_tc_sncc_fused_status(L.ptr(ws), C, R, nv, ctypes.byref(st), 1) == 0
    assert st.value == FVR_ERR_TIMEOUT
    assert lib.fvr_tc_sncc_fused_status(L.ptr(ws), C, R, nv, ctypes.byref(st), 0) == 0 and st.value == 0
    # the same workspace afterwards, twice, against a fresh one
    fresh_loss, fresh_grad = full_call(torch.zeros(wsb, dtype=torch.uint8, device=dev))
    for _ in range(2):
        l2, g2 = full_call(ws)
        assert torch.equal(l2, fresh_loss) and torch.equal(g2, fresh_grad)
    assert lib.fvr_tc_sncc_fused_status(L.ptr(ws), C, R, nv, ctypes.byref(st), 0) == 0 and st.value == 0
    assert np.isfinite(fresh_loss.cpu().numpy()).all()
