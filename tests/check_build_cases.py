"""Small cases of every instrumented kernel family, run in a child process by
test_gpu_check_build.py with FVR_B200_LIB naming either the normal library or
the bounds-checked debug build.  Prints one JSON object: the outputs (as
lists) and, for the debug build, the check words."""
import ctypes
import json
import sys
from pathlib import Path

import numpy as np
import torch

REPO = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(REPO / "diff-fvr_b200"))
sys.path.insert(0, str(REPO))

import fvr  # noqa: E402
from fvr import _lib as L  # noqa: E402
from fvr.cone_beam_fvr import PerspectiveSlabFVR  # noqa: E402
from fvr.diff_fvr import DifferentiableFourierVolumeRenderer  # noqa: E402
from fvr.gradients import SpectralGradientEngine  # noqa: E402
from fvr.synthetic import make_ellipsoid_volume, make_pinhole_mats, make_poses  # noqa: E402
from fvr.triton_slice import fourier_slice_3d, pou_pinhole_warp_sum  # noqa: E402


def main():
    dev = torch.device("cuda", 0)
    out = {}
    vol = make_ellipsoid_volume(24, 1)
    poses = torch.from_numpy(make_poses(5, 2)).to(dev)
    tp = torch.from_numpy(make_poses(1, 3)).to(dev)
    for name, dt in (("f32", torch.float32), ("bf16", torch.bfloat16), ("f16", torch.float16)):
        eng = fvr.TorchDiffFVREngine(torch.from_numpy(vol), device=dev)
        fa = eng.prepare_spectral_target(eng(tp, view="ap", out_res=20))
        fl = eng.prepare_spectral_target(eng(tp, view="lateral", out_res=20))
        if dt != torch.float32:
            eng.to_precision(dt)
        p = poses.clone().requires_grad_(True)
        loss = eng.forward_spectral_ncc(p, fa, view="ap") + eng.forward_spectral_ncc(p, fl, view="lateral")
        loss.backward()
        img = eng(poses, view="lateral", out_res=20)
        out[f"sncc_{name}"] = [float(loss)] + p.grad.flatten().tolist()
        out[f"img_{name}"] = img.flatten().tolist()
    g = torch.Generator().manual_seed(5)
    vri = torch.randn((2, 2, 10, 12, 9), generator=g).to(dev)
    u = (torch.randn((3, 3), generator=g) * 4).to(dev).requires_grad_(True)
    v = (torch.randn((3, 3), generator=g) * 4).to(dev).requires_grad_(True)
    f = torch.linspace(-0.6, 0.6, 7, device=dev)
    fy, fx = torch.meshgrid(f, f, indexing="ij")
    s = fourier_slice_3d(vri, u, v, fx.reshape(-1), fy.reshape(-1), (4.5, 5.5, 4.0))
    (s * s).sum().backward()
    out["slice3d"] = s.flatten().tolist() + u.grad.flatten().tolist() + v.grad.flatten().tolist()
    for name, dt in (("f32", torch.float32), ("bf16", torch.bfloat16)):
        m = PerspectiveSlabFVR.from_volume(make_ellipsoid_volume(40, 4), vox_mm=2.0, grid_blocks=(2, 2, 2),
                                           block_res=32, overlap=0.5, dtype=dt, device=dev)
        k_inv = torch.tensor([[1 / 300.0, 0.0, -0.1], [0.0, 1 / 300.0, -0.1], [0.0, 0.0, 1.0]], device=dev)
        lat = m.make_pinhole_lattice(k_inv, 600.0, 60, 60)
        mats = make_pinhole_mats(3, 6, sad_mm=300.0, device=dev).requires_grad_(True)
        o = m.forward_pinhole(mats, lat)
        (o * o).sum().backward()
        out[f"pou_{name}"] = o.flatten().tolist()[::7] + mats.grad.flatten().tolist()
        m.fused_warp_adjoint = False  # the two-kernel backward (warp adjoint + block-image adjoint)
        mats3 = mats.detach().clone().requires_grad_(True)
        (m.forward_pinhole(mats3, lat) ** 2).sum().backward()
        out[f"pou_two_kernel_{name}"] = mats3.grad.flatten().tolist()
        m.fused_warp_adjoint = True
        mats2 = mats.detach().clone().requires_grad_(True)
        o2 = m.forward_pinhole(mats2, lat[:5])
        o2.sum().backward()
        out[f"pou_rays_{name}"] = o2.flatten().tolist()[::7] + mats2.grad.flatten().tolist()
    imgs = torch.randn((3, 2, 16, 16), generator=g).to(dev).requires_grad_(True)
    db = (300 + torch.randn((3, 2), generator=g) * 10).to(dev).requires_grad_(True)
    cu = (torch.randn((3, 2), generator=g) * 6).to(dev).requires_grad_(True)
    cv = (torch.randn((3, 2), generator=g) * 6).to(dev).requires_grad_(True)
    rx = torch.linspace(-0.05, 0.05, 30, device=dev).view(1, 30).expand(20, 30).contiguous()
    ry = torch.linspace(-0.05, 0.05, 20, device=dev).view(20, 1).expand(20, 30).contiguous()
    ic = torch.ones((20, 30), device=dev)
    w = pou_pinhole_warp_sum(imgs, db, cu, cv, rx, ry, ic, rx.reshape(-1), ry.reshape(-1), ic.reshape(-1), 0.5, 8.0)
    (w * w).sum().backward()
    out["warp"] = w.flatten().tolist()[::5] + imgs.grad.flatten().tolist()[::5] + db.grad.flatten().tolist()
    ren = DifferentiableFourierVolumeRenderer(make_ellipsoid_volume(16, 7).astype(np.float64), device=dev)
    ta = ren.extract_frequency_slice(2.0, -1.0, 0.5, 0.3, 0.2, view="ap")
    tl = ren.extract_frequency_slice(2.0, -1.0, 0.5, -0.4, 0.2, view="lateral")
    lo, gr = SpectralGradientEngine(ren).compute_biplanar_loss_and_gradients(np.array([1.0, 0.5, -1, 0.2, 0.1, 0.3]),
                                                                             ta, tl)
    out["numpy"] = [lo] + list(gr) + ren.render_drr(3.0, 1.0, -2.0, view="ap").flatten().tolist()[::3]
    torch.cuda.synchronize()
    words = (ctypes.c_ulonglong * 4)()
    rc = L.load().fvr_check_words(words, 4, 1)
    out["check_rc"] = rc
    out["check_words"] = [int(x) for x in words]
    print(json.dumps(out))


if __name__ == "__main__":
    main()
