"""The benchmark's secondary configurations checked against the float64
oracle at the size they are timed.

* PoU-FVR cone beam: seeded 192^3 ellipsoid volume (1 mm), 4x4x4 blocks at
  50 % overlap, block_res 64 (P = 128), pinhole SDD 1020 / SAD 765 mm,
  256^2 detector at 0.8 mm; two poses, forward and pose-matrix gradient
  (the reference's cone_beam_fvr.py:480-573 restated in oracle/pou.py).
* Large torch-convention case: seeded 256^3 volume (spacing 0.8 x 0.8 x 1.5:
  voxel-unit spectrum, spacing[0] in the phase) -> 512^3 spectrum, R = 192,
  two candidates x AP + lateral: image and spectral-NCC pose gradient
  (torch_engine.py:176-307 restated in oracle/torch_convention.py and the C
  oracle).

Bounds: f32 1e-5 relative L2 forward / 1e-4 gradient; 16-bit storage at the
bounds stated for it (f16 with brick scales 1e-3, the PoU block spectra
included; bf16 1e-2 for the images and the spectral-NCC gradient, 3e-2 for
the PoU pose gradient).  Each test
prints the measured errors.
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu

F_PITCH = 1020.0 / 0.8


@pytest.fixture(scope="module")
def pou_case():
    from oracle import pou as opou
    from fvr import synthetic

    vol = synthetic.make_ellipsoid_volume(192, 0)
    om = opou.PoUModel(vol, vox_mm=1.0, grid_blocks=(4, 4, 4), block_res=64, overlap=0.5)
    H = 256
    k_inv = np.array([[1 / F_PITCH, 0, -0.5 * H / F_PITCH], [0, 1 / F_PITCH, -0.5 * H / F_PITCH], [0, 0, 1.0]])
    olat = opou.make_pinhole_lattice(k_inv, 1020.0, H, H)
    mats = synthetic.make_pinhole_mats(2, 1, sad_mm=765.0).numpy().astype(np.float64)
    w = np.random.default_rng(5).standard_normal((2, 1, H, H))
    ref = opou.forward_pinhole(om, mats, olat)
    gref = opou.forward_pinhole_grad(om, mats, olat, w)
    blocks = om.B
    del om
    return vol, k_inv, mats, w, ref, gref, blocks


@pytest.mark.parametrize("dtype,fwd_bound,grad_bound", [(torch.float32, 1e-5, 1e-4),
                                                        (torch.float16, 1e-3, 1e-3),
                                                        (torch.bfloat16, 1e-2, 3e-2)])
def test_pou_cone_beam_timed_geometry_vs_fp64(pou_case, dtype, fwd_bound, grad_bound):
    from fvr.cone_beam_fvr import PerspectiveSlabFVR

    vol, k_inv, mats, w, ref, gref, blocks = pou_case
    m = PerspectiveSlabFVR.from_volume(vol, vox_mm=1.0, grid_blocks=(4, 4, 4), block_res=64, overlap=0.5,
                                       dtype=dtype)
    assert m.B == blocks and m.P == 128
    lat = m.make_pinhole_lattice(torch.tensor(k_inv, dtype=torch.float32, device="cuda"), 1020.0, 256, 256)
    mm = torch.tensor(mats, dtype=torch.float32, device="cuda").requires_grad_(True)
    out = m.forward_pinhole(mm, lat)
    (out * torch.tensor(w, dtype=torch.float32, device="cuda")).sum().backward()
    e_fwd = rel_l2(out.detach().cpu().numpy(), ref)
    e_grad = rel_l2(mm.grad.cpu().numpy(), gref)
    print(f"PoU 192^3 4x4x4 P=128 256^2 {dtype}: forward {e_fwd:.3e}, mats gradient {e_grad:.3e} vs fp64")
    assert e_fwd < fwd_bound
    assert e_grad < grad_bound


@pytest.fixture(scope="module")
def large_case():
    from oracle import c_oracle
    from oracle import torch_convention as tc
    from fvr import synthetic

    vol = synthetic.make_ellipsoid_volume(256, 0)
    poses = synthetic.make_poses(2, 1)
    tpose = synthetic.make_poses(1, 2)
    R, sp0 = 192, 0.8
    spec = tc.spectrum(vol, 2.0)
    hp = tc.hp_filter(R, R, 4.0)
    out = {"vol": vol, "poses": poses, "R": R}
    loss, grad = 0.0, np.zeros((2, 6))
    for v in ("ap", "lateral"):
        ft = tc.prepare_spectral_target(tc.forward_image(spec, tpose, v, R, sp0))
        out[f"ft_{v}"] = ft
        out[f"img_{v}"] = tc.forward_image(spec, poses, v, R, sp0)
        lo, _, gr = c_oracle.sncc(spec, poses, ft, v, hp, sp0)
        loss += lo
        grad += gr
    out["loss"], out["grad"] = loss, grad
    del spec
    return out


@pytest.mark.parametrize("storage,img_bound,grad_bound", [("f32", 1e-5, 1e-4), ("f16", 1e-3, 1e-3),
                                                          ("bf16", 1e-2, 1e-2)])
def test_large_volume_spectrum512_vs_fp64(large_case, storage, img_bound, grad_bound):
    import fvr

    c = large_case
    R = c["R"]
    dev = torch.device("cuda", 0)
    eng = fvr.TorchDiffFVREngine(torch.from_numpy(c["vol"]), spacing=(0.8, 0.8, 1.5), pad_factor=2.0, device=dev)
    if storage != "f32":
        eng.to_precision(torch.float16 if storage == "f16" else torch.bfloat16)
    poses = torch.from_numpy(c["poses"]).to(dev)
    e_img = max(rel_l2(eng(poses, view=v, out_res=R).cpu().numpy(), c[f"img_{v}"]) for v in ("ap", "lateral"))
    fts = [torch.from_numpy(c[f"ft_{v}"]).to(dev) for v in ("ap", "lateral")]
    loss, grad = eng.spectral_ncc_value_and_grad(poses, fts, views=("ap", "lateral"))
    g = grad.cpu().numpy()
    e_grad = rel_l2(g[:, :5], c["grad"][:, :5])  # tz is never read by the reference (zero gradient)
    e_loss = abs(float(loss) - c["loss"])
    print(f"256^3 -> 512^3 R=192 {storage}: image {e_img:.3e}, gradient {e_grad:.3e}, loss {e_loss:.3e} vs fp64")
    assert e_img < img_bound
    assert e_grad < grad_bound
    assert np.all(g[:, 5] == 0.0)
