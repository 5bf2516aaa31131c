"""Generate golden vectors by running the reference implementation on CPU.

Usage (needs the reference checkout; run from the repository root):

    python tests/golden/make_golden.py <reference checkout> [name,name,...]

(names: slice_warp, torch_engine, pou, numpy_renderer, articulated,
ingest_targets, phantom, registration; all of them when none is given)

It imports the reference's ``fvr`` package (``src/fvr``) with empty stand-ins
for ``pydicom`` / ``SimpleITK`` (only ``dicom_loader`` needs them, and nothing
on the rendering path calls it), runs seeded small cases through the
reference's public entry points and its autograd, and writes the inputs and
outputs to ``tests/golden/*.npz``.  The fixtures are committed; the tests never
read the reference checkout.
"""
from __future__ import annotations

import math
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


def _import_reference(ref_root: Path):
    for name in ("pydicom", "SimpleITK"):
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.path.insert(0, str(ref_root / "src"))
    import fvr  # noqa: F401
    from fvr import cone_beam_fvr, diff_fvr, gradients, torch_engine, triton_slice

    return torch_engine, triton_slice, cone_beam_fvr, diff_fvr, gradients


def _ellipsoids(n, seed, shape=None):
    sys.path.insert(0, str(REPO))
    from oracle.torch_convention import make_ellipsoid_volume

    return make_ellipsoid_volume(n, seed, shape=shape)


def gen_slice_and_warp(ts):
    import torch

    out = {}
    # trilinear gather + adjoint (mirrors tests/test_cone_beam_fvr.py:152-177 set-up)
    torch.manual_seed(11)
    B_vol, D, H, W, N_pose, P = 3, 24, 20, 22, 4, 20
    vol = torch.randn(B_vol, 2, D, H, W, dtype=torch.float32)
    coords = torch.linspace(-0.45, 0.45, P)
    fy, fx = torch.meshgrid(coords, coords, indexing="ij")
    fx_flat, fy_flat = fx.reshape(-1).contiguous(), fy.reshape(-1).contiguous()
    u0 = torch.randn(N_pose, 3) * 8.0
    v0 = torch.randn(N_pose, 3) * 8.0
    c = (11.0, 9.5, 10.5)
    u = u0.clone().requires_grad_(True)
    v = v0.clone().requires_grad_(True)
    s = ts.fourier_slice_3d_torch(vol, u, v, fx_flat, fy_flat, c)
    w_out = torch.randn_like(s)
    (s * w_out).sum().backward()
    out.update(
        slice_vol=vol.numpy(), slice_u=u0.numpy(), slice_v=v0.numpy(), slice_fx=fx_flat.numpy(),
        slice_fy=fy_flat.numpy(), slice_center=np.array(c), slice_out=s.detach().numpy(),
        slice_wout=w_out.numpy(), slice_gu=u.grad.numpy(), slice_gv=v.grad.numpy(),
    )
    # pinhole warp-sum + adjoint (mirrors tests/test_cone_beam_fvr.py:179-205 set-up)
    torch.manual_seed(17)
    B_blk, N_pose, P, H, W = 4, 3, 24, 18, 20
    imgs0 = torch.randn(B_blk, N_pose, P, P, dtype=torch.float32)
    d_b0 = torch.full((B_blk, N_pose), 300.0) + torch.randn(B_blk, N_pose) * 15.0
    cu0 = torch.randn(B_blk, N_pose) * 4.0
    cv0 = torch.randn(B_blk, N_pose) * 4.0
    rx_hw = torch.linspace(-0.08, 0.08, W).view(1, W).expand(H, W).contiguous()
    ry_hw = torch.linspace(-0.07, 0.07, H).view(H, 1).expand(H, W).contiguous()
    ic_hw = 1.0 / torch.sqrt((1.0 + rx_hw ** 2 + ry_hw ** 2)).clamp(min=0.1)
    inv_ds, c_idx = 0.25, 12.0
    t = [x.clone().requires_grad_(True) for x in (imgs0, d_b0, cu0, cv0)]
    o = ts.pou_pinhole_warp_sum_torch(t[0], t[1], t[2], t[3], rx_hw, ry_hw, ic_hw, inv_ds, c_idx)
    w2 = torch.randn_like(o)
    (o * w2).sum().backward()
    out.update(
        warp_imgs=imgs0.numpy(), warp_db=d_b0.numpy(), warp_cu=cu0.numpy(), warp_cv=cv0.numpy(),
        warp_rx=rx_hw.numpy(), warp_ry=ry_hw.numpy(), warp_ic=ic_hw.numpy(), warp_inv_ds=np.array(inv_ds),
        warp_c_idx=np.array(c_idx), warp_out=o.detach().numpy(), warp_wout=w2.numpy(),
        warp_g_imgs=t[0].grad.numpy(), warp_g_db=t[1].grad.numpy(), warp_g_cu=t[2].grad.numpy(),
        warp_g_cv=t[3].grad.numpy(),
    )
    np.savez_compressed(HERE / "slice_warp.npz", **out)


def gen_torch_engine(te):
    import torch

    out = {}
    vol = _ellipsoids(20, 5, shape=(20, 18, 22))
    spacing = (1.5, 1.5, 1.5)
    eng = te.TorchDiffFVREngine(torch.from_numpy(vol), spacing=spacing, pad_factor=2.0, use_triton=False)
    out["vol"] = vol
    out["spacing0"] = np.array(spacing[0])
    out["spectrum"] = eng.f_vol_5d[0].numpy()
    poses = torch.tensor(
        [[0.0, 0.0, 0.0, 0.0, 0.0, 0.0], [5.0, -3.0, 2.0, 4.0, -2.0, 1.0], [-7.5, 6.0, -4.0, -3.0, 2.5, -5.0]],
        dtype=torch.float32,
    )
    out["poses"] = poses.numpy()
    for view in ("ap", "lateral"):
        for R in (20, 16):
            with torch.no_grad():
                out[f"slice_{view}_{R}"] = eng._extract_slice_spectrum(poses, view=view, out_res=R).numpy()
                out[f"image_{view}_{R}"] = eng(poses, view=view, out_res=R).numpy()
        # image-path autograd
        p = poses.clone().requires_grad_(True)
        img = eng(p, view=view, out_res=20)
        w = torch.from_numpy(np.random.default_rng(3).standard_normal(img.shape).astype(np.float32))
        (img * w).sum().backward()
        out[f"image_w_{view}"] = w.numpy()
        out[f"image_grad_{view}"] = p.grad.numpy()
        # target + spectral NCC with autograd
        tpose = torch.tensor([[2.0, -1.0, 1.5, 1.0, -0.5, 0.0]], dtype=torch.float32)
        with torch.no_grad():
            target = eng(tpose, view=view, out_res=20)
            f_targ = eng.prepare_spectral_target(target, high_pass=True)
            f_targ_nohp = eng.prepare_spectral_target(target, high_pass=False)
        out[f"target_{view}"] = target.numpy()
        out[f"ftarg_{view}"] = f_targ.numpy()
        out[f"ftarg_nohp_{view}"] = f_targ_nohp.numpy()
        p = poses.clone().requires_grad_(True)
        loss = eng.forward_spectral_ncc(p, f_targ, view=view, high_pass=True)
        loss.backward()
        out[f"sncc_loss_{view}"] = loss.detach().numpy()
        out[f"sncc_grad_{view}"] = p.grad.numpy()
        p = poses.clone().requires_grad_(True)
        loss = eng.forward_spectral_ncc(p, f_targ_nohp, view=view, high_pass=False)
        loss.backward()
        out[f"sncc_nohp_loss_{view}"] = loss.detach().numpy()
        out[f"sncc_nohp_grad_{view}"] = p.grad.numpy()
        # image-domain spectral NCC
        pred = eng(poses, view=view, out_res=20).detach().requires_grad_(True)
        l2 = eng.spectral_ncc_loss(pred, target, high_pass=True)
        l2.backward()
        out[f"incc_loss_{view}"] = l2.detach().numpy()
        out[f"incc_grad_{view}"] = pred.grad.numpy()
    # bf16 storage (CPU semantics: the stored spectrum is rounded, the slice is not)
    eb = te.TorchDiffFVREngine(torch.from_numpy(vol), spacing=spacing, pad_factor=2.0, use_triton=False).to_precision(
        torch.bfloat16
    )
    with torch.no_grad():
        out["bf16_image_ap"] = eb(poses, view="ap", out_res=20).numpy()
        out["bf16_spectrum"] = eb.f_vol_5d[0].float().numpy()
    np.savez_compressed(HERE / "torch_engine.npz", **out)


def gen_pou(cb):
    import torch

    out = {}
    # PoU windows (cone_beam_fvr.py:42-61)
    for length, k, ov in [(64, 2, 0.25), (96, 3, 0.25), (128, 4, 0.25), (192, 4, 0.5), (50, 3, 0.4)]:
        ws, step = cb._make_pou_1d(length, k, ov)
        out[f"pou1d_{length}_{k}_{ov}"] = torch.stack(ws).numpy()
        out[f"pou1d_step_{length}_{k}_{ov}"] = np.array(step)
    out["sinc2_12_24"] = cb._sinc2_precomp_1d(12, 24).numpy()

    vol = _ellipsoids(28, 9, shape=(28, 26, 30))
    out["vol"] = vol
    fvr = cb.PerspectiveSlabFVR.from_volume(vol, vox_mm=2.0, grid_blocks=(2, 2, 2), block_res=12, overlap=0.25,
                                            use_triton=False)
    out["B"] = np.array(fvr.B)
    out["P"] = np.array(fvr.P)
    out["ds_block"] = np.array(fvr.ds_block)
    out["centers"] = fvr.centers.numpy()
    out["F_blk_ri"] = fvr.F_blk_ri.numpy()
    out["FX_flat"] = fvr.FX_flat.numpy()
    # a grid_center / 3-axis-different block grid build (centres only)
    fvr2 = cb.PerspectiveSlabFVR.from_volume(vol, vox_mm=1.5, grid_blocks=(3, 2, 1), block_res=10, overlap=0.5,
                                             center_mode="grid_center", use_triton=False)
    out["g2_B"] = np.array(fvr2.B)
    out["g2_centers"] = fvr2.centers.numpy()
    out["g2_ds_block"] = np.array(fvr2.ds_block)
    out["g2_F_blk_ri_sum"] = fvr2.F_blk_ri.double().sum(dim=(2, 3, 4)).numpy()

    H, W = 24, 20
    k_inv = torch.tensor(
        [[1.0 / 300.0, 0.0, -W / 600.0], [0.0, 1.0 / 300.0, -H / 600.0], [0.0, 0.0, 1.0]], dtype=torch.float32
    )
    out["k_inv"] = k_inv.numpy()
    lattice = fvr.make_pinhole_lattice(k_inv, sdd_mm=600.0, height=H, width=W)
    for i, name in enumerate(["src0", "trg0", "u0", "v0", "n0", "rx", "ry", "ic"]):
        out[f"lat_{name}"] = lattice[i].numpy()

    def se3(rot_vec, trans):
        skew = torch.zeros((rot_vec.shape[0], 3, 3), dtype=rot_vec.dtype)
        skew[:, 0, 1], skew[:, 1, 0] = -rot_vec[:, 2], rot_vec[:, 2]
        skew[:, 0, 2], skew[:, 2, 0] = rot_vec[:, 1], -rot_vec[:, 1]
        skew[:, 1, 2], skew[:, 2, 1] = -rot_vec[:, 0], rot_vec[:, 0]
        m = torch.eye(4, dtype=rot_vec.dtype).unsqueeze(0).repeat(rot_vec.shape[0], 1, 1)
        m[:, :3, :3] = torch.matrix_exp(skew)
        m[:, :3, 3] = trans
        return m

    rot0 = torch.tensor([[0.12, -0.08, 0.05], [-0.15, 0.10, -0.04], [0.0, 0.0, 0.0]], dtype=torch.float32)
    xyz0 = torch.tensor([[4.0, -3.0, -300.0], [-2.0, 5.0, -310.0], [0.0, 0.0, -300.0]], dtype=torch.float32)
    mats = se3(rot0, xyz0).detach()
    out["mats"] = mats.numpy()
    for tag, lat in (("inv", lattice), ("exp", lattice[:5])):
        m = mats.clone().requires_grad_(True)
        img = fvr.forward_pinhole(m, lat)
        w = torch.from_numpy(np.random.default_rng(4).standard_normal(img.shape).astype(np.float32))
        (img * w).sum().backward()
        out[f"pin_{tag}_out"] = img.detach().numpy()
        out[f"pin_{tag}_w"] = w.numpy()
        out[f"pin_{tag}_gmats"] = m.grad.numpy()
    # C-arm front-end (explicit rays) with autograd on the 6 scalars
    for view in ("ap", "lateral"):
        params = [torch.tensor(v, requires_grad=True) for v in (3.0, -2.0, 1.5, 1.0, -1.0, 0.5)]
        img = fvr.forward_carm_view(*params, sad_mm=300.0, sdd_mm=600.0, det_px=20, det_fov_mm=70.0, view=view)
        w = torch.from_numpy(np.random.default_rng(5).standard_normal(img.shape).astype(np.float32))
        (img * w).sum().backward()
        out[f"carm_{view}_out"] = img.detach().numpy()
        out[f"carm_{view}_w"] = w.numpy()
        out[f"carm_{view}_grad"] = np.array([float(p.grad) for p in params])
    # edge-dominant NCC (fine only at H=48, multiscale at H=96)
    rng = np.random.default_rng(6)
    for Hs in (48, 96):
        a = torch.from_numpy(rng.standard_normal((3, 1, Hs, Hs)).astype(np.float32)).cumsum(-1).requires_grad_(True)
        a_leaf = a.detach().clone().requires_grad_(True)
        b = torch.from_numpy(rng.standard_normal((3, 1, Hs, Hs)).astype(np.float32)).cumsum(-2)
        val = cb.edge_dominant_ncc(a_leaf, b, reduction="none")
        val.sum().backward()
        out[f"edge_{Hs}_a"] = a_leaf.detach().numpy()
        out[f"edge_{Hs}_b"] = b.numpy()
        out[f"edge_{Hs}_val"] = val.detach().numpy()
        out[f"edge_{Hs}_grad"] = a_leaf.grad.numpy()
    np.savez_compressed(HERE / "pou.npz", **out)


def gen_numpy(df, gr):
    out = {}
    vol = _ellipsoids(16, 7, shape=(16, 14, 18)).astype(np.float64)
    out["vol"] = vol
    ren = df.DifferentiableFourierVolumeRenderer(vol, pad_factor=2.0)
    out["f_3d"] = ren.f_3d
    ren_np = df.DifferentiableFourierVolumeRenderer(vol, pad_factor=2.0, apply_premultiplication=False)
    out["f_3d_nopremult"] = ren_np.f_3d
    pose = (3.0, -2.0, 1.5, 1.25, -0.75)
    out["pose5"] = np.array(pose)
    for view in ("ap", "lateral", "axial"):
        out[f"slice_{view}"] = ren.extract_frequency_slice(*pose, view=view)
        out[f"drr_{view}"] = ren.render_drr(*pose, view=view)
        out[f"drr_nocrop_{view}"] = ren.render_drr(*pose, view=view, crop_to_roi=False)
    t_ap = ren.extract_frequency_slice(0, 0, 0, view="ap")
    t_lat = ren.extract_frequency_slice(0, 0, 0, view="lateral")
    out["ncc_ap"] = np.array(ren.compute_spectral_ncc(out["slice_ap"], t_ap))
    eng = gr.SpectralGradientEngine(ren)
    test_pose = np.array([1.0, -1.0, 0.5, 1.5, -1.0, 2.0])
    loss, grad = eng.compute_biplanar_loss_and_gradients(test_pose, t_ap, t_lat)
    out["bip_pose"] = test_pose
    out["bip_loss"] = np.array(loss)
    out["bip_grad"] = grad
    ncc, du, dv = eng.compute_spectral_ncc_and_grad_translation(out["slice_lateral"], t_lat, view="lateral")
    out["tgrad"] = np.array([ncc, du, dv])
    np.savez_compressed(HERE / "numpy_renderer.npz", **out)


def gen_articulated(ref_root: Path):
    """ArticulatedSpineModel (articulated_spine.py): three segments of one
    shape, spectra and DRRs at an articulated pose, the biplanar objective's
    building blocks at two poses."""
    from fvr import articulated_spine as asp

    out = {}
    segs = []
    for k in range(3):
        sub = _ellipsoids(16, 30 + k, shape=(12, 14, 16)).astype(np.float64)
        out[f"sub{k}"] = sub
        segs.append(asp.VertebralSegment(f"L{3 + k}", sub, nominal_offset_z=12.0 * k))
    model = asp.ArticulatedSpineModel(segs)
    base = np.array([2.0, -1.5, 1.0, 0.75, -0.5, 1.25])
    arts = [np.array([1.5, -0.5, 0.8, 0.3, -0.2, 0.4]), np.array([-1.0, 1.2, -0.6, -0.25, 0.35, -0.3])]
    out["base"] = base
    out["arts"] = np.stack(arts)
    for view in ("ap", "lateral"):
        out[f"spec_{view}"] = model.render_articulated_spectrum(base, arts, view=view)
        out[f"drr_{view}"] = model.render_drr(base, arts, view=view)
    out["spec_ap_noart"] = model.render_articulated_spectrum(base, [], view="ap")
    t_ap = model.render_articulated_spectrum(np.zeros(6), [np.zeros(6)] * 2, view="ap")
    t_lat = model.render_articulated_spectrum(np.zeros(6), [np.zeros(6)] * 2, view="lateral")
    out["ncc_ap"] = np.array(segs[0].renderer.compute_spectral_ncc(out["spec_ap"], t_ap))
    out["ncc_lat"] = np.array(segs[0].renderer.compute_spectral_ncc(out["spec_lateral"], t_lat))
    np.savez_compressed(HERE / "articulated.npz", **out)


def gen_ingest_and_targets(ref_root: Path):
    """resample_isotropic_cube / hu_to_attenuation (dicom_loader.py) on a small
    anisotropic HU volume, and RobustDiffFVREngine._prepare_spectrum
    (core_engine.py:71-85) for the three views."""
    from fvr import core_engine, diff_fvr, dicom_loader

    out = {}
    rng = np.random.default_rng(11)
    hu = (rng.uniform(-1000.0, 1500.0, size=(9, 13, 11))).astype(np.float32)
    spacing = (2.5, 0.8, 1.1)
    out["hu"] = hu
    out["spacing"] = np.array(spacing)
    for n in (16, 23):
        res, sp = dicom_loader.resample_isotropic_cube(hu, spacing, n)
        out[f"resampled_{n}"] = res
        out[f"voxel_mm_{n}"] = np.array(sp[0])
        out[f"mu_{n}"] = dicom_loader.hu_to_attenuation(res)
    vol = _ellipsoids(16, 9, shape=(14, 12, 16)).astype(np.float64)
    out["vol"] = vol
    ren = diff_fvr.DifferentiableFourierVolumeRenderer(vol, pad_factor=2.0)
    holder = type("Holder", (), {})()
    holder.renderer = ren
    for view, shape in (("ap", (14, 16)), ("lateral", (13, 11)), ("axial", (12, 16))):
        img = rng.uniform(0.0, 1.0, size=shape)
        out[f"img_{view}"] = img
        out[f"target_{view}"] = core_engine.RobustDiffFVREngine._prepare_spectrum(holder, img, view)
    np.savez_compressed(HERE / "ingest_targets.npz", **out)


def gen_registration(ref_root: Path):
    """GradientRegistrationOptimizer.register_adam (gradient_optimizer.py:24-90)
    and RobustDiffFVREngine.register_biplanar_robust (core_engine.py:109-224,
    clean and metal branches) on a seeded 32^3 ellipsoid cube: trajectories,
    final poses, losses and evaluation counts."""
    from fvr import core_engine, diff_fvr, gradient_optimizer

    out = {}
    vol = _ellipsoids(32, 21).astype(np.float64)
    out["vol"] = vol
    truth = np.array([1.5, -1.0, 0.8, 0.6, -0.4, 0.5])
    out["truth"] = truth
    ren = diff_fvr.DifferentiableFourierVolumeRenderer(vol, pad_factor=2.0)
    f_ap = ren.extract_frequency_slice(*truth[:3], tx=truth[3], ty=truth[5], view="ap")
    f_lat = ren.extract_frequency_slice(*truth[:3], tx=truth[4], ty=truth[5], view="lateral")
    opt = gradient_optimizer.GradientRegistrationOptimizer(ren)
    r = opt.register_adam(f_ap, f_lat, np.zeros(6), max_iter=12)
    out["adam_losses"] = np.array([t[1] for t in r["trajectory"]])
    out["adam_poses"] = np.stack([t[2] for t in r["trajectory"]])
    out["adam_final_pose"] = r["final_pose"]
    out["adam_final_loss"] = np.array(r["final_loss"])
    out["adam_iterations"] = np.array(r["iterations"])
    eng = core_engine.RobustDiffFVREngine(vol, spacing=(1.0, 1.0, 1.0))
    t_ap = eng.render_calibrated_drr(*truth[:3], tx=truth[3], ty=truth[5], view="ap")
    t_lat = eng.render_calibrated_drr(*truth[:3], tx=truth[4], ty=truth[5], view="lateral")
    out["target_ap"], out["target_lat"] = t_ap, t_lat
    for tag, (a, b) in (("clean", (t_ap, t_lat)), ("metal", (t_ap.copy(), t_lat.copy()))):
        if tag == "metal":
            a[3:10, 20:27] = a.max() * 3.0
            b[22:29, 4:11] = b.max() * 3.0
            out["metal_target_ap"], out["metal_target_lat"] = a, b
        res = eng.register_biplanar_robust(a, b, initial_pose=(0.5, 0.0, -0.3, 0.0, 0.2, 0.0), max_iter=2)
        out[f"robust_{tag}_pose"] = np.asarray(res["final_pose"])
        out[f"robust_{tag}_loss"] = np.array(res["final_loss"])
        out[f"robust_{tag}_evals"] = np.array(res["evaluations"])
        out[f"robust_{tag}_metal"] = np.array(res["metal_detected"])
    np.savez_compressed(HERE / "registration.npz", **out)


def gen_phantom(ref_root: Path):
    """create_spine_phantom (dicom_loader.py:114-176) at the size the
    reference's engine test uses (64) and at odd and non-power-of-two sizes;
    stored as int16 HU (every label is an integer)."""
    from fvr import dicom_loader

    out = {}
    for n in (64, 37, 50, 96):
        vol, sp = dicom_loader.create_spine_phantom(n)
        assert vol.dtype == np.float32 and np.array_equal(vol, np.round(vol))
        out[f"hu_{n}"] = vol.astype(np.int16)
        out[f"spacing_{n}"] = np.array(sp)
    np.savez_compressed(HERE / "phantom.npz", **out)


def main():
    if len(sys.argv) < 2:
        sys.exit("usage: make_golden.py <reference checkout> [name,name,...]")
    ref_root = Path(sys.argv[1])
    only = set(sys.argv[2].split(",")) if len(sys.argv) > 2 else None
    import torch

    torch.set_num_threads(4)
    te, ts, cb, df, gr = _import_reference(ref_root)
    gens = {"slice_warp": lambda: gen_slice_and_warp(ts), "torch_engine": lambda: gen_torch_engine(te),
            "pou": lambda: gen_pou(cb), "numpy_renderer": lambda: gen_numpy(df, gr),
            "articulated": lambda: gen_articulated(ref_root),
            "ingest_targets": lambda: gen_ingest_and_targets(ref_root),
            "phantom": lambda: gen_phantom(ref_root),
            "registration": lambda: gen_registration(ref_root)}
    for name, gen in gens.items():
        if only is None or name in only:
            gen()
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
