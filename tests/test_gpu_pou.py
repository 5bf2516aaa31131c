"""GPU parity of the PoU-FVR cone-beam path (PerspectiveSlabFVR drop-in) and
the pinhole warp-sum against the reference's golden vectors and the float64
oracle, plus mirrors of the reference's tests/test_cone_beam_fvr.py cases.

Tolerances: forward 2e-5 relative L2 against the reference's float32
outputs (its own float32 noise is ~1e-5), 1e-5 against the float64 oracle;
gradients 1e-4 (entries at lattice-point kinks excluded, see
test_oracle_golden.py).
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import pou as opou

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _t(a, dtype=torch.float32):
    return torch.as_tensor(np.asarray(a), dtype=dtype, device=DEV)


@pytest.fixture(scope="module")
def model(golden):
    from fvr.cone_beam_fvr import PerspectiveSlabFVR

    g = golden("pou")
    return PerspectiveSlabFVR.from_volume(g["vol"], vox_mm=2.0, grid_blocks=(2, 2, 2), block_res=12, overlap=0.25)


@pytest.fixture(scope="module")
def lattice(golden):
    from fvr.cone_beam_fvr import PerspectiveSlabFVR

    g = golden("pou")
    return PerspectiveSlabFVR.make_pinhole_lattice(_t(g["k_inv"]), 600.0, 24, 20)


def test_block_decomposition_and_spectra(model, golden):
    g = golden("pou")
    assert model.B == int(g["B"]) and model.P == int(g["P"])
    assert abs(model.ds_block - float(g["ds_block"])) < 1e-12
    assert np.allclose(model.centers.cpu().numpy(), g["centers"], atol=1e-4)
    assert rel_l2(model.F_blk_ri.cpu().numpy(), g["F_blk_ri"]) < 2e-6
    assert np.allclose(model.FX_flat.cpu().numpy(), g["FX_flat"], rtol=1e-6)


def test_block_decomposition_other_grid(golden):
    from fvr.cone_beam_fvr import PerspectiveSlabFVR

    g = golden("pou")
    m2 = PerspectiveSlabFVR.from_volume(g["vol"], vox_mm=1.5, grid_blocks=(3, 2, 1), block_res=10, overlap=0.5,
                                        center_mode="grid_center")
    assert m2.B == int(g["g2_B"])
    assert np.allclose(m2.centers.cpu().numpy(), g["g2_centers"], atol=1e-4)
    assert rel_l2(m2.F_blk_ri.double().sum(dim=(2, 3, 4)).cpu().numpy(), g["g2_F_blk_ri_sum"]) < 2e-6


def test_lattice(lattice, golden):
    g = golden("pou")
    for i, name in enumerate(["src0", "trg0", "u0", "v0", "n0", "rx", "ry", "ic"]):
        assert np.allclose(lattice[i].cpu().numpy(), g[f"lat_{name}"], rtol=1e-5, atol=1e-5), name


@pytest.mark.parametrize("tag", ["inv", "exp"])
def test_forward_pinhole_and_mats_grad(model, lattice, golden, tag):
    g = golden("pou")
    lat = lattice if tag == "inv" else lattice[:5]
    mats = _t(g["mats"]).requires_grad_(True)
    out = model.forward_pinhole(mats, lat)
    assert tuple(out.shape) == g[f"pin_{tag}_out"].shape
    (out * _t(g[f"pin_{tag}_w"])).sum().backward()
    assert rel_l2(out.detach().cpu().numpy(), g[f"pin_{tag}_out"]) < 2e-5
    om = opou.PoUModel(g["vol"], vox_mm=2.0, grid_blocks=(2, 2, 2), block_res=12, overlap=0.25)
    olat = opou.make_pinhole_lattice(g["k_inv"], 600.0, 24, 20)
    ref = opou.forward_pinhole(om, g["mats"], olat) if tag == "inv" else opou.forward_explicit(om, g["mats"], olat)
    assert rel_l2(out.detach().cpu().numpy(), ref) < 1e-5
    gm = mats.grad.cpu().numpy()
    mask = np.ones(gm.shape, bool)
    mask[2, :3, :3] = False  # identity rotation: lattice-point kinks
    assert rel_l2(gm[mask], g[f"pin_{tag}_gmats"][mask]) < 1e-4
    if tag == "inv":
        assert rel_l2(gm[mask], opou.forward_pinhole_grad(om, g["mats"], olat, g["pin_inv_w"])[mask]) < 1e-4


@pytest.mark.parametrize("view", ["ap", "lateral"])
def test_carm_view_and_grads(model, golden, view):
    g = golden("pou")
    params = [torch.tensor(v, requires_grad=True) for v in (3.0, -2.0, 1.5, 1.0, -1.0, 0.5)]
    img = model.forward_carm_view(*params, sad_mm=300.0, sdd_mm=600.0, det_px=20, det_fov_mm=70.0, view=view)
    assert img.device == params[0].device  # results come back on the pose scalars' device
    (img * torch.as_tensor(g[f"carm_{view}_w"], dtype=torch.float32)).sum().backward()
    assert rel_l2(img.detach().cpu().numpy(), g[f"carm_{view}_out"]) < 2e-5
    grads = np.array([float(p.grad) for p in params])
    assert rel_l2(grads, g[f"carm_{view}_grad"]) < 1e-4


def test_warp_sum_dropin(golden):
    from fvr.triton_slice import pou_pinhole_warp_sum

    g = golden("slice_warp")
    t = [_t(g[k]).requires_grad_(True) for k in ("warp_imgs", "warp_db", "warp_cu", "warp_cv")]
    rx, ry, ic = (_t(g[k]) for k in ("warp_rx", "warp_ry", "warp_ic"))
    out = pou_pinhole_warp_sum(t[0], t[1], t[2], t[3], rx, ry, ic, rx.reshape(-1), ry.reshape(-1), ic.reshape(-1),
                               float(g["warp_inv_ds"]), float(g["warp_c_idx"]))
    (out * _t(g["warp_wout"])).sum().backward()
    assert rel_l2(out.detach().cpu().numpy(), g["warp_out"]) < 2e-6
    for x, k in zip(t, ("warp_g_imgs", "warp_g_db", "warp_g_cu", "warp_g_cv")):
        assert rel_l2(x.grad.cpu().numpy(), g[k]) < 1e-5, k


# ------------------------------------------- mirrors of tests/test_cone_beam_fvr.py


def test_pou_windows_sum_to_unity():
    from fvr.cone_beam_fvr import _make_pou_1d

    for length, k in [(64, 2), (96, 3), (128, 4)]:
        ws, _ = _make_pou_1d(length, k, overlap=0.25)
        assert torch.allclose(torch.stack(ws, dim=0).sum(dim=0), torch.ones(length), atol=1e-5)


def test_front_vs_back_magnification():
    from fvr.cone_beam_fvr import PerspectiveSlabFVR

    n, vox = 64, 2.0
    vol = np.zeros((n, n, n), dtype=np.float32)
    zz, yy, xx = np.meshgrid(*(((np.arange(n) - (n - 1) / 2.0) * vox),) * 3, indexing="ij")
    vol[((zz - 16.0) ** 2 + (yy + 32.0) ** 2 + (xx - 24.0) ** 2) < 81.0] = 1.0
    vol[((zz + 16.0) ** 2 + (yy - 32.0) ** 2 + (xx - 24.0) ** 2) < 81.0] = 1.0
    fvr = PerspectiveSlabFVR.from_volume(vol, vox_mm=vox, grid_blocks=(2, 4, 2), block_res=48)
    z0 = torch.tensor(0.0)
    img = fvr.forward_carm_view(z0, z0, z0, z0, z0, z0, sad_mm=300.0, sdd_mm=600.0, det_px=96,
                                det_fov_mm=n * vox, view="ap").cpu()
    u = torch.linspace(-0.5, 0.5, 96) * (n * vox)
    top, bot = img[48:, :], img[:48, :]
    x_front = float((top.sum(dim=0) * u).sum() / top.sum())
    x_back = float((bot.sum(dim=0) * u).sum() / bot.sum())
    assert x_front > x_back + 7.0


def test_cone_beam_gradients_finite_nonzero():
    from fvr.cone_beam_fvr import PerspectiveSlabFVR

    n = 48
    vol = np.zeros((n, n, n), dtype=np.float32)
    zz, yy, xx = np.ogrid[:n, :n, :n]
    vol[((zz - 24) ** 2 + (yy - 24) ** 2 + (xx - 24) ** 2) < 144] = 0.05
    cb = PerspectiveSlabFVR.from_volume(vol, vox_mm=2.0, grid_blocks=(2, 2, 2), block_res=40)
    target = cb.forward_carm_view(*(torch.tensor(v) for v in (3.0, -2.0, 1.5, 1.0, -1.0, 0.5)), sad_mm=600.0,
                                  sdd_mm=900.0, det_px=48, det_fov_mm=96.0, view="ap").detach()
    params = [torch.tensor(0.0, requires_grad=True) for _ in range(6)]
    pred = cb.forward_carm_view(*params, sad_mm=600.0, sdd_mm=900.0, det_px=48, det_fov_mm=96.0, view="ap")
    a0, b0 = pred - pred.mean(), target - target.mean()
    (1.0 - (a0 * b0).sum() / (a0.norm() * b0.norm() + 1e-8)).backward()
    assert all(bool(torch.isfinite(p.grad)) for p in params)
    assert any(abs(float(p.grad)) > 1e-4 for p in params)


def test_grid_vs_pixel_centre():
    from fvr.cone_beam_fvr import PerspectiveSlabFVR

    vol = np.ones((32, 32, 32), dtype=np.float32)
    a = PerspectiveSlabFVR.from_volume(vol, vox_mm=2.5, grid_blocks=(2, 2, 2), block_res=32, center_mode="pixel_center")
    b = PerspectiveSlabFVR.from_volume(vol, vox_mm=2.5, grid_blocks=(2, 2, 2), block_res=32, center_mode="grid_center")
    d = a.centers - b.centers
    assert torch.allclose(d, torch.full_like(d, 1.25), atol=1e-4)
    with pytest.raises(ValueError):
        PerspectiveSlabFVR.from_volume(vol, vox_mm=1.0, center_mode="invalid")


def test_batched_equals_single_and_bf16_parity():
    from fvr.cone_beam_fvr import PerspectiveSlabFVR

    n = 32
    vol = np.zeros((n, n, n), dtype=np.float32)
    zz, yy, xx = np.ogrid[:n, :n, :n]
    vol[((zz - 14) ** 2 + (yy - 17) ** 2 + (xx - 16) ** 2) < 81] = 0.08
    fvr = PerspectiveSlabFVR.from_volume(vol, vox_mm=2.0, grid_blocks=(2, 2, 2), block_res=32)
    H = W = 48
    k_inv = torch.tensor([[[1 / 300.0, 0.0, -W / 600.0], [0.0, 1 / 300.0, -H / 600.0], [0.0, 0.0, 1.0]]])
    lat = fvr.make_pinhole_lattice(k_inv, sdd_mm=600.0, height=H, width=W)
    mats = torch.eye(4).unsqueeze(0).repeat(4, 1, 1)
    mats[:, 2, 3] = -300.0
    mats[:, 0, 3] = torch.tensor([0.0, 4.0, -3.0, 6.0])
    mats[:, 1, 3] = torch.tensor([0.0, -2.0, 5.0, 1.0])
    mats = mats.to(DEV).requires_grad_(True)
    batched = fvr.forward_pinhole(mats, lat)
    assert batched.shape == (4, 1, H, W)
    for b in range(4):
        assert torch.allclose(batched[b:b + 1], fvr.forward_pinhole(mats[b:b + 1].detach(), lat), atol=1e-4)
    batched.sum().backward()
    assert bool(torch.all(torch.isfinite(mats.grad))) and float(mats.grad.abs().sum()) > 1e-4
    f16 = PerspectiveSlabFVR.from_volume(vol, vox_mm=2.0, grid_blocks=(2, 2, 2), block_res=32).to_precision(
        torch.bfloat16)
    m2 = mats.detach().clone().requires_grad_(True)
    out = f16.forward_pinhole(m2, lat)
    out.sum().backward()
    assert out.dtype == torch.float32
    assert torch.allclose(out, batched.detach(), atol=0.15, rtol=0.05)
    assert float(m2.grad.abs().sum()) > 1e-4


@pytest.mark.parametrize("W,pinhole", [(256, False), (384, False), (512, False), (320, False), (256, True)])
def test_warp_row_strips_match_oracle(W, pinhole):
    """Detector rows of 256 pixels (one CTA each) take the row-strip warp:
    exactly uniform rows, widths whose CTAs alternate between one-row and
    two-row (per-pixel) paths (384), cover half a row each (512) or end in a
    partly filled one-row CTA (320: the last CTA holds 192 pixels), and the
    pinhole lattice whose rows agree only to float rounding.  20 blocks span two strip rounds; positions fall
    inside, on and beyond every image edge.  Same bounds as the golden
    warp case: 2e-6 forward, 1e-5 gradients against the float64 oracle."""
    from fvr.cone_beam_fvr import PerspectiveSlabFVR
    from fvr.triton_slice import pou_pinhole_warp_sum

    rng = np.random.default_rng(31)
    B, N, P, H = 20, 2, 24, 6
    imgs = rng.standard_normal((B, N, P, P)).astype(np.float32)
    db = rng.uniform(260.0, 320.0, (B, N)).astype(np.float32)
    cu = rng.uniform(-10.0, 10.0, (B, N)).astype(np.float32)
    cv = rng.uniform(-10.0, 10.0, (B, N)).astype(np.float32)
    inv_ds, c_idx = 0.4, 12.0
    if pinhole:
        k_inv = torch.tensor([[1 / 2000.0, 0.0, -W / 4000.0], [0.0, 1 / 1500.0, -0.1], [0.0, 0.0, 1.0]])
        lat = PerspectiveSlabFVR.make_pinhole_lattice(k_inv, 1000.0, H, W)
        rx, ry, ic = (t.cpu().numpy().astype(np.float32) for t in lat[5:8])
    else:
        rx = np.broadcast_to(np.linspace(-0.12, 0.12, W, dtype=np.float32), (H, W)).copy()
        ry = np.broadcast_to(np.array([-0.1, -0.06, -0.01, 0.03, 0.07, 0.11], np.float32)[:, None], (H, W)).copy()
        ic = rng.uniform(0.95, 1.0, (H, W)).astype(np.float32)
    t = [_t(a).requires_grad_(True) for a in (imgs, db, cu, cv)]
    out = pou_pinhole_warp_sum(t[0], t[1], t[2], t[3], _t(rx), _t(ry), _t(ic), _t(rx).reshape(-1),
                               _t(ry).reshape(-1), _t(ic).reshape(-1), inv_ds, c_idx)
    wout = rng.standard_normal((N, H, W)).astype(np.float32)
    (out * _t(wout)).sum().backward()
    f64 = [a.astype(np.float64) for a in (imgs, db, cu, cv, rx, ry, ic)]
    ref = opou.warp_sum(*f64, inv_ds, c_idx)
    assert rel_l2(out.detach().cpu().numpy(), ref) < 2e-6
    grads = opou.warp_sum_adjoint(*f64, inv_ds, c_idx, wout.astype(np.float64))
    for x, r, k in zip(t, grads, ("imgs", "db", "cu", "cv")):
        assert rel_l2(x.grad.cpu().numpy(), r) < 1e-5, k


def test_invariant_matches_explicit_rays():
    from fvr.cone_beam_fvr import PerspectiveSlabFVR

    vol = torch.zeros((48, 48, 48))
    vol[14:34, 16:32, 18:30] = 1.5
    fvr = PerspectiveSlabFVR.from_volume(vol, vox_mm=2.0, grid_blocks=(2, 2, 2), block_res=32)
    H = W = 28
    k_inv = torch.tensor([[1 / 300.0, 0.0, -W / 600.0], [0.0, 1 / 300.0, -H / 600.0], [0.0, 0.0, 1.0]])
    lat11 = fvr.make_pinhole_lattice(k_inv, sdd_mm=600.0, height=H, width=W)

    def se3(rv, tr):
        skew = torch.zeros((rv.shape[0], 3, 3), dtype=rv.dtype, device=rv.device)
        skew[:, 0, 1], skew[:, 1, 0] = -rv[:, 2], rv[:, 2]
        skew[:, 0, 2], skew[:, 2, 0] = rv[:, 1], -rv[:, 1]
        skew[:, 1, 2], skew[:, 2, 1] = -rv[:, 0], rv[:, 0]
        m = torch.eye(4, dtype=rv.dtype, device=rv.device).unsqueeze(0).repeat(rv.shape[0], 1, 1)
        m[:, :3, :3] = torch.matrix_exp(skew)
        m[:, :3, 3] = tr
        return m

    rot0 = torch.tensor([[0.15, -0.10, 0.08], [-0.20, 0.12, -0.05]])
    xyz0 = torch.tensor([[5.0, -4.0, -300.0], [-3.0, 6.0, -310.0]])
    r1, t1 = rot0.clone().requires_grad_(True), xyz0.clone().requires_grad_(True)
    o1 = fvr.forward_pinhole(se3(r1, t1), lat11)
    w = torch.randn_like(o1)
    (o1 * w).sum().backward()
    r2, t2 = rot0.clone().requires_grad_(True), xyz0.clone().requires_grad_(True)
    o2 = fvr.forward_pinhole(se3(r2, t2), lat11[:5])
    (o2 * w).sum().backward()
    assert torch.allclose(o1, o2, atol=1e-4, rtol=1e-4)
    assert torch.allclose(r1.grad, r2.grad, atol=5e-4, rtol=1e-3)
    assert torch.allclose(t1.grad, t2.grad, atol=5e-4, rtol=1e-3)


def test_presets_and_parity_offsets():
    from fvr.cone_beam_fvr import SLAB_PRESETS, PerspectiveSlabFVR, sample_isocenter_parity_offsets

    assert SLAB_PRESETS["isotropic"]["grid_blocks"] == (4, 4, 4) and SLAB_PRESETS["isotropic"]["block_res"] == 64
    vol = np.zeros((32, 32, 32), dtype=np.float32)
    vol[8:24, 8:24, 8:24] = 0.5
    iso = PerspectiveSlabFVR.from_volume(vol, vox_mm=2.0, preset="isotropic", block_res=16)
    assert iso.B == 64 and iso.F_blk_ri.dtype == torch.bfloat16
    with pytest.raises(ValueError):
        PerspectiveSlabFVR.resolve_slab_preset("nonexistent")
    offs = sample_isocenter_parity_offsets((1.0, 2.0, 4.0))
    assert offs.shape == (27, 3)
    assert torch.allclose(offs.abs().max(dim=0).values, torch.tensor([0.5, 1.0, 2.0]))


@pytest.mark.parametrize("block_res,det,dtype,grid", [(32, 64, torch.float32, 3), (48, 96, torch.bfloat16, 3),
                                                      (64, 256, torch.float32, 3), (64, 128, torch.float16, 3),
                                                      (32, 256, torch.float32, 3), (32, 256, torch.float32, 2)])
def test_fused_warp_adjoint_matches_two_kernel_path(block_res, det, dtype, grid):
    """On a separable pinhole lattice the backward takes the fused warp +
    block-image adjoint (fvr_pou_warp_image_adjoint: dL/dimgs formed in shared
    memory by a gather along detector rows); its pose gradient equals the
    two-kernel path's (fvr_pou_warp_bwd scatter + fvr_pou_slice_image_adjoint).
    The last two cases put about five and seven detector columns on each image
    column: the kernel's 12-tap register layout, then (more taps than that)
    its column loops."""
    import fvr._lib as L
    from fvr import synthetic
    from fvr.cone_beam_fvr import PerspectiveSlabFVR, _prepared_lattice

    vol = synthetic.make_ellipsoid_volume(96, 0)
    m = PerspectiveSlabFVR.from_volume(vol, vox_mm=2.0, grid_blocks=(grid,) * 3, block_res=block_res, overlap=0.5,
                                       dtype=dtype)
    f = 1020.0 / (3.2 * 64 / det)
    k_inv = np.array([[1 / f, 0, -0.5 * det / f], [0, 1 / f, -0.5 * det / f], [0, 0, 1.0]])
    lat = m.make_pinhole_lattice(_t(k_inv), 1020.0, det, det)
    assert _prepared_lattice(lat, m._dev)[4] is not None
    assert L.query("fvr_pou_warp_image_adjoint_supported", m.P, det, det) == 1
    mats = synthetic.make_pinhole_mats(4, 3, sad_mm=765.0)
    grads, outs = [], []
    for fused in (True, False):
        m.fused_warp_adjoint = fused
        mm = mats.to(DEV).requires_grad_(True)
        out = m.forward_pinhole(mm, lat)
        w = torch.from_numpy(np.random.default_rng(5).standard_normal(out.shape).astype(np.float32)).to(DEV)
        (out * w).sum().backward()
        grads.append(mm.grad.cpu().numpy())
        outs.append(out.detach().cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
    assert np.abs(grads[1]).max() > 0
    assert rel_l2(grads[0], grads[1]) < 1e-5


def test_full_geometry_subset_vs_oracle():
    """4x4x4 blocks, 50 % overlap, block_res 32 on a seeded 96^3 volume, 256x... pinhole
    at SDD 1020 / SAD 765: forward and mats gradient against the float64 oracle."""
    from fvr import synthetic
    from fvr.cone_beam_fvr import PerspectiveSlabFVR

    vol = synthetic.make_ellipsoid_volume(96, 0)
    fvr = PerspectiveSlabFVR.from_volume(vol, vox_mm=2.0, grid_blocks=(4, 4, 4), block_res=32, overlap=0.5)
    om = opou.PoUModel(vol, vox_mm=2.0, grid_blocks=(4, 4, 4), block_res=32, overlap=0.5)
    assert fvr.B == om.B
    H = 64
    f = 1020.0 / 3.2
    k_inv = np.array([[1 / f, 0, -0.5 * H / f], [0, 1 / f, -0.5 * H / f], [0, 0, 1.0]])
    lat = fvr.make_pinhole_lattice(_t(k_inv), 1020.0, H, H)
    olat = opou.make_pinhole_lattice(k_inv, 1020.0, H, H)
    mats = synthetic.make_pinhole_mats(3, 1, sad_mm=765.0)
    m = mats.to(DEV).requires_grad_(True)
    out = fvr.forward_pinhole(m, lat)
    w = np.random.default_rng(2).standard_normal(out.shape).astype(np.float32)
    (out * _t(w)).sum().backward()
    ref = opou.forward_pinhole(om, mats.numpy(), olat)
    assert rel_l2(out.detach().cpu().numpy(), ref) < 1e-5
    gref = opou.forward_pinhole_grad(om, mats.numpy(), olat, w)
    assert rel_l2(m.grad.cpu().numpy(), gref) < 1e-4


# ----------------------------------------------------- edge-dominant NCC (a17)


def _edge_torch64(pred, target, crop, w):
    """Plain PyTorch float64 statement of the edge-dominant NCC per item [B]
    (test reference for the CUDA kernel's values and autograd gradients)."""
    import torch.nn.functional as F

    kx = torch.tensor([[-1.0, 0, 1], [-2, 0, 2], [-1, 0, 1]], dtype=torch.float64, device=pred.device)
    kx = kx.view(1, 1, 3, 3).repeat(pred.shape[1], 1, 1, 1)
    ky = kx.transpose(-1, -2).contiguous()
    C = pred.shape[1]

    def resp(x, k):
        r = F.conv2d(x, k, padding=1, groups=C)
        return r[..., crop:r.shape[-2] - crop, crop:r.shape[-1] - crop]

    def ncc(u, v):
        u0 = u - u.mean((-2, -1), keepdim=True)
        v0 = v - v.mean((-2, -1), keepdim=True)
        den = ((u0 * u0).sum((-2, -1)) * (v0 * v0).sum((-2, -1))).clamp(min=1e-12).sqrt()
        return ((u0 * v0).sum((-2, -1)) / den).mean(1)

    def scale(a, b):
        return 0.5 * (ncc(resp(a, kx), resp(b, kx)) + ncc(resp(a, ky), resp(b, ky)))

    val = scale(pred, target.expand_as(pred))
    if w > 0 and pred.shape[-1] >= 96:
        box = lambda x: F.avg_pool2d(x, 3, stride=1, padding=1)  # noqa: E731
        val = (1 - w) * val + w * scale(box(pred), box(target.expand_as(pred)))
    return val


@pytest.mark.parametrize("H", [48, 96])
def test_edge_dominant_ncc_golden(golden, H):
    from fvr.cone_beam_fvr import edge_dominant_ncc

    g = golden("pou")
    a = _t(g[f"edge_{H}_a"]).requires_grad_(True)
    b = _t(g[f"edge_{H}_b"])
    val = edge_dominant_ncc(a, b, reduction="none")
    val.sum().backward()
    assert rel_l2(val.detach().cpu().numpy(), g[f"edge_{H}_val"]) < 1e-5
    assert rel_l2(a.grad.cpu().numpy(), g[f"edge_{H}_grad"]) < 1e-4
    ref = opou.edge_dominant_ncc(g[f"edge_{H}_a"], g[f"edge_{H}_b"], reduction="none")
    assert np.allclose(val.detach().cpu().numpy(), ref, rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("B,Bt,C,H,W,crop,w,mean", [
    (3, 1, 1, 64, 112, None, 0.25, True),     # broadcast target, rectangular, blurred scale on
    (2, 2, 2, 100, 96, 0, 0.4, False),        # no crop: zero-padded borders enter the moments
    (4, 4, 1, 130, 70, 7, 0.25, False),       # last dim < 96: fine scale only
    (1, 1, 1, 256, 256, None, 0.25, True),    # detector size of the PoU workload
])
def test_edge_dominant_ncc_vs_torch64(B, Bt, C, H, W, crop, w, mean):
    from fvr.cone_beam_fvr import edge_dominant_ncc

    rng = np.random.default_rng(B * 100 + H)
    pa = rng.standard_normal((B, C, H, W)).cumsum(-1).cumsum(-2)
    pb = pa[:Bt] + 0.3 * rng.standard_normal((Bt, C, H, W)).cumsum(-2)
    a = _t(pa).requires_grad_(True)
    b = _t(pb).requires_grad_(True)
    val = edge_dominant_ncc(a, b, border_crop=crop, multiscale_weight=w, reduction="mean" if mean else "none")
    (val * torch.arange(1, val.numel() + 1, device=DEV, dtype=torch.float32).reshape(val.shape)).sum().backward()
    a64 = torch.tensor(pa, dtype=torch.float64, device=DEV, requires_grad=True)
    b64 = torch.tensor(pb, dtype=torch.float64, device=DEV, requires_grad=True)
    c = max(4, W // 8) if crop is None else crop
    ref = _edge_torch64(a64, b64, c, w)
    ref = ref.mean() if mean else ref
    (ref * torch.arange(1, ref.numel() + 1, device=DEV, dtype=torch.float64).reshape(ref.shape)).sum().backward()
    assert rel_l2(val.detach().double().cpu().numpy(), ref.detach().cpu().numpy()) < 1e-6
    assert rel_l2(a.grad.double().cpu().numpy(), a64.grad.cpu().numpy()) < 1e-4
    assert rel_l2(b.grad.double().cpu().numpy(), b64.grad.cpu().numpy()) < 1e-4


# ------------------------------------------------ fused block-image kernels


@pytest.mark.parametrize("block_res,dtype", [(32, torch.float32), (48, torch.bfloat16), (48, torch.float16),
                                             (64, torch.float32), (64, torch.bfloat16), (80, torch.float32),
                                             (80, torch.float16)])
def test_fused_block_images_match_slice_plus_fft(block_res, dtype):
    """fvr_pou_slice_image (slice + inverse FFT in one CTA) and its adjoint
    equal the unfused slice kernel + batched FFT path, P = 2 x block_res in
    {64, 96, 128, 160}.

    The fused kernels read one sample of each Hermitian pair (S(-k) =
    conj S(k)) where the unfused path reads both.  The two are separate
    roundings of conjugate spectrum values: identical in f32 up to the FFT's
    own rounding, and one 16-bit step apart wherever that rounding moves a
    value across a 16-bit boundary (block spectra of lengths with a factor 3
    or 5), hence the looser 16-bit bounds."""
    import ctypes

    import fvr._lib as L
    from fvr import _runtime as RT
    from fvr.cone_beam_fvr import PerspectiveSlabFVR
    from fvr.synthetic import make_ellipsoid_volume, make_pinhole_mats

    vol = make_ellipsoid_volume(64, 3)
    m = PerspectiveSlabFVR.from_volume(vol, vox_mm=1.5, grid_blocks=(2, 2, 2), block_res=block_res, overlap=0.5,
                                       dtype=dtype)
    B, P, N = m.B, m.P, 3
    assert L.query("fvr_pou_image_supported", P) == 1
    dev = m._dev
    mats = make_pinhole_mats(N, 4, sad_mm=400.0, device=dev).to(torch.float32).contiguous()
    geo = torch.empty((N, int(L.query("fvr_pou_geo_stride"))), dtype=torch.float64, device=dev)
    offs = torch.empty((B, N, 3), dtype=torch.float64, device=dev)
    base = (ctypes.c_double * 12)(*([0.0] * 3 + [1.0, 0, 0] + [0, 1.0, 0] + [0, 0, 1.0]))
    s = L.stream_ptr(dev)
    L.call("fvr_pou_pose", L.ptr(mats), None, N, base, float(P) * m.ds_block, L.ptr(m.centers), B, L.ptr(geo),
           L.ptr(offs), s)
    st = m._stencil
    fused = torch.empty((B, N, P, P), dtype=torch.float32, device=dev)
    L.call("fvr_pou_slice_image", st.code, L.ptr(st.data), L.ptr(st.scales), B, P, L.ptr(geo), N,
           L.ptr(m._freqs), L.ptr(fused), s)
    slices = torch.empty((B, N, P, P), dtype=torch.complex64, device=dev)
    L.call("fvr_pou_slice", st.code, L.ptr(st.data), L.ptr(st.scales), B, P, L.ptr(geo), N, L.ptr(m._freqs),
           L.ptr(slices), s)
    ref = RT.fft2d(slices, inverse=True, out_shift=RT.SHIFT_FFT, scale=1.0 / (P * P), out_mode=RT.OUT_REAL)
    tol_fwd, tol_adj = (2e-6, 2e-5) if dtype == torch.float32 else (1e-5, 2e-4)
    assert rel_l2(fused.cpu().numpy(), ref.cpu().numpy()) < tol_fwd
    # adjoint against the unfused FFT + slice adjoint (tile sums)
    g = torch.from_numpy(np.random.default_rng(1).standard_normal((B, N, P, P)).astype(np.float32)).to(dev)
    wsb = L.query("fvr_pou_slice_image_adjoint_workspace", B, N)
    ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
    L.call("fvr_pou_slice_image_adjoint", st.code, L.ptr(st.data), L.ptr(st.scales), B, P, L.ptr(geo), N,
           L.ptr(m._freqs), L.ptr(g), L.ptr(ws), wsb, s)
    got = ws[: N * B * 6 * 8].view(torch.float64).view(N, B, 6).cpu().numpy()
    G = RT.fft2d(g, inverse=False, in_shift=RT.SHIFT_IFFT, out_shift=RT.SHIFT_FFT, scale=1.0 / (P * P))
    wsb2 = L.query("fvr_pou_slice_adjoint_workspace", B, P, N)
    ws2 = torch.empty(wsb2, dtype=torch.uint8, device=dev)
    L.call("fvr_pou_slice_adjoint", st.code, L.ptr(st.data), L.ptr(st.scales), B, P, L.ptr(geo), N,
           L.ptr(m._freqs), L.ptr(G), L.ptr(ws2), wsb2, s)
    tiles = (P * P + 255) // 256
    want = ws2[: N * B * tiles * 6 * 8].view(torch.float64).view(N, B, tiles, 6).sum(2).cpu().numpy()
    assert rel_l2(got, want) < tol_adj
