"""The reference's tests hand the drop-in CPU tensors and NumPy arrays
(tests/test_torch_engine.py, tests/test_cone_beam_fvr.py of the reference).
These cases run the same calls with CPU inputs: the work runs on the CUDA
device and results and gradients come back on the inputs' device.  Also the
spine phantom of the engine test's fixture, exact against the reference's
own output.

Tolerances: the golden cases keep the bounds of their CUDA-input twins
(slice 1e-5 / gradients 1e-4 against the reference's float32 output, warp
2e-6 / 1e-5); the phantom's HU labels are compared exactly.
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [64, 37, 50, 96])
def test_spine_phantom_exact(golden, n):
    from fvr.dicom_loader import create_spine_phantom

    vol, spacing = create_spine_phantom(n)
    g = golden("phantom")
    assert isinstance(vol, np.ndarray) and vol.dtype == np.float32 and vol.shape == (n, n, n)
    assert tuple(spacing) == tuple(g[f"spacing_{n}"])
    assert np.array_equal(vol, g[f"hu_{n}"].astype(np.float32))


def test_spine_phantom_engine_fixture():
    """The reference engine test's set-up: phantom(64) -> attenuation ->
    engine with spacing 1.5; batched AP / lateral images of four poses are
    finite and non-negative, and the pose gradient is finite and non-zero."""
    from fvr import TorchDiffFVREngine
    from fvr.dicom_loader import create_spine_phantom, hu_to_attenuation

    vol_hu, _ = create_spine_phantom(size=64)
    vol = torch.from_numpy(hu_to_attenuation(vol_hu)).float()
    eng = TorchDiffFVREngine(vol, spacing=(1.5, 1.5, 1.5), pad_factor=2.0)
    poses = torch.tensor([[0.0] * 6, [5.0, 0, 0, 0, 0, 0], [0, 5.0, 0, 0, 0, 0], [2.0, -3.0, 1.5, 4.0, -2.0, 1.0]])
    for view in ("ap", "lateral"):
        img = eng(poses, view=view, out_res=64)
        assert img.shape == (4, 1, 64, 64)
        assert bool(torch.all(torch.isfinite(img))) and bool(torch.all(img >= 0.0))
    p = torch.tensor([[3.0, -2.0, 1.0, 5.0, -3.0, 2.0]], requires_grad=True)
    (eng(p, view="ap", out_res=64) ** 2).sum().backward()
    assert p.grad.shape == (1, 6) and p.grad.device.type == "cpu"
    assert bool(torch.all(torch.isfinite(p.grad))) and not bool(torch.all(p.grad == 0))


def test_slice_cpu_inputs(golden):
    from fvr.triton_slice import fourier_slice_3d_torch, trilinear_slice_analytical_ref

    g = golden("slice_warp")
    vol = torch.from_numpy(g["slice_vol"])
    fx, fy = torch.from_numpy(g["slice_fx"]), torch.from_numpy(g["slice_fy"])
    c = tuple(float(x) for x in g["slice_center"])
    wout = torch.from_numpy(g["slice_wout"])
    for fn in (fourier_slice_3d_torch, trilinear_slice_analytical_ref):
        u = torch.from_numpy(g["slice_u"]).clone().requires_grad_(True)
        v = torch.from_numpy(g["slice_v"]).clone().requires_grad_(True)
        out = fn(vol, u, v, fx, fy, c)
        assert out.device.type == "cpu" and out.dtype == torch.float32
        (out * wout).sum().backward()
        assert u.grad.device.type == "cpu"
        assert rel_l2(out.detach().numpy(), g["slice_out"]) < 1e-5
        assert rel_l2(u.grad.numpy(), g["slice_gu"]) < 1e-4
        assert rel_l2(v.grad.numpy(), g["slice_gv"]) < 1e-4


def test_warp_cpu_inputs(golden):
    from fvr.triton_slice import pou_pinhole_warp_sum_analytical_ref, pou_pinhole_warp_sum_torch

    g = golden("slice_warp")
    rx, ry, ic = (torch.from_numpy(g[k]) for k in ("warp_rx", "warp_ry", "warp_ic"))
    for fn in (pou_pinhole_warp_sum_torch, pou_pinhole_warp_sum_analytical_ref):
        t = [torch.from_numpy(g[k]).clone().requires_grad_(True) for k in ("warp_imgs", "warp_db", "warp_cu",
                                                                             "warp_cv")]
        out = fn(t[0], t[1], t[2], t[3], rx, ry, ic, float(g["warp_inv_ds"]), float(g["warp_c_idx"]))
        assert out.device.type == "cpu"
        (out * torch.from_numpy(g["warp_wout"])).sum().backward()
        assert rel_l2(out.detach().numpy(), g["warp_out"]) < 2e-6
        for x, k in zip(t, ("warp_g_imgs", "warp_g_db", "warp_g_cu", "warp_g_cv")):
            assert x.grad.device.type == "cpu"
            assert rel_l2(x.grad.numpy(), g[k]) < 1e-5, k


def test_edge_ncc_cpu_inputs():
    """The reference's vignetting-invariance case with CPU images."""
    from fvr.cone_beam_fvr import edge_dominant_ncc

    H = 96
    yy, xx = torch.meshgrid(torch.linspace(-1, 1, H), torch.linspace(-1, 1, H), indexing="ij")
    img = torch.exp(-((xx - 0.1) ** 2 + (yy + 0.05) ** 2) / 0.04) + 0.5 * ((xx ** 2 + yy ** 2) < 0.25).float()
    ref = img[None, None]
    vig = ref.clone() + 0.8 * xx[None, None]
    vig[:, :, :6, :] = -10.0
    vig[:, :, -6:, :] = -10.0
    shifted = torch.roll(ref, shifts=(4, 4), dims=(-2, -1))
    same = edge_dominant_ncc(ref, ref)
    assert same.device.type == "cpu"
    assert float(same) > 0.999
    assert float(edge_dominant_ncc(ref, vig)) > 0.98
    assert float(edge_dominant_ncc(shifted, vig)) < 0.50


def test_pinhole_cpu_mats_and_lattice(golden):
    """forward_pinhole with a CPU lattice and CPU pose matrices: the result and
    the matrices' gradient on the CPU, equal to the CUDA-input call."""
    from fvr.cone_beam_fvr import PerspectiveSlabFVR

    g = golden("pou")
    model = PerspectiveSlabFVR.from_volume(g["vol"], vox_mm=2.0, grid_blocks=(2, 2, 2), block_res=12, overlap=0.25)
    lat_cpu = model.make_pinhole_lattice(torch.from_numpy(g["k_inv"]).float(), 600.0, 24, 20)
    assert all(t.device.type == "cpu" for t in lat_cpu)
    m_cpu = torch.from_numpy(g["mats"]).float().requires_grad_(True)
    out_cpu = model.forward_pinhole(m_cpu, lat_cpu)
    (out_cpu * torch.from_numpy(g["pin_inv_w"]).float()).sum().backward()
    assert out_cpu.device.type == "cpu" and m_cpu.grad.device.type == "cpu"
    assert rel_l2(out_cpu.detach().numpy(), g["pin_inv_out"]) < 2e-5
    lat_gpu = model.make_pinhole_lattice(torch.from_numpy(g["k_inv"]).float().cuda(), 600.0, 24, 20)
    m_gpu = torch.from_numpy(g["mats"]).float().cuda().requires_grad_(True)
    out_gpu = model.forward_pinhole(m_gpu, lat_gpu)
    (out_gpu * torch.from_numpy(g["pin_inv_w"]).float().cuda()).sum().backward()
    assert torch.equal(out_cpu.detach(), out_gpu.detach().cpu())
    # the warp adjoint accumulates with atomics: equal up to the order of float additions
    assert rel_l2(m_cpu.grad.numpy(), m_gpu.grad.cpu().numpy()) < 1e-5


def test_empty_batches_follow_torch_semantics():
    """No candidate poses: empty image batches, and the spectral NCC of an
    empty batch is NaN (1 - the mean over nothing, as the reference's torch
    code gives); gradients flow to the empty pose tensors."""
    from fvr import TorchDiffFVREngine
    from fvr.cone_beam_fvr import PerspectiveSlabFVR
    from fvr.synthetic import make_ellipsoid_volume

    eng = TorchDiffFVREngine(torch.from_numpy(make_ellipsoid_volume(16, 2)))
    p0 = torch.zeros((0, 6), requires_grad=True)
    img = eng(p0, view="ap", out_res=16)
    assert img.shape == (0, 1, 16, 16)
    ft = eng.prepare_spectral_target(eng(torch.zeros((1, 6)), view="ap", out_res=16))
    loss = eng.forward_spectral_ncc(p0, ft, view="ap")
    assert bool(torch.isnan(loss))
    (img.sum() + 0.0 * loss.nan_to_num()).backward()
    assert p0.grad is not None and p0.grad.shape == (0, 6)
    m = PerspectiveSlabFVR.from_volume(make_ellipsoid_volume(32, 3), vox_mm=2.0, grid_blocks=(2, 2, 2), block_res=16)
    k_inv = torch.tensor([[1 / 300.0, 0.0, -0.05], [0.0, 1 / 300.0, -0.05], [0.0, 0.0, 1.0]])
    lat = m.make_pinhole_lattice(k_inv, 600.0, 30, 30)
    out = m.forward_pinhole(torch.zeros((0, 4, 4)), lat)
    assert out.shape == (0, 1, 30, 30)
