"""GPU parity of the NumPy-convention renderer and gradient engine
(``DifferentiableFourierVolumeRenderer``, src/fvr/diff_fvr.py;
``SpectralGradientEngine``, src/fvr/gradients.py) against the golden vectors
and the float64 NumPy oracle.  Everything here is fp64 end to end, so the
bar is 1e-10 relative."""
import numpy as np
import pytest

from conftest import rel_l2
from oracle import numpy_convention as nc

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.fixture(scope="module")
def fvr_np():
    import fvr.diff_fvr as df
    import fvr.gradients as gr

    return df, gr


def _ellipsoids(shape, seed):
    from oracle.torch_convention import make_ellipsoid_volume

    return make_ellipsoid_volume(max(shape), seed, shape=shape).astype(np.float64)


def test_spectrum_golden(fvr_np, golden):
    df, _ = fvr_np
    g = golden("numpy_renderer")
    ren = df.DifferentiableFourierVolumeRenderer(g["vol"], pad_factor=2.0)
    assert (ren.pz, ren.py, ren.px) == g["f_3d"].shape
    assert rel_l2(ren.f_3d, g["f_3d"]) < TOL
    ren2 = df.DifferentiableFourierVolumeRenderer(g["vol"], pad_factor=2.0, apply_premultiplication=False)
    assert rel_l2(ren2.f_3d, g["f_3d_nopremult"]) < TOL


@pytest.mark.parametrize("view", ["ap", "lateral", "axial"])
def test_slices_and_drr_golden(fvr_np, golden, view):
    df, _ = fvr_np
    g = golden("numpy_renderer")
    ren = df.DifferentiableFourierVolumeRenderer(g["vol"], pad_factor=2.0)
    pose = tuple(float(x) for x in g["pose5"])
    assert rel_l2(ren.extract_frequency_slice(*pose, view=view), g[f"slice_{view}"]) < TOL
    drr = ren.render_drr(*pose, view=view)
    assert drr.shape == g[f"drr_{view}"].shape
    assert rel_l2(drr, g[f"drr_{view}"]) < TOL
    assert rel_l2(ren.render_drr(*pose, view=view, crop_to_roi=False), g[f"drr_nocrop_{view}"]) < TOL


def test_ncc_and_gradients_golden(fvr_np, golden):
    df, gr = fvr_np
    g = golden("numpy_renderer")
    ren = df.DifferentiableFourierVolumeRenderer(g["vol"], pad_factor=2.0)
    t_ap = ren.extract_frequency_slice(0, 0, 0, view="ap")
    t_lat = ren.extract_frequency_slice(0, 0, 0, view="lateral")
    assert abs(ren.compute_spectral_ncc(g["slice_ap"], t_ap) - float(g["ncc_ap"])) < 1e-12
    eng = gr.SpectralGradientEngine(ren)
    loss, grad = eng.compute_biplanar_loss_and_gradients(g["bip_pose"], t_ap, t_lat)
    assert abs(loss - float(g["bip_loss"])) < 1e-12
    assert np.allclose(grad, g["bip_grad"], rtol=1e-8, atol=1e-12)
    tg = eng.compute_spectral_ncc_and_grad_translation(g["slice_lateral"], t_lat, view="lateral")
    assert np.allclose(tg, g["tgrad"], rtol=1e-9, atol=1e-13)


@pytest.mark.parametrize("shape,pad", [((20, 17, 23), 1.5), ((24, 24, 24), 2.0), ((9, 31, 12), 2.5)])
def test_ragged_sizes_vs_oracle(fvr_np, shape, pad):
    """Odd, non-power-of-two padded sizes (generic radices), large rotations
    that push samples over the strict map_coordinates edge."""
    df, gr = fvr_np
    vol = _ellipsoids(shape, 11)
    ren = df.DifferentiableFourierVolumeRenderer(vol, pad_factor=pad)
    f3d = nc.spectrum(vol, pad)
    assert rel_l2(ren.f_3d, f3d) < TOL
    rng = np.random.default_rng(3)
    for view in ("ap", "lateral", "axial"):
        pose = tuple(rng.uniform(-40, 40, 3)) + tuple(rng.uniform(-3, 3, 2))
        assert rel_l2(ren.extract_frequency_slice(*pose, view=view),
                      nc.extract_frequency_slice(f3d, *pose, view=view)) < TOL
        for crop in (True, False):
            assert rel_l2(ren.render_drr(*pose, view=view, crop_to_roi=crop),
                          nc.render_drr(f3d, shape, *pose, view=view, crop_to_roi=crop)) < TOL
    t_ap = nc.extract_frequency_slice(f3d, view="ap")
    t_lat = nc.extract_frequency_slice(f3d, view="lateral")
    pose6 = np.array([2.0, -3.0, 1.0, 0.7, -1.2, 0.4])
    loss, grad = gr.SpectralGradientEngine(ren).compute_biplanar_loss_and_gradients(pose6, t_ap, t_lat)
    loss_o, grad_o = nc.biplanar_loss_and_gradients(f3d, pose6, t_ap, t_lat)
    assert abs(loss - loss_o) < 1e-12
    assert np.allclose(grad, grad_o, rtol=1e-8, atol=1e-11)


def test_cube_translation_gradient_matches_finite_differences(fvr_np):
    """Mirror of tests/test_gradient_numerical.py: 32^3 cube, the closed-form
    translation gradient against central differences of the loss."""
    df, gr = fvr_np
    cube = np.zeros((32, 32, 32))
    cube[10:22, 10:22, 10:22] = 1.0
    ren = df.DifferentiableFourierVolumeRenderer(cube, pad_factor=2.0)
    eng = gr.SpectralGradientEngine(ren)
    t_ap = ren.extract_frequency_slice(0, 0, 0, view="ap")
    t_lat = ren.extract_frequency_slice(0, 0, 0, view="lateral")
    pose = np.array([1.0, -1.0, 0.5, 1.5, -1.0, 2.0])
    _, grad = eng.compute_biplanar_loss_and_gradients(pose, t_ap, t_lat)

    def loss(p):
        yaw, pitch, roll, tx, ty, tz = p
        a = ren.extract_frequency_slice(yaw, pitch, roll, tx=tx, ty=tz, view="ap")
        b = ren.extract_frequency_slice(yaw, pitch, roll, tx=ty, ty=tz, view="lateral")
        return 0.5 * (1 - ren.compute_spectral_ncc(a, t_ap)) + 0.5 * (1 - ren.compute_spectral_ncc(b, t_lat))

    eps = 1e-4
    for i in range(3, 6):
        pp, pm = pose.copy(), pose.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (loss(pp) - loss(pm)) / (2 * eps)
        assert abs(fd - grad[i]) < 1e-6 * max(1.0, abs(fd))


def test_zero_norm_gives_zero(fvr_np):
    df, gr = fvr_np
    vol = _ellipsoids((12, 12, 12), 2)
    ren = df.DifferentiableFourierVolumeRenderer(vol)
    t = ren.extract_frequency_slice(view="ap")
    z = np.zeros_like(t)
    assert ren.compute_spectral_ncc(z, t) == 0.0
    assert gr.SpectralGradientEngine(ren).compute_spectral_ncc_and_grad_translation(z, t) == (0.0, 0.0, 0.0)
    with pytest.raises(ValueError):
        ren.compute_spectral_ncc(t, t[:-1])
