"""The NumPy-convention registration engines on the B200 renderer against
trajectories of the reference's own engines (tests/golden/registration.npz,
written by tests/golden/make_golden.py from the reference):

* GradientRegistrationOptimizer.register_adam (gradient_optimizer.py:24-90):
  every iteration's loss (1e-9 absolute) and pose (1e-7), the iteration
  count and the best pose;
* RobustDiffFVREngine.register_biplanar_robust (core_engine.py:109-224), the
  clean spectral-NCC branch and the masked-metal branch: the metal flag, the
  evaluation count, the final pose (1e-6) and loss (1e-9).

The renderer computes in fp64 like the reference, so the optimisers follow
the same paths.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_register_adam_trajectory(golden):
    from fvr.diff_fvr import DifferentiableFourierVolumeRenderer
    from fvr.gradient_optimizer import GradientRegistrationOptimizer

    g = golden("registration")
    ren = DifferentiableFourierVolumeRenderer(g["vol"], pad_factor=2.0)
    t = g["truth"]
    f_ap = ren.extract_frequency_slice(*t[:3], tx=t[3], ty=t[5], view="ap")
    f_lat = ren.extract_frequency_slice(*t[:3], tx=t[4], ty=t[5], view="lateral")
    r = GradientRegistrationOptimizer(ren).register_adam(f_ap, f_lat, np.zeros(6), max_iter=12)
    assert r["iterations"] == int(g["adam_iterations"])
    losses = np.array([x[1] for x in r["trajectory"]])
    poses = np.stack([x[2] for x in r["trajectory"]])
    np.testing.assert_allclose(losses, g["adam_losses"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(poses, g["adam_poses"], rtol=0, atol=1e-7)
    np.testing.assert_allclose(r["final_pose"], g["adam_final_pose"], rtol=0, atol=1e-7)
    assert abs(r["final_loss"] - float(g["adam_final_loss"])) < 1e-9
    assert r["evaluations"] == 7 * r["iterations"]


@pytest.mark.parametrize("tag", ["clean", "metal"])
def test_register_biplanar_robust(golden, tag):
    from fvr.core_engine import RobustDiffFVREngine

    g = golden("registration")
    eng = RobustDiffFVREngine(g["vol"], spacing=(1.0, 1.0, 1.0))
    a, b = (g["target_ap"], g["target_lat"]) if tag == "clean" else (g["metal_target_ap"], g["metal_target_lat"])
    res = eng.register_biplanar_robust(a, b, initial_pose=(0.5, 0.0, -0.3, 0.0, 0.2, 0.0), max_iter=2)
    assert res["metal_detected"] == bool(g[f"robust_{tag}_metal"])
    assert res["evaluations"] == int(g[f"robust_{tag}_evals"])
    np.testing.assert_allclose(res["final_pose"], g[f"robust_{tag}_pose"], rtol=0, atol=1e-6)
    assert abs(res["final_loss"] - float(g[f"robust_{tag}_loss"])) < 1e-9


def test_robust_engine_argument_checks():
    from fvr.core_engine import RobustDiffFVREngine, detect_radio_opaque_metal

    vol = np.zeros((16, 16, 16))
    vol[4:12, 5:11, 6:10] = 1.0
    with pytest.raises(ValueError):
        RobustDiffFVREngine(vol, sdd_mm=1000.0)
    with pytest.raises(ValueError):
        RobustDiffFVREngine(vol, spacing=(1.0, 1.0, 2.0))
    with pytest.raises(ValueError):
        RobustDiffFVREngine(np.zeros((16, 16, 8)))
    eng = RobustDiffFVREngine(vol)
    with pytest.raises(ValueError):
        eng.register_biplanar_robust(np.ones((16, 16)), np.random.rand(16, 16))
    with pytest.raises(ValueError):
        eng.register_biplanar_robust(np.random.rand(8, 8), np.random.rand(16, 16))
    img = np.zeros((10, 10))
    img[0, 0] = 1.0
    img[1, 1] = 0.985
    m = detect_radio_opaque_metal(img)
    assert m.dtype == bool and int(m.sum()) == 2
    assert np.array_equal(eng.detect_metal_hardware_mask(img), ~m)
