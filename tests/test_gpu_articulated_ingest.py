"""GPU parity of the callers and data formats around the NumPy-convention path:
articulated multi-segment spectra (``ArticulatedSpineModel``,
src/fvr/articulated_spine.py), volume ingest (``resample_isotropic_cube`` /
``hu_to_attenuation``, src/fvr/dicom_loader.py) and the target-spectrum
preparation of ``RobustDiffFVREngine._prepare_spectrum``
(src/fvr/core_engine.py:71-85), against the reference's golden vectors and
the float64 oracle.  fp64 paths: 1e-10 relative; the float32 resample: one
float32 rounding of the fp64 interpolation."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import numpy_convention as nc

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.fixture(scope="module")
def spine(golden):
    from fvr.articulated_spine import ArticulatedSpineModel, VertebralSegment

    g = golden("articulated")
    segs = [VertebralSegment(f"L{3 + k}", g[f"sub{k}"], nominal_offset_z=12.0 * k) for k in range(3)]
    return ArticulatedSpineModel(segs), g


def test_articulated_spectra_and_drr_golden(spine):
    model, g = spine
    arts = list(g["arts"])
    for view in ("ap", "lateral"):
        assert rel_l2(model.render_articulated_spectrum(g["base"], arts, view=view), g[f"spec_{view}"]) < TOL
        assert rel_l2(model.render_drr(g["base"], arts, view=view), g[f"drr_{view}"]) < TOL
    # fewer articulations than joints: the upper segments keep the last accumulated pose
    assert rel_l2(model.render_articulated_spectrum(g["base"], [], view="ap"), g["spec_ap_noart"]) < TOL


def test_articulated_matches_per_segment_sum_and_oracle(spine):
    """One launch for all segments equals the sum of the segments' own
    extract_frequency_slice calls, and the oracle, on ragged joint lists."""
    model, g = spine
    f3ds = [nc.spectrum(g[f"sub{k}"], 2.0) for k in range(3)]
    base = np.array([-4.0, 3.0, 2.5, -1.5, 2.0, 0.5])
    arts = [np.array([0.5, 1.0, -2.0, 0.2, 0.1, -0.4])]
    for view in ("ap", "lateral"):
        got = model.render_articulated_spectrum(base, arts, view=view)
        assert rel_l2(got, nc.articulated_spectrum(f3ds, base, arts, view)) < TOL
        per_seg = None
        curr = base.copy()
        for k, seg in enumerate(model.segments):
            if k > 0 and len(arts) >= k:
                curr = curr + arts[k - 1]
            yaw, pitch, roll, tx, ty, tz = curr
            a, b = (ty, tz) if view == "lateral" else (tx, tz)
            s = seg.renderer.extract_frequency_slice(yaw, pitch, roll, a, b, view=view)
            per_seg = s if per_seg is None else per_seg + s
        assert rel_l2(got, per_seg) < 1e-13


def test_articulated_registration_recovers_pose(spine):
    """Two-stage Powell registration on device-resident spectra: the rigid
    stage recovers a small base offset and the loss drops to near zero."""
    model, _ = spine
    truth = np.array([2.0, -1.0, 1.5, 0.5, -0.5, 0.25])
    arts = [np.zeros(6), np.zeros(6)]
    t_ap = model.render_articulated_spectrum(truth, arts, view="ap")
    t_lat = model.render_articulated_spectrum(truth, arts, view="lateral")
    res = model.register_articulated_biplanar(t_ap, t_lat, np.zeros(6), max_iter_global=20, max_iter_local=2)
    assert res["final_loss"] < 1e-3
    assert np.abs(res["base_pose"] - truth).max() < 0.5
    assert len(res["articulations"]) == 2


def test_articulated_rejects_mismatched_segments():
    from fvr.articulated_spine import ArticulatedSpineModel, VertebralSegment

    a = VertebralSegment("a", np.ones((8, 8, 8)), 0.0)
    b = VertebralSegment("b", np.ones((8, 8, 10)), 0.0)
    with pytest.raises(ValueError):
        ArticulatedSpineModel([a, b])


@pytest.mark.parametrize("n", [16, 23])
def test_resample_and_attenuation_golden(golden, n):
    from fvr import dicom_loader as dl

    g = golden("ingest_targets")
    res, sp = dl.resample_isotropic_cube(g["hu"], tuple(g["spacing"]), n)
    ref = g[f"resampled_{n}"]
    assert res.dtype == np.float32 and res.shape == (n, n, n)
    assert sp == (float(g[f"voxel_mm_{n}"]),) * 3
    assert np.max(np.abs(res - ref)) <= 2e-4  # at most a float32 ulp of the largest HU values
    assert np.array_equal(dl.hu_to_attenuation(ref), g[f"mu_{n}"])
    mu, sp2 = dl.attenuation_cube(g["hu"], tuple(g["spacing"]), n)
    assert sp2 == sp
    assert np.array_equal(mu.cpu().numpy(), dl.hu_to_attenuation(res))


def test_resample_edges_and_errors():
    """Edge semantics on an anisotropic grid (points past the last sample get
    air) against the oracle; the reference's argument checks."""
    from fvr import dicom_loader as dl

    rng = np.random.default_rng(3)
    hu = rng.uniform(-1200.0, 2000.0, size=(5, 17, 9)).astype(np.float32)
    for spacing, n in (((3.0, 0.7, 1.9), 12), ((1.0, 1.0, 1.0), 17), ((0.5, 2.0, 1.0), 7)):
        res, sp = dl.resample_isotropic_cube(hu, spacing, n)
        ref, sp_ref = nc.resample_isotropic_cube(hu, spacing, n)
        assert sp == sp_ref
        assert np.max(np.abs(res - ref)) <= 2e-4
    with pytest.raises(ValueError):
        dl.resample_isotropic_cube(hu[:1], (1.0, 1.0, 1.0), 8)
    with pytest.raises(ValueError):
        dl.resample_isotropic_cube(hu, (1.0, -1.0, 1.0), 8)
    with pytest.raises(ValueError):
        dl.resample_isotropic_cube(hu, (1.0, 1.0, 1.0), 1)


def test_attenuation_cube_feeds_the_engine(golden):
    """The device attenuation cube goes straight into the torch-convention
    engine and renders the same images as the host round trip."""
    from fvr import dicom_loader as dl
    from fvr.torch_engine import TorchDiffFVREngine

    g = golden("ingest_targets")
    mu, sp = dl.attenuation_cube(g["hu"], tuple(g["spacing"]), 16)
    poses = torch.tensor([[3.0, -2.0, 1.0, 1.0, -1.0, 0.0]], device=mu.device)
    e1 = TorchDiffFVREngine(mu, spacing=sp)
    e2 = TorchDiffFVREngine(torch.from_numpy(dl.hu_to_attenuation(dl.resample_isotropic_cube(
        g["hu"], tuple(g["spacing"]), 16)[0])), spacing=sp)
    a, b = e1(poses, view="ap", out_res=16), e2(poses, view="ap", out_res=16)
    assert torch.equal(a, b) and bool(torch.isfinite(a).all())


def test_target_spectrum_golden(golden):
    from fvr.diff_fvr import DifferentiableFourierVolumeRenderer, prepare_target_spectrum

    g = golden("ingest_targets")
    ren = DifferentiableFourierVolumeRenderer(g["vol"], pad_factor=2.0)
    for view in ("ap", "lateral", "axial"):
        got = prepare_target_spectrum(ren, g[f"img_{view}"], view)
        assert rel_l2(got, g[f"target_{view}"]) < TOL
        dev = prepare_target_spectrum(ren, g[f"img_{view}"], view, keep_on_device=True)
        assert dev.is_cuda and dev.dtype == torch.complex128
    with pytest.raises(ValueError):
        prepare_target_spectrum(ren, np.zeros((ren.pz + 1, 4)), "ap")
