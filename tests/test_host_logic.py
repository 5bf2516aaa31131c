"""Host-side logic of the package that runs without a GPU: argument checks
that mirror the reference's, pose bookkeeping, seeding and the capture
guard.  (The kernels themselves are covered by the -m gpu suite.)"""
import gc
from types import SimpleNamespace

import numpy as np
import pytest
import torch


def test_ingest_checks_match_the_reference():
    """dicom_loader.py:11-30: the same ValueError cases, raised before any
    device work."""
    from fvr.dicom_loader import _check

    good = np.zeros((4, 5, 6), np.float32)
    _check(good, (1.0, 1.0, 2.0), 8)
    bad = [
        (np.zeros((4, 5), np.float32), (1, 1, 1), 8),
        (np.zeros((1, 5, 6), np.float32), (1, 1, 1), 8),
        (np.full((4, 5, 6), np.nan, np.float32), (1, 1, 1), 8),
        (good, (1, 1), 8),
        (good, (1, 0, 1), 8),
        (good, (1, np.inf, 1), 8),
        (good, (1, 1, 1), 1),
        (good, (1, 1, 1), 8.0),
    ]
    for vol, sp, res in bad:
        with pytest.raises(ValueError):
            _check(vol, sp, res)


def test_articulated_segment_poses_accumulate():
    """articulated_spine.py:55-59: segment i's pose is the base pose plus the
    first i relative articulations; missing articulations leave it unchanged."""
    from fvr.articulated_spine import ArticulatedSpineModel

    model = SimpleNamespace(num_segments=3)
    base = np.array([1.0, 2.0, 3.0, 4.0, 5.0, 6.0])
    arts = [np.full(6, 0.5), np.full(6, 0.25)]
    poses = ArticulatedSpineModel._segment_poses(model, base, arts)
    assert np.allclose(poses[0], base)
    assert np.allclose(poses[1], base + 0.5)
    assert np.allclose(poses[2], base + 0.75)
    short = ArticulatedSpineModel._segment_poses(model, base, arts[:1])
    assert np.allclose(short[2], base + 0.5)


def test_articulated_view_spec():
    """articulated_spine.py:60-68: lateral slices use (ty, tz), AP (tx, tz),
    anything else the axial slice with (tx, ty)."""
    from fvr.articulated_spine import _view_spec

    pose = (10.0, 20.0, 30.0, 1.0, 2.0, 3.0)
    assert _view_spec(pose, "lateral") == (10.0, 20.0, 30.0, 2.0, 3.0, "lateral")
    assert _view_spec(pose, "ap") == (10.0, 20.0, 30.0, 1.0, 3.0, "ap")
    assert _view_spec(pose, "axial") == (10.0, 20.0, 30.0, 1.0, 2.0, "axial")


def test_multistart_seeds():
    """exp30:108-117: candidate 0 starts at the unperturbed pose, the others
    uniformly within the rotation and translation limits, reproducibly."""
    from fvr.registration import sample_multistart_theta

    th = sample_multistart_theta(64, torch.device("cpu"), 7)
    assert th.shape == (64, 6) and th.dtype == torch.float32
    assert torch.all(th[0] == 0)
    assert float(th[1:, :3].abs().max()) <= np.radians(12.0) + 1e-6
    assert float(th[1:, 3:].abs().max()) <= 15.0 + 1e-5
    assert torch.equal(th, sample_multistart_theta(64, torch.device("cpu"), 7))
    assert not torch.equal(th, sample_multistart_theta(64, torch.device("cpu"), 8))


def test_synthetic_poses_and_volume():
    from fvr import synthetic

    p = synthetic.make_poses(32, 3)
    assert p.shape == (32, 6) and p.dtype == np.float32
    assert np.abs(p[:, :3]).max() <= 10.0 and np.abs(p[:, 3:]).max() <= 5.0
    v = synthetic.make_ellipsoid_volume(16, 0, shape=(8, 16, 12))
    assert v.shape == (8, 16, 12) and v.dtype == np.float32 and v.min() >= 0.0 and v.max() > 0.0
    assert np.array_equal(v, synthetic.make_ellipsoid_volume(16, 0, shape=(8, 16, 12)))


def test_capture_guard_restores_the_collector():
    from fvr.graphs import no_gc_during_capture

    was = gc.isenabled()
    gc.enable()
    try:
        with no_gc_during_capture():
            assert not gc.isenabled()
        assert gc.isenabled()
        gc.disable()
        with no_gc_during_capture():
            assert not gc.isenabled()
        assert not gc.isenabled()
    finally:
        (gc.enable if was else gc.disable)()


def test_separable_ray_tables():
    """Host logic of the fused PoU warp adjoint: a pinhole lattice whose rays
    agree per detector column (rx) and per row (ry) up to float rounding gives
    the per-column and per-row midpoints; a skewed lattice gives None (the
    two-kernel backward then runs)."""
    from fvr.cone_beam_fvr import _SEPARABLE_REL, _separable_rays

    H, W = 6, 8
    cols = torch.linspace(-0.1, 0.1, W)
    rows = torch.linspace(-0.08, 0.08, H)
    rx = cols.repeat(H, 1).clone()
    ry = rows[:, None].repeat(1, W).clone()
    rx[2, 3] = torch.nextafter(rx[2, 3], torch.tensor(1.0))  # one float step, as the lattice's rounding
    out = _separable_rays(rx, ry)
    assert out is not None
    rxc, ryr = out
    assert rxc.shape == (W,) and ryr.shape == (H,)
    assert torch.allclose(rxc, cols, rtol=0, atol=1e-8) and torch.equal(ryr, rows)
    skew = rx + 1e-3 * torch.arange(H, dtype=torch.float32)[:, None]  # rx moves along a column
    assert _separable_rays(skew, ry) is None
    assert _separable_rays(rx, ry + 1e-3 * torch.arange(W, dtype=torch.float32)[None, :]) is None
    assert _separable_rays(rx.reshape(-1), ry.reshape(-1)) is None
    assert 0 < _SEPARABLE_REL < 1e-5
