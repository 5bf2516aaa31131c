"""SE(3) exponential map (rows a18) and the batched multi-start registration
driver on the PoU-FVR renderer (the loop of the reference's
experiments/exp30_gpu_multistart_registration.py)."""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _se3_torch64(theta):
    """Plain PyTorch float64 statement: matrix_exp of the rotation vector's
    skew matrix, translation in the last column (the reference's _se3_exp)."""
    w, t = theta[:, :3], theta[:, 3:]
    K = torch.zeros((theta.shape[0], 3, 3), dtype=theta.dtype, device=theta.device)
    K[:, 0, 1], K[:, 1, 0] = -w[:, 2], w[:, 2]
    K[:, 0, 2], K[:, 2, 0] = w[:, 1], -w[:, 1]
    K[:, 1, 2], K[:, 2, 1] = -w[:, 0], w[:, 0]
    T = torch.eye(4, dtype=theta.dtype, device=theta.device).repeat(theta.shape[0], 1, 1)
    T[:, :3, :3] = torch.matrix_exp(K)
    T[:, :3, 3] = t
    return T


def test_se3_exp_and_adjoint_vs_matrix_exp():
    from fvr.registration import se3_exp

    rng = np.random.default_rng(0)
    th = rng.standard_normal((64, 6)) * np.array([0.6, 0.6, 0.6, 20.0, 20.0, 20.0])
    th[0, :3] = 0.0           # identity rotation
    th[1, :3] = [1e-7, -2e-7, 5e-8]  # below the series switch
    th[2, :3] = [math.pi - 1e-3, 0.0, 0.0]
    t32 = torch.tensor(th, dtype=torch.float32, device=DEV, requires_grad=True)
    t64 = torch.tensor(th, dtype=torch.float64, device=DEV, requires_grad=True)
    m = se3_exp(t32)
    ref = _se3_torch64(t64)
    assert torch.allclose(m.double(), ref, atol=2e-6, rtol=1e-6)
    w = torch.randn((64, 4, 4), dtype=torch.float64, device=DEV)
    (m * w.float()).sum().backward()
    (ref * w).sum().backward()
    assert torch.allclose(t32.grad.double(), t64.grad, atol=5e-5, rtol=1e-4)


def _setup(block_res=32, H=64, n_cand=8, seed=5):
    from fvr import synthetic
    from fvr.cone_beam_fvr import PerspectiveSlabFVR
    from fvr.registration import sample_multistart_theta, se3_exp

    vol = synthetic.make_ellipsoid_volume(48, seed)
    model = PerspectiveSlabFVR.from_volume(vol, vox_mm=2.0, grid_blocks=(2, 2, 2), block_res=block_res,
                                           overlap=0.5)
    sdd, pix = 600.0, 1.6
    f = sdd / pix
    k_inv = torch.tensor([[1.0 / f, 0.0, -0.5 * H / f], [0.0, 1.0 / f, -0.5 * H / f], [0.0, 0.0, 1.0]],
                         device=DEV)
    lattice = model.make_pinhole_lattice(k_inv, sdd, H, H)
    initA = synthetic.make_pinhole_mats(1, 0, sad_mm=400.0, rot_deg=0.0, trans_mm=0.0, device=DEV)
    Ry90 = torch.tensor([[0.0, 0.0, 1.0, 0.0], [0.0, 1.0, 0.0, 0.0], [-1.0, 0.0, 0.0, 0.0], [0.0, 0.0, 0.0, 1.0]],
                        device=DEV)
    initB = Ry90 @ initA

    def render_pair(dT):
        return model.forward_pinhole(dT @ initA, lattice), model.forward_pinhole(dT @ initB, lattice)

    theta_gt = torch.tensor([[0.05, -0.04, 0.03, 3.0, -2.0, 2.5]], device=DEV)
    with torch.no_grad():
        refA, refB = render_pair(se3_exp(theta_gt))
    theta0 = sample_multistart_theta(n_cand, DEV, seed, rot_deg_lim=6.0, trans_mm_lim=6.0)
    return render_pair, refA, refB, theta0, theta_gt


def test_registration_graph_replay_equals_eager_iterations():
    from fvr.registration import MultistartRegistration

    render_pair, refA, refB, theta0, _ = _setup()
    eager = MultistartRegistration(render_pair, refA, refB, theta0, steps=20, graph=False)
    graph = MultistartRegistration(render_pair, refA, refB, theta0, steps=20, graph=True)
    eager.run(6)
    graph.run(6)
    torch.cuda.synchronize()
    assert torch.allclose(eager.theta, graph.theta, atol=1e-5, rtol=1e-5)
    assert torch.allclose(eager.m, graph.m, atol=1e-6, rtol=1e-4)


def test_registration_descends_towards_ground_truth():
    from fvr.registration import MultistartRegistration

    render_pair, refA, refB, theta0, theta_gt = _setup()
    reg = MultistartRegistration(render_pair, refA, refB, theta0, steps=60, graph=True)
    l0, _ = reg.evaluate()
    reg.run(60)
    l1, best = reg.evaluate()
    assert float(l1.min()) < float(l0.min())
    assert float(l1.mean()) < float(l0.mean())
    err_t = float((best[0, 3:] - theta_gt[0, 3:]).norm())
    err0 = float((theta0[:, 3:] - theta_gt[:, 3:]).norm(dim=1).min())
    assert err_t < err0


def test_multi_volume_registration_equals_separate_runs():
    """Two volumes of different size and block count, two initialisations
    each: MultiVolumeRegistration (one graph replay per iteration for all of
    them) gives every candidate the Adam trajectory that a separate
    MultistartRegistration of its own (volume, initialisation) gives it."""
    from fvr import synthetic
    from fvr.cone_beam_fvr import PerspectiveSlabFVR
    from fvr.registration import MultistartRegistration, MultiVolumeRegistration, sample_multistart_theta, se3_exp

    H, sdd = 48, 600.0
    f = sdd / 2.0
    k_inv = torch.tensor([[1.0 / f, 0.0, -0.5 * H / f], [0.0, 1.0 / f, -0.5 * H / f], [0.0, 0.0, 1.0]], device=DEV)
    initA = synthetic.make_pinhole_mats(1, 0, sad_mm=400.0, rot_deg=0.0, trans_mm=0.0, device=DEV)
    Ry90 = torch.tensor([[0.0, 0.0, 1.0, 0.0], [0.0, 1.0, 0.0, 0.0], [-1.0, 0.0, 0.0, 0.0], [0.0, 0.0, 0.0, 1.0]],
                        device=DEV)
    initB = Ry90 @ initA
    problems, separate = [], []
    for vi, shape in enumerate(((40, 40, 40), (32, 48, 40))):
        vol = synthetic.make_ellipsoid_volume(max(shape), 11 + vi, shape=shape)
        m = PerspectiveSlabFVR.from_volume(vol, vox_mm=2.0, grid_blocks=(2, 2, 2), block_res=32, overlap=0.5)
        lat = m.make_pinhole_lattice(k_inv, sdd, H, H)
        refsA, refsB, thetas = [], [], []
        for ii in range(2):
            gt = torch.tensor([[0.03 * (ii + 1), -0.02, 0.01 * vi, 2.0 - ii, -1.0, 1.5 * vi]], device=DEV)
            with torch.no_grad():
                dT = se3_exp(gt)
                rA, rB = m.forward_pinhole(dT @ initA, lat), m.forward_pinhole(dT @ initB, lat)
            th0 = sample_multistart_theta(6, DEV, 20 + 3 * vi + ii, rot_deg_lim=5.0, trans_mm_lim=5.0)
            refsA.append(rA)
            refsB.append(rB)
            thetas.append(th0)

            def render_pair(d, m=m, lat=lat):
                return m.forward_pinhole(d @ initA, lat), m.forward_pinhole(d @ initB, lat)

            separate.append(MultistartRegistration(render_pair, rA, rB, th0, steps=10, graph=True))
        problems.append((m, lat, initA, initB, torch.cat(refsA), torch.cat(refsB), torch.cat(thetas)))
    multi = MultiVolumeRegistration(problems, steps=10)
    multi.run(5)
    for r in separate:
        r.run(5)
    torch.cuda.synchronize()
    got = multi.reg.theta.view(4, 6, 6)
    for k, r in enumerate(separate):
        assert torch.allclose(got[k], r.theta, atol=2e-5, rtol=1e-4), k
    best = multi.evaluate()
    assert len(best) == 2 and all(len(v) == 2 for v in best)
