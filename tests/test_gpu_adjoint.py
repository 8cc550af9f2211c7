"""Forward + adjoint of the masked CC (emc_cc_adjoint) against the FP64 oracle and finite differences."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(built_lib, cuda):
    from emclarity_b200 import api, synthetic
    rng = np.random.default_rng(31)
    n = 64
    ref = synthetic.blob_reference(rng, n)
    mask = synthetic.soft_sphere_mask(n, 28)
    truth = api.define_matrix([12.0, 25.0, -40.0], "inv")
    w = api.wedge_ctf_weight(n, -60, 60, synthetic.ctf_dict(25000.0))
    part = synthetic.make_particle(torch.from_numpy(ref).cuda(), rng, truth, (1, -2, 0), w, 1.0)
    q, e = api.particle_spectrum(part, w)
    h = api.particle_template(q)
    s = api.Search()
    rid = s.add_reference(torch.from_numpy(ref).cuda(), torch.from_numpy(mask).cuda())
    s.set_orientations(np.zeros((1, 3)))
    return dict(s=s, rid=rid, h=h, e=e.item(), ref=ref, mask=mask, n=n, truth=truth)


def test_template_is_inverse_fft(setup):
    h = setup["h"].cpu().numpy()
    assert h.shape == (64, 64, 64) and np.isfinite(h).all()


def test_adjoint_matches_oracle(setup):
    from emclarity_b200 import api
    s, h = setup["s"], setup["h"]
    prior = api.define_matrix([10.0, 20.0, -35.0], "inv")
    poses = np.array([[2.0, 5.0, -4.0, 1.2, -1.7, 0.3], [0.0, 0.0, 0.0, 0.0, 0.0, 0.0],
                      [-3.0, 4.0, 2.5, 0.9, -2.2, 0.1]])
    cc, grad = s.cc_adjoint(setup["rid"], h, setup["e"], prior, poses)
    hn = h.cpu().numpy()
    for i, p in enumerate(poses):
        D = api.define_matrix([p[0], p[1], p[2] - p[0]], "inv")
        M = (prior @ D).T
        cco, dM, dt = O.cc_pose(setup["ref"], hn, setup["e"], M, p[3:], mask=setup["mask"])
        assert abs(cc[i] - cco) <= 1e-4 * abs(cco) + 1e-6
        # shift gradient
        assert np.allclose(grad[i, 3:], dt, rtol=2e-3, atol=2e-4 * np.abs(dt).max())
        # angle gradient: chain dM through M(angles) by central differences of the matrix
        eps = 1e-4
        ga = []
        for k in range(3):
            pp = p.copy(); pp[k] += eps
            pm = p.copy(); pm[k] -= eps
            Mp = (prior @ api.define_matrix([pp[0], pp[1], pp[2] - pp[0]], "inv")).T
            Mm = (prior @ api.define_matrix([pm[0], pm[1], pm[2] - pm[0]], "inv")).T
            ga.append(np.sum(dM * (Mp - Mm) / (2 * eps)))
        assert np.allclose(grad[i, :3], ga, rtol=2e-3, atol=2e-4 * np.abs(ga).max())


def test_adjoint_finite_differences_on_gpu(setup):
    """The GPU gradient against central differences of the GPU forward value."""
    from emclarity_b200 import api
    s, h = setup["s"], setup["h"]
    prior = np.eye(3)
    p0 = np.array([3.0, 7.0, -2.0, 0.4, -0.6, 0.8])
    cc0, g0 = s.cc_adjoint(setup["rid"], h, setup["e"], prior, p0[None])
    steps = np.array([0.05, 0.05, 0.05, 0.02, 0.02, 0.02])
    poses = []
    for k in range(6):
        for sg in (1, -1):
            p = p0.copy(); p[k] += sg * steps[k]
            poses.append(p)
    cc, _ = s.cc_adjoint(setup["rid"], h, setup["e"], prior, np.array(poses))
    fd = (cc[0::2] - cc[1::2]) / (2 * steps)
    assert np.allclose(g0[0], fd, rtol=3e-2, atol=3e-2 * np.abs(fd).max())


def test_gradient_ascent_recovers_pose(setup):
    """A few gradient steps from a 4-degree / 1-voxel offset move towards the truth."""
    from emclarity_b200 import api
    s, h = setup["s"], setup["h"]
    truth = setup["truth"]
    start = np.array([14.0, 28.0, -37.0, 0.0, 0.0, 0.0])
    prior = np.eye(3)
    p = start.copy()
    lr = np.array([200.0, 200.0, 200.0, 20.0, 20.0, 20.0])
    cc_first = None
    for _ in range(30):
        cc, g = s.cc_adjoint(setup["rid"], h, setup["e"], prior, p[None])
        cc_first = cc[0] if cc_first is None else cc_first
        p = p + lr * g[0]
    cc_last, _ = s.cc_adjoint(setup["rid"], h, setup["e"], prior, p[None])
    assert cc_last[0] > cc_first


def test_bad_arguments(setup):
    from emclarity_b200 import EmcError
    s, h = setup["s"], setup["h"]
    with pytest.raises(EmcError):
        s.cc_adjoint(setup["rid"] + 3, h, setup["e"], np.eye(3), np.zeros((1, 6)))
    with pytest.raises(EmcError):
        s.cc_adjoint(setup["rid"], h, 0.0, np.eye(3), np.zeros((1, 6)))


def _batch(setup, poses, interp, prior=None):
    from emclarity_b200 import refine
    k = len(poses)
    prior = np.eye(3) if prior is None else prior
    obj = refine.BatchObjective(setup["s"], [setup["rid"]] * k, [setup["h"]] * k, [setup["e"]] * k, [prior] * k,
                                interp=interp)
    f, g = obj(np.asarray(poses))
    return -f, -g


def test_linear_cell_adjoint_matches_oracle(setup):
    """The trilinear forward + adjoint through the corner cells against the FP64 trilinear oracle."""
    from emclarity_b200 import api
    poses = np.array([[2.0, 5.0, -4.0, 1.2, -1.7, 0.3], [-3.0, 4.0, 2.5, 0.9, -2.2, 0.1]])
    cc, grad = _batch(setup, poses, "linear")
    hn = setup["h"].cpu().numpy()
    for i, p in enumerate(poses):
        M = api.define_matrix([p[0], p[1], p[2] - p[0]], "inv").T
        cco, dM, dt = O.cc_pose(setup["ref"], hn, setup["e"], M, p[3:], mask=setup["mask"], interp=0)
        assert abs(cc[i] - cco) <= 1e-4 * abs(cco) + 1e-6
        assert np.allclose(grad[i, 3:], dt, rtol=5e-3, atol=5e-4 * np.abs(dt).max())


def test_batched_adjoint_matches_single(setup):
    poses = np.array([[1.0, 2.0, 3.0, 0.1, 0.2, 0.3], [4.0, 5.0, 6.0, -0.3, 0.0, 0.5]])
    cc_b, g_b = _batch(setup, poses, "cubic")
    cc_s, g_s = setup["s"].cc_adjoint(setup["rid"], setup["h"], setup["e"], np.eye(3), poses)
    assert np.allclose(cc_b, cc_s, rtol=1e-12) and np.allclose(g_b, g_s, rtol=1e-12)


def test_lbfgs_refinement_reduces_pose_error(setup):
    """L-BFGS from a 3-degree / 1-voxel perturbation converges to the planted pose."""
    from emclarity_b200 import api, refine
    truth = setup["truth"]
    rng = np.random.default_rng(5)
    starts = []
    for _ in range(4):
        # truth: defineMatrix([12, 25, -40], 'inv') = D(phi = 12, theta = 25, psi - phi = -40)
        starts.append([12.0 + rng.uniform(-3, 3), 25.0 + rng.uniform(-3, 3), -28.0 + rng.uniform(-3, 3),
                       1.0 + rng.uniform(-1, 1), -2.0 + rng.uniform(-1, 1), rng.uniform(-1, 1)])
    starts = np.array(starts)
    k = len(starts)
    obj = refine.BatchObjective(setup["s"], [setup["rid"]] * k, [setup["h"]] * k, [setup["e"]] * k,
                                [np.eye(3)] * k, interp="cubic")
    x, f, hist = refine.lbfgs(obj, starts, n_iter=25)
    R = np.array([api.define_matrix([p[0], p[1], p[2] - p[0]], "inv") for p in x])
    err = refine.geodesic_deg(R, truth[None])
    R0 = np.array([api.define_matrix([p[0], p[1], p[2] - p[0]], "inv") for p in starts])
    err0 = refine.geodesic_deg(R0, truth[None])
    assert np.all(hist[-1] <= hist[0] + 1e-12)
    assert np.median(err) < 0.5 < np.median(err0)
    assert np.allclose(x[:, 3:], [1, -2, 0], atol=0.3)


def _poses50(seed=50):
    """50 seeded poses around the planted one (truth = defineMatrix([12, 25, -40], 'inv'), shift (1, -2, 0)):
    angles within +/-6 degrees, shifts within +/-1.5 voxels."""
    rng = np.random.default_rng(seed)
    base = np.array([12.0, 25.0, -28.0, 1.0, -2.0, 0.0])
    return base + np.concatenate([rng.uniform(-6, 6, (50, 3)), rng.uniform(-1.5, 1.5, (50, 3))], axis=1)


def _angle_grad_from_dM(prior, p, dM):
    """Chain dCC/dM (the oracle's matrix gradient) through M(angles) = (prior D(phi, theta, psi - phi))'."""
    from emclarity_b200 import api
    eps = 1e-5
    out = []
    for k in range(3):
        pp = p.copy(); pp[k] += eps
        pm = p.copy(); pm[k] -= eps
        Mp = (prior @ api.define_matrix([pp[0], pp[1], pp[2] - pp[0]], "inv")).T
        Mm = (prior @ api.define_matrix([pm[0], pm[1], pm[2] - pm[0]], "inv")).T
        out.append(np.sum(dM * (Mp - Mm) / (2 * eps)))
    return np.array(out)


@pytest.mark.parametrize("interp,oracle_interp", [("cubic", 1), ("linear", 0)])
def test_adjoint_on_50_poses_against_the_fp64_gradient(setup, interp, oracle_interp):
    """CC and the full 6-vector gradient of the device adjoint against the FP64 oracle's analytic
    gradient (orc_cc_pose_interp) on 50 seeded poses with a non-trivial prior."""
    from emclarity_b200 import api
    prior = api.define_matrix([-20.0, 10.0, 35.0], "inv")
    poses = _poses50()
    cc, grad = _batch(setup, poses, interp, prior=prior)
    hn = setup["h"].cpu().numpy()
    rel = []
    for i, p in enumerate(poses):
        M = (prior @ api.define_matrix([p[0], p[1], p[2] - p[0]], "inv")).T
        cco, dM, dt = O.cc_pose(setup["ref"], hn, setup["e"], M, p[3:], mask=setup["mask"], interp=oracle_interp)
        assert abs(cc[i] - cco) <= 1e-4 * abs(cco) + 1e-6, (i, cc[i], cco)
        go = np.concatenate([_angle_grad_from_dM(prior, p, dM), dt])
        for part in (slice(0, 3), slice(3, 6)):
            rel.append(np.linalg.norm(grad[i, part] - go[part]) / max(np.linalg.norm(go[part]), 1e-12))
    rel = np.array(rel)
    assert np.median(rel) < 1e-3 and rel.max() < 5e-3, (np.median(rel), rel.max())


def test_adjoint_on_50_poses_against_finite_differences(setup):
    """The tricubic gradient against central differences of the device forward value on 50 poses, all
    600 displaced poses evaluated in one batched launch."""
    from emclarity_b200 import api
    prior = api.define_matrix([-20.0, 10.0, 35.0], "inv")
    poses = _poses50(seed=51)
    _, g0 = _batch(setup, poses, "cubic", prior=prior)
    steps = np.array([0.02, 0.02, 0.02, 0.01, 0.01, 0.01])
    disp = []
    for p in poses:
        for k in range(6):
            for sg in (1, -1):
                q = p.copy(); q[k] += sg * steps[k]
                disp.append(q)
    cc, _ = _batch(setup, np.array(disp), "cubic", prior=prior)
    fd = ((cc[0::2] - cc[1::2]).reshape(50, 6)) / (2 * steps)
    rel = []
    for i in range(50):
        for part in (slice(0, 3), slice(3, 6)):
            rel.append(np.linalg.norm(g0[i, part] - fd[i, part]) / max(np.linalg.norm(fd[i, part]), 1e-12))
    rel = np.array(rel)
    assert np.median(rel) < 5e-3 and rel.max() < 3e-2, (np.median(rel), rel.max())


def test_autograd_function_shim(setup):
    """refine.CCPose (torch.autograd.Function over emc_cc_adjoint_batch): values equal the batched call,
    backward scales the adjoint gradient by grad_out, and torch.autograd.gradcheck's finite differences
    agree with the analytic Jacobian (tricubic objective, FP32 forward)."""
    from emclarity_b200 import api, refine
    k = 4
    prior = api.define_matrix([-20.0, 10.0, 35.0], "inv")
    obj = refine.BatchObjective(setup["s"], [setup["rid"]] * k, [setup["h"]] * k, [setup["e"]] * k, [prior] * k,
                                interp="cubic")
    x = torch.tensor(_poses50(seed=52)[:k], dtype=torch.float64, requires_grad=True)
    cc = refine.CCPose.apply(x, obj)
    # a second launch: the FP64 reductions' atomic order may differ in the last bits
    cc_ref, g_ref = obj.cc_grad(x.detach().numpy())
    assert np.allclose(cc.detach().numpy(), cc_ref, rtol=1e-12, atol=0)
    w = torch.tensor([1.0, -2.0, 0.5, 3.0], dtype=torch.float64)
    (w * cc).sum().backward()
    assert np.allclose(x.grad.numpy(), w.numpy()[:, None] * g_ref, rtol=1e-9, atol=1e-12 * np.abs(g_ref).max())
    atol = 2e-2 * float(np.abs(g_ref).max())
    assert torch.autograd.gradcheck(lambda t: refine.CCPose.apply(t, obj), (x.detach().requires_grad_(),),
                                    eps=1e-2, atol=atol, rtol=2e-2, raise_exception=True)
