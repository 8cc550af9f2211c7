"""The MATLAB-facing boundary: our MEX gateways (built against the MEX stand-in) keep the
reference call signatures, and agree with the C-ABI and with the reference's own MEX kernels."""
import numpy as np
import pytest
import torch

import mexcall
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gateways(built_lib, cuda):
    from emclarity_b200 import build
    build.build_mex()
    return {n: mexcall.ours(n) for n in build.GATEWAYS}


def smooth(shape, seed):
    import importlib.util
    import os
    spec = importlib.util.spec_from_file_location("mk", os.path.join(os.path.dirname(__file__), "golden",
                                                                     "make_ref_fixtures.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    return mk.smooth_volume(shape, seed)


def test_mexXform3d_gateway_create_reuse_destroy(gateways):
    from emclarity_b200 import api
    g = gateways["mexXform3d_b200"]
    vol = torch.from_numpy(smooth((32, 28, 24), 1)).cuda()
    size = np.array([24, 28, 32], np.uint64)
    R = api.define_matrix([10, 20, 30], "forward").astype(np.float32)
    out, h, dummy = g(3, size, vol, R, np.array([1.0, -0.5, 0.25], np.float32), np.array(True))
    ip = api.Interpolator(vol, interp="linear_border")
    ref = ip.interp3d(R.astype(np.float64), (1.0, -0.5, 0.25), "forward")
    assert torch.allclose(out, ref, atol=1e-6)
    # reuse through the handle with a 2x2x2 dummy volume (interpolator.m:114-119)
    R2 = api.define_matrix([-40, 15, 5], "inv").astype(np.float32)
    (out2,) = g(1, size, vol[:2, :2, :2].contiguous(), R2, np.zeros(3, np.float32), np.array(False), h)
    ref2 = ip.interp3d(R2.astype(np.float64), (0, 0, 0), "inv")
    assert torch.allclose(out2, ref2, atol=1e-6)
    g(0, h, dummy)  # destroy


def test_mexFFT_gateway_roundtrip(gateways):
    g = gateways["mexFFT_b200"]
    x = torch.randn(80, 84, 90, device="cuda")   # sizes of BH_multi_iterator's "nextBest" list
    X, pf, pi = g(3, x, np.int16(2))
    assert torch.allclose(X, torch.fft.rfftn(x), atol=2e-6 * torch.fft.rfftn(x).abs().max().item())
    (y,) = g(1, X, np.int16(2), pf, pi)
    assert torch.allclose(y / x.numel(), x, atol=1e-5)
    g(0, torch.zeros(1, device="cuda"), np.int16(2), pf, pi)


def test_mexCTF_and_mexSF3D_gateways(gateways):
    from emclarity_b200 import api
    (c,) = gateways["mexCTF_b200"](1, np.array(True), np.array(False), np.int16(64), np.int16(48), np.float32(2.17),
                                   np.float32(0.0197), np.float32(2.7), np.float32(26000), np.float32(24000),
                                   np.float32(35), np.float32(0.085))
    ref = api.ctf2d(64, 48, 2.17, 0.0197, 2.7, 26000, 24000, 35, 0.085, True, False, False)
    assert torch.allclose(c, ref, atol=1e-6)
    tilts = np.arange(-60, 61, 15.0).astype(np.float32)
    nt = len(tilts)
    f = lambda v: np.full(nt, v, np.float32)  # noqa: E731
    (sf,) = gateways["mexSF3D_b200"](1, np.array(False), np.array(True), np.array([32, 32, 32], np.uint32),
                                     f(2.0), f(0.0197), f(2.7), f(12000), f(12000), f(0), f(0.1), np.uint32(nt),
                                     tilts, f(20.0), f(1.0), np.int16(1))
    ref = api.sf3d((32, 32, 32), 2.0, 0.0197, 2.7, 12000, 12000, 0, 0.1, tilts, 20.0, 1.0)
    assert torch.allclose(sf, ref, atol=1e-6)


def test_mexEmcSearch_gateway(gateways):
    from emclarity_b200 import api, synthetic
    case = synthetic.PlainCase(seed=4)
    gd = case.to_gpu()
    grid = case.grid[::10]
    # argument 4 is wdgMask (the particle's wedge, on the rotated reference), the optional 8th refWdg
    ref_wdg = (0.5 + 0.5 * gd["weight"].abs()).contiguous()
    for extra in ((), (ref_wdg,)):
        cc, pk, best = gateways["mexEmcSearch"](3, gd["ref"], gd["mask"], gd["particle"], gd["weight"], np.eye(3),
                                                grid, np.int32(7), *extra)
        q, e = api.particle_spectrum(gd["particle"], *extra)
        s = api.Search(peak_radius=7)
        rid = s.add_reference(gd["ref"], gd["mask"])
        s.set_orientations(grid)
        cc2, pk2, best2 = s.run_host([s.particle(q, e.item(), rid, orient_count=len(grid), wedge=gd["weight"])])
        s.close()
        assert np.allclose(cc.reshape(-1), cc2, atol=1e-6)
        assert np.array_equal(pk, pk2)
        assert int(best[0, 1]) == best2[0][1] + 1


# ------------------------------------------------------------------ the reference's own kernels
need_ref = pytest.mark.skipif(not mexcall.have_reference(), reason="oracle/_ref not built (needs the reference tree)")


@need_ref
def test_rotation_matches_reference_mexXform3d(built_lib, cuda):
    """Our trilinear with a zero border against the reference texture kernel; the only expected
    difference is the texture unit's 8-bit fractional weights.  A transposed matrix (wrong
    rotation sense) or a flipped shift sign would be orders of magnitude further off."""
    from emclarity_b200 import api
    ref = mexcall.reference("mexXform3d")
    vol_np = smooth((40, 40, 40), 7)
    vol = torch.from_numpy(vol_np).cuda()
    size = np.array([40, 40, 40], np.uint64)
    ip = api.Interpolator(vol, interp="linear_border")
    for ang, sh, fwd in [([20, 35, -50], (1.5, -0.75, 2.0), True), ([-70, 10, 130], (0, 0, 0), False),
                         ([5, 60, 15], (0.3, 2.0, -1.0), False)]:
        R = api.define_matrix(ang, "forward" if fwd else "inv")
        r_out, tex, arr = ref(3, size, vol, R.astype(np.float32), np.asarray(sh, np.float32), np.array(fwd))
        ref(0, tex, arr)
        ours = ip.interp3d(R, sh, "forward" if fwd else "inv")
        d = (ours - r_out).abs()
        assert d.max().item() < 1e-2 and d.mean().item() < 1e-3
        wrong = ip.interp3d(R.T, sh, "forward" if fwd else "inv")
        assert (wrong - r_out).abs().mean().item() > 10 * d.mean().item()


@need_ref
def test_ctf_matches_reference_mexCTF(built_lib, cuda):
    from emclarity_b200 import api
    ref = mexcall.reference("mexCTF")
    for half, sq, centred in [(True, False, None), (False, True, True), (True, True, False)]:
        args = [np.array(half), np.array(sq), np.int32(96), np.int32(80), np.float32(2.17), np.float32(0.01968697),
                np.float32(2.7), np.float32(26000), np.float32(24000), np.float32(35), np.float32(0.085)]
        if centred is not None:
            args.append(np.array(centred))
        (r_out,) = ref(1, *args)
        ours = api.ctf2d(96, 80, 2.17, 0.01968697, 2.7, 26000, 24000, 35, 0.085, half, sq, bool(centred))
        assert (ours - r_out).abs().max().item() < 2e-5


@need_ref
def test_fft_matches_reference_mexFFT(built_lib, cuda):
    from emclarity_b200 import api
    ref = mexcall.reference("mexFFT")
    x = torch.randn(48, 64, 96, device="cuda")
    X, pf, pi = ref(3, x, np.int32(2))
    ours = api.FourierTransformer((48, 64, 96)).fwd_fft(x)
    assert (ours - X).abs().max().item() < 2e-6 * X.abs().max().item()
    (y,) = ref(1, X, np.int32(2), pf, pi)
    ref(0, torch.zeros(1, device="cuda"), np.int32(2), pf, pi)
    yo = api.FourierTransformer((48, 64, 96)).inv_fft(ours)
    assert (yo - y).abs().max().item() < 1e-5 * y.abs().max().item()


def test_mexEmcAverage_gateway(gateways):
    """create / add / result / free through the gateway give the same half-set averages as the
    C-ABI (MATLAB layout: particles n x n x n x p, rotations 9 x p, 1-based wedge indices)."""
    from emclarity_b200 import api, synthetic
    rng = np.random.default_rng(8)
    n, p, nw = 32, 6, 24
    mask = torch.from_numpy(synthetic.soft_sphere_mask(n, 11)).cuda()
    parts = torch.randn((p, n, n, n), device="cuda")
    wedges = torch.rand((2, nw, nw, nw), device="cuda")
    rots = np.array([api.define_matrix(synthetic.random_euler(rng), "inv") for _ in range(p)])
    shifts = rng.uniform(-1, 1, (p, 3)).astype(np.float32)
    wts = rng.uniform(0.5, 1, p).astype(np.float32)
    halves = np.array([1, 2, 1, 2, 2, 1], np.int32)
    widx = np.array([0, 1, 1, 0, 0, 1], np.int32)
    sym = api.symmetry_matrices("C2")
    g = gateways["mexEmcAverage"]
    symcm = np.stack([m for m in sym], axis=-1)  # 3 x 3 x k, each a MATLAB matrix
    (h,) = g(1, mask, symcm, np.int32(nw), np.float32(0.01))
    rots_cm = np.stack([r.flatten(order="F") for r in rots], axis=1)  # 9 x p
    (kept,) = g(1, h, parts, rots_cm, shifts.T.copy(), wts, halves, wedges, widx + 1)
    assert kept.reshape(-1).tolist() == [1] * p
    outs = [g(3, h, np.int32(hf)) for hf in (1, 2)]
    g(0, h)
    avg = api.Average(mask, symmetry="C2", wedge_box=nw)
    avg.add(parts, rots, halves, shifts=shifts, weights=wts, wedges=wedges, wedge_index=widx)
    for hf, (a, w, c) in zip((1, 2), outs):
        ra, rw, rc = avg.result(hf)
        assert int(c.reshape(-1)[0]) == rc == 3
        assert torch.equal(a, ra) and torch.equal(w, rw)
    avg.close()
