"""Pad/taper, bandpass, band-limit-centre-normalise and the two xcf operators against the oracle."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("pl,pt,taper", [((2, 3, 4), (1, -2, 0), True), ((0, 0, 0), (0, 0, 0), False),
                                         ((-3, 5, 1), (4, 0, -6), False), ((8, 8, 8), (8, 8, 8), True)])
def test_pad3d(built_lib, cuda, pl, pt, taper):
    from emclarity_b200 import api
    a = np.random.default_rng(1).standard_normal((20, 22, 24)).astype(np.float32)
    got = api.pad3d(torch.from_numpy(a).cuda(), pl, pt, 0.25, taper).cpu().numpy()
    ref = O.pad3d_np(a, pl, pt, 0.25, taper)
    assert got.shape == ref.shape
    assert np.abs(got - ref).max() < 1e-6


@pytest.mark.parametrize("args", [((64, 64, 64), 1e-3, 40.0, 10.0, 2.5), ((96, 80, 48), 0.0, 0.0, 12.0, 2.17),
                                  ((64, 64, 64), 0.0, 0.0, 0.0, 0.0), ((48, 48, 48), 0.0, 0.0, 0.0, -1.0),
                                  ((64, 64, 1), 1e-3, 50.0, 8.0, 2.0)])
def test_bandpass3d(built_lib, cuda, args):
    from emclarity_b200 import api
    shape, ht, hc, lc, pix = args
    got = api.bandpass3d(shape, ht, hc, lc, pix).cpu().numpy()
    ref = O.bandpass3d_np(shape, ht, hc, lc, pix)
    assert np.abs(got - ref).max() < 2e-6


def test_band_limit_center_normalize(built_lib, cuda):
    from emclarity_b200 import api
    a = np.random.default_rng(2).standard_normal((40, 44, 48)).astype(np.float32) + 0.3
    bp_np = O.bandpass3d_np((64, 64, 64), 1e-3, 40.0, 10.0, 2.5)
    got = api.band_limit_center_normalize(torch.from_numpy(a).cuda(), (8, 10, 12), (8, 10, 12), True,
                                          torch.from_numpy(bp_np.astype(np.float32)).cuda()).cpu().numpy()
    ref = O.band_limit_center_normalize_np(a, (8, 10, 12), (8, 10, 12), True, bp_np)
    assert np.abs(got - ref).max() < 2e-5 * np.abs(ref).max()


def test_xcf_rotational(built_lib, cuda):
    from emclarity_b200 import api
    rng = np.random.default_rng(3)
    P = (rng.standard_normal((32, 32, 17)) + 1j * rng.standard_normal((32, 32, 17))).astype(np.complex64)
    R = (P + 0.5 * (rng.standard_normal(P.shape) + 1j * rng.standard_normal(P.shape))).astype(np.complex64)
    wm = rng.uniform(0, 1, P.shape).astype(np.float32)
    rw = rng.uniform(0, 1, P.shape).astype(np.float32)
    t = lambda x: torch.from_numpy(x).cuda()  # noqa: E731
    got = api.xcf_rotational(t(P), t(R), t(wm), t(rw))
    ref = O.xcf_rotational_np(P.astype(np.complex128), R.astype(np.complex128), wm, rw)
    assert abs(got - ref) < 1e-5 * abs(ref)
    got = api.xcf_rotational(t(P), t(R))
    ref = O.xcf_rotational_np(P.astype(np.complex128), R.astype(np.complex128))
    assert abs(got - ref) < 1e-5 * abs(ref)


def test_xcf_translational_matches_oracle(built_lib, cuda):
    """Map, masked argmax and centre of mass against the FP64 oracle on a search-like input."""
    from emclarity_b200 import api, synthetic
    rng = np.random.default_rng(4)
    n = 32
    ref = synthetic.blob_reference(rng, n, n_blobs=10)
    part = np.roll(ref, (1, -2, 3), axis=(0, 1, 2)) + 0.05 * rng.standard_normal(ref.shape).astype(np.float32)
    q, e = O.particle_spectrum(part)
    M = np.eye(3)
    c = n // 2
    ax = np.arange(n) - c
    zz, yy, xx = np.meshgrid(ax, ax, ax, indexing="ij")
    pmask = ((xx ** 2 + yy ** 2 + zz ** 2) <= 36).astype(np.float32)
    v_o, peak_o, map_o = O.xcf_translational(ref, q, M, peak_mask=pmask)
    R = np.fft.rfftn(ref.astype(np.float64))
    R.flat[0] = 0
    A = torch.from_numpy(q.astype(np.complex64)).cuda()
    B = torch.from_numpy(np.conj(R).astype(np.complex64)).cuda()
    peak, mv, mp = api.xcf_translational(A, B, torch.from_numpy(pmask).cuda(), 3, return_map=True)
    assert np.allclose(peak, peak_o, atol=1e-3)
    # without the centre-of-mass passes the integer argmax is the planted shift
    peak0, _ = api.xcf_translational(A, B, torch.from_numpy(pmask).cuda(), 0)
    assert np.array_equal(peak0, [3, -2, 1])
    scale = np.sqrt(np.sum(np.abs(R) ** 2 * np.where(np.arange(n // 2 + 1) % (n // 2) == 0, 1, 2)) * e)
    assert np.allclose(mp.cpu().numpy() * n ** 3 / scale, map_o, atol=1e-5 * np.abs(map_o).max())
