"""Wedge, mask and filter builders (emc_binary_wedge, emc_mask_sphere, emc_cref_filter) against the FP64
restatements of BH_weightMask3d's binary wedge, EMC_maskShape('sphere') and BH_multi_cRef."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,tmin,tmax", [(64, -60.0, 60.0), (48, -55.0, 62.0), (33, -45.0, 70.0)])
@pytest.mark.parametrize("smooth", [True, False])
def test_binary_wedge(built_lib, cuda, n, tmin, tmax, smooth):
    from emclarity_b200 import api
    for half in (True, False):
        got = api.binary_wedge(n, tmin, tmax, smooth=smooth, half=half).cpu().numpy()
        want = O.binary_wedge_np(n, tmin, tmax, smooth=smooth, half=half)
        assert got.shape == want.shape
        assert np.abs(got - want).max() < 2e-6, np.abs(got - want).max()
    if not smooth:
        # the unsmoothed half spectrum is the search's wedge weight without a CTF (min 0, max 1)
        w = api.wedge_ctf_weight(n, tmin, tmax, None).cpu().numpy()
        assert np.abs(w - api.binary_wedge(n, tmin, tmax, smooth=False).cpu().numpy()).max() < 2e-6


@pytest.mark.parametrize("shape,radius,shift,kernel", [
    ((64, 64, 64), 28.0, (0, 0, 0), 0.04),
    ((48, 64, 80), (20.0, 17.5, 14.0), (1.5, -2.0, 0.25), 0.04),
    ((512 // 4, 96, 100), (30.0, 30.0, 30.0), (0, 0, 0), 0.1),
    ((64, 64, 64), 20.0, (3, 0, -2), 0.0),
    ((1, 80, 72), (25.0, 30.0, 1.0), (0.5, 0.5, 0.0), 0.04),
])
def test_mask_sphere(built_lib, cuda, shape, radius, shift, kernel):
    from emclarity_b200 import api
    got = api.mask_sphere(shape, radius, shift, kernel).cpu().numpy()
    want = O.mask_sphere_np(shape, radius, shift, kernel)
    assert np.abs(got - want).max() < 1e-6, np.abs(got - want).max()
    if kernel == 0:
        assert np.array_equal(got, want)


def test_synthetic_mask_is_the_device_mask(built_lib, cuda):
    """The input generator's host mask equals emc_mask_sphere."""
    from emclarity_b200 import api, synthetic
    for n, r in ((64, 28.0), (96, 42.0)):
        assert np.abs(api.mask_sphere((n, n, n), r).cpu().numpy() - synthetic.soft_sphere_mask(n, r)).max() < 1e-6


def _fsc_case(rng, pixel, n_shells=40):
    f = np.sort(rng.uniform(0.0, 0.5, n_shells - 1)) / pixel
    f = np.concatenate([[0.0], f])
    fsc = 1.0 / (1.0 + np.exp((f * pixel - 0.3) / 0.03)) + 0.02 * rng.standard_normal(n_shells)
    os_freq = np.arange(0, 501) * 0.001 / pixel
    force = np.where(os_freq * pixel < 0.35, 1.0, np.exp(-((os_freq * pixel - 0.35) / 0.03) ** 2))
    return f, fsc, os_freq, force


@pytest.mark.parametrize("shape,mtf", [((64, 64, 64), 0.0), ((48, 64, 80), 1.0), ((96, 96, 96), 2.0),
                                       ((64, 64, 64), 30.06)])
def test_cref_filter(built_lib, cuda, shape, mtf):
    from emclarity_b200 import api
    rng = np.random.default_rng(int(mtf * 10) + shape[0])
    pixel = 2.5
    f, fsc, os_freq, force = _fsc_case(rng, pixel)
    got = api.cref_filter(f, fsc, os_freq, shape, pixel, force_mask=force, mtf=mtf).cpu().numpy()
    want = O.cref_filter_np(f, fsc, os_freq, shape, pixel, force_mask=force, mtf=mtf)
    assert got.shape == want.shape
    assert np.abs(got - want).max() < 1e-5 * max(1.0, np.abs(want).max()), np.abs(got - want).max()


def test_builders_reject_bad_arguments(built_lib, cuda):
    from emclarity_b200 import EmcError, api
    with pytest.raises(EmcError):
        api.binary_wedge(64, 60.0, -60.0)
    with pytest.raises(EmcError):
        api.mask_sphere((64, 64, 64), 0.5)
    with pytest.raises(EmcError):
        api.cref_filter([0.0, 0.1, 0.05], [1.0, 0.5, 0.2], np.arange(10) * 0.01, (32, 32, 32), 2.0)
