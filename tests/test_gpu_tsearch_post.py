"""Template-search pre / post-processing: moving average, local normalisation and the peak loop."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fs", [6, 9])
def test_moving_average_matches_restatement(built_lib, cuda, fs):
    from emclarity_b200 import api
    rng = np.random.default_rng(fs)
    v = rng.standard_normal((30, 36, 40)).astype(np.float32)
    got = api.moving_average(torch.from_numpy(v).cuda(), fs).cpu().numpy()
    ref = O.moving_average_np(v, fs)
    assert np.abs(got - ref).max() < 2e-6 * np.abs(v).max()


def test_local_normalize_matches_restatement(built_lib, cuda):
    from emclarity_b200 import api
    rng = np.random.default_rng(3)
    v = (rng.standard_normal((32, 40, 48)) * 2 + 5).astype(np.float32)
    d = torch.from_numpy(v).cuda()
    api.local_normalize(d, 12)
    ref = O.local_normalize_np(v, 12)
    assert np.abs(d.cpu().numpy() - ref).max() < 2e-4 * np.abs(ref).max()


def _peak_case(seed, n_angles=30):
    from emclarity_b200 import synthetic
    rng = np.random.default_rng(seed)
    nz, ny, nx = 72, 80, 96
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    mag = 0.05 * rng.standard_normal((nz, ny, nx))
    for _ in range(40):
        c = rng.uniform([8, 8, 8], [nz - 8, ny - 8, nx - 8])
        h = rng.uniform(0.5, 3.0)
        mag += h * np.exp(-((z - c[0]) ** 2 + (y - c[1]) ** 2 + (x - c[2]) ** 2) / (2 * 1.5 ** 2))
    ang = rng.integers(1, n_angles + 1, (nz, ny, nx)).astype(np.float32)
    ang[:, :, :4] = 0  # a padded margin with no angle
    ang[10:14, 10:14, 10:14] = -1
    angle_list = np.stack([rng.uniform(0, 360, n_angles), rng.uniform(0, 180, n_angles),
                           rng.uniform(-180, 180, n_angles)], axis=1)
    rm = 6
    r = 2 * rm + 1
    g = np.arange(r) - rm
    zz, yy, xx = np.meshgrid(g, g, g, indexing="ij")
    removal = ((xx ** 2 / 25.0 + yy ** 2 / 16.0 + zz ** 2 / 9.0) <= 1.0).astype(np.float32)  # anisotropic
    return mag.astype(np.float32), ang, angle_list, removal, rm


def test_peak_loop_matches_restatement(built_lib, cuda):
    from emclarity_b200 import api
    mag, ang, al, removal, rm = _peak_case(7)
    d_mag = torch.from_numpy(mag).cuda()
    d_ang = torch.from_numpy(ang).cuda()
    got = api.tsearch_peaks(d_mag, d_ang, removal, rm, al, max_peaks=25, high_thr=0.2, sampling=2.0)
    ref = O.tsearch_peaks_np(mag, ang, removal, rm, al, max_peaks=25, high_thr=0.2, sampling=2.0)
    assert got.shape == ref.shape and got.shape[0] == 25
    assert np.allclose(got[:, :3], ref[:, :3], atol=1e-5)
    assert np.array_equal(got[:, 3:6], ref[:, 3:6])
    assert np.allclose(got[:, 9], ref[:, 9], rtol=1e-6)
    assert np.all(np.diff(got[:, 9]) <= 1e-6)  # non-increasing scores


def test_peak_loop_stops_at_threshold_and_tries(built_lib, cuda):
    from emclarity_b200 import api
    mag, ang, al, removal, rm = _peak_case(8)
    ref_hi = O.tsearch_peaks_np(mag, ang, removal, rm, al, max_peaks=1000, high_thr=1.0)
    got_hi = api.tsearch_peaks(torch.from_numpy(mag).cuda(), torch.from_numpy(ang).cuda(), removal, rm, al,
                               max_peaks=1000, high_thr=1.0)
    assert len(got_hi) == len(ref_hi) and np.all(got_hi[:, 9] > 1.0)
    got_t = api.tsearch_peaks(torch.from_numpy(mag).cuda(), torch.from_numpy(ang).cuda(), removal, rm, al,
                              max_peaks=1000, max_tries=5)
    assert len(got_t) <= 5
