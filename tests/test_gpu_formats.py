"""Device MRC reads, window extraction and per-particle SF3D weights against their restatements."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode,big", [(2, False), (1, True), (0, False), (6, True)])
def test_mrc_read_device_matches_host(built_lib, cuda, tmp_path, mode, big):
    from emclarity_b200 import api
    rng = np.random.default_rng(mode)
    shape = (200, 192, 160)
    lo, hi = {0: (-128, 127), 1: (-3000, 3000), 2: (-1, 1), 6: (0, 65535)}[mode]
    v = rng.uniform(lo, hi, shape)
    v = v.astype(np.float32) if mode == 2 else np.round(v).astype(O._MRC_DTYPES[mode])
    p = str(tmp_path / "t.mrc")
    O.mrc_write_np(p, v, mode=mode, big_endian=big)
    d = api.mrc_read_device(p)
    assert torch.equal(d.cpu(), torch.from_numpy(O.mrc_read_np(p)))
    box = (11, 150, 1, 192, 3, 198)
    assert torch.equal(api.mrc_read_device(p, box).cpu(), torch.from_numpy(O.mrc_read_np(p, box)))


def test_large_read_streams_in_blocks(built_lib, cuda, tmp_path):
    from emclarity_b200 import api
    v = np.arange(96 * 256 * 384, dtype=np.float32).reshape(96, 256, 384) * 0.5  # 37.7 MB, 2 blocks
    p = str(tmp_path / "big.mrc")
    O.mrc_write_np(p, v)
    assert torch.equal(api.mrc_read_device(p).cpu(), torch.from_numpy(v))


def test_extract_windows_matches_restatement(built_lib, cuda):
    from emclarity_b200 import api
    rng = np.random.default_rng(5)
    vol = rng.standard_normal((70, 90, 110)).astype(np.float32)
    ws = (48, 40, 36)
    centers = [(55.4, 45.2, 35.9), (3.2, 88.7, 1.0), (109.9, 2.5, 69.99), (20.0, 60.0, 50.0)]
    out, sh, ok = api.extract_windows(torch.from_numpy(vol).cuda(), ws, centers, 10.0)
    for i, c in enumerate(centers):
        w, s, v = O.extract_window_np(vol, ws, c, 10.0)
        assert np.array_equal(out[i].cpu().numpy(), w)
        assert np.allclose(sh[i], s) and ok[i] == v


def _tilt_table(rng, n=9):
    t = np.zeros((n, 22))
    t[:, 0] = rng.permutation(n) + 1
    t[:, 3] = np.linspace(-60, 60, n)
    t[:, 10] = np.linspace(0, 120, n)
    t[:, 11] = 4.1e-8
    t[:, 12] = -1.05
    t[:, 13] = rng.uniform(0.8, 1.2, n)
    t[:, 14] = -rng.uniform(2.5e-6, 3.5e-6, n)
    t[:, 15] = 2.17e-10
    t[:, 16] = 2.7e-3
    t[:, 17] = 1.968697e-12
    t[:, 18] = 0.085
    return t


def test_sf3d_particles_match_restatement(built_lib, cuda):
    from emclarity_b200 import api
    rng = np.random.default_rng(6)
    t = _tilt_table(rng)
    size = (32, 32, 32)
    xyz = np.array([[100.0, 200.0, 50.0], [400.0, 30.0, 140.0]])
    rg = np.array([[512, 512, 256], [0.0, 1.0, -2.0]])
    got = api.sf3d_particles(size, 2.0, t, xyz, rg).cpu().numpy()
    ref = O.sf3d_particles_np(size, 2.0, t, xyz, rg)
    assert got.shape == ref.shape == (2, 32, 32, 32)
    for g, r in zip(got, ref):
        assert abs(g.min() - 1e-4) < 1e-6
        assert np.abs(g - r).max() <= 2e-4 * np.abs(r).max(), np.abs(g - r).max()
    # the two positions differ in height, so their defocus and weights differ
    assert np.abs(got[0] - got[1]).max() > 1e-3 * np.abs(got[0]).max()


def test_sf3d_particles_batched_equals_one_at_a_time(built_lib, cuda):
    """One call over 1,700 particles (two chunks of tilt images) gives every particle the volume a
    one-particle call gives it."""
    from emclarity_b200 import api
    rng = np.random.default_rng(7)
    t = _tilt_table(rng)
    size = (32, 32, 32)
    rg = np.array([[512, 512, 256], [0.0, 1.0, -2.0]])
    xyz = np.column_stack([rng.uniform(0, 512, 1700), rng.uniform(0, 512, 1700), rng.uniform(0, 256, 1700)])
    batch = api.sf3d_particles(size, 2.0, t, xyz, rg)
    for i in (0, 1, 911, 1597, 1598, 1699):
        one = api.sf3d_particles(size, 2.0, t, xyz[i:i + 1], rg)[0]
        assert torch.equal(batch[i], one), i


def test_sf3d_weight_as_the_search_wedge(built_lib, cuda):
    """The per-particle SF3D weight, ifftshift-ed to a half spectrum (iMaxWedgeIfft), as the search's
    wdgMask: the search against the FP64 oracle with the same weight."""
    from emclarity_b200 import api, synthetic
    from tests.searchcheck import check_best, check_cc_and_peaks
    rng = np.random.default_rng(8)
    n = 64
    t = _tilt_table(rng)
    rg = np.array([[512, 512, 256], [0.0, 0.0, 0.0]])
    sf = api.sf3d_particles((n, n, n), 4.0, t, np.array([[256.0, 300.0, 90.0]]), rg)
    w = api.centred_to_half(sf)[0].contiguous()
    assert torch.equal(w.cpu(), torch.from_numpy(np.fft.ifftshift(sf[0].cpu().numpy())[:, :, : n // 2 + 1].copy()))
    ref = synthetic.blob_reference(rng, n)
    mask = synthetic.soft_sphere_mask(n, 28)
    truth = api.define_matrix([10.0, 20.0, -15.0], "inv")
    part = synthetic.make_particle(torch.from_numpy(ref).cuda(), rng, truth, (2, -1, 0), w, 0.2)
    grid = synthetic.local_grid(64, 8.0, 2.0)
    prior = api.define_matrix([10.0, 20.0, -15.0], "inv") @ api.define_matrix([3.0, 2.0, -1.0], "inv").T
    s = api.Search(peak_radius=6)
    rid = s.add_reference(torch.from_numpy(ref).cuda(), torch.from_numpy(mask).cuda())
    s.set_orientations(grid)
    q, e = api.particle_spectrum(part)
    cc, pk, best = s.run_host([s.particle(q, e.item(), rid, prior=prior, orient_count=len(grid), wedge=w)])
    s.close()
    P, _ = O.particle_spectrum(part.cpu().numpy())
    mats = api.search_matrices(grid, prior)
    kw = dict(mask=mask, wdg_mask=w.cpu().numpy())
    cc_o, pk_o = O.search(ref, P, mats, radius=6, **kw)
    check_cc_and_peaks(cc, pk, cc_o, pk_o, lambda o: O.xcf_translational(ref, P, mats[o], **kw)[2], "sf3d wedge")
    check_best(best[0][1], cc_o, what="sf3d wedge")
