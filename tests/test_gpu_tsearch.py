"""Template search (per-voxel max of std-normalised CC maps and argmax angle) against the oracle."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def make_tomo(shape, tmpl, positions, rng):
    from emclarity_b200 import api
    tomo = rng.standard_normal(shape).astype(np.float32)
    t = tmpl.shape[0]
    for (z, y, x), ang in positions:
        M = api.define_matrix(ang, "forward")
        rot = O.rotate(tmpl, M, (0, 0, 0), "forward")
        tomo[z - t // 2:z - t // 2 + t, y - t // 2:y - t // 2 + t, x - t // 2:x - t // 2 + t] -= 3.0 * rot
    return tomo


def oracle_maps(tomo, tmpl, mats):
    """The oracle's std-normalised CC map of every orientation (a one-orientation MIP is the map itself)
    and the MIP / first-argmax angle derived from them (strict '<' update: the first orientation wins)."""
    maps = np.stack([O.tsearch(tomo, tmpl, [M])[0] for M in mats])
    return maps, maps.max(axis=0), maps.argmax(axis=0).astype(np.float64) + 1


def check_mip(peak, ang, maps, peak_o, ang_o):
    """MIP values within 1e-4; a voxel whose winning orientation differs from the oracle's must be a
    near-tie: the oracle's own CC of the GPU's orientation there equals its maximum within tolerance."""
    tol = 1e-4 * np.abs(peak_o) + 2e-5 * np.abs(peak_o).max()
    assert np.all(np.abs(peak - peak_o) <= tol), np.abs(peak - peak_o).max()
    bad = np.flatnonzero((ang != ang_o).ravel())
    if bad.size:
        k = ang.ravel()[bad].astype(int) - 1
        assert np.all((k >= 0) & (k < maps.shape[0]))
        got = maps.reshape(maps.shape[0], -1)[k, bad]
        assert np.all(np.abs(got - peak_o.ravel()[bad]) <= tol.ravel()[bad]), (
            "%d angle mismatches, worst gap %.3g" % (bad.size, np.abs(got - peak_o.ravel()[bad]).max()))
    return bad.size


@pytest.mark.parametrize("shape,t", [((48, 64, 64), 16), ((32, 48, 96), 12), ((48, 72, 80), 15)])
def test_template_search_against_oracle(built_lib, cuda, shape, t):
    from emclarity_b200 import api, synthetic
    rng = np.random.default_rng(41)
    tmpl = synthetic.blob_reference(rng, t, n_blobs=8)
    grid = api.euler_search("C1", 60, 30, 60, 30)[:12]
    pos = [((shape[0] // 2, shape[1] // 3, shape[2] // 3), grid[3]),
           ((shape[0] // 2 + 4, 2 * shape[1] // 3, 2 * shape[2] // 3), grid[7])]
    tomo = make_tomo(shape, tmpl, pos, rng)
    ts = api.TemplateSearch(torch.from_numpy(tomo).cuda())
    peak, ang = ts.run(torch.from_numpy(tmpl).cuda(), grid)
    peak, ang = peak.cpu().numpy(), ang.cpu().numpy()
    mats = [api.define_matrix([p, th, ps - p], "forward") for p, th, ps in grid]
    maps, peak_o, ang_o = oracle_maps(tomo, tmpl, mats)
    # the derived MIP is the oracle's own MIP
    peak_m, ang_m = O.tsearch(tomo, tmpl, mats)
    assert np.array_equal(peak_m, peak_o) and np.array_equal(ang_m, ang_o)
    check_mip(peak, ang, maps, peak_o, ang_o)
    ts.close()


def test_template_search_full_size_against_oracle(built_lib, cuda):
    """The template-search configuration's size: a 512 x 512 x 256 tomogram (noise plus planted copies of
    a 48^3 blob template at seeded non-overlapping positions and orientations) on 4 orientations of the
    12-degree grid, every voxel's MIP value and winning orientation against the FP64 oracle."""
    from emclarity_b200 import api, synthetic
    rng = np.random.default_rng(512)
    t = 48
    tmpl = synthetic.blob_reference(rng, 64)[8:56, 8:56, 8:56].copy()
    grid = api.euler_search("C1", 180, 12, 48, 12)
    sel = grid[[0, 411, 1207, 2001]]
    shape = (256, 512, 512)
    pos = []
    while len(pos) < 24:
        c = tuple(int(v) for v in (rng.integers(t, shape[0] - t), rng.integers(t, shape[1] - t),
                                   rng.integers(t, shape[2] - t)))
        if all(sum((a - b) ** 2 for a, b in zip(c, q)) >= t * t for q, _ in pos):
            pos.append((c, sel[len(pos) % 4]))
    tomo = make_tomo(shape, tmpl, pos, rng)
    ts = api.TemplateSearch(torch.from_numpy(tomo).cuda())
    peak, ang = ts.run(torch.from_numpy(tmpl).cuda(), sel)
    peak, ang = peak.cpu().numpy(), ang.cpu().numpy()
    ts.close()
    mats = [api.define_matrix([p, th, ps - p], "forward") for p, th, ps in sel]
    maps, peak_o, ang_o = oracle_maps(tomo, tmpl, mats)
    check_mip(peak, ang, maps, peak_o, ang_o)


def test_template_search_finds_planted_particles(built_lib, cuda):
    """Planted (dark) copies give the top MIP values at their centres with their orientation."""
    from emclarity_b200 import api, synthetic
    rng = np.random.default_rng(42)
    t = 16
    tmpl = synthetic.blob_reference(rng, t, n_blobs=8)
    grid = api.euler_search("C1", 60, 30, 60, 30)
    shape = (48, 64, 64)
    pos = [((20, 20, 20), grid[5]), ((28, 44, 40), grid[11])]
    tomo = make_tomo(shape, tmpl, pos, rng) * 0.3
    ts = api.TemplateSearch(torch.from_numpy(tomo).cuda())
    peak, ang = ts.run(torch.from_numpy(tmpl).cuda(), grid)
    peak, ang = peak.cpu().numpy(), ang.cpu().numpy()
    for (z, y, x), _ in pos:
        win = peak[z - 2:z + 3, y - 2:y + 3, x - 2:x + 3]
        assert win.max() > np.percentile(peak, 99.9)
