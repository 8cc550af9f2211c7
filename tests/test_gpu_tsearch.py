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
    peak_o, ang_o = O.tsearch(tomo, tmpl, mats)
    assert np.allclose(peak, peak_o, rtol=1e-4, atol=2e-5 * np.abs(peak_o).max())
    # winning orientation identical wherever the runner-up is not within tolerance
    mism = ang != ang_o
    assert mism.mean() < 1e-3
    ts.close()


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
