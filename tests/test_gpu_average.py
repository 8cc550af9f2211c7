"""Subtomogram averaging on the GPU against the FP64 restatement of BH_average3d's loop."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _case(seed, n=40, k=10, nw=36, n_wedges=2):
    from emclarity_b200 import api, synthetic
    rng = np.random.default_rng(seed)
    ref = synthetic.blob_reference(rng, n)
    parts, rots, shifts, weights, halves, widx = [], [], [], [], [], []
    for i in range(k):
        R = api.define_matrix(synthetic.random_euler(rng), "inv")
        t = rng.uniform(-1.5, 1.5, 3)
        # the window holds the reference rotated forward by R and shifted; the average rotates it back
        vol = O.rotate(ref, R.T, t, "forward", interp=2) + 0.3 * rng.standard_normal((n, n, n))
        parts.append(vol.astype(np.float32))
        rots.append(R)
        shifts.append(t)
        weights.append(rng.uniform(0.5, 1.0))
        halves.append(1 + (i % 2))
        widx.append(i % n_wedges)
    mask = synthetic.soft_sphere_mask(n, 0.35 * n)
    wedges = [np.abs(rng.standard_normal((nw, nw, nw))).astype(np.float32) for _ in range(n_wedges)]
    return dict(parts=np.array(parts), rots=np.array(rots), shifts=np.array(shifts, np.float32),
                weights=np.array(weights, np.float32), halves=np.array(halves), widx=np.array(widx),
                mask=mask, wedges=np.array(wedges), ref=ref)


def _run_gpu(c, symmetry="C1", batch=0, wedges=True):
    from emclarity_b200 import api
    nw = c["wedges"].shape[-1] if wedges else 0
    avg = api.Average(torch.from_numpy(c["mask"]).cuda(), symmetry=symmetry, wedge_box=nw, batch=batch)
    kept = avg.add(torch.from_numpy(c["parts"]).cuda(), c["rots"], c["halves"], shifts=c["shifts"],
                   weights=c["weights"], wedges=torch.from_numpy(c["wedges"]).cuda() if wedges else None,
                   wedge_index=c["widx"] if wedges else None)
    out = {h: avg.result(h) for h in (1, 2)}
    avg.close()
    return out, kept


def _run_oracle(c, symmetry=None, wedges=True):
    return O.average_np(list(c["parts"]), c["mask"], list(c["rots"]), c["halves"], shifts=c["shifts"],
                        weights=c["weights"], wedges=list(c["wedges"]) if wedges else None,
                        wedge_index=c["widx"] if wedges else None, symmetry=symmetry)


@pytest.mark.parametrize("symmetry", ["C1", "C3"])
def test_average_matches_oracle(built_lib, cuda, symmetry):
    from emclarity_b200 import api
    c = _case(11)
    g, kept = _run_gpu(c, symmetry)
    o, kept_o = _run_oracle(c, O.symmetry_matrices_np(symmetry))
    assert kept.all() and kept_o.all()
    for h in (1, 2):
        avg, wsum, cnt = g[h]
        oa, ow, oc = o[h]
        assert cnt == oc == 5
        a = avg.cpu().numpy()
        assert np.abs(a - oa).max() <= 2e-5 * np.abs(oa).max(), np.abs(a - oa).max()
        w = wsum.cpu().numpy()
        assert np.abs(w - ow).max() <= 2e-5 * np.abs(ow).max()


def test_average_recovers_the_reference(built_lib, cuda):
    """Aligned, noisy copies average back to (a masked, normalised) reference."""
    c = _case(12, k=16)
    g, _ = _run_gpu(c, wedges=False)
    a = (g[1][0].cpu().numpy() + g[2][0].cpu().numpy()) / 2
    r = c["ref"] * c["mask"]
    cc = np.sum((a - a.mean()) * (r - r.mean())) / np.sqrt(np.sum((a - a.mean()) ** 2) * np.sum((r - r.mean()) ** 2))
    assert cc > 0.9, cc


def test_batches_give_identical_sums(built_lib, cuda):
    """Particles are added in order whatever the batch split: bit-identical results."""
    c = _case(13, k=7)
    a, _ = _run_gpu(c, batch=0)
    b, _ = _run_gpu(c, batch=3)
    for h in (1, 2):
        assert torch.equal(a[h][0], b[h][0]) and torch.equal(a[h][1], b[h][1]) and a[h][2] == b[h][2]


def test_non_finite_particle_is_dropped(built_lib, cuda):
    c = _case(14, k=4)
    c["parts"][2, 20, 20, 20] = np.nan
    g, kept = _run_gpu(c)
    o, kept_o = _run_oracle(c)
    assert list(kept) == list(kept_o) == [True, True, False, True]
    for h in (1, 2):
        assert g[h][2] == o[h][2]
        assert np.isfinite(g[h][0].cpu().numpy()).all()


def test_empty_half_set_is_nan_and_bad_arguments(built_lib, cuda):
    from emclarity_b200 import EmcError, api
    c = _case(15, k=2)
    c["halves"][:] = 1
    g, _ = _run_gpu(c, wedges=False)
    assert g[2][2] == 0 and torch.isnan(g[2][0]).all()
    avg = api.Average(torch.from_numpy(c["mask"]).cuda())
    with pytest.raises(EmcError):
        avg.add(torch.from_numpy(c["parts"]).cuda(), c["rots"], [1, 3])
    with pytest.raises(EmcError):
        avg.result(0)
    with pytest.raises(EmcError):
        api.Average(torch.zeros(8, 8, 8, device="cuda"))  # no voxel above the threshold
    avg.close()
