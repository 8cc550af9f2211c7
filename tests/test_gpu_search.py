"""Fused orientation search against the FP64 oracle (same inputs, same orientation list).

Operands follow BH_multi_xcf_Translational_2.m:35-38 with BH_multi_xcf_Rotational's binding
(BH_alignRaw3d_v2.m:1376-1383): the particle's own wedge.CTF weight is wdgMask and multiplies the
rotated reference (the search descriptor's `wedge`); the reference's weight refWdg multiplies the
particle (folded into its spectrum; 1 unless a test sets it).  Every peak or best-orientation
difference must be a near-tie in the oracle's own map (tests/searchcheck.py)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.searchcheck import check_best, check_cc_and_peaks

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def plain_case(built_lib, cuda):
    from emclarity_b200 import synthetic
    case = synthetic.PlainCase(seed=3)
    g = case.to_gpu()
    return case, g


def run_gpu(case, g, grid, interp="linear", store="f32", wref=None, prior=None, ref_wdg=None, radius=None):
    from emclarity_b200 import api
    q, e = api.particle_spectrum(g["particle"], ref_wdg)
    s = api.Search(peak_radius=radius or case.peak_radius, interp=interp)
    rid = s.add_reference(g["ref"], g["mask"], wref, store=store)
    s.set_orientations(grid)
    pdesc = s.particle(q, e.item(), rid, prior=prior, orient_count=len(grid), wedge=g["weight"])
    cc, pk, best = s.run_host([pdesc])
    s.close()
    return cc, pk, best


class OracleRun:
    """The FP64 oracle on the same operands; .map(o) gives orientation o's full map for tie checks."""

    def __init__(self, case, g, grid, interp=0, ref=None, wref=None, prior=None, ref_wdg=None, radius=None):
        from emclarity_b200 import api
        self.P, _ = O.particle_spectrum(g["particle"].cpu().numpy())
        self.kw = dict(mask=case.mask, wref=wref, ref_wdg=ref_wdg, wdg_mask=g["weight"].cpu().numpy(), interp=interp)
        self.ref = case.ref if ref is None else ref
        self.mats = api.search_matrices(grid, prior)
        self.cc, self.pk = O.search(self.ref, self.P, self.mats, radius=radius or case.peak_radius, **self.kw)

    def map(self, o):
        return O.xcf_translational(self.ref, self.P, self.mats[o], **self.kw)[2]


def compare(cc_g, pk_g, orc, what=""):
    return check_cc_and_peaks(cc_g, pk_g, orc.cc, orc.pk, orc.map, what)


def test_plain_search_parity_and_truth(plain_case):
    case, g = plain_case
    grid = case.grid
    cc_g, pk_g, best = run_gpu(case, g, grid)
    orc = OracleRun(case, g, grid)
    compare(cc_g, pk_g, orc, "plain")
    check_best(best[0][1], orc.cc, what="plain")
    b = int(np.argmax(orc.cc))
    if best[0][1] == b:
        assert tuple(best[0][2]) == tuple(orc.pk[b])
    # the planted shift is recovered at the best orientation
    assert tuple(best[0][2]) == tuple(int(v) for v in case.shift)
    # and the best orientation is the grid point nearest the truth
    from emclarity_b200 import api
    mats = api.search_matrices(grid)
    ang = np.degrees(np.arccos(np.clip((np.einsum("kij,ij->k", mats, case.truth_matrix) - 1) / 2, -1, 1)))
    assert ang[best[0][1]] <= np.sort(ang)[2] + 1e-9


def test_wedges_on_both_sides_and_bandpass(plain_case):
    """Different non-unit weights on both sides of the CC (refWdg on the particle, the particle's
    wedge.CTF as wdgMask on the reference) plus a bandpass on the reference; swapping the two
    weights' roles gives other CCs, so the binding is tested, not only the product."""
    case, g = plain_case
    n = case.n
    rng = np.random.default_rng(17)
    ref_wdg = O.even_weight_np(rng, n, 0.3, 1.4)[:, :, : n // 2 + 1].astype(np.float32)
    k = np.fft.fftfreq(n)
    kz, ky, kx = np.meshgrid(k, k, np.fft.rfftfreq(n), indexing="ij")
    bp = np.exp(-(kx ** 2 + ky ** 2 + kz ** 2) / (2 * 0.2 ** 2)).astype(np.float32)
    grid = case.grid[::6]
    cc_g, pk_g, best = run_gpu(case, g, grid, wref=torch.from_numpy(bp).cuda(),
                               ref_wdg=torch.from_numpy(ref_wdg).cuda())
    orc = OracleRun(case, g, grid, wref=bp, ref_wdg=ref_wdg)
    compare(cc_g, pk_g, orc, "two wedges")
    check_best(best[0][1], orc.cc, what="two wedges")
    swapped, _ = O.search(case.ref, orc.P, orc.mats, radius=case.peak_radius, mask=case.mask, wref=bp,
                          ref_wdg=g["weight"].cpu().numpy(), wdg_mask=ref_wdg)
    assert np.abs(swapped - orc.cc).max() > 1e-2 * np.abs(orc.cc).max()


def test_cubic_and_border_modes(plain_case):
    case, g = plain_case
    grid = case.grid[::9]
    for interp, mode in (("cubic", 1), ("linear_border", 2)):
        cc_g, pk_g, best = run_gpu(case, g, grid, interp=interp)
        orc = OracleRun(case, g, grid, interp=mode)
        compare(cc_g, pk_g, orc, interp)
        check_best(best[0][1], orc.cc, what=interp)


def test_reference_weight_path(plain_case):
    """A real half-spectrum bandpass on the rotated reference and no particle wedge: the weighted
    E_R comes from one weight only."""
    case, g = plain_case
    n = case.n
    k = np.fft.fftfreq(n)
    kz, ky, kx = np.meshgrid(k, k, np.fft.rfftfreq(n), indexing="ij")
    bp = np.exp(-(kx ** 2 + ky ** 2 + kz ** 2) / (2 * 0.18 ** 2)).astype(np.float32)
    grid = case.grid[::7]
    from emclarity_b200 import api
    q, e = api.particle_spectrum(g["particle"], g["weight"])
    s = api.Search(peak_radius=case.peak_radius)
    rid = s.add_reference(g["ref"], g["mask"], torch.from_numpy(bp).cuda())
    s.set_orientations(grid)
    cc_g, pk_g, best = s.run_host([s.particle(q, e.item(), rid, orient_count=len(grid))])
    s.close()
    P, _ = O.particle_spectrum(g["particle"].cpu().numpy())
    kw = dict(mask=case.mask, wref=bp, ref_wdg=g["weight"].cpu().numpy())
    mats = api.search_matrices(grid)
    cc_o, pk_o = O.search(case.ref, P, mats, radius=case.peak_radius, **kw)
    check_cc_and_peaks(cc_g, pk_g, cc_o, pk_o, lambda o: O.xcf_translational(case.ref, P, mats[o], **kw)[2], "wref")
    check_best(best[0][1], cc_o, what="wref")


def test_bf16_reference_storage(plain_case):
    case, g = plain_case
    grid = case.grid[::5]
    cc_g, pk_g, best = run_gpu(case, g, grid, store="bf16")
    ref_bf = torch.from_numpy(case.ref).to(torch.bfloat16).float().numpy()
    orc = OracleRun(case, g, grid, ref=ref_bf)
    compare(cc_g, pk_g, orc, "bf16")
    check_best(best[0][1], orc.cc, what="bf16")


def test_prior_composition(plain_case):
    """RotMat = R_prior * D (FP64 on the device) matches the host composition."""
    from emclarity_b200 import api
    case, g = plain_case
    prior = api.define_matrix([33.0, 21.0, -48.0], "inv")
    grid = case.grid[::11]
    cc_g, pk_g, best = run_gpu(case, g, grid, prior=prior)
    orc = OracleRun(case, g, grid, prior=prior)
    compare(cc_g, pk_g, orc, "prior")
    check_best(best[0][1], orc.cc, what="prior")


def _uneven_batch(rng, s, boxes, grid, radius, slices=True, store="f32"):
    """Particles of the given boxes (C2 recipe: seeded prior, truth within a few degrees of it,
    integer shift, defocus U[1.5, 4] um, tilt range +/-U[50, 65] deg, SNR 0.1) registered on s."""
    from emclarity_b200 import api, synthetic
    refs, descs, keep, oracle_in = {}, [], [], []
    for n in sorted(set(boxes)):
        ref = synthetic.blob_reference(rng, n)
        mask = synthetic.soft_sphere_mask(n, 28 * n / 64)
        refs[n] = (ref, mask, s.add_reference(torch.from_numpy(ref).cuda(), torch.from_numpy(mask).cuda(), store=store))
    for i, n in enumerate(boxes):
        ref, mask, rid = refs[n]
        prior = api.define_matrix(synthetic.random_euler(rng), "inv")
        truth = prior @ api.define_matrix([rng.uniform(-6, 6), rng.uniform(0, 6), rng.uniform(-6, 6)], "inv")
        shift = rng.integers(-4, 5, 3)
        wt = api.wedge_ctf_weight(n, -rng.uniform(50, 65), rng.uniform(50, 65),
                                  synthetic.ctf_dict(rng.uniform(15000, 40000)))
        part = synthetic.make_particle(torch.from_numpy(ref).cuda(), rng, truth, shift, wt, 0.1)
        q, e = api.particle_spectrum(part)
        keep += [q, wt]
        begin = (3 * i) % 8 if slices else 0
        descs.append(s.particle(q, e.item(), rid, prior=prior, orient_begin=begin, orient_count=len(grid) - begin,
                                wedge=wt))
        oracle_in.append((ref, mask, part.cpu().numpy(), wt.cpu().numpy(), prior, begin))
    return descs, keep, oracle_in


def _check_uneven(grid, descs, oracle_in, cc_g, pk_g, best, radius, ref_override=None):
    from emclarity_b200 import api
    off = 0
    for k, ((ref, mask, part, wt, prior, begin), hit) in enumerate(zip(oracle_in, best)):
        ref = ref_override(ref) if ref_override else ref
        P, _ = O.particle_spectrum(part)
        mats = api.search_matrices(grid[begin:], prior)
        kw = dict(mask=mask, wdg_mask=wt)
        cc_o, pk_o = O.search(ref, P, mats, radius=radius, **kw)
        m = len(grid) - begin
        check_cc_and_peaks(cc_g[off:off + m], pk_g[off:off + m], cc_o, pk_o,
                           lambda o: O.xcf_translational(ref, P, mats[o], **kw)[2], "particle %d" % k)
        if check_best(hit[1], cc_o, offset=begin, what="particle %d" % k):
            assert tuple(hit[2]) == tuple(pk_o[hit[1] - begin])
        off += m


def test_batched_uneven_matches_oracle(built_lib, cuda):
    """Several particles of 64^3 and 96^3 (and one 128^3) in one call, each with its own slice."""
    from emclarity_b200 import api, synthetic
    rng = np.random.default_rng(21)
    grid = synthetic.local_grid(24, 8.0, 2.0)
    s = api.Search(peak_radius=5)
    s.set_orientations(grid)
    descs, keep, oracle_in = _uneven_batch(rng, s, [64, 96, 64, 128, 96], grid, 5)
    cc_g, pk_g, best = s.run_host(descs)
    _check_uneven(grid, descs, oracle_in, cc_g, pk_g, best, 5)
    # the same request again replays the captured graph and gives identical results
    cc2, pk2, best2 = s.run_host(descs)
    assert np.array_equal(cc2, cc_g) and np.array_equal(pk2, pk_g)


def test_batched_uneven_c2_shape(built_lib, cuda):
    """The batched uneven configuration at parity scale: 20 particles (12 x 64^3, 6 x 96^3, 2 x 128^3,
    the 60/30/10 split) x 256 local orientations within 8 degrees of each particle's prior, peak
    radius 7, one call; every CC, peak and best orientation against the FP64 oracle."""
    from emclarity_b200 import api, synthetic
    rng = np.random.default_rng(2000)
    grid = synthetic.local_grid(256, 8.0, 2.0)
    boxes = [int(b) for b in synthetic.batched_sizes(20, seed=3)]
    assert sorted(boxes).count(64) == 12 and boxes.count(96) == 6 and boxes.count(128) == 2
    s = api.Search(peak_radius=7)
    s.set_orientations(grid)
    descs, keep, oracle_in = _uneven_batch(rng, s, boxes, grid, 7, slices=False)
    cc_g, pk_g, best = s.run_host(descs)
    _check_uneven(grid, descs, oracle_in, cc_g, pk_g, best, 7)
    s.close()


def test_graph_replay_device_outputs(plain_case):
    from emclarity_b200 import api
    case, g = plain_case
    q, e = api.particle_spectrum(g["particle"], g["weight"])
    s = api.Search(peak_radius=7)
    rid = s.add_reference(g["ref"], g["mask"])
    s.set_orientations(case.grid)
    d = s.particle(q, e.item(), rid, orient_count=len(case.grid))
    cc = torch.empty(len(case.grid), device="cuda")
    pk = torch.empty(len(case.grid), 3, dtype=torch.int32, device="cuda")
    best = torch.empty(1, 5, dtype=torch.int32, device="cuda")
    s.run([d], cc, pk, best)
    a = (cc.clone(), pk.clone(), best.clone())
    for _ in range(3):
        s.run([d], cc, pk, best)
    torch.cuda.synchronize()
    assert torch.equal(a[0], cc) and torch.equal(a[1], pk) and torch.equal(a[2], best)


def test_bad_requests_are_rejected(plain_case):
    from emclarity_b200 import EmcError, api
    case, g = plain_case
    q, e = api.particle_spectrum(g["particle"], g["weight"])
    s = api.Search(peak_radius=7)
    rid = s.add_reference(g["ref"], g["mask"])
    s.set_orientations(case.grid)
    with pytest.raises(EmcError):
        s.run_host([s.particle(q, e.item(), rid, orient_begin=530, orient_count=20)])
    with pytest.raises(EmcError):
        s.run_host([s.particle(q, e.item(), rid + 5, orient_count=3)])
    with pytest.raises(EmcError):
        s.run_host([s.particle(q, 0.0, rid, orient_count=3)])
    with pytest.raises(EmcError):
        s.configure(peak_radius=-1)
    with pytest.raises(EmcError):
        s.add_reference(torch.zeros(80, 80, 80, device="cuda"))


def test_nan_particle_does_not_win(plain_case):
    """A NaN in the particle spectrum gives NaN CCs, never a spurious best orientation."""
    from emclarity_b200 import api
    case, g = plain_case
    q, e = api.particle_spectrum(g["particle"], g["weight"])
    qn = q.clone()
    qn[3, 4, 5] = float("nan")
    s = api.Search(peak_radius=7)
    rid = s.add_reference(g["ref"], g["mask"])
    s.set_orientations(case.grid[:10])
    cc, pk, best = s.run_host([s.particle(qn, e.item(), rid, orient_count=10)])
    assert np.all(np.isnan(cc))
    assert best[0][1] == -1


@pytest.mark.parametrize("store", ["f32", "bf16"])
def test_planes_per_cta_options_agree(built_lib, cuda, store):
    """Pass A with 1, 2, 4 or 8 z-planes per CTA computes the same CCs and peaks; the tuner
    picks one of the options it timed."""
    from emclarity_b200 import EmcError, api, synthetic
    rng = np.random.default_rng(41)
    grid = synthetic.local_grid(30, 8.0, 2.0)
    s = api.Search(peak_radius=4)
    descs, keep = [], []
    for n in (64, 96, 128):
        ref = synthetic.blob_reference(rng, n)
        mask = synthetic.soft_sphere_mask(n, 28 * n / 64)
        rid = s.add_reference(torch.from_numpy(ref).cuda(), torch.from_numpy(mask).cuda(), store=store)
        wt = api.wedge_ctf_weight(n, -55, 62, synthetic.ctf_dict(25000.0))
        truth = api.define_matrix([2.0, 4.0, -3.0], "inv")
        part = synthetic.make_particle(torch.from_numpy(ref).cuda(), rng, truth, (1, 0, -1), wt, 0.5)
        q, e = api.particle_spectrum(part)
        keep += [q, wt]
        descs.append(s.particle(q, e.item(), rid, orient_count=len(grid), wedge=wt))
    s.set_orientations(grid)
    cc0, pk0, best0 = s.run_host(descs)
    for n in (64, 96, 128):
        g, ms = s.planes(n, store)
        assert g in ms and ms[g] == min(ms.values())
        assert set(ms) <= {1, 2, 4, 8} and 1 in ms
    options = {64: (1, 2, 4, 8), 96: (1, 2, 4), 128: (1, 2)}
    for k in range(4):
        for n in (64, 96, 128):
            opts = options[n]
            s.set_planes(n, opts[min(k, len(opts) - 1)])
        cc, pk, best = s.run_host(descs)
        assert np.allclose(cc, cc0, rtol=1e-6, atol=1e-7)
        assert np.array_equal(pk, pk0)
        assert [b[1] for b in best] == [b[1] for b in best0]
    with pytest.raises(EmcError):
        s.set_planes(128, 4)
    with pytest.raises(EmcError):
        s.set_planes(96, 8)
    with pytest.raises(EmcError):
        s.set_planes(64, 3)
    s.set_planes(64, 0)
    assert s.planes(64, store)[0] == 0
    s.close()


@pytest.mark.parametrize("radius", [12, 15])
def test_large_peak_radius_matches_oracle(plain_case, radius):
    """Peak windows up to the largest supported radius (15: 31 rows / 16 row pairs in pass C)."""
    case, g = plain_case
    grid = case.grid[::20]
    cc, pk, best = run_gpu(case, g, grid, radius=radius)
    orc = OracleRun(case, g, grid, radius=radius)
    compare(cc, pk, orc, "radius %d" % radius)
    check_best(best[0][1], orc.cc, what="radius %d" % radius)
    assert np.all(np.sum(pk.astype(float) ** 2, axis=1) <= radius * radius)


def test_device_energies_match_host_energies(plain_case):
    """emc_search_run_energies reads E_P from device memory; the descriptors' energies are ignored
    (here deliberately wrong), and the results equal those of emc_search_run with host energies."""
    from emclarity_b200 import api
    case, g = plain_case
    grid = case.grid[::4]
    shifts = [(0, 0, 0), (1, -2, 0), (0, 3, -1)]
    qs, es = [], []
    for k in range(3):
        part = torch.roll(g["particle"], shifts=shifts[k], dims=(0, 1, 2)).contiguous()
        q, e = api.particle_spectrum(part, g["weight"])
        qs.append(q)
        es.append(e)
    energies = torch.cat(es)
    s = api.Search(peak_radius=case.peak_radius)
    rid = s.add_reference(g["ref"], g["mask"])
    s.set_orientations(grid)
    n_or = len(grid)
    outs = []
    cc = torch.empty(3 * n_or, device="cuda")
    pk = torch.empty((3 * n_or, 3), dtype=torch.int32, device="cuda")
    best = torch.empty((3, 5), dtype=torch.int32, device="cuda")
    for use_dev in (False, True, True):  # the second device run replays the cached graph
        descs = [s.particle(qs[k], 1.0 if use_dev else es[k].item(), rid, orient_count=n_or) for k in range(3)]
        cc.fill_(-5.0)
        s.run(descs, cc=cc, peak=pk, best=best, energies=energies if use_dev else None)
        torch.cuda.synchronize()
        outs.append((cc.cpu().numpy(), pk.cpu().numpy(), best.cpu().numpy()))
    with pytest.raises(ValueError):
        s.run(descs, energies=energies.float())
    s.close()
    for o in outs[1:]:
        assert np.array_equal(o[0], outs[0][0])
        assert np.array_equal(o[1], outs[0][1])
        assert np.array_equal(o[2], outs[0][2])


def test_batched_particle_spectra_match_single(plain_case):
    """emc_particle_spectra over a batch equals emc_particle_spectrum particle by particle (same FFT
    passes per line; energies are FP64 sums whose order may differ)."""
    from emclarity_b200 import api
    case, g = plain_case
    parts = torch.stack([torch.roll(g["particle"], shifts=(k, -k, 2 * k), dims=(0, 1, 2)) for k in range(5)])
    weights = torch.stack([g["weight"] * (1.0 + 0.1 * k) for k in range(5)]).contiguous()
    for bp in (None, weights[4].contiguous()):
        qs, es = api.particle_spectra(parts.contiguous(), weights, bandpass=bp)
        for k in range(5):
            q1, e1 = api.particle_spectrum(parts[k].contiguous(), weights[k].contiguous(), bandpass=bp)
            assert torch.equal(torch.view_as_real(qs[k]), torch.view_as_real(q1))
            assert abs(es[k].item() - e1.item()) <= 1e-12 * abs(e1.item())
    qn, en = api.particle_spectra(parts[:2].contiguous())
    q0, e0 = api.particle_spectrum(parts[1].contiguous())
    assert torch.equal(torch.view_as_real(qn[1]), torch.view_as_real(q0))


def test_bf16_storage_against_fp64_oracle_on_unrounded_reference(built_lib, cuda):
    """Mixed precision (BF16 reference storage, FP32 interpolation and FFT) against the FP64 oracle on the
    unrounded reference: 30 particles of the uneven mix x 16 orientations.  Storage rounding is the only
    difference, so CCs agree to the BF16 level and every best-orientation difference is a near-tie."""
    from emclarity_b200 import api, synthetic
    rng = np.random.default_rng(303)
    grid = synthetic.local_grid(256, 8.0, 2.0)[::16]
    boxes = [int(b) for b in synthetic.batched_sizes(30, seed=5)]
    s = api.Search(peak_radius=7)
    s.set_orientations(grid)
    descs, keep, oracle_in = _uneven_batch(rng, s, boxes, grid, 7, slices=False, store="bf16")
    cc_g, pk_g, best = s.run_host(descs)
    s.close()
    rel, gaps = [], []
    off = 0
    for k, (ref, mask, part, wt, prior, begin) in enumerate(oracle_in):
        P, _ = O.particle_spectrum(part)
        cc_o, _ = O.search(ref, P, api.search_matrices(grid, prior), mask=mask, wdg_mask=wt, radius=7)
        m = len(grid)
        rel.append(np.abs(cc_g[off:off + m] - cc_o) / np.abs(cc_o))
        b = int(np.argmax(cc_o))
        gaps.append(abs(cc_o[best[k][1]] - cc_o[b]) / abs(cc_o[b]))
        off += m
    rel = np.concatenate(rel)
    gaps = np.array(gaps)
    assert np.median(rel) < 1e-3 and rel.max() < 1e-2, (np.median(rel), rel.max())
    assert np.all(gaps <= 2e-3), gaps.max()


def test_chunk_overlap_gives_identical_results(built_lib, cuda):
    """Two scratch slots (consecutive chunks on two graph branches) and one slot (chunks in order) give
    bit-identical CCs, peaks and best orientations over many small chunks of uneven boxes."""
    from emclarity_b200 import api, synthetic
    rng = np.random.default_rng(77)
    grid = synthetic.local_grid(40, 8.0, 2.0)
    s = api.Search(peak_radius=5, chunk_evals=37)
    s.set_orientations(grid)
    descs, keep, _ = _uneven_batch(rng, s, [64, 96, 64, 128, 64, 96], grid, 5)
    total = sum(d.orient_count for d in descs)
    out = {}
    for slots in (1, 2):
        s.set_overlap(slots)
        cc = torch.empty(total, device="cuda")
        pk = torch.empty((total, 3), dtype=torch.int32, device="cuda")
        best = torch.empty((len(descs), 5), dtype=torch.int32, device="cuda")
        for _ in range(2):  # recorded, then replayed
            cc.fill_(-7.0)
            s.run(descs, cc=cc, peak=pk, best=best)
            torch.cuda.synchronize()
            out.setdefault(slots, []).append((cc.cpu().numpy(), pk.cpu().numpy(), best.cpu().numpy()))
    s.close()
    ref = out[1][0]
    for cc, pk, best in out[1][1:] + out[2]:
        assert np.array_equal(cc, ref[0]) and np.array_equal(pk, ref[1]) and np.array_equal(best, ref[2])


def _aligned_run(s, rid, q, e, w, grid):
    return s.run_host([s.particle(q, e, rid, orient_count=len(grid), wedge=w)])


def test_z_pass_copies_any_alignment(plain_case):
    """64^3 pass B copies the slabs in 16-byte rows from the boundary below each row start; a spectrum
    or weight at an odd element offset (no 16-byte aligned base) is copied element by element.  Every
    placement gives the same bits."""
    from emclarity_b200 import api
    case, g = plain_case
    grid = case.grid[:24]
    q, e = api.particle_spectrum(g["particle"])
    w = g["weight"].contiguous()
    s = api.Search(peak_radius=case.peak_radius)
    rid = s.add_reference(g["ref"], g["mask"])
    s.set_orientations(grid)
    cc0, pk0, best0 = _aligned_run(s, rid, q, e.item(), w, grid)
    for qo, wo in ((1, 0), (0, 1), (1, 2), (0, 3), (1, 3)):
        qb = torch.zeros(q.numel() + 2, dtype=q.dtype, device=q.device)
        qb[qo:qo + q.numel()] = q.flatten()
        wb = torch.zeros(w.numel() + 4, dtype=w.dtype, device=w.device)
        wb[wo:wo + w.numel()] = w.flatten()
        q2, w2 = qb[qo:qo + q.numel()].view(q.shape), wb[wo:wo + w.numel()].view(w.shape)
        assert (q2.data_ptr() % 16 != 0) == (qo == 1) and (w2.data_ptr() % 16 != 0) == (wo != 0)
        cc, pk, best = _aligned_run(s, rid, q2, e.item(), w2, grid)
        assert np.array_equal(cc, cc0) and np.array_equal(pk, pk0) and best == best0, (qo, wo)
    s.close()


def test_bounded_wait_reports_timeout_and_context_stays_usable(plain_case):
    """A pass-B wait that runs out (the test hook announces 16 bytes that are never copied) is
    reported as EMC_E_TIMEOUT by run_host and by status() after a device-output run; with the
    defaults restored the same handle gives the same results as before."""
    from emclarity_b200 import _lib as L
    from emclarity_b200 import api
    case, g = plain_case
    grid = case.grid[:16]
    q, e = api.particle_spectrum(g["particle"])
    s = api.Search(peak_radius=case.peak_radius)
    rid = s.add_reference(g["ref"], g["mask"])
    s.set_orientations(grid)
    desc = [s.particle(q, e.item(), rid, orient_count=len(grid), wedge=g["weight"])]
    cc0, pk0, best0 = s.run_host(desc)
    s.test_wait(wait_cycles=100_000, phantom_bytes=16)
    with pytest.raises(L.EmcError) as ei:
        s.run_host(desc)
    assert ei.value.status == L.EMC_E_TIMEOUT
    cc_d = torch.empty(len(grid), device="cuda")
    s.run(desc, cc=cc_d)
    with pytest.raises(L.EmcError) as ei:
        s.status()
    assert ei.value.status == L.EMC_E_TIMEOUT
    s.status()  # the report was cleared
    s.test_wait()
    cc1, pk1, best1 = s.run_host(desc)
    assert np.array_equal(cc1, cc0) and np.array_equal(pk1, pk0) and best1 == best0
    s.run(desc, cc=cc_d)
    s.status()
    assert np.array_equal(cc_d.cpu().numpy(), cc0)
    s.close()
