"""CPU checks of the oracle itself: its FFT against numpy, its host math against the
numpy restatements and the committed golden vectors, and internal consistency."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.mark.parametrize("shape", [(8, 12, 16), (16, 16, 16), (6, 24, 9), (64, 64, 64), (5, 7, 3)])
def test_oracle_fft_matches_numpy(shape):
    x = np.random.default_rng(1).standard_normal(shape)
    X = O.rfftn(x)
    ref = np.fft.rfftn(x)
    assert np.abs(X - ref).max() <= 1e-11 * np.abs(ref).max()
    back = O.irfftn(X, shape) / x.size
    assert np.abs(back - x).max() < 1e-12


@pytest.mark.parametrize("n", [2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512, 7, 25])
def test_oracle_fft1_lengths(n):
    x = np.random.default_rng(n).standard_normal((3, n)) + 1j * np.random.default_rng(n + 1).standard_normal((3, n))
    assert np.abs(O.fft1(x, -1) - np.fft.fft(x, axis=-1)).max() < 1e-10 * n
    assert np.abs(O.fft1(x, 1) - np.fft.ifft(x, axis=-1) * n).max() < 1e-10 * n


def test_define_matrix_matches_numpy_restatement():
    rng = np.random.default_rng(2)
    for _ in range(50):
        a = rng.uniform(-360, 360, 3)
        for d in ("forward", "inv"):
            M = O.define_matrix(a, d)
            assert np.abs(M - O.define_matrix_np(a, d)).max() < 1e-14
            assert np.abs(M @ M.T - np.eye(3)).max() < 1e-14
    # 'forward' and 'inv' of the same triple are inverse rotations (BH_defineMatrix.m:85-102)
    a = [30.0, 50.0, -70.0]
    assert np.abs(O.define_matrix(a, "forward") @ O.define_matrix(a, "inv") - np.eye(3)).max() < 1e-14


def test_define_matrix_known_values():
    # pure Z rotation by 90 degrees: Rz(90) with 'inv' ordering of [90, 0, 0]
    M = O.define_matrix([90, 0, 0], "inv")
    assert np.allclose(M, [[0, -1, 0], [1, 0, 0], [0, 0, 1]], atol=1e-15)
    # pure X rotation by the second angle
    M = O.define_matrix([0, 90, 0], "inv")
    assert np.allclose(M, [[1, 0, 0], [0, 0, -1], [0, 1, 0]], atol=1e-15)


@pytest.mark.parametrize("args,count", [
    (("C1", 40, 10, 40, 10), 540),     # the 10-degree grid of the single-subtomogram workload
    (("C1", 180, 12, 48, 12), 2592),   # the 12-degree template-search grid
    (("C1", 180, 15, 180, 15), 4600),  # the full 15-degree grid
    (("C1", 0, 0, 0, 0), 1),
    (("C2", 20, 10, 180, 10), None),
    (("O", 90, 15, 90, 15), None),
    (("I", 30, 10, 90, 10), None),
    (("C1", -20, 10, 20, 10), None),   # bipolar
])
def test_euler_grid_counts(args, count):
    g = O.euler_search_np(*args)
    if count is not None:
        assert len(g) == count
    assert np.all(g[:, 1] >= 0) and np.all(g[:, 1] <= 180)


def test_rotate_identity_and_inverse():
    rng = np.random.default_rng(3)
    v = rng.standard_normal((16, 16, 16))
    for interp in (0, 1, 2):
        out = O.rotate(v, np.eye(3), interp=interp)
        assert np.abs(out - v).max() < 1e-12
    # a 90 degree rotation about z permutes voxels exactly (origin floor(n/2))
    M = O.define_matrix([90, 0, 0], "inv")
    out = O.rotate(v, M, interp=0)
    c = 8
    for (z, y, x) in [(3, 4, 5), (10, 2, 7), (8, 8, 8)]:
        s = M @ np.array([x - c, y - c, z - c]) + c
        sx, sy, sz = np.rint(s).astype(int)
        if 0 <= sx < 16 and 0 <= sy < 16 and 0 <= sz < 16:
            assert abs(out[z, y, x] - v[sz, sy, sx]) < 1e-12


def test_rotate_shift_semantics():
    """'forward' applies -shift before the rotation, 'inv' adds it after (mexXform3d.cu:45-65)."""
    rng = np.random.default_rng(4)
    v = rng.standard_normal((12, 12, 12))
    sh = (1.0, -2.0, 3.0)
    out_f = O.rotate(v, np.eye(3), sh, "forward")
    out_i = O.rotate(v, np.eye(3), sh, "inv")
    assert abs(out_f[6, 6, 6] - v[6 - 3, 6 + 2, 6 - 1]) < 1e-12
    assert abs(out_i[6, 6, 6] - v[6 + 3, 6 - 2, 6 + 1]) < 1e-12


def test_interpn_linear_boundary():
    """interpn(...,'linear',0): exact at the last grid point, 0 just outside."""
    v = np.arange(4 * 4 * 4, dtype=np.float64).reshape(4, 4, 4)
    # identity with a shift of -1 ('inv'): s = p - 1; at p = 0 -> s = -1 -> 0
    out = O.rotate(v, np.eye(3), (-1, 0, 0), "inv", interp=0)
    assert out[0, 0, 0] == 0.0
    assert out[0, 0, 1] == v[0, 0, 0]
    # border mode interpolates towards zero inside (-1, 0)
    out = O.rotate(v, np.eye(3), (-0.5, 0, 0), "inv", interp=2)
    assert abs(out[0, 0, 0] - 0.5 * v[0, 0, 0]) < 1e-12


def test_ctf_oracle_formula():
    """mexCTF (ctf.cu:45-62) against a direct numpy evaluation of the same formula."""
    nx, ny, pix, wl, cs, df1, df2, ast, ac = 64, 48, 2.5, 0.019687, 2.7, 26000.0, 24000.0, 30.0, 0.07
    out = O.ctf2d(nx, ny, pix, wl, cs, df1, df2, ast, ac, half=True)
    x = np.arange(nx // 2 + 1)
    y = np.arange(ny)
    y = np.where(y > ny // 2, y - ny, y)
    fx = x[None, :] / (pix * nx)
    fy = y[:, None] / (pix * ny)
    phi = np.arctan2(fy, fx)
    r2 = fx * fx + fy * fy
    amp = np.arctan(ac / np.sqrt(1 - ac * ac))
    a = np.radians(ast) - np.pi * np.rint(ast / 180)
    val = np.sin(np.pi * 0.5 * cs * 1e7 * wl ** 3 * r2 * r2
                 - np.pi * wl * r2 * (0.5 * (df1 + df2) + 0.5 * (df1 - df2) * np.cos(2 * (phi - a))) - amp)
    assert np.abs(out - val).max() < 1e-12


def test_search_oracle_finds_planted_shift():
    """A particle that is the reference rolled by d correlates best at shift d (sign check)."""
    rng = np.random.default_rng(5)
    n = 16
    ref = np.zeros((n, n, n))
    ref[4:12, 5:11, 6:10] = rng.standard_normal((8, 6, 4))
    d = (2, -1, 3)
    part = np.roll(ref, (d[2], d[1], d[0]), axis=(0, 1, 2))
    q, e = O.particle_spectrum(part)
    cc, pk = O.search(ref, q, [np.eye(3)], radius=5)
    assert tuple(pk[0]) == d
    assert abs(cc[0] - 1.0) < 1e-9


def test_search_oracle_matches_full_map():
    """The windowed argmax equals the argmax of the full fftshifted map under a spherical mask."""
    rng = np.random.default_rng(6)
    n = 16
    ref = rng.standard_normal((n, n, n))
    part = rng.standard_normal((n, n, n))
    q, e = O.particle_spectrum(part)
    M = O.define_matrix([10, 20, 30], "inv")
    cc, pk = O.search(ref, q, [M], radius=4)
    c = n // 2
    ax = np.arange(n) - c
    zz, yy, xx = np.meshgrid(ax, ax, ax, indexing="ij")
    pmask = ((xx ** 2 + yy ** 2 + zz ** 2) <= 16).astype(np.float64)
    v, peak, full = O.xcf_translational(ref, q, M, peak_mask=pmask)
    full_masked = np.where(pmask > 0.5, full, -np.inf)
    idx = np.unravel_index(np.argmax(full_masked), full.shape)
    assert (idx[2] - c, idx[1] - c, idx[0] - c) == tuple(pk[0])
    assert abs(full_masked[idx] - cc[0]) < 1e-12


def _xcf2_case(seed, n=16):
    """Reference, particle, mask, bandpasses and two different non-unit even weights."""
    rng = np.random.default_rng(seed)
    ax = np.arange(n) - n // 2
    zz, yy, xx = np.meshgrid(ax, ax, ax, indexing="ij")
    ref = np.exp(-((xx - 1) ** 2 + (yy + 2) ** 2 + zz ** 2) / 6.0) + 0.7 * np.exp(-((xx + 3) ** 2 + yy ** 2 + (zz - 2) ** 2) / 3.0)
    ref += 0.1 * rng.standard_normal(ref.shape)
    mask = np.clip(1.2 - np.sqrt(xx ** 2 + yy ** 2 + zz ** 2) / 6.0, 0, 1)
    part = np.roll(ref, (1, -2, 2), axis=(0, 1, 2)) + 0.3 * rng.standard_normal(ref.shape)
    k = np.fft.fftfreq(n)
    kz, ky, kx = np.meshgrid(k, k, k, indexing="ij")
    s2 = kx ** 2 + ky ** 2 + kz ** 2
    bp_part = np.exp(-s2 / (2 * 0.22 ** 2))         # bandpassFilt (particle)
    bp_ref = np.exp(-s2 / (2 * 0.3 ** 2))           # bandpassFiltREF (rotated reference)
    w_part = O.even_weight_np(rng, n, 0.1, 2.0)     # wdgMask (multiplies the reference)
    w_ref = O.even_weight_np(rng, n, 0.5, 1.5)      # refWdg (multiplies the particle)
    return ref, mask, part, bp_part, bp_ref, w_part, w_ref


def test_search_oracle_is_the_literal_translational_2_formula():
    """orc_xcf_translational's map equals a numpy transcription of BH_multi_xcf_Translational_2.m:35-38
    on full spectra, with different non-unit weights on both sides, a reference bandpass, a mask, a
    rotation and a shift; its zero-lag value equals BH_multi_xcf_Rotational (:71-78) of the same
    operands; orc_search's windowed peak is the map's masked maximum."""
    n = 16
    ref, mask, part, bp_part, bp_ref, w_part, w_ref = _xcf2_case(9, n)
    h = n // 2 + 1
    M = O.define_matrix([12.0, 25.0, -40.0], "inv")
    shift = (0.5, -1.0, 0.25)
    # operands as at BH_alignRaw3d_v2.m:1287-1330 (the reference through RotMat', 'forward')
    P_full = np.fft.fftn(part)
    P_full.flat[0] = 0
    P_full *= bp_part
    r = O.rotate(ref, M.T, shift, "forward") * mask
    R_full = np.fft.fftn(r) * bp_ref
    R_full.flat[0] = 0
    want = O.xcf_translational_2_np(P_full, np.conj(R_full), w_part, w_ref)
    P_half, _ = O.particle_spectrum(part, bandpass=bp_part[:, :, :h])
    c = n // 2
    zz, yy, xx = np.meshgrid(*(np.arange(n) - c,) * 3, indexing="ij")
    pmask = ((xx ** 2 + yy ** 2 + zz ** 2) <= 9).astype(np.float64)
    v, peak, got = O.xcf_translational(ref, P_half, M, mask=mask, wref=bp_ref[:, :, :h], ref_wdg=w_ref[:, :, :h],
                                       wdg_mask=w_part[:, :, :h], shift=shift, peak_mask=pmask)
    assert np.abs(got - want).max() < 1e-12 * np.abs(want).max()
    rot = O.xcf_rotational_np(P_half, np.conj(R_full[:, :, :h]), w_part[:, :, :h], w_ref[:, :, :h], nx=n)
    assert abs(got[c, c, c] - rot) < 1e-12 * abs(rot)
    cc, pk = O.search(ref, P_half, [M], mask=mask, wref=bp_ref[:, :, :h], ref_wdg=w_ref[:, :, :h],
                      wdg_mask=w_part[:, :, :h], shift=shift, radius=3)
    masked = np.where(pmask > 0.5, want, -np.inf)
    idx = np.unravel_index(np.argmax(masked), masked.shape)
    assert (idx[2] - c, idx[1] - c, idx[0] - c) == tuple(pk[0])
    assert abs(masked[idx] - cc[0]) < 1e-12 * abs(cc[0])
    # the wedges matter: swapping their roles changes the normalisation (so a test that used only one
    # binding could not tell them apart)
    v_sw, _, got_sw = O.xcf_translational(ref, P_half, M, mask=mask, wref=bp_ref[:, :, :h], ref_wdg=w_part[:, :, :h],
                                          wdg_mask=w_ref[:, :, :h], shift=shift)
    assert abs(got_sw[c, c, c] - got[c, c, c]) > 1e-3 * abs(got[c, c, c])


def test_f32_port_agrees_with_f64_oracle():
    rng = np.random.default_rng(7)
    n = 32
    ref = np.zeros((n, n, n), np.float32)
    ref[8:24, 8:24, 8:24] = rng.standard_normal((16, 16, 16))
    part = np.roll(ref, 2, axis=0) + 0.5 * rng.standard_normal((n, n, n)).astype(np.float32)
    mats = [O.define_matrix([a, 10, -a], "inv") for a in (0, 20, 40)]
    q64, e64 = O.particle_spectrum(part)
    q32, e32 = O.particle_spectrum(part, precision="f32")
    w64 = O.even_weight_np(rng, n)[:, :, : n // 2 + 1]
    cc64, pk64 = O.search(ref, q64, mats, radius=4, wdg_mask=w64)
    cc32, pk32 = O.search(ref, q32, mats, radius=4, wdg_mask=w64, precision="f32")
    assert np.allclose(cc32, cc64, rtol=1e-4, atol=1e-6)
    assert np.array_equal(pk32, pk64)


def test_cc_pose_gradient_matches_finite_differences():
    rng = np.random.default_rng(8)
    n = 16
    ax = np.arange(n) - n // 2
    zz, yy, xx = np.meshgrid(ax, ax, ax, indexing="ij")
    ref = np.exp(-((xx - 1) ** 2 + (yy + 1) ** 2 + zz ** 2) / 8.0) + 0.5 * np.exp(-((xx + 2) ** 2 + (yy - 2) ** 2 + (zz - 1) ** 2) / 4.0)
    h = rng.standard_normal((n, n, n))
    M = O.define_matrix([5, 8, -3], "inv")
    t = np.array([0.3, -0.2, 0.1])
    cc, dM, dt = O.cc_pose(ref, h, 2.0, M, t)
    eps = 1e-6
    for i in range(3):
        for j in range(3):
            Mp = M.copy(); Mp[i, j] += eps
            Mm = M.copy(); Mm[i, j] -= eps
            fd = (O.cc_pose(ref, h, 2.0, Mp, t)[0] - O.cc_pose(ref, h, 2.0, Mm, t)[0]) / (2 * eps)
            assert abs(fd - dM[i, j]) < 1e-6 * max(1.0, abs(fd)) + 1e-8
    for j in range(3):
        tp = t.copy(); tp[j] += eps
        tm = t.copy(); tm[j] -= eps
        fd = (O.cc_pose(ref, h, 2.0, M, tp)[0] - O.cc_pose(ref, h, 2.0, M, tm)[0]) / (2 * eps)
        assert abs(fd - dt[j]) < 1e-6 * max(1.0, abs(fd)) + 1e-8


def test_pocketfft_arm_matches_oracle():
    """The second CPU arm (numpy + scipy.fft in spawned processes) computes the oracle's CCs and peaks."""
    from oracle import pocketfft_arm as PF
    n = 16
    ref, mask, part, bp_part, bp_ref, w_part, w_ref = _xcf2_case(13, n)
    h = n // 2 + 1
    P, _ = O.particle_spectrum(part, bandpass=bp_part[:, :, :h])
    mats = [O.define_matrix([a, 15.0, -2 * a], "inv") for a in range(0, 90, 15)]
    kw = dict(mask=mask, wref=bp_ref[:, :, :h], ref_wdg=w_ref[:, :, :h], wdg_mask=w_part[:, :, :h], shift=(1, 0, -1))
    cc, pk = O.search(ref, P, mats, radius=3, **kw)
    with PF.Pool(ref, P, radius=3, processes=2, **kw) as pool:
        cc2, pk2 = pool.search(mats)
    assert np.allclose(cc2, cc, rtol=1e-4, atol=1e-6)
    assert np.array_equal(pk2, pk)


def test_synthetic_mask_matches_the_emc_maskshape_restatement():
    """The input generator's soft sphere is EMC_maskShape('sphere') (kernel 4 %, single-precision test)."""
    from emclarity_b200 import synthetic
    for n, r in ((64, 28.0), (32, 10.5)):
        assert np.abs(synthetic.soft_sphere_mask(n, r) - O.mask_sphere_np((n, n, n), r)).max() < 1e-6


def test_unsmoothed_wedge_restatement_is_the_binary_wedge():
    """Without smoothing, BH_weightMask3d's wedge is the binary cone test times the Nyquist window (its
    min / max normalisation is the identity); the half layout is the ifftshifted centred grid."""
    n = 24
    w = O.binary_wedge_np(n, -50.0, 65.0, smooth=False, half=False)
    assert w.min() == 0.0 and abs(w.max() - 1.0) < 1e-15
    h = O.binary_wedge_np(n, -50.0, 65.0, smooth=False, half=True)
    assert np.array_equal(h, np.fft.ifftshift(w)[:, :, : n // 2 + 1])
    c = n // 2
    assert w[c, c, c] == 1.0  # the origin slab is kept
