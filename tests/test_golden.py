"""The CPU oracle against golden vectors produced by the reference's own MEX kernels
(mexFiles/mexXform3d.cu, mexFiles/mexCTF.cu + utils/ctf.cu, mexFiles/mexFFT.cu) run on a B200 by
tests/golden/make_ref_fixtures.py.  This pins the oracle's rotation convention (origin, matrix
orientation, shift sign and order), its CTF formula and its FFT layout to the reference itself."""
import os

import numpy as np
import pytest

from oracle import oracle as O

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_mex.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(FIX)


def test_rotation_convention_pinned_to_reference(golden):
    """Texture trilinear (8-bit fractional weights) against the exact trilinear of the oracle in
    border mode: agreement to texture precision; a transposed matrix or a flipped shift is far off."""
    for k in range(int(golden["xform_n"])):
        vol = golden["xform_vol_%d" % int(golden["xform_%d_vol" % k])]
        R = golden["xform_%d_R" % k].astype(np.float64)
        sh = golden["xform_%d_shift" % k].astype(np.float64)
        fwd = bool(golden["xform_%d_fwd" % k])
        ref = golden["xform_%d_out" % k]
        ours = O.rotate(vol, R, sh, "forward" if fwd else "inv", interp=2)
        d = np.abs(ours - ref)
        assert d.max() < 1e-2 and d.mean() < 1e-3, (k, d.max(), d.mean())
        wrong_r = O.rotate(vol, R.T, sh, "forward" if fwd else "inv", interp=2)
        wrong_s = O.rotate(vol, R, -sh, "forward" if fwd else "inv", interp=2)
        if np.abs(R - R.T).max() > 1e-6:
            assert np.abs(wrong_r - ref).mean() > 5 * d.mean()
        if np.abs(sh).max() > 0:
            assert np.abs(wrong_s - ref).mean() > 5 * d.mean()


def test_ctf_pinned_to_reference(golden):
    for i in range(int(golden["ctf_n"])):
        nx, ny, pix, wl, cs, d1, d2, ast, ac, half, sq, centred = golden["ctf_%d_params" % i]
        ours = O.ctf2d(int(nx), int(ny), pix, wl, cs, d1, d2, ast, ac, bool(half), bool(sq), centred > 0)
        ref = golden["ctf_%d_out" % i]
        assert ours.shape == ref.shape
        assert np.abs(ours - ref).max() < 5e-5, i


def test_fft_pinned_to_reference(golden):
    for i in range(int(golden["fft_n"])):
        x = golden["fft_%d_in" % i]
        X = O.rfftn(x)
        if "fft_%d_fwd_ok" % i in golden:
            ref = golden["fft_%d_fwd" % i]
            assert np.abs(X - ref).max() < 2e-6 * np.abs(ref).max()
        y = O.irfftn(X, x.shape)
        assert np.abs(y - golden["fft_%d_inv" % i]).max() < 2e-5 * np.abs(y).max()
