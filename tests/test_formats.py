"""MRC volumes, tilt tables and window bounds (host code, CPU)."""
import os

import numpy as np
import pytest

from oracle import oracle as O

# The reference's own tilt tables, where its tree is available: EMC_REFERENCE_DIR names its root.
REF_DIR = os.environ.get("EMC_REFERENCE_DIR", "")
REF_TLT = os.path.join(REF_DIR, "docs", "anticipatedTiltAlignment", "ctf", "riboNew05_ali1_ctf.tlt") if REF_DIR else ""


@pytest.mark.parametrize("mode", [0, 1, 2, 6])
@pytest.mark.parametrize("big_endian", [False, True])
def test_mrc_read_matches_restatement(built_lib, tmp_path, mode, big_endian):
    from emclarity_b200 import api
    rng = np.random.default_rng(mode + 10 * big_endian)
    lo, hi = {0: (-128, 127), 1: (-3000, 3000), 2: (-1, 1), 6: (0, 65535)}[mode]
    v = rng.uniform(lo, hi, (5, 7, 9))
    v = v.astype(np.float32) if mode == 2 else np.round(v).astype(O._MRC_DTYPES[mode])
    p = str(tmp_path / "v.mrc")
    O.mrc_write_np(p, v, mode=mode, big_endian=big_endian, ext_bytes=64 if big_endian else 0, pixel=3.0)
    h = api.mrc_header(p)
    assert (h["nx"], h["ny"], h["nz"], h["mode"]) == (9, 7, 5, mode)
    assert h["byte_swapped"] == int(big_endian) and h["data_offset"] == 1024 + (64 if big_endian else 0)
    assert np.allclose(h["pixel_size"], 3.0)
    assert np.array_equal(api.mrc_read(p), O.mrc_read_np(p))
    box = (2, 8, 3, 7, 2, 4)
    assert np.array_equal(api.mrc_read(p, box), O.mrc_read_np(p, box))
    assert np.array_equal(api.mrc_read(p, (0, 0, 4, 4, 0, 0)), O.mrc_read_np(p, (0, 0, 4, 4, 0, 0)))


def test_mrc_write_roundtrip_and_header_stats(built_lib, tmp_path):
    from emclarity_b200 import api
    rng = np.random.default_rng(2)
    v = rng.standard_normal((6, 5, 8)).astype(np.float32)
    p = str(tmp_path / "w.mrc")
    api.mrc_write(p, v, pixel_size=(1.5, 2.0, 2.5), origin=(1, 2, 3))
    assert np.array_equal(O.mrc_read_np(p), v)
    h = api.mrc_header(p)
    assert np.allclose(h["pixel_size"], (1.5, 2.0, 2.5)) and np.allclose(h["origin"], (1, 2, 3))
    assert h["dmin"] == v.min() and h["dmax"] == v.max() and abs(h["dmean"] - v.mean()) < 1e-6
    # SAVE_IMG's rms: std(std(std(vol))) along x, then y, then z, n - 1 normalisation
    s = np.std(np.std(np.std(v.astype(np.float64), axis=2, ddof=1), axis=1, ddof=1), ddof=1)
    assert abs(h["rms"] - s) < 1e-6


def test_mrc_errors(built_lib, tmp_path):
    from emclarity_b200 import EmcError, api
    with pytest.raises(EmcError):
        api.mrc_header(str(tmp_path / "missing.mrc"))
    p = str(tmp_path / "bad.mrc")
    O.mrc_write_np(p, np.zeros((2, 2, 2), np.float32))
    raw = bytearray(open(p, "rb").read())
    raw[12] = 4  # complex float mode, not read
    open(p, "wb").write(bytes(raw))
    with pytest.raises(EmcError):
        api.mrc_read(p)
    O.mrc_write_np(p, np.zeros((2, 2, 2), np.float32))
    with pytest.raises(EmcError):
        api.mrc_read(p, (1, 3, 1, 2, 1, 2))


def test_tilt_table_parsing(built_lib, tmp_path):
    from emclarity_b200 import api
    rng = np.random.default_rng(3)
    t = rng.standard_normal((7, 22)) * np.logspace(-12, 3, 22)
    p = tmp_path / "a_ctf.tlt"
    with open(p, "w") as f:
        for row in t:
            f.write("\t".join("%.9e" % x for x in row) + "\n")
        f.write("\n")
    got = api.tlt_read(p)
    assert got.shape == (7, 22) and np.allclose(got, t, rtol=1e-9)
    bad = tmp_path / "bad.tlt"
    bad.write_text("1 2 3\n4 5\n")
    from emclarity_b200 import EmcError
    with pytest.raises(EmcError):
        api.tlt_read(bad)


@pytest.mark.skipif(not REF_TLT or not os.path.exists(REF_TLT), reason="EMC_REFERENCE_DIR not set or tree absent")
def test_reference_tilt_table_parses(built_lib):
    from emclarity_b200 import api
    t = api.tlt_read(REF_TLT)
    assert t.shape == (41, 22)
    assert np.all(np.abs(t[:, 3]) <= 90) and np.allclose(t[:, 17], 1.968697e-12)


def test_window_bounds_match_restatement(built_lib):
    from emclarity_b200 import api
    rng = np.random.default_rng(4)
    for _ in range(300):
        vs = rng.integers(40, 300, 3)
        ws = rng.integers(16, 96, 3)
        c = rng.uniform(-5, vs + 5)
        r = rng.uniform(4, 30)
        start, pl, pt, sh, ok = api.window_bounds(vs, ws, r, c)
        s2, pl2, pt2, sh2, ok2 = O.window_bounds_np(vs, ws, r, c)
        assert tuple(s2) == start and tuple(pl2) == pl and tuple(pt2) == pt and ok == ok2
        assert np.allclose(sh, sh2)
