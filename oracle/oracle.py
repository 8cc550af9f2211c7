"""Python access to the CPU oracle of the orientation-search path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg as the checker; the product never imports it.

``lib(precision)`` loads oracle/liboracle_f64.so (the FP64 oracle) or liboracle_f32.so
(the single-precision CPU port used as the timed baseline), building them with make when
missing.  The numpy helpers below restate the host-side parts of the reference that are
plain arithmetic (grid enumeration, rotation matrices, masks and wedges).
"""
import ctypes as C
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_libs = {}


def build():
    r = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)


def lib(precision="f64"):
    if precision in _libs:
        return _libs[precision]
    path = os.path.join(HERE, "liboracle_%s.so" % precision)
    src = os.path.join(HERE, "emc_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        build()
    L = C.CDLL(path)
    sfx = "_" + precision
    R = C.c_double if precision == "f64" else C.c_float
    pR = C.POINTER(R)
    pd, pi = C.POINTER(C.c_double), C.POINTER(C.c_int)
    sig = {
        "orc_define_matrix": (None, [pd, C.c_int, pd]),
        "orc_rotate": (None, [pR, C.c_int, C.c_int, C.c_int, pd, C.c_int, pd, C.c_int, C.c_int, pR]),
        "orc_fft3_r2c": (None, [pR, C.c_int, C.c_int, C.c_int, pR]),
        "orc_fft3_c2r": (None, [pR, C.c_int, C.c_int, C.c_int, pR]),
        "orc_fft1": (None, [pR, C.c_int, C.c_int, C.c_int]),
        "orc_ctf2d": (None, [R, R, R, R, R, R, R, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, R, R, pR]),
        "orc_sf3d": (None, [C.c_int, C.c_int, C.c_int, C.c_int, pR, pR, pR, pR, pR, pR, pR, C.c_int, pR, pR, pR, pR]),
        "orc_particle_spectrum": (C.c_double, [pR, pR, pR, C.c_int, pR]),
        "orc_search": (None, [pR, pR, pR, C.c_int, pR, pR, pR, pd, C.c_int, pd, C.c_int, C.c_int, C.c_int, pd, pi]),
        "orc_xcf_translational": (C.c_double, [pR, pR, pR, C.c_int, pR, pR, pR, pd, pd, pR, C.c_int, pR, pd]),
        "orc_tsearch": (None, [pR, C.c_int, C.c_int, C.c_int, pR, C.c_int, pd, C.c_int, pR, pR]),
        "orc_cc_pose": (C.c_double, [pR, pR, C.c_int, pR, C.c_double, pd, pd, pd, pd]),
        "orc_cc_pose_interp": (C.c_double, [pR, pR, C.c_int, pR, C.c_double, pd, pd, C.c_int, pd, pd]),
    }
    funcs = {}
    for name, (res, args) in sig.items():
        f = getattr(L, name + sfx)
        f.restype = res
        f.argtypes = args
        funcs[name] = f
    obj = type("OracleLib", (), {})()
    obj.__dict__.update(funcs)
    obj.dtype = np.float64 if precision == "f64" else np.float32
    obj.ptr = lambda a, _p=pR: a.ctypes.data_as(_p)
    _libs[precision] = obj
    return obj


def _p(a, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t))


def _arr(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype) if a is not None else None


# ----------------------------------------------------------------------------- wrappers
def define_matrix(angles, direction="inv"):
    out = np.zeros(9)
    a = np.ascontiguousarray(angles, dtype=np.float64)
    lib().orc_define_matrix(_p(a), 0 if direction == "forward" else 1, _p(out))
    return out.reshape(3, 3, order="F")


def rotate(vol, M, shift=(0, 0, 0), direction="forward", interp=0, precision="f64", symmetry=None):
    L = lib(precision)
    v = _arr(vol, L.dtype)
    nz, ny, nx = v.shape
    mats = [np.asarray(M, dtype=np.float64)] if symmetry is None else [np.asarray(M) @ s for s in symmetry]
    mp = np.ascontiguousarray(np.concatenate([m.reshape(3, 3).flatten(order="F") for m in mats]))
    sh = np.ascontiguousarray(shift, dtype=np.float64)
    out = np.zeros_like(v)
    L.orc_rotate(L.ptr(v), nx, ny, nz, _p(mp), len(mats), _p(sh), 1 if direction == "forward" else 0, interp,
                 L.ptr(out))
    return out


def rfftn(vol, precision="f64"):
    L = lib(precision)
    v = _arr(vol, L.dtype)
    nz, ny, nx = v.shape
    out = np.zeros((nz, ny, nx // 2 + 1), dtype=np.complex128 if precision == "f64" else np.complex64)
    L.orc_fft3_r2c(L.ptr(v), nx, ny, nz, L.ptr(out.view(L.dtype)))
    return out


def irfftn(spec, shape, precision="f64"):
    L = lib(precision)
    s = np.ascontiguousarray(spec, dtype=np.complex128 if precision == "f64" else np.complex64)
    nz, ny, nx = shape
    out = np.zeros(shape, dtype=L.dtype)
    L.orc_fft3_c2r(L.ptr(s.view(L.dtype)), nx, ny, nz, L.ptr(out))
    return out


def fft1(data, sign=-1, precision="f64"):
    L = lib(precision)
    d = np.ascontiguousarray(data, dtype=np.complex128 if precision == "f64" else np.complex64).copy()
    n = d.shape[-1]
    L.orc_fft1(L.ptr(d.view(L.dtype)), n, d.size // n, sign)
    return d


def ctf2d(nx, ny, pixel_size, wavelength, cs_mm, defocus1, defocus2, astig_deg, amp_contrast, half=True,
          squared=False, centred=False, radial_weight=None, exposure=None, precision="f64"):
    L = lib(precision)
    out = np.zeros((ny, nx // 2 + 1 if half else nx), dtype=L.dtype)
    L.orc_ctf2d(pixel_size, wavelength, cs_mm, defocus1, defocus2, astig_deg, amp_contrast, nx, ny, int(half),
                int(squared), int(centred), int(radial_weight is not None), radial_weight or 0.0, exposure or 0.0,
                L.ptr(out))
    return out


def sf3d(size, pixel_size, wavelength, cs_mm, df1, df2, astig_deg, amp_contrast, tilt_deg, exposure, occupancy,
         squared=True, precision="f64"):
    L = lib(precision)
    nt = len(tilt_deg)
    arrs = [np.ascontiguousarray(np.broadcast_to(np.asarray(x, dtype=L.dtype), (nt,))) for x in
            (pixel_size, wavelength, cs_mm, df1, df2, astig_deg, amp_contrast, tilt_deg, exposure, occupancy)]
    nx, ny, nz = size
    out = np.zeros((nz, ny, nx), dtype=L.dtype)
    L.orc_sf3d(int(squared), nx, ny, nz, *[L.ptr(a) for a in arrs[:7]], nt, L.ptr(arrs[7]), L.ptr(arrs[8]),
               L.ptr(arrs[9]), L.ptr(out))
    return out


def particle_spectrum(particle, weight=None, bandpass=None, precision="f64"):
    L = lib(precision)
    p = _arr(particle, L.dtype)
    n = p.shape[0]
    w = _arr(weight, L.dtype)
    b = _arr(bandpass, L.dtype)
    q = np.zeros((n, n, n // 2 + 1), dtype=np.complex128 if precision == "f64" else np.complex64)
    e = L.orc_particle_spectrum(L.ptr(p), L.ptr(w) if w is not None else None, L.ptr(b) if b is not None else None,
                                n, L.ptr(q.view(L.dtype)))
    return q, e


def search(ref, P, matrices, mask=None, wref=None, ref_wdg=None, wdg_mask=None, shift=(0, 0, 0), radius=7, interp=0,
           nthreads=0, precision="f64"):
    """Per-orientation (cc, peak) of the normalised translational CC (BH_multi_xcf_Translational_2.m:35-38)
    over the spherical peak window.  ``matrices``: RotMat per orientation (the reference is sampled
    through RotMat', 'forward'); ``P``: particle half spectrum (rotPART_FT, P(0) = 0); ``wref``: the
    reference bandpass; ``ref_wdg`` / ``wdg_mask``: the formula's refWdg (multiplies P) and wdgMask
    (multiplies the reference), real half spectra or None (= 1)."""
    L = lib(precision)
    r = _arr(ref, L.dtype)
    n = r.shape[0]
    m, wr, rw, wm = (_arr(a, L.dtype) for a in (mask, wref, ref_wdg, wdg_mask))
    pp = np.ascontiguousarray(P, dtype=np.complex128 if precision == "f64" else np.complex64)
    mats = np.ascontiguousarray(np.stack([np.asarray(M).T.flatten(order="F") for M in matrices]))
    sh = np.ascontiguousarray(shift, dtype=np.float64)
    no = len(matrices)
    cc = np.zeros(no)
    pk = np.zeros((no, 3), dtype=np.int32)
    opt = lambda a: L.ptr(a) if a is not None else None  # noqa: E731
    L.orc_search(L.ptr(r), opt(m), opt(wr), n, L.ptr(pp.view(L.dtype)), opt(rw), opt(wm), _p(mats), no, _p(sh),
                 int(radius), int(interp), int(nthreads), _p(cc), _p(pk, C.c_int))
    return cc, pk


def xcf_translational(ref, P, matrix, mask=None, wref=None, ref_wdg=None, wdg_mask=None, shift=(0, 0, 0),
                      peak_mask=None, interp=0):
    """(max inside the peak mask, subvoxel peak, fftshifted normalised map) for one matrix; operands as
    ``search``."""
    L = lib("f64")
    r = _arr(ref, L.dtype)
    n = r.shape[0]
    m, wr, rw, wm, pm = (_arr(a, L.dtype) for a in (mask, wref, ref_wdg, wdg_mask, peak_mask))
    pp = np.ascontiguousarray(P, dtype=np.complex128)
    M = np.ascontiguousarray(np.asarray(matrix).T.flatten(order="F"))
    sh = np.ascontiguousarray(shift, dtype=np.float64)
    out = np.zeros((n, n, n))
    peak = np.zeros(3)
    opt = lambda a: L.ptr(a) if a is not None else None  # noqa: E731
    v = L.orc_xcf_translational(L.ptr(r), opt(m), opt(wr), n, L.ptr(pp.view(L.dtype)), opt(rw), opt(wm), _p(M),
                                _p(sh), opt(pm), int(interp), L.ptr(out), _p(peak))
    return v, peak, out


def tsearch(tomo, tmpl, matrices, precision="f64"):
    """Template search MIP; ``matrices``: defineMatrix([phi,theta,psi-phi],'forward') per orientation."""
    L = lib(precision)
    t = _arr(tomo, L.dtype)
    g = _arr(tmpl, L.dtype)
    nz, ny, nx = t.shape
    mats = np.ascontiguousarray(np.stack([np.asarray(M).flatten(order="F") for M in matrices]))
    peak = np.zeros_like(t)
    ang = np.zeros_like(t)
    L.orc_tsearch(L.ptr(t), nx, ny, nz, L.ptr(g), g.shape[0], _p(mats), len(matrices), L.ptr(peak), L.ptr(ang))
    return peak, ang


def cc_pose(ref, h, energy, matrix, t, mask=None, interp=1):
    """Zero-lag normalised CC of the rotated reference (tricubic interp=1 or trilinear interp=0,
    sampled through matrix, 'forward', shift t) against the real-space template h; returns
    (cc, dM (3x3), dt (3))."""
    L = lib("f64")
    r = _arr(ref, L.dtype)
    hh = _arr(h, L.dtype)
    m = _arr(mask, L.dtype)
    M = np.ascontiguousarray(np.asarray(matrix).flatten(order="F"))
    tt = np.ascontiguousarray(t, dtype=np.float64)
    dM = np.zeros(9)
    dt = np.zeros(3)
    cc = L.orc_cc_pose_interp(L.ptr(r), L.ptr(m) if m is not None else None, r.shape[0], L.ptr(hh), float(energy),
                              _p(M), _p(tt), int(interp), _p(dM), _p(dt))
    return cc, dM.reshape(3, 3, order="F"), dt


# ----------------------------------------------------------------------------- numpy restatements
def define_matrix_np(angles, direction="inv"):
    """BH_defineMatrix 'Bah' (coordinates/BH_defineMatrix.m:85-126) in numpy."""
    a = np.radians(np.asarray(angles, dtype=np.float64))
    a = -a if direction == "forward" else a[::-1]
    c, s = np.cos(a), np.sin(a)
    rz3 = np.array([[c[2], -s[2], 0], [s[2], c[2], 0], [0, 0, 1]])
    rx2 = np.array([[1, 0, 0], [0, c[1], -s[1]], [0, s[1], c[1]]])
    rz1 = np.array([[c[0], -s[0], 0], [s[0], c[0], 0], [0, 0, 1]])
    return rz3 @ rx2 @ rz1


def _colon(a, d, b):
    if not d > 0 or b < a:
        return []
    n = int(math.floor((b - a) / d + 1e-10 * (1 + abs((b - a) / d)))) + 1
    return [a + k * d for k in range(n)]


def euler_search_np(symmetry, theta_max, theta_step, psi_max, psi_step):
    """eulerSearch (coordinates/eulerSearch.m:38-177) walked as BH_alignRaw3d_v2.m:1119-1170."""
    bipolar = theta_max < 0
    theta_max = abs(theta_max)
    psi_w = 2.0 * psi_max
    k, num = symmetry[0], symmetry[1:]
    if k == "C":
        psi_w = min(psi_w, 360.0 / float(num)); theta_max = min(180.0, theta_max); phi_max = 360.0
    elif k == "D":
        psi_w = 360.0 / float(num); theta_max = min(theta_max, 90.0); phi_max = 360.0
    elif k == "O":
        psi_w = min(psi_w, 90.0); theta_max = min(theta_max, 54.7); phi_max = 90.0
    elif k == "I":
        psi_w = min(psi_w, 180.0); theta_max = 31.7; phi_max = 180.0
    else:
        raise ValueError(symmetry)
    psi = _colon(-psi_w / 2, psi_step, psi_w / 2) or [0.0]
    theta = _colon(0.0, theta_step, theta_max) or [0.0]
    if bipolar:
        theta = theta + [180.0 - t for t in reversed(theta)]
    out = []
    for th in theta:
        if th in (0.0, 180.0):
            step = phi_max
        else:
            step = abs(theta_step / math.sin(math.radians(th)))
            step = phi_max if step > phi_max else phi_max / math.floor(phi_max / step + 0.5)
        for ph in _colon(0.0, step, phi_max - 1):
            for ps in psi:
                out.append((math.fmod(ph, 360.0), th, ps))
    return np.array(out)


def pad3d_np(img, pad_low, pad_top, fill=0.0, taper=False):
    """BH_padZeros3d (masking/BH_padZeros3d.m:79-229), numeric fill, 'single' / 'singleTaper'.
    Arrays are (z, y, x); pads are given (x, y, z)."""
    img = np.asarray(img, dtype=np.float64)
    pl = list(pad_low)[::-1]
    pt = list(pad_top)[::-1]
    sl = tuple(slice(max(-l, 0), img.shape[a] - max(-t, 0)) for a, (l, t) in enumerate(zip(pl, pt)))
    im = img[sl].copy()
    if taper:
        tap = 0.5 + 0.5 * np.cos(np.arange(7) * np.pi / 7)     # 1 ... 0.0495
        for a in range(3):
            n = im.shape[a]
            t = np.ones(n)
            k = min(7, n)
            t[:k] *= tap[::-1][:k]           # low side: first slice gets the smallest weight
            t[n - k:] *= tap[:k]                 # high side: last slice gets the smallest weight
            shape = [1, 1, 1]
            shape[a] = n
            t = t.reshape(shape)
            im = im * t + fill * (1 - t)
    out = np.full(tuple(s + max(l, 0) + max(t, 0) for s, l, t in zip(im.shape, pl, pt)), fill, dtype=np.float64)
    out[max(pl[0], 0):max(pl[0], 0) + im.shape[0], max(pl[1], 0):max(pl[1], 0) + im.shape[1],
        max(pl[2], 0):max(pl[2], 0) + im.shape[2]] = im
    return out


def bandpass3d_np(shape_xyz, high_thresh, high_cut, low_cut, pixel_size):
    """BH_bandpass3d (masking/BH_bandpass3d.m:54-170) on the half spectrum, returned (z, y, x//2+1).
    pixel_size > 0 numeric, 0 -> 'nyquist', < 0 -> 'nyquistHigh'."""
    nx, ny, nz = shape_xyz
    mn = min(nx, ny, nz) if nz > 1 else min(nx, ny)
    hc = hr = 0.0
    if pixel_size > 0:
        if high_cut != 0:
            hc = pixel_size / high_cut
        lc = pixel_size / low_cut
        if lc > 0:
            lr = 2.0 / mn
        else:
            lc = abs(lc)
            lr = math.sqrt(-(0.5 - lc) ** 2 / (2 * math.log(1e-3)))
        if high_cut != 0:
            hr = math.sqrt(-hc ** 2 / (2 * math.log(high_thresh)))
    else:
        if pixel_size < 0:
            hc = 7.0 / mn
            hr = math.sqrt(-hc ** 2 / (2 * math.log(1e-6)))
        lr = 1.5 / mn
        lc = 0.485 + low_cut
    fz = np.fft.fftfreq(nz)[:, None, None] if nz > 1 else np.zeros((1, 1, 1))
    fy = np.fft.fftfreq(ny)[None, :, None]
    fx = (np.arange(nx // 2 + 1) / nx)[None, None, :]
    r = np.sqrt(fx ** 2 + fy ** 2 + fz ** 2)
    w = np.where(r < lc, 1.0, np.exp(-(r - lc) ** 2 / (2 * lr * lr)))
    if hc != 0:
        w = np.where(r <= hc, np.exp(-(r - hc) ** 2 / (2 * hr * hr)), w)
    return w


def band_limit_center_normalize_np(img, pad_low, pad_top, taper=False, bandpass=None):
    """BH_bandLimitCenterNormalize (masking/BH_bandLimitCenterNormalize.m:40-61), half spectrum."""
    p = pad3d_np(img, pad_low, pad_top, float(np.mean(np.asarray(img, dtype=np.float64))), taper)
    F = np.fft.rfftn(p)
    F.flat[0] = 0
    if bandpass is not None:
        F = F * bandpass
    nx = p.shape[2]
    hw = np.full(F.shape[2], 2.0)
    hw[0] = 1.0
    if nx % 2 == 0:
        hw[-1] = 1.0
    e = float(np.sum(hw[None, None, :] * np.abs(F) ** 2))
    return F / (math.sqrt(e) / p.size)


def xcf_rotational_np(P, R, wdg_mask=None, ref_wdg=None, nx=None):
    """BH_multi_xcf_Rotational (statistics/BH_multi_xcf_Rotational.m:71-78) on half spectra."""
    wm = 1.0 if wdg_mask is None else wdg_mask
    rw = 1.0 if ref_wdg is None else ref_wdg
    nx = nx if nx is not None else 2 * (P.shape[2] - 1)
    hw = np.full(P.shape[2], 2.0)
    hw[0] = 1.0
    if nx % 2 == 0:
        hw[-1] = 1.0
    hw = hw[None, None, :]
    num = np.sum(hw * np.real(rw * P * R * wm))
    den = np.sum(hw * np.abs(R * wm) ** 2) * np.sum(hw * np.abs(P * rw) ** 2)
    return num / math.sqrt(den)


def xcf_translational_2_np(rotPART_FT, REF_FT, wdgMask, refWdg):
    """statistics/BH_multi_xcf_Translational_2.m:35-38 as written, on FULL spectra (numpy fftn order):
    fftshift(real(ifftn((refWdg .* rotPART_FT .* REF_FT .* wdgMask) ./
    (sqrt(sum(abs(REF_FT .* wdgMask).^2) .* sum(abs(rotPART_FT .* refWdg).^2)) ./ numel(wdgMask)))))."""
    num = refWdg * rotPART_FT * REF_FT * wdgMask
    den = np.sqrt(np.sum(np.abs(REF_FT * wdgMask) ** 2) * np.sum(np.abs(rotPART_FT * refWdg) ** 2)) / np.size(wdgMask)
    return np.fft.fftshift(np.real(np.fft.ifftn(num / den)))


def even_weight_np(rng, n, lo=0.2, hi=1.5):
    """A random real full-grid weight with W(-k) = W(k) (as every wedge / CTF weight is), numpy fftn order."""
    a = rng.uniform(lo, hi, (n, n, n))
    flip = np.roll(a[::-1, ::-1, ::-1], 1, axis=(0, 1, 2))
    return 0.5 * (a + flip)


def _conv_same_np(v, taps):
    """convn(v, taps along each axis, 'same') with zero padding (a symmetric, odd-length kernel)."""
    out = np.asarray(v, dtype=np.float64)
    for axis in range(out.ndim):
        if out.shape[axis] > 1:
            out = np.apply_along_axis(lambda r: np.convolve(r, taps, mode="same"), axis, out)
    return out


def binary_wedge_np(n, tilt_min, tilt_max, smooth=True, half=True):
    """BH_weightMask3d(.., 'binaryWedgeGPU') (masking/BH_weightMask3d.m:99-143), Y tilt axis, FP64:
    theta = atan2d(X, Z) on the centred grid, cones of +/-(90 - |tilt|) removed, |X|, |Z| <= 2 kept,
    convn with BH_multi_gaussian3d(9, 1.5), times fftshift(BH_bandpass3d(.., 'nyquist')), then
    (W - min) / max(W - min).  half: the ifftshifted half spectrum (z, y, x <= n/2)."""
    c = n // 2
    ax = np.arange(n) - c
    Z, Y, X = np.meshgrid(ax, ax, ax, indexing="ij")
    max_cone, min_cone = 90.0 - abs(tilt_min), 90.0 - abs(tilt_max)
    th = np.degrees(np.arctan2(X, Z))
    excl = ((180 - min_cone <= th) | (th <= max_cone - 180)) | ((-min_cone <= th) & (th <= max_cone))
    w = np.where(excl, 0.0, 1.0)
    w[(np.abs(X) <= 2) & (np.abs(Z) <= 2)] = 1.0
    if smooth:
        t = np.exp(-0.5 * ((np.arange(9) - 4) / 1.5) ** 2)
        w = _conv_same_np(w, t / t.sum())
    rn = np.sqrt(X ** 2 + Y ** 2 + Z ** 2) / n
    w = w * np.where(rn < 0.485, 1.0, np.exp(-(rn - 0.485) ** 2 / (2 * (1.5 / n) ** 2)))
    w = w - w.min()
    w = w / w.max()
    return np.fft.ifftshift(w)[:, :, : n // 2 + 1] if half else w


def mask_sphere_np(shape_zyx, radius_xyz, shift_xyz=(0.0, 0.0, 0.0), kernel=0.04):
    """EMC_maskShape('sphere', SIZE, RADIUS, .., {'shift', shift; 'kernel', kernel})
    (masking/EMC_maskShape.m:95-224): coordinates i - floor(n/2) - shift (EMC_coordVectors, origin 1),
    the ellipsoid test in single precision, the outer ceil(k/2) voxels of every face zeroed
    (EMC_resize 'force_taper' with a zero taper), EMC_convn with the separable EMC_gaussianKernel
    ([1, k], sigma), / max, <= 0.001 -> 0."""
    nz, ny, nx = shape_zyx
    r = np.broadcast_to(np.asarray(radius_xyz, np.float64), (3,)).copy()
    sh = np.asarray(shift_xyz, np.float64)
    k = 0
    if kernel > 0:
        mn = min(nx, ny, nz) if nz > 1 else min(nx, ny)
        v = (mn * kernel - 1) / 2
        k = int(np.floor(abs(v) + 0.5) * np.sign(v)) * 2 + 1  # MATLAB round: half away from zero
        k = max(k, 9)
        r = r + math.ceil(k / 2)
    f32 = np.float32
    vx = ((np.arange(nx) - nx // 2).astype(f32) - f32(sh[0])) / f32(r[0])
    vy = ((np.arange(ny) - ny // 2).astype(f32) - f32(sh[1])) / f32(r[1])
    if nz > 1:
        vz = ((np.arange(nz) - nz // 2).astype(f32) - f32(sh[2])) / f32(r[2])
    else:
        vz = np.zeros(1, f32)
    q = (vx[None, None, :] * vx[None, None, :] + vy[None, :, None] * vy[None, :, None]) + vz[:, None, None] * vz[:, None, None]
    m = (q <= f32(1)).astype(np.float64)
    if not k:
        return m
    t = math.ceil(k / 2)
    m[:, :, :t] = 0
    m[:, :, nx - t:] = 0
    m[:, :t, :] = 0
    m[:, ny - t:, :] = 0
    if nz > 1:
        m[:t] = 0
        m[nz - t:] = 0
    sigma = math.sqrt(-(math.ceil(k / 2) / 2) ** 2 / (2 * math.log(0.5)))
    g = np.exp(-0.5 * ((np.arange(k) - (k - 1) / 2) / sigma) ** 2)
    m = _conv_same_np(m, g / g.sum())
    m = m / m.max()
    m[m <= 0.001] = 0
    return m


def cref_filter_np(shell_freq, shell_fsc, os_freq, shape_zyx, pixel_size, force_mask=None, mtf=0.0):
    """BH_multi_cRef (statistics/BH_multi_cRef.m:55-145, the isotropic filter) with scipy's not-a-knot
    CubicSpline for MATLAB's fit(.., 'cubicSpline'): cRef(|k| / pixel) on the half spectrum (FFT order),
    the radius formed in single precision as the reference's single radialGrid."""
    from scipy.interpolate import CubicSpline
    fsc = CubicSpline(np.asarray(shell_freq, float), np.maximum(np.asarray(shell_fsc, float), 0.0), bc_type="not-a-knot")
    ox = np.asarray(os_freq, float)
    if mtf == 0:
        m = np.ones_like(ox)
    else:
        det, cap = {1.0: (-100.0, 0.05), 2.0: (-25.0, 0.06)}.get(float(mtf), (-np.round(mtf), mtf - np.round(mtf)))
        m = 1.0 / ((np.exp(det * ox ** 1.25) + cap) / cap)
    F = fsc(ox)
    vals = np.sqrt(np.abs(2 * F / (1 + F))) * m * (1.0 if force_mask is None else np.asarray(force_mask, float))
    cref = CubicSpline(ox, vals, bc_type="not-a-knot")
    nz, ny, nx = shape_zyx
    f32 = np.float32
    kx = np.arange(nx // 2 + 1).astype(f32) / f32(nx)
    ky = (np.fft.fftfreq(ny) * ny).astype(f32) / f32(ny)
    kz = (np.fft.fftfreq(nz) * nz).astype(f32) / f32(nz)
    r2 = (kx[None, None, :] * kx[None, None, :] + ky[None, :, None] * ky[None, :, None]) + kz[:, None, None] * kz[:, None, None]
    rad = np.sqrt(r2.astype(f32)) / f32(pixel_size)
    return cref(rad.astype(np.float64))


def symmetry_matrices_np(symmetry):
    """interpolator.check_symmetry operators as applied by interp3d (testScripts/interpolator.m:172-214):
    C<n> / D<n>: defineMatrix([0, 0, k 360/n], 'Bah', 'forward') for k < n (for D<n> nSymMats = n, so the
    stored mirrored copies are never applied); O: the 24 proper signed permutation matrices."""
    kind = symmetry[0]
    if kind in "CD":
        n = int(symmetry[1:])
        return np.array([define_matrix_np([0.0, 0.0, k * 360.0 / n], "forward") for k in range(n)])
    if symmetry == "O":
        import itertools
        out = []
        for perm in itertools.permutations(range(3)):
            for signs in itertools.product((1, -1), repeat=3):
                m = np.zeros((3, 3))
                for i in range(3):
                    m[i, perm[i]] = signs[i]
                if round(np.linalg.det(m)) == 1:
                    out.append(m)
        return np.array(out)
    raise ValueError("symmetry %s" % symmetry)


def average_np(particles, mask, rotations, halves, shifts=None, weights=None, wedges=None, wedge_index=None,
               symmetry=None, bin_threshold=0.01):
    """FP64 restatement of the accumulation loop of transformations/BH_average3d.m:1417-1482 and the
    final division (:1703-1707).  Per particle: r = interpolator(particle, R, shift, 'inv', symmetry)
    (testScripts/interpolator.m:29-78: zero-border trilinear of mexXform3d, the sum over R S_k divided
    by the number of operators); r = (r - mean(r(B))) / rms(r(B) - mean) .* mask with B = mask >
    bin_threshold (:1087-1092, :1439-1441); skipped when mean(r(:)) is not finite (:1450-1456); r .*
    weight added to the sum of its half set, and the rotated wedge (zero shift) times weight to the
    half set's wedge sum.  Returns {half: (average, wedge_sum or None, count)} and the kept flags."""
    k = len(particles)
    syms = [np.eye(3)] if symmetry is None else list(symmetry)
    n = particles[0].shape[-1]
    B = mask > bin_threshold
    sums = {1: np.zeros((n,) * 3), 2: np.zeros((n,) * 3)}
    nw = wedges[0].shape[-1] if wedges is not None else 0
    wsums = {1: np.zeros((nw,) * 3), 2: np.zeros((nw,) * 3)} if nw else None
    counts = {1: 0, 2: 0}
    kept = np.zeros(k, dtype=bool)
    for p in range(k):
        R = np.asarray(rotations[p], dtype=np.float64).reshape(3, 3)
        sh = (0.0, 0.0, 0.0) if shifts is None else tuple(float(v) for v in shifts[p])
        w = 1.0 if weights is None else float(weights[p])
        r = rotate(np.asarray(particles[p], np.float64), R, sh, "inv", interp=2, symmetry=syms)
        mu = r[B].mean()
        r = r - mu
        r = r / np.sqrt(np.mean(r[B] ** 2))
        r = r * mask
        if not np.isfinite(r.mean()):
            continue
        kept[p] = True
        h = int(halves[p])
        sums[h] += r * w
        counts[h] += 1
        if nw:
            wv = rotate(np.asarray(wedges[int(wedge_index[p])], np.float64), R, (0.0, 0.0, 0.0), "inv", interp=2,
                        symmetry=syms)
            wsums[h] += wv * w
    out = {}
    for h in (1, 2):
        avg = sums[h] / counts[h] if counts[h] else np.full((n,) * 3, np.nan)
        out[h] = (avg, wsums[h] if nw else None, counts[h])
    return out, kept


# ------------------------------------------------------------------ data formats
_MRC_DTYPES = {0: "i1", 1: "i2", 2: "f4", 6: "u2"}


def mrc_write_np(path, vol, mode=2, big_endian=False, ext_bytes=0, pixel=1.0):
    """Writes an MRC file with numpy (any of the modes getVolume reads), for tests; header words at
    the offsets @MRCImage/private/readHeader.m reads them."""
    e = ">" if big_endian else "<"
    v = np.asarray(vol)
    nz, ny, nx = v.shape
    hdr = bytearray(1024)
    import struct
    struct.pack_into(e + "10i", hdr, 0, nx, ny, nz, mode, 0, 0, 0, nx, ny, nz)
    struct.pack_into(e + "6f", hdr, 40, nx * pixel, ny * pixel, nz * pixel, 90, 90, 90)
    struct.pack_into(e + "3i", hdr, 64, 1, 2, 3)
    struct.pack_into(e + "3f", hdr, 76, float(v.min()), float(v.max()), float(v.mean()))
    struct.pack_into(e + "i", hdr, 92, ext_bytes)
    hdr[208:212] = b"MAP "
    with open(path, "wb") as f:
        f.write(bytes(hdr))
        f.write(b"\0" * ext_bytes)
        f.write(np.ascontiguousarray(v, dtype=e + _MRC_DTYPES[mode]).tobytes())


def mrc_read_np(path, box=None):
    """Restatement of getVolume (@MRCImage/getVolume.m:150-298) with readHeader's byte-order test
    (@MRCImage/private/readHeader.m:18-40) and data offset 1024 + extended bytes (:176)."""
    import struct
    raw = open(path, "rb").read()
    e = "<"
    nx, ny, nz = struct.unpack_from("<3i", raw, 0)
    if nx < 0 or ny < 0 or nz < 0 or (nx > 65535 and ny > 65535 and nz > 65535):
        e = ">"
        nx, ny, nz = struct.unpack_from(">3i", raw, 0)
    mode = struct.unpack_from(e + "i", raw, 12)[0]
    ext = struct.unpack_from(e + "i", raw, 92)[0]
    data = np.frombuffer(raw, dtype=e + _MRC_DTYPES[mode], count=nx * ny * nz, offset=1024 + ext)
    v = data.reshape(nz, ny, nx).astype(np.float32)
    if box is not None:
        x1, x2, y1, y2, z1, z2 = [int(b) for b in box]
        x1, y1, z1 = x1 or 1, y1 or 1, z1 or 1
        x2, y2, z2 = x2 or nx, y2 or ny, z2 or nz
        v = v[z1 - 1:z2, y1 - 1:y2, x1 - 1:x2]
    return v


def window_bounds_np(volume_size, window_size, mask_radius, center):
    """BH_isWindowValid (logicals/BH_isWindowValid.m): 0-based start of the window, pads, shift, valid."""
    vs, ws = np.asarray(volume_size, float), np.asarray(window_size, float)
    min_size = (mask_radius + 6) * 2
    win_low = np.ceil((ws - 1) / 2)
    win_top = win_low - np.mod(ws - 1, 2)
    c = np.floor(center)
    low = c - win_low
    top = vs - (c + win_top)
    pad_low = (np.abs(low) + 1) * (low <= 0)
    pad_top = np.abs(top) * (top <= 0)
    valid = not np.any(ws - pad_low - pad_top - min_size < -2)
    return (low - 1).astype(int), pad_low.astype(int), pad_top.astype(int), np.asarray(center) - c, valid


def extract_window_np(vol, window_size, center, mask_radius):
    """Crop [LOW, TOP] of BH_isWindowValid and BH_padZeros3d with zeros (BH_average3d.m:1304-1341)."""
    nz, ny, nx = vol.shape
    start, pl, pt, sh, ok = window_bounds_np((nx, ny, nz), window_size, mask_radius, center)
    wx, wy, wz = window_size
    out = np.zeros((wz, wy, wx), dtype=vol.dtype)
    for k in range(wz):
        z = start[2] + k
        if not 0 <= z < nz:
            continue
        for j in range(wy):
            y = start[1] + j
            if not 0 <= y < ny:
                continue
            x0, x1 = max(0, start[0]), min(nx, start[0] + wx)
            if x1 > x0:
                out[k, j, x0 - start[0]:x1 - start[0]] = vol[z, y, x0:x1]
    return out, sh, ok


def sf3d_particles_np(size, sampling, tlt, xyz, recon_geometry):
    """BH_weightMaskMex (masking/BH_weightMaskMex.m:1-60) restated: single-precision host arithmetic,
    the SF3D volume from the C oracle of mexSF3D, then SF3D - (min - 1e-4)."""
    order = np.argsort(np.asarray(tlt)[:, 0], kind="stable")
    T = np.asarray(tlt)[order].astype(np.float32)
    f = np.float32
    pix = T[:, 15] * f(sampling) * f(1e10)
    cs = T[:, 16] * f(1e3)
    lam = T[:, 17] * f(1e10)
    ac = T[:, 18]
    def0 = -T[:, 14] * f(1e10)
    ddf = T[:, 11] * f(1e10)
    dphi = T[:, 12] * f(180.0) / f(np.pi)
    tilt = T[:, 3]
    expo = T[:, 10]
    dose = T[:, 13] / np.mean(T[:, 13], dtype=np.float32)
    el = np.exp(f(-75.0) / (np.cos(tilt * f(np.pi / 180)) * f(400.0)))
    el = el / el.max()
    occ = el * dose
    rg = np.asarray(recon_geometry, dtype=np.float64).reshape(2, 3)
    origin = np.ceil((rg[0] + 1) / 2)
    out = []
    for p in np.asarray(xyz, dtype=np.float64).reshape(-1, 3):
        v = p - origin + rg[1]
        a = tilt * f(np.pi / 180)
        z = -np.sin(a) * f(v[0]) + np.cos(a) * f(v[2])
        d = def0 - z * pix
        vol = sf3d(size, pix, lam, cs, d + ddf, d - ddf, dphi, ac, tilt, expo, occ, squared=True)
        out.append(vol - (vol.min() - 1e-4))
    return np.array(out)


# ------------------------------------------------------------------ template-search pre / post
def moving_average_np(img, feature_size):
    """BH_movingAverage_2 (statistics/BH_movingAverage_2.m): padarray(img, ceil(L/2), 'both', 'symmetric'),
    separable convn(..., 'same') with the EMC_gaussianKernel([1, L], 3) row kernel along x, y, z, crop."""
    L = int(feature_size)
    t = np.arange(L) - (L - 1) / 2.0
    w = np.exp(-0.5 * (t / 3.0) ** 2)
    w /= w.sum()
    p = int(np.ceil(L / 2))
    v = np.pad(np.asarray(img, dtype=np.float64), p, mode="symmetric")
    h = L // 2
    for axis in (2, 1, 0):  # x, y, z of a (z, y, x) array
        full = np.apply_along_axis(lambda r: np.convolve(r, w, mode="full"), axis, v)
        idx = [slice(None)] * 3
        idx[axis] = slice(h, h + v.shape[axis])  # 'same': central part starting at floor(L/2)
        v = full[tuple(idx)]
    return v[p:-p, p:-p, p:-p]


def local_normalize_np(img, feature_size):
    """BH_templateSearch3d_2.m:558-561: (x - avg) ./ sqrt(avg(x.^2) - avg.^2)."""
    x = np.asarray(img, dtype=np.float64)
    a = moving_average_np(x, feature_size)
    a2 = moving_average_np(x * x, feature_size)
    return (x - a) / np.sqrt(a2 - a * a)


def tsearch_peaks_np(mag, ang, removal, rm_dim, angle_list, max_peaks, max_tries=10000, high_thr=0.0, sampling=1.0,
                     mask_cutoff=0.98):
    """The peak loop of alignment/BH_templateSearch3d_2.m:1100-1275 with nPeaks = 1 (FP64 restatement)."""
    mag = np.array(mag, dtype=np.float64)
    ang = np.asarray(ang)
    nz, ny, nx = mag.shape
    peaks = []
    tries = 0
    while len(peaks) < max_peaks and tries < max_tries:
        flat = mag.ravel()
        if np.all(np.isnan(flat)):
            break
        coord = int(np.nanargmax(flat))
        mx = flat[coord]
        if not mx > high_thr:
            break
        tries += 1
        z, y, x = np.unravel_index(coord, mag.shape)
        a = ang[z, y, x]
        if a > 0:
            box = mag[max(0, z - 1):z + 2, max(0, y - 1):y + 2, max(0, x - 1):x + 2]
            zz, yy, xx = np.meshgrid(np.arange(max(0, z - 1), min(nz, z + 2)) - z,
                                     np.arange(max(0, y - 1), min(ny, y + 2)) - y,
                                     np.arange(max(0, x - 1), min(nx, x + 2)) - x, indexing="ij")
            sw = box.sum()
            cm = np.array([(box * xx).sum(), (box * yy).sum(), (box * zz).sum()]) / sw
            e = np.asarray(angle_list[int(a) - 1], dtype=np.float64)
            row = np.zeros(10)
            row[0:3] = sampling * (np.array([x + 1, y + 1, z + 1]) + cm - rm_dim)
            row[3:6] = e
            row[9] = mx
            peaks.append(row)
            R = define_matrix_np(e, "forward")
            rmask = rotate(removal, R, (0, 0, 0), "forward", interp=2)
            r = 2 * rm_dim + 1
            for bz in range(r):
                for by in range(r):
                    for bx in range(r):
                        X, Y, Z = x - rm_dim + bx, y - rm_dim + by, z - rm_dim + bz
                        if 0 <= X < nx and 0 <= Y < ny and 0 <= Z < nz and not rmask[bz, by, bx] < mask_cutoff:
                            mag[Z, Y, X] = 0.0
        else:
            mag[z, y, x] = 0.0
    return np.array(peaks).reshape(-1, 10)
