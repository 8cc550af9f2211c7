"""Python mirror of the reference's operator interface for the orientation-search path.

Each class or function wraps one C-ABI entry point of libemc_b200.so and keeps the
argument meaning of the reference call it replaces:

* ``Interpolator``        testScripts/interpolator.m (mexXform3d)
* ``FourierTransformer``  testScripts/fourierTransformer.m (mexFFT)
* ``ctf2d`` / ``sf3d``    mexFiles/mexCTF.cu, mexFiles/mexSF3D.cu
* ``Search``              the orientation loop of alignment/BH_alignRaw3d_v2.m:1119-1423
                          with the normalised translational CC of
                          statistics/BH_multi_xcf_Translational_2.m
* ``TemplateSearch``      alignment/BH_templateSearch3d_2.m:633-887
* ``Average``             transformations/BH_average3d.m:1207-1707 (half-set sums)

Tensors are torch CUDA tensors used as device buffers only; volumes have shape
(nz, ny, nx) (x fastest, the reference's column-major order), half spectra are complex64
of shape (nz, ny, nx//2+1).  Every computation runs in the CUDA library; a missing
library or a CPU tensor raises.
"""
import ctypes as C

import numpy as np
import torch

from . import _lib as L


def _stream(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _need_cuda(t, name, dtype=torch.float32):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError("%s must be a CUDA tensor" % name)
    if t.dtype != dtype:
        raise TypeError("%s must be %s, got %s" % (name, dtype, t.dtype))
    if not t.is_contiguous():
        raise ValueError("%s must be contiguous" % name)
    return C.c_void_p(t.data_ptr())


def _dptr(arr):
    arr = np.ascontiguousarray(arr, dtype=np.float64)
    return arr, arr.ctypes.data_as(C.POINTER(C.c_double))


# --------------------------------------------------------------------------- host math
def define_matrix(angles, direction="inv"):
    """BH_defineMatrix(angles, 'Bah', direction) as a (3, 3) float64 array (row i, col j)."""
    d = {"forward": 0, "inv": 1}[direction]
    a, ap = _dptr(angles)
    out = np.zeros(9)
    L.call("emc_define_matrix", ap, d, out.ctypes.data_as(C.POINTER(C.c_double)))
    return out.reshape(3, 3, order="F")


def euler_search(symmetry, theta_max, theta_step, psi_max, psi_step):
    """eulerSearch grid as an (n, 3) array of (phi, theta, psi) in degrees, walk order."""
    cnt = C.c_int(0)
    L.call("emc_euler_search", symmetry.encode(), theta_max, theta_step, psi_max, psi_step, None, C.byref(cnt))
    out = np.zeros((cnt.value, 3))
    L.call("emc_euler_search", symmetry.encode(), theta_max, theta_step, psi_max, psi_step,
           out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(cnt))
    return out


def search_matrices(phi_theta_psi, prior=None):
    """RotMat = prior * defineMatrix([phi, theta, psi-phi], 'inv') for every orientation (FP64)."""
    prior = np.eye(3) if prior is None else np.asarray(prior, dtype=np.float64)
    out = []
    for phi, theta, psi in np.asarray(phi_theta_psi, dtype=np.float64):
        out.append(prior @ define_matrix([phi, theta, psi - phi], "inv"))
    return np.array(out)


# --------------------------------------------------------------------------- interpolator
class Interpolator:
    """Rotate / shift / interpolate a volume (mexXform3d through interpolator.m).

    ``interp3d(angles, shifts, direction, symmetry_matrices)``: ``angles`` is an Euler
    triple (converted with defineMatrix(angles, 'Bah', direction)) or a 3x3 matrix used as
    is; 'forward' negates the shift and applies it before the rotation, 'inv' after it.
    """

    def __init__(self, volume, store="f32", interp="linear"):
        self.shape = tuple(volume.shape)
        nz, ny, nx = self.shape
        h = C.c_void_p()
        dt = {"f32": L.DTYPE_F32, "bf16": L.DTYPE_BF16}[store]
        L.call("emc_xform3d_create", _need_cuda(volume, "volume"), nx, ny, nz, dt, C.byref(h), _stream())
        self._h = h
        self.interp = {"linear": L.INTERP_LINEAR, "cubic": L.INTERP_CUBIC,
                       "linear_border": L.INTERP_LINEAR_BORDER}[interp]

    def interp3d(self, angles, shifts=(0.0, 0.0, 0.0), direction="forward", symmetry=None, out=None):
        m = np.asarray(angles, dtype=np.float64)
        if m.size == 3:
            m = define_matrix(m, direction)
        m = m.reshape(3, 3)
        mats = [m] if symmetry is None else [m @ s for s in symmetry]
        packed = np.concatenate([np.asarray(x, dtype=np.float64).reshape(3, 3).flatten(order="F") for x in mats])
        packed, pp = _dptr(packed)
        sh = (C.c_float * 3)(*[float(v) for v in shifts])
        if out is None:
            out = torch.empty(self.shape, dtype=torch.float32, device="cuda")
        fwd = 1 if direction == "forward" else 0
        L.call("emc_xform3d_apply", self._h, pp, len(mats), sh, fwd, self.interp, _need_cuda(out, "out"), _stream())
        return out

    def close(self):
        if getattr(self, "_h", None):
            L.load().emc_xform3d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------------- FFT
class FourierTransformer:
    """Unnormalised R2C / C2R transforms with a cached plan (mexFFT through fourierTransformer.m)."""

    def __init__(self, shape, batch=1):
        shape = tuple(shape)
        self.shape = shape
        dims = list(reversed(shape))  # x fastest
        rank = len(dims)
        arr = (C.c_int * 3)(*(dims + [1] * (3 - rank)))
        h = C.c_void_p()
        L.call("emc_fft_plan", rank, arr, batch, C.byref(h))
        self._h = h
        self.batch = batch
        self.half_shape = shape[:-1] + (shape[-1] // 2 + 1,)
        # fourierTransformer.m:63-66
        self.inv_trim = 1 if shape[-1] % 2 else 2

    def fwd_fft(self, vol, out=None):
        if out is None:
            out = torch.empty(((self.batch,) if self.batch > 1 else ()) + self.half_shape, dtype=torch.complex64,
                              device="cuda")
        L.call("emc_fft_r2c", self._h, _need_cuda(vol, "vol"), _need_cuda(out, "out", torch.complex64), _stream())
        return out

    def inv_fft(self, ft, out=None):
        if out is None:
            out = torch.empty(((self.batch,) if self.batch > 1 else ()) + self.shape, dtype=torch.float32,
                              device="cuda")
        L.call("emc_fft_c2r", self._h, _need_cuda(ft, "ft", torch.complex64), _need_cuda(out, "out"), _stream())
        return out

    def close(self):
        if getattr(self, "_h", None):
            L.load().emc_fft_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------------- CTF
def _ctfp(pixel_size, wavelength, cs_mm, defocus1, defocus2, astig_deg, amp_contrast):
    return L.CtfParams(pixel_size, wavelength, cs_mm, amp_contrast, defocus1, defocus2, astig_deg)


def ctf2d(nx, ny, pixel_size, wavelength, cs_mm, defocus1, defocus2, astig_deg, amp_contrast, half=True,
          squared=False, centred=False, radial_weight=None, exposure=None):
    """mexCTF(half, sq, nX, nY, pix, lambda, Cs, df1, df2, ast, AC[, centred]) -> (ny, nx') tensor."""
    p = _ctfp(pixel_size, wavelength, cs_mm, defocus1, defocus2, astig_deg, amp_contrast)
    out = torch.empty((ny, nx // 2 + 1 if half else nx), dtype=torch.float32, device="cuda")
    if radial_weight is None:
        L.call("emc_ctf2d", C.byref(p), nx, ny, int(half), int(squared), int(centred), _need_cuda(out, "out"),
               _stream())
    else:
        L.call("emc_ctf2d_exposure", C.byref(p), nx, ny, int(half), int(squared), int(centred),
               float(radial_weight), float(exposure), _need_cuda(out, "out"), _stream())
    return out


def sf3d(size, pixel_size, wavelength, cs_mm, df1, df2, astig_deg, amp_contrast, tilt_deg, exposure, occupancy,
         squared=True):
    """mexSF3D: sum over tilts of the exposure-weighted CTF^2 on the tilted central slab.

    ``size`` is (nx, ny, nz); per-tilt arrays have one entry per tilt.  Returns (nz, ny, nx)."""
    nt = len(tilt_deg)

    def fa(x):
        a = np.ascontiguousarray(np.broadcast_to(np.asarray(x, dtype=np.float32), (nt,)))
        return a, a.ctypes.data_as(C.POINTER(C.c_float))

    arrs = [fa(x) for x in (pixel_size, wavelength, cs_mm, df1, df2, astig_deg, amp_contrast, tilt_deg, exposure,
                            occupancy)]
    sz = (C.c_uint * 3)(*[int(v) for v in size])
    out = torch.empty((size[2], size[1], size[0]), dtype=torch.float32, device="cuda")
    L.call("emc_sf3d", 0, int(squared), sz, *[a[1] for a in arrs[:7]], nt, arrs[7][1], arrs[8][1], arrs[9][1],
           _need_cuda(out, "out"), _stream())
    return out


def wedge_ctf_weight(n, tilt_min=-60.0, tilt_max=60.0, ctf=None, squared=False):
    """Half-spectrum (n, n, n//2+1) weight: binary Y-axis missing wedge times the 3-D CTF.

    ``ctf``: dict(pixel_size, wavelength, cs_mm, defocus, amp_contrast) or None."""
    out = torch.empty((n, n, n // 2 + 1), dtype=torch.float32, device="cuda")
    p = None
    if ctf is not None:
        p = C.byref(_ctfp(ctf["pixel_size"], ctf["wavelength"], ctf["cs_mm"], ctf["defocus"], ctf["defocus"], 0.0,
                          ctf["amp_contrast"]))
    L.call("emc_wedge_ctf_weight", int(n), float(tilt_min), float(tilt_max), p, int(squared),
           _need_cuda(out, "out"), _stream())
    return out


# --------------------------------------------------------------------------- particle prep
def binary_wedge(n, tilt_min=-60.0, tilt_max=60.0, smooth=True, half=True):
    """BH_weightMask3d 'binaryWedgeGPU' for a Y tilt axis (smoothed, Nyquist-windowed, normalised to
    [0, 1]): the half spectrum in FFT order ((n, n, n/2+1), the search's wdgMask form) or the centred
    n^3 volume the reference returns (half=False)."""
    shape = (n, n, n // 2 + 1) if half else (n, n, n)
    out = torch.empty(shape, dtype=torch.float32, device="cuda")
    L.call("emc_binary_wedge", int(n), float(tilt_min), float(tilt_max), int(bool(smooth)), int(bool(half)),
           _need_cuda(out, "out"), _stream())
    return out


def centred_to_half(vol):
    """ifftshift of centred weight volumes ((count,) nz, ny, nx) cropped to half spectra ((count,) nz, ny,
    nx/2+1) in FFT order: the reference's centred SF3D / wedge volumes in the form the search's wedge takes."""
    v = vol if vol.dim() == 4 else vol.unsqueeze(0)
    count, nz, ny, nx = v.shape
    out = torch.empty((count, nz, ny, nx // 2 + 1), dtype=torch.float32, device="cuda")
    L.call("emc_centred_to_half", _need_cuda(v, "vol"), nx, ny, nz, count, _need_cuda(out, "out"), _stream())
    return out if vol.dim() == 4 else out[0]


def mask_sphere(shape_zyx, radius, shift=(0.0, 0.0, 0.0), kernel=0.04):
    """EMC_maskShape('sphere', SIZE, RADIUS, 'gpu', {'shift', shift; 'kernel', kernel}): shape and the
    returned tensor are (z, y, x); radius and shift are (x, y, z) like the reference's vectors (a
    scalar radius is isotropic)."""
    nz, ny, nx = shape_zyx
    r = np.broadcast_to(np.asarray(radius, dtype=np.float64), (3,)).copy()
    size = (C.c_int * 3)(int(nx), int(ny), int(nz))
    ra, rp = _dptr(r)
    sa, sp = _dptr(np.asarray(shift, dtype=np.float64).reshape(3))
    out = torch.empty((nz, ny, nx), dtype=torch.float32, device="cuda")
    L.call("emc_mask_sphere", size, rp, sp, float(kernel), _need_cuda(out, "out"), _stream())
    return out


def cref_filter(shell_freq, shell_fsc, os_freq, shape_zyx, pixel_size, force_mask=None, mtf=0.0):
    """BH_multi_cRef's isotropic filter sqrt(2 FSC / (1 + FSC)) . MTF . forceMask as a half spectrum
    (z, y, x/2+1) in FFT order; frequencies in 1/Angstrom."""
    nz, ny, nx = shape_zyx
    sf, sfp = _dptr(shell_freq)
    fs, fsp = _dptr(shell_fsc)
    ox, oxp = _dptr(os_freq)
    fm, fmp = _dptr(force_mask) if force_mask is not None else (None, None)
    size = (C.c_int * 3)(int(nx), int(ny), int(nz))
    out = torch.empty((nz, ny, nx // 2 + 1), dtype=torch.float32, device="cuda")
    L.call("emc_cref_filter", sfp, fsp, len(sf), oxp, fmp, len(ox), float(mtf), size, float(pixel_size),
           _need_cuda(out, "out"), _stream())
    return out


def particle_spectrum(particle, weight=None, bandpass=None):
    """Q = weight .* bandpass .* fftn(particle), Q(0) = 0, and E_P = sum |Q|^2 (full spectrum)."""
    n = particle.shape[-1]
    q = torch.empty((n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    e = torch.zeros(1, dtype=torch.float64, device="cuda")
    L.call("emc_particle_spectrum", n, _need_cuda(particle, "particle"),
           _need_cuda(weight, "weight") if weight is not None else None,
           _need_cuda(bandpass, "bandpass") if bandpass is not None else None,
           _need_cuda(q, "q", torch.complex64), _need_cuda(e, "energy", torch.float64), _stream())
    return q, e


def particle_spectra(particles, weights=None, bandpass=None, out=None, energies=None):
    """particle_spectrum over a batch: particles [B, n, n, n], weights [B, n, n, n/2+1] or None,
    bandpass one shared half spectrum or None.  Returns (spectra [B, n, n, n/2+1] complex64,
    energies [B] float64), written into `out` / `energies` when given."""
    count, n = particles.shape[0], particles.shape[-1]
    if weights is not None and (weights.shape[0] != count or weights[0].numel() != n * n * (n // 2 + 1)):
        raise ValueError("weights must hold one half spectrum per particle")
    if out is None:
        out = torch.empty((count, n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    if energies is None:
        energies = torch.empty(count, dtype=torch.float64, device="cuda")
    if out.shape[0] < count or energies.numel() < count:
        raise ValueError("out / energies hold fewer than %d particles" % count)
    L.call("emc_particle_spectra", n, count, _need_cuda(particles, "particles"),
           _need_cuda(weights, "weights") if weights is not None else None,
           _need_cuda(bandpass, "bandpass") if bandpass is not None else None,
           _need_cuda(out, "out", torch.complex64), _need_cuda(energies, "energies", torch.float64), _stream())
    return out, energies


def particle_template(q):
    """h = unnormalised inverse transform of Q (the real-space particle template)."""
    n = q.shape[0]
    h = torch.empty((n, n, n), dtype=torch.float32, device="cuda")
    L.call("emc_particle_template", n, _need_cuda(q, "q", torch.complex64), _need_cuda(h, "h"), _stream())
    return h


# --------------------------------------------------------------------------- search
class Search:
    """Fused orientation search: rotate the reference, FFT, conj-multiply with the particle
    spectrum, normalised CC map over the peak window, argmax, best orientation."""

    def __init__(self, peak_radius=0, interp="linear", chunk_evals=0):
        h = C.c_void_p()
        L.call("emc_search_create", C.byref(h))
        self._h = h
        self._keep = []
        self.configure(peak_radius, interp, chunk_evals)

    def configure(self, peak_radius=0, interp="linear", chunk_evals=0):
        mode = {"linear": L.INTERP_LINEAR, "cubic": L.INTERP_CUBIC, "linear_border": L.INTERP_LINEAR_BORDER}[interp]
        L.call("emc_search_configure", self._h, int(peak_radius), mode, int(chunk_evals))

    def add_reference(self, ref, mask=None, wref=None, store="f32"):
        n = ref.shape[-1]
        rid = C.c_int(-1)
        dt = {"f32": L.DTYPE_F32, "bf16": L.DTYPE_BF16}[store]
        L.call("emc_search_add_reference", self._h, _need_cuda(ref, "ref"), n,
               _need_cuda(mask, "mask") if mask is not None else None,
               _need_cuda(wref, "wref") if wref is not None else None, dt, C.byref(rid), _stream())
        return rid.value

    def set_orientations(self, phi_theta_psi):
        a, ap = _dptr(np.asarray(phi_theta_psi, dtype=np.float64).reshape(-1, 3))
        L.call("emc_search_set_orientations", self._h, ap, a.shape[0])
        self.n_orient = a.shape[0]

    @staticmethod
    def particle(spectrum, energy, ref_id, prior=None, shift=(0, 0, 0), orient_begin=0, orient_count=0, wedge=None):
        """Search item.  spectrum = refWdg .* B .* F(particle) (particle_spectrum with weight = refWdg) and
        energy its sum |.|^2; wedge: wdgMask, the real half-spectrum weight applied to the rotated
        reference (BH_multi_xcf_Translational_2.m:35-38), or None (= 1).  The tensors must stay alive
        while the search runs."""
        d = L.ParticleDesc()
        d.spectrum = spectrum.data_ptr()
        if wedge is not None:
            if tuple(wedge.shape) != tuple(spectrum.shape):
                raise ValueError("wedge must be a real half spectrum of the spectrum's shape")
            d.wedge = _need_cuda(wedge, "wedge").value
        d.energy = float(energy)
        pr = np.eye(3) if prior is None else np.asarray(prior, dtype=np.float64).reshape(3, 3)
        d.prior[:] = list(pr.flatten(order="F"))
        d.shift[:] = [float(v) for v in shift]
        d.box = spectrum.shape[0]
        d.ref_id = int(ref_id)
        d.orient_begin = int(orient_begin)
        d.orient_count = int(orient_count)
        return d

    def run(self, particles, cc=None, peak=None, best=None, stream=None, energies=None):
        """Device outputs: cc (float32 [pairs]), peak (int32 [pairs, 3]), best (int32 [np, 5] view of hits).
        energies: optional CUDA float64 [np] (as written by particle_spectrum); when given, the
        search reads particle p's energy from it on the device and ignores the descriptors' values."""
        if energies is not None and (not isinstance(energies, torch.Tensor) or energies.dtype != torch.float64
                                     or energies.numel() < len(particles)):
            raise ValueError("energies must be a float64 tensor with one value per particle")
        arr = (L.ParticleDesc * len(particles))(*particles)
        self._keep = [arr]
        outs = (_need_cuda(cc, "cc") if cc is not None else None,
                _need_cuda(peak, "peak", torch.int32) if peak is not None else None,
                _need_cuda(best, "best", torch.int32) if best is not None else None, _stream(stream))
        if energies is None:
            L.call("emc_search_run", self._h, arr, len(particles), *outs)
        else:
            L.call("emc_search_run_energies", self._h, arr, len(particles),
                   _need_cuda(energies, "energies", torch.float64), *outs)

    def run_host(self, particles):
        """Host outputs: (cc [pairs], peak [pairs, 3], best list of (cc, orient, peak))."""
        total = sum(p.orient_count for p in particles)
        arr = (L.ParticleDesc * len(particles))(*particles)
        cc = np.zeros(total, dtype=np.float32)
        pk = np.zeros((total, 3), dtype=np.int32)
        hits = (L.SearchHit * len(particles))()
        L.call("emc_search_run_host", self._h, arr, len(particles), cc.ctypes.data_as(C.POINTER(C.c_float)),
               pk.ctypes.data_as(C.POINTER(C.c_int)), hits, _stream())
        best = [(h.cc, h.orient, tuple(h.peak)) for h in hits]
        return cc, pk, best

    def set_profiling(self, enable=True):
        L.call("emc_search_set_profiling", self._h, int(bool(enable)))

    def timings(self, reset=False):
        """Per-pass device time (ms) and launch counts since the last reset, CC evaluations,
        and the number of kernels launched by the most recent run."""
        ms = (C.c_double * 4)()
        ln = (C.c_long * 4)()
        ev = C.c_long(0)
        last = C.c_long(0)
        L.call("emc_search_timings", self._h, ms, ln, C.byref(ev), C.byref(last), int(bool(reset)))
        names = ("fwd_xy", "z_mul", "inv_peak", "decode")
        return {"ms": dict(zip(names, list(ms))), "launches": dict(zip(names, list(ln))), "evals": ev.value,
                "launches_last_run": last.value}

    def set_planes(self, box, planes):
        """Fixes pass A's z-planes per CTA for `box` (1, 2, 4 or 8); 0 returns it to timing-based tuning."""
        L.call("emc_search_set_planes", self._h, int(box), int(planes))

    def set_overlap(self, slots):
        """Chunk scratch slots of recorded runs: 2 (default) runs consecutive 64^3 chunks concurrently,
        1 in order (larger boxes always run in order)."""
        L.call("emc_search_set_overlap", self._h, int(slots))

    def status(self):
        """Synchronises the current stream; raises EmcError (EMC_E_TIMEOUT) if a device-side wait of a
        run since the last check gave up (those runs' results are invalid)."""
        L.call("emc_search_status", self._h, _stream())

    def test_wait(self, wait_cycles=1 << 31, phantom_bytes=0):
        """Test hook: bound later runs' device-side waits at wait_cycles SM cycles and announce
        phantom_bytes more bytes than they copy (> 0 makes every such wait run out)."""
        L.call("emc_search_test_wait", self._h, int(wait_cycles), int(phantom_bytes))

    def planes(self, box, dtype="f32"):
        """(planes in use, {planes option: pass-A ms per launch at tuning}) for (box, dtype); 0 = not tuned yet."""
        g = C.c_int(0)
        ms = (C.c_float * 4)()
        L.call("emc_search_get_planes", self._h, int(box), {"f32": L.DTYPE_F32, "bf16": L.DTYPE_BF16}[dtype],
               C.byref(g), ms)
        return g.value, {1 << k: float(ms[k]) for k in range(4) if ms[k] >= 0}

    def cc_adjoint(self, ref_id, h, energy_p, prior, poses):
        """CC and gradient (dphi, dtheta, dpsi per degree; dtx, dty, dtz per voxel) per pose."""
        poses = np.ascontiguousarray(np.asarray(poses, dtype=np.float64).reshape(-1, 6))
        pr, pp = _dptr(np.asarray(prior, dtype=np.float64).reshape(3, 3).flatten(order="F"))
        n = poses.shape[0]
        cc = np.zeros(n)
        grad = np.zeros((n, 6))
        L.call("emc_cc_adjoint", self._h, int(ref_id), _need_cuda(h, "h"), float(energy_p), pp,
               poses.ctypes.data_as(C.POINTER(C.c_double)), n, cc.ctypes.data_as(C.POINTER(C.c_double)),
               grad.ctypes.data_as(C.POINTER(C.c_double)), _stream())
        return cc, grad

    def close(self):
        if getattr(self, "_h", None):
            L.load().emc_search_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TemplateSearch:
    """Template matching over a whole tomogram: per-voxel max of std-normalised CC maps and
    the 1-based index of the winning orientation (BH_templateSearch3d_2.m:633-887)."""

    def __init__(self, tomogram):
        nz, ny, nx = tomogram.shape
        self.shape = (nz, ny, nx)
        h = C.c_void_p()
        L.call("emc_tsearch_create", _need_cuda(tomogram, "tomogram"), nx, ny, nz, C.byref(h), _stream())
        self._h = h

    def run(self, template, phi_theta_psi, peak=None, angle=None):
        t = template.shape[-1]
        a, ap = _dptr(np.asarray(phi_theta_psi, dtype=np.float64).reshape(-1, 3))
        if peak is None:
            peak = torch.empty(self.shape, dtype=torch.float32, device="cuda")
        if angle is None:
            angle = torch.empty(self.shape, dtype=torch.float32, device="cuda")
        L.call("emc_tsearch_run", self._h, _need_cuda(template, "template"), t, ap, a.shape[0],
               _need_cuda(peak, "peak"), _need_cuda(angle, "angle"), _stream())
        return peak, angle

    def close(self):
        if getattr(self, "_h", None):
            L.load().emc_tsearch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tsearch_peaks(mag, ang, removal_mask, rm_dim, angle_list, max_peaks, max_tries=10000, high_thr=0.0,
                  sampling=1.0, mask_cutoff=0.98):
    """Greedy peak picking of BH_templateSearch3d_2 (nPeaks = 1) on CUDA maps (mag is modified);
    returns the (k, 10) rows (x, y, z, e1, e2, e3, 0, 0, 0, score)."""
    nz, ny, nx = mag.shape
    rm = np.ascontiguousarray(removal_mask, dtype=np.float32)
    al = np.ascontiguousarray(angle_list, dtype=np.float64).reshape(-1, 3)
    out = np.zeros((max(1, int(max_peaks)), 10))
    nf = C.c_int(0)
    L.call("emc_tsearch_peaks", _need_cuda(mag, "mag"), _need_cuda(ang, "ang"), nx, ny, nz,
           rm.ctypes.data_as(C.POINTER(C.c_float)), int(rm_dim), float(mask_cutoff),
           al.ctypes.data_as(C.POINTER(C.c_double)), al.shape[0], int(max_peaks), int(max_tries), float(high_thr),
           float(sampling), out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(nf), _stream())
    return out[:nf.value]


def moving_average(vol, feature_size, out=None):
    """BH_movingAverage_2(vol, featureSize) on a CUDA volume."""
    nz, ny, nx = vol.shape
    if out is None:
        out = torch.empty_like(vol)
    L.call("emc_moving_average", _need_cuda(vol, "vol"), nx, ny, nz, int(feature_size), _need_cuda(out, "out"),
           _stream())
    return out


def local_normalize(vol, feature_size):
    """In place (x - avg) / sqrt(avg(x^2) - avg^2) (BH_templateSearch3d_2.m:558-561)."""
    nz, ny, nx = vol.shape
    L.call("emc_local_normalize", _need_cuda(vol, "vol"), nx, ny, nz, int(feature_size), _stream())
    return vol


# --------------------------------------------------------------------------- averaging
def symmetry_matrices(symmetry):
    """The operators interpolator applies for 'C<n>', 'D<n>' or 'O' as (k, 3, 3) float64 arrays
    (testScripts/interpolator.m:172-214)."""
    cnt = C.c_int(0)
    L.call("emc_symmetry_matrices", symmetry.encode(), None, C.byref(cnt))
    out = np.zeros(9 * cnt.value)
    L.call("emc_symmetry_matrices", symmetry.encode(), out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(cnt))
    return out.reshape(cnt.value, 3, 3).transpose(0, 2, 1).copy()  # column-major -> (row, col)


class Average:
    """Odd / even half-set subtomogram sums of BH_average3d (transformations/BH_average3d.m:1207-1707).

    ``add(particles, rotations, shifts, weights, halves, wedges=None, wedge_index=None)`` rotates each
    extracted window back with interpolator(..., 'inv', symmetry), normalises it inside
    ``mask > bin_threshold``, multiplies by the soft mask and adds it (times its peak weight) to
    its half set; ``result(half)`` returns (sum / count, summed rotated weights, count).
    """

    def __init__(self, mask, symmetry="C1", wedge_box=0, bin_threshold=0.01, batch=0):
        n = mask.shape[-1]
        self.n, self.nw = n, int(wedge_box)
        sym = symmetry_matrices(symmetry) if isinstance(symmetry, str) else np.asarray(symmetry, np.float64)
        packed, pp = _dptr(np.concatenate([m.flatten(order="F") for m in sym.reshape(-1, 3, 3)]))
        h = C.c_void_p()
        L.call("emc_average_create", n, _need_cuda(mask, "mask"), float(bin_threshold), self.nw, pp, len(sym),
               int(batch), C.byref(h), _stream())
        self._h = h
        self._keep = packed

    def add(self, particles, rotations, halves, shifts=None, weights=None, wedges=None, wedge_index=None):
        k = particles.shape[0]
        rot = np.ascontiguousarray(np.concatenate([np.asarray(r, np.float64).reshape(3, 3).flatten(order="F")
                                                   for r in np.asarray(rotations).reshape(-1, 3, 3)]))
        hv = np.ascontiguousarray(halves, dtype=np.int32).reshape(k)
        sh = None if shifts is None else np.ascontiguousarray(shifts, dtype=np.float32).reshape(k, 3)
        wt = None if weights is None else np.ascontiguousarray(weights, dtype=np.float32).reshape(k)
        kept = np.zeros(k, dtype=np.int32)
        wp, nwdg, wi = None, 0, None
        if wedges is not None:
            wp, nwdg = _need_cuda(wedges, "wedges"), wedges.shape[0]
            wi = np.ascontiguousarray(wedge_index, dtype=np.int32).reshape(k)
        fp = lambda a: None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))
        ip = lambda a: None if a is None else a.ctypes.data_as(C.POINTER(C.c_int))
        L.call("emc_average_add", self._h, _need_cuda(particles, "particles"), k,
               rot.ctypes.data_as(C.POINTER(C.c_double)), fp(sh), fp(wt), ip(hv), wp, nwdg, ip(wi), ip(kept),
               _stream())
        return kept.astype(bool)

    def result(self, half):
        avg = torch.empty((self.n,) * 3, dtype=torch.float32, device="cuda")
        wsum = torch.empty((self.nw,) * 3, dtype=torch.float32, device="cuda") if self.nw else None
        cnt = C.c_long(0)
        L.call("emc_average_result", self._h, int(half), _need_cuda(avg, "avg"),
               None if wsum is None else _need_cuda(wsum, "wedge_sum"), C.byref(cnt), _stream())
        return avg, wsum, cnt.value

    def reset(self):
        L.call("emc_average_reset", self._h, _stream())

    def close(self):
        if getattr(self, "_h", None):
            L.load().emc_average_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------------- data formats
def _box(box):
    if box is None:
        return None
    b = np.ascontiguousarray(np.asarray(box, dtype=np.int32).reshape(6))
    return b


def mrc_header(path):
    """MRCImage header fields (@MRCImage/private/readHeader.m) as a dict."""
    h = L.MrcHeader()
    L.call("emc_mrc_read_header", str(path).encode(), C.byref(h))
    out = {f: getattr(h, f) for f, _ in L.MrcHeader._fields_}
    for k in ("cell", "pixel_size", "origin"):
        out[k] = tuple(out[k])
    return out


def mrc_read(path, box=None):
    """getVolume(MRCImage(path), [x1 x2], [y1 y2], [z1 z2]) as a float32 (nz, ny, nx) numpy array;
    box = (x1, x2, y1, y2, z1, z2), 1-based inclusive, 0 = whole axis."""
    h = mrc_header(path)
    b = _box(box)
    lo = [(b[2 * d] if b is not None and b[2 * d] else 1) for d in range(3)]
    hi = [(b[2 * d + 1] if b is not None and b[2 * d + 1] else (h["nx"], h["ny"], h["nz"])[d]) for d in range(3)]
    out = np.empty((hi[2] - lo[2] + 1, hi[1] - lo[1] + 1, hi[0] - lo[0] + 1), dtype=np.float32)
    L.call("emc_mrc_read", str(path).encode(), None if b is None else b.ctypes.data_as(C.POINTER(C.c_int)),
           out.ctypes.data_as(C.POINTER(C.c_float)))
    return out


def mrc_read_device(path, box=None, out=None):
    """The same box read straight into a CUDA tensor (pinned double-buffered staging)."""
    h = mrc_header(path)
    b = _box(box)
    lo = [(b[2 * d] if b is not None and b[2 * d] else 1) for d in range(3)]
    hi = [(b[2 * d + 1] if b is not None and b[2 * d + 1] else (h["nx"], h["ny"], h["nz"])[d]) for d in range(3)]
    shape = (hi[2] - lo[2] + 1, hi[1] - lo[1] + 1, hi[0] - lo[0] + 1)
    if out is None:
        out = torch.empty(shape, dtype=torch.float32, device="cuda")
    L.call("emc_mrc_read_device", str(path).encode(), None if b is None else b.ctypes.data_as(C.POINTER(C.c_int)),
           _need_cuda(out, "out"), _stream())
    return out


def mrc_write(path, vol, pixel_size=1.0, origin=None):
    """SAVE_IMG for a float32 (nz, ny, nx) volume (mode 2)."""
    v = np.ascontiguousarray(vol, dtype=np.float32)
    nz, ny, nx = v.shape
    px = (C.c_float * 3)(*([float(pixel_size)] * 3 if np.isscalar(pixel_size) else [float(p) for p in pixel_size]))
    org = None if origin is None else (C.c_float * 3)(*[float(o) for o in origin])
    L.call("emc_mrc_write", str(path).encode(), v.ctypes.data_as(C.POINTER(C.c_float)), nx, ny, nz, px, org)


def tlt_read(path):
    """A whitespace-separated tilt table (e.g. <tilt>_ctf.tlt) as a (rows, cols) float64 array."""
    r, c = C.c_int(0), C.c_int(0)
    L.call("emc_tlt_read", str(path).encode(), None, 0, C.byref(r), C.byref(c))
    out = np.zeros((r.value, c.value))
    L.call("emc_tlt_read", str(path).encode(), out.ctypes.data_as(C.POINTER(C.c_double)), r.value, C.byref(r),
           C.byref(c))
    return out


def window_bounds(volume_size, window_size, mask_radius, center):
    """BH_isWindowValid: (start0 (x, y, z), pad_low, pad_top, shift, valid)."""
    vs = (C.c_int * 3)(*[int(v) for v in volume_size])
    ws = (C.c_int * 3)(*[int(v) for v in window_size])
    cen = (C.c_double * 3)(*[float(v) for v in center])
    st, pl, pt = (C.c_int * 3)(), (C.c_int * 3)(), (C.c_int * 3)()
    sh = (C.c_double * 3)()
    ok = C.c_int(0)
    L.call("emc_window_bounds", vs, ws, float(mask_radius), cen, st, pl, pt, sh, C.byref(ok))
    return tuple(st), tuple(pl), tuple(pt), tuple(sh), bool(ok.value)


def extract_windows(volume, window_size, centers, mask_radius):
    """Windows of a (nz, ny, nx) CUDA volume around 1-based (x, y, z) centres, zero padded:
    returns (windows [count, wz, wy, wx], fractional shifts [count, 3], valid [count])."""
    nz, ny, nx = volume.shape
    ws = (C.c_int * 3)(*[int(v) for v in window_size])
    cen = np.ascontiguousarray(centers, dtype=np.float64).reshape(-1, 3)
    k = cen.shape[0]
    out = torch.empty((k, int(window_size[2]), int(window_size[1]), int(window_size[0])), dtype=torch.float32,
                      device="cuda")
    sh = np.zeros((k, 3))
    ok = np.zeros(k, dtype=np.int32)
    L.call("emc_extract_windows", _need_cuda(volume, "volume"), nx, ny, nz, ws,
           cen.ctypes.data_as(C.POINTER(C.c_double)), k, float(mask_radius), _need_cuda(out, "out"),
           sh.ctypes.data_as(C.POINTER(C.c_double)), ok.ctypes.data_as(C.POINTER(C.c_int)), _stream())
    return out, sh, ok.astype(bool)


def sf3d_particles(size, sampling, tlt, xyz, recon_geometry):
    """BH_weightMaskMex for each particle position: (count, nz, ny, nx) CUDA tensor."""
    t = np.ascontiguousarray(tlt, dtype=np.float64)
    p = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    rg = np.ascontiguousarray(recon_geometry, dtype=np.float64).reshape(2, 3)
    sz = (C.c_uint * 3)(*[int(v) for v in size])
    out = torch.empty((p.shape[0], int(size[2]), int(size[1]), int(size[0])), dtype=torch.float32, device="cuda")
    L.call("emc_sf3d_particles", sz, float(sampling), t.ctypes.data_as(C.POINTER(C.c_double)), t.shape[0],
           t.shape[1], p.ctypes.data_as(C.POINTER(C.c_double)), rg.ctypes.data_as(C.POINTER(C.c_double)),
           p.shape[0], _need_cuda(out, "out"), _stream())
    return out


# --------------------------------------------------------------------------- volume / spectrum operators
def pad3d(img, pad_low, pad_top, fill=0.0, taper=False):
    """BH_padZeros3d(img, padLow, padTop, 'GPU', 'single'|'singleTaper', fill); pads given (x, y, z)."""
    nz, ny, nx = img.shape
    pl = (C.c_int * 3)(*[int(v) for v in pad_low])
    pt = (C.c_int * 3)(*[int(v) for v in pad_top])
    out_shape = tuple(s + l + t for s, l, t in zip((nz, ny, nx), reversed(pad_low), reversed(pad_top)))
    out = torch.empty(out_shape, dtype=torch.float32, device="cuda")
    L.call("emc_pad3d", _need_cuda(img, "img"), nx, ny, nz, pl, pt, float(fill), int(bool(taper)),
           _need_cuda(out, "out"), _stream())
    return out


def bandpass3d(shape_xyz, high_thresh, high_cut, low_cut, pixel_size):
    """BH_bandpass3d on the half spectrum (z, y, x//2+1); pixel_size 0 -> 'nyquist', < 0 -> 'nyquistHigh'."""
    nx, ny, nz = shape_xyz
    out = torch.empty((nz, ny, nx // 2 + 1), dtype=torch.float32, device="cuda")
    L.call("emc_bandpass3d", nx, ny, nz, float(high_thresh), float(high_cut), float(low_cut), float(pixel_size),
           _need_cuda(out, "out"), _stream())
    return out


def band_limit_center_normalize(img, pad_low=(0, 0, 0), pad_top=(0, 0, 0), taper=False, bandpass=None):
    """BH_bandLimitCenterNormalize: half spectrum of the mean-padded image, F(0) = 0, bandpassed,
    scaled to sqrt(sum |F|^2) / numel = 1."""
    nz, ny, nx = img.shape
    od = [s + l + t for s, l, t in zip((nx, ny, nz), pad_low, pad_top)]
    out = torch.empty((od[2], od[1], od[0] // 2 + 1), dtype=torch.complex64, device="cuda")
    pl = (C.c_int * 3)(*[int(v) for v in pad_low])
    pt = (C.c_int * 3)(*[int(v) for v in pad_top])
    L.call("emc_band_limit_center_normalize", _need_cuda(img, "img"), nx, ny, nz, pl, pt, int(bool(taper)),
           _need_cuda(bandpass, "bandpass") if bandpass is not None else None,
           _need_cuda(out, "out", torch.complex64), _stream())
    return out


def xcf_rotational(part_ft, ref_ft_conj, wdg_mask=None, ref_wdg=None, nx=None):
    """BH_multi_xcf_Rotational on half spectra (z, y, x//2+1)."""
    nz, ny, nxh = part_ft.shape
    nx = nx if nx is not None else 2 * (nxh - 1)
    cc = C.c_double(0)
    L.call("emc_xcf_rotational", _need_cuda(part_ft, "part_ft", torch.complex64),
           _need_cuda(ref_ft_conj, "ref_ft", torch.complex64),
           _need_cuda(wdg_mask, "wdg_mask") if wdg_mask is not None else None,
           _need_cuda(ref_wdg, "ref_wdg") if ref_wdg is not None else None, nx, ny, nz, C.byref(cc), _stream())
    return cc.value


def xcf_translational(a, b, peak_mask=None, peak_com=3, nx=None, return_map=False):
    """BH_multi_xcf_Translational(A, B, peakMask, peakCOM): subvoxel peak (x, y, z) of
    fftshift(real(ifftn(A .* B))) and the peak value (scaled like MATLAB ifftn)."""
    nz, ny, nxh = a.shape
    nx = nx if nx is not None else 2 * (nxh - 1)
    peak = (C.c_double * 3)()
    mv = C.c_double(0)
    mp = torch.empty((nz, ny, nx), dtype=torch.float32, device="cuda") if return_map else None
    L.call("emc_xcf_translational", _need_cuda(a, "a", torch.complex64), _need_cuda(b, "b", torch.complex64),
           nx, ny, nz, _need_cuda(peak_mask, "peak_mask") if peak_mask is not None else None, int(peak_com), peak,
           C.byref(mv), _need_cuda(mp, "map") if mp is not None else None, _stream())
    res = (np.array(list(peak)), mv.value)
    return res + (mp,) if return_map else res
