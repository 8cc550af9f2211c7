"""Seeded synthetic inputs for the orientation-search workloads.

The reference publishes no benchmark data for this path, so every workload is generated
here from a single numpy ``Generator(PCG64(seed))`` stream per configuration:

* reference: sum of 40 isotropic Gaussian blobs (sigma ~ U[2, 4] px, amplitude 1) with centres
  uniform in a radius-24 ball (scaled with the box), pixel 2.5 A;
* particle: the reference rotated by a seeded ZXZ orientation, integer-shifted by
  U{-4..4}^3, multiplied in Fourier space by the binary Y-axis missing wedge and the CTF
  (300 kV, Cs 2.7 mm, amplitude contrast 0.07, seeded or fixed defocus), plus Gaussian noise
  with variance var(signal) / SNR.

Host-side generation uses numpy; the volume work (rotation, FFTs, weights) runs on the GPU
through the library's own kernels.
"""
import math

import numpy as np
import torch

from . import api

WAVELENGTH_300KV = 0.019687  # Angstrom
PIXEL = 2.5                  # Angstrom


def ctf_dict(defocus_A, pixel=PIXEL):
    return dict(pixel_size=pixel, wavelength=WAVELENGTH_300KV, cs_mm=2.7, defocus=defocus_A, amp_contrast=0.07)


def blob_reference(rng, n=64, n_blobs=40, radius=None, sigma=(2.0, 4.0)):
    """Sum of isotropic Gaussians on an n^3 grid (x fastest, origin floor(n/2))."""
    scale = n / 64.0
    radius = 24.0 * scale if radius is None else radius
    centres = []
    while len(centres) < n_blobs:
        p = rng.uniform(-radius, radius, size=3)
        if p @ p <= radius * radius:
            centres.append(p)
    sig = rng.uniform(sigma[0], sigma[1], size=n_blobs) * scale
    c = n // 2
    ax = np.arange(n, dtype=np.float64) - c
    z, y, x = np.meshgrid(ax, ax, ax, indexing="ij")
    vol = np.zeros((n, n, n))
    for (px, py, pz), s in zip(centres, sig):
        vol += np.exp(-((x - px) ** 2 + (y - py) ** 2 + (z - pz) ** 2) / (2.0 * s * s))
    return vol.astype(np.float32)


def soft_sphere_mask(n, radius, kernel=0.04):
    """Soft spherical mask of EMC_maskShape('sphere', [n n n], radius, ..) (masking/EMC_maskShape.m:
    95-224), the input generator's host copy of emc_mask_sphere: a ball of radius + ceil(k/2) about
    floor(n/2) (single-precision test), the outer ceil(k/2) voxels of every face zeroed, a separable
    Gaussian of k = max(9, round((0.04 n - 1)/2)*2+1) taps and sigma = sqrt(-(ceil(k/2)/2)^2/(2 ln 0.5)),
    rescaled to max 1, values <= 0.001 set to 0."""
    v = (n * kernel - 1) / 2
    k = max(9, int(math.floor(abs(v) + 0.5) * (1 if v >= 0 else -1)) * 2 + 1)
    m = math.ceil(k / 2)
    r = np.float32(radius + m)
    ax = (np.arange(n) - n // 2).astype(np.float32) / r
    q = (ax[None, None, :] * ax[None, None, :] + ax[None, :, None] * ax[None, :, None]) + ax[:, None, None] * ax[:, None, None]
    ball = (q <= np.float32(1)).astype(np.float64)
    ball[:m] = 0
    ball[n - m:] = 0
    ball[:, :m] = 0
    ball[:, n - m:] = 0
    ball[:, :, :m] = 0
    ball[:, :, n - m:] = 0
    sigma = math.sqrt(-(m / 2) ** 2 / (2 * math.log(0.5)))
    g = np.exp(-0.5 * ((np.arange(k) - (k - 1) / 2) / sigma) ** 2)
    g /= g.sum()
    out = ball
    for axis in range(3):
        out = np.apply_along_axis(lambda v_: np.convolve(v_, g, mode="same"), axis, out)
    out /= out.max()
    out[out <= 0.001] = 0.0
    return out.astype(np.float32)


def random_euler(rng, theta_max=180.0):
    """Seeded ZXZ triple (phi, theta, psi) in degrees with theta in [0, theta_max]."""
    return np.array([rng.uniform(0, 360), rng.uniform(0, theta_max), rng.uniform(-180, 180)])


def make_particle(ref_gpu, rng, truth_matrix, shift, weight_gpu, snr, ft=None):
    """Particle = wedge.CTF-filtered (reference through truth_matrix', 'forward'), rolled by
    `shift` voxels, plus Gaussian noise of variance var(signal)/snr.  Returns a CUDA tensor."""
    n = ref_gpu.shape[-1]
    interp = api.Interpolator(ref_gpu)
    rot = interp.interp3d(np.asarray(truth_matrix).T, (0, 0, 0), "forward")
    interp.close()
    rot = torch.roll(rot, shifts=(int(shift[2]), int(shift[1]), int(shift[0])), dims=(0, 1, 2)).contiguous()
    ft = ft or api.FourierTransformer((n, n, n))
    spec = ft.fwd_fft(rot)
    spec *= weight_gpu
    sig = ft.inv_fft(spec) / float(n ** 3)
    var = float(sig.double().var())
    g = torch.Generator(device="cuda")
    g.manual_seed(int(rng.integers(0, 2 ** 62)))
    noise = torch.randn(sig.shape, generator=g, device="cuda", dtype=torch.float32) * math.sqrt(var / snr)
    return (sig + noise).contiguous()


class PlainCase:
    """Single-subtomogram search (64^3, 10 degree grid, soft mask radius 28)."""

    def __init__(self, seed=0, n=64, snr=0.1, grid=("C1", 40.0, 10.0, 40.0, 10.0), mask_radius=28, peak_radius=7,
                 defocus=25000.0, tilt=(-60.0, 60.0)):
        rng = np.random.default_rng(seed)
        self.n = n
        self.ref = blob_reference(rng, n)
        self.mask = soft_sphere_mask(n, mask_radius * n / 64.0)
        self.grid = api.euler_search(*grid)
        # truth: a seeded orientation inside the grid's range with off-grid jitter
        k = int(rng.integers(0, len(self.grid)))
        phi, theta, psi = self.grid[k]
        jitter = rng.uniform(-2.0, 2.0, size=3)
        self.truth_euler = np.array([phi, max(theta + jitter[1], 0.0), psi]) + np.array([jitter[0], 0, jitter[2]])
        self.truth_index_hint = k
        self.truth_matrix = api.search_matrices([self.truth_euler])[0]
        self.shift = rng.integers(-4, 5, size=3)
        self.peak_radius = peak_radius
        self.ctf = ctf_dict(defocus)
        self.tilt = tilt
        self.snr = snr
        self.rng = rng

    def to_gpu(self):
        d = {}
        d["ref"] = torch.from_numpy(self.ref).cuda()
        d["mask"] = torch.from_numpy(self.mask).cuda()
        d["weight"] = api.wedge_ctf_weight(self.n, self.tilt[0], self.tilt[1], self.ctf)
        d["particle"] = make_particle(d["ref"], self.rng, self.truth_matrix, self.shift, d["weight"], self.snr)
        return d


def batched_sizes(n_particles=2000, seed=0):
    """60% 64^3, 30% 96^3, 10% 128^3 in a seeded order."""
    rng = np.random.default_rng(seed + 7)
    n64 = int(round(0.6 * n_particles))
    n96 = int(round(0.3 * n_particles))
    n128 = n_particles - n64 - n96
    sizes = np.array([64] * n64 + [96] * n96 + [128] * n128)
    rng.shuffle(sizes)
    return sizes


def local_grid(n_orient=256, max_angle=8.0, step=2.0):
    """Local search around a prior: eulerSearch(C1, max, step, max, step) truncated to the
    n_orient orientations closest to identity (geodesic angle)."""
    g = api.euler_search("C1", max_angle, step, max_angle, step)
    mats = api.search_matrices(g)
    ang = np.degrees(np.arccos(np.clip((np.trace(mats, axis1=1, axis2=2) - 1) / 2, -1, 1)))
    order = np.argsort(ang, kind="stable")[:n_orient]
    return g[np.sort(order)]
