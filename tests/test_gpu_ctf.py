"""CTF images (mexCTF), the SF3D wedge (mexSF3D) and the wedge.CTF weight against the oracle."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

P = dict(pixel_size=2.17, wavelength=0.01968697, cs_mm=2.7, defocus1=26000.0, defocus2=24000.0, astig_deg=35.0,
         amp_contrast=0.085)


@pytest.mark.parametrize("half", [True, False])
@pytest.mark.parametrize("centred", [False, True])
@pytest.mark.parametrize("squared", [False, True])
@pytest.mark.parametrize("nx,ny", [(64, 64), (96, 80), (65, 33)])
def test_ctf2d(built_lib, cuda, half, centred, squared, nx, ny):
    from emclarity_b200 import api
    got = api.ctf2d(nx, ny, P["pixel_size"], P["wavelength"], P["cs_mm"], P["defocus1"], P["defocus2"],
                    P["astig_deg"], P["amp_contrast"], half, squared, centred).cpu().numpy()
    ref = O.ctf2d(nx, ny, P["pixel_size"], P["wavelength"], P["cs_mm"], P["defocus1"], P["defocus2"],
                  P["astig_deg"], P["amp_contrast"], half, squared, centred)
    assert got.shape == ref.shape
    assert np.abs(got - ref).max() < 2e-4


def test_ctf2d_exposure(built_lib, cuda):
    from emclarity_b200 import api
    got = api.ctf2d(64, 64, P["pixel_size"], P["wavelength"], P["cs_mm"], P["defocus1"], P["defocus2"],
                    P["astig_deg"], P["amp_contrast"], False, True, True, radial_weight=0.7, exposure=40.0)
    ref = O.ctf2d(64, 64, P["pixel_size"], P["wavelength"], P["cs_mm"], P["defocus1"], P["defocus2"],
                  P["astig_deg"], P["amp_contrast"], False, True, True, radial_weight=0.7, exposure=40.0)
    got = got.cpu().numpy()
    assert np.abs(got - ref).max() < 2e-4 * max(1.0, np.abs(ref).max())


def test_sf3d(built_lib, cuda):
    from emclarity_b200 import api
    tilts = np.arange(-60, 61, 3.0)
    nt = len(tilts)
    expo = np.abs(tilts) / 3.0 * 3.0 + 3.0
    occ = np.exp(-75.0 / (np.cos(np.radians(tilts)) * 400.0))
    occ = occ / occ.max()
    args = ((48, 48, 48), 2.0, 0.01969, 2.7, 12000.0 + 100 * np.arange(nt), 12000.0 + 100 * np.arange(nt), 0.0, 0.1,
            tilts, expo, occ)
    got = api.sf3d(*args).cpu().numpy()
    ref = O.sf3d(*args)
    assert np.abs(got - ref).max() < 2e-4 * np.abs(ref).max()


def test_wedge_ctf_weight(built_lib, cuda):
    from emclarity_b200 import api
    n = 64
    # an asymmetric range (-55, 62): the cones are 35 and 28 degrees; the half spectrum is the
    # ifftshifted centred grid, so the Nyquist index of every axis is the frequency -n/2
    w = api.wedge_ctf_weight(n, -55, 62, None).cpu().numpy()
    k = np.fft.fftfreq(n) * n
    kxs = np.where(np.arange(n // 2 + 1) == n // 2, -n // 2, np.arange(n // 2 + 1))
    kz, ky, kx = np.meshgrid(k, k, kxs, indexing="ij")
    th = np.degrees(np.arctan2(kx, kz))
    excl = (180 - 28 <= th) | (th <= 35 - 180) | ((-28 <= th) & (th <= 35))
    ref = np.where(excl, 0.0, 1.0)
    ref[(np.abs(kx) <= 2) & (np.abs(kz) <= 2)] = 1.0
    # BH_bandpass3d 'nyquist' window: 1 below 0.485 cycles/px, Gaussian roll-off of width 1.5/n
    rn = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2) / n
    ref = ref * np.where(rn < 0.485, 1.0, np.exp(-(rn - 0.485) ** 2 / (2 * (1.5 / n) ** 2)))
    assert np.abs(w - ref).max() < 5e-6
    ctf = dict(pixel_size=2.5, wavelength=0.019687, cs_mm=2.7, defocus=25000.0, amp_contrast=0.07)
    wc = api.wedge_ctf_weight(n, -55, 62, ctf).cpu().numpy()
    s2 = (kx ** 2 + ky ** 2 + kz ** 2) / (n * 2.5) ** 2
    amp = np.arctan(0.07 / np.sqrt(1 - 0.07 ** 2))
    c = np.sin(np.pi * 0.5 * 2.7e7 * 0.019687 ** 3 * s2 * s2 - np.pi * 0.019687 * s2 * 25000.0 - amp)
    assert np.abs(wc - ref * c).max() < 2e-4
