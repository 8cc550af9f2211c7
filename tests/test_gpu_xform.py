"""Rotation / interpolation (mexXform3d replacement) against the FP64 oracle."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def smooth_volume(shape, seed):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(shape)
    # low-pass so interpolation differences stay at FP32 level, zero near the border
    V = np.fft.rfftn(v)
    kz = np.fft.fftfreq(shape[0])[:, None, None]
    ky = np.fft.fftfreq(shape[1])[None, :, None]
    kx = np.fft.rfftfreq(shape[2])[None, None, :]
    V *= np.exp(-(kx ** 2 + ky ** 2 + kz ** 2) / (2 * 0.08 ** 2))
    v = np.fft.irfftn(V, shape)
    c = np.array(shape) // 2
    zz, yy, xx = np.meshgrid(*[np.arange(s) - cc for s, cc in zip(shape, c)], indexing="ij")
    r = np.sqrt((xx / c[2]) ** 2 + (yy / c[1]) ** 2 + (zz / c[0]) ** 2)
    v *= np.clip((0.85 - r) / 0.1, 0, 1)
    return (v / np.abs(v).max()).astype(np.float32)


@pytest.mark.parametrize("interp,mode", [("linear", 0), ("cubic", 1), ("linear_border", 2)])
@pytest.mark.parametrize("shape", [(64, 64, 64), (33, 40, 48), (96, 96, 96)])
@pytest.mark.parametrize("direction", ["forward", "inv"])
def test_rotate_against_oracle(built_lib, cuda, interp, mode, shape, direction):
    from emclarity_b200 import api
    v = smooth_volume(shape, 11)
    rng = np.random.default_rng(12)
    ang = rng.uniform(-180, 180, 3)
    sh = rng.uniform(-3, 3, 3)
    M = api.define_matrix(ang, direction)
    ip = api.Interpolator(torch.from_numpy(v).cuda(), interp=interp)
    got = ip.interp3d(M, sh, direction).cpu().numpy()
    ref = O.rotate(v, M, sh, direction, interp=mode)
    assert np.abs(got - ref).max() < 2e-5


def test_bf16_storage(built_lib, cuda):
    from emclarity_b200 import api
    v = smooth_volume((64, 64, 64), 13)
    M = api.define_matrix([20, 30, 40], "inv")
    vb = torch.from_numpy(v).to(torch.bfloat16).float().numpy()
    ip = api.Interpolator(torch.from_numpy(v).cuda(), store="bf16")
    got = ip.interp3d(M).cpu().numpy()
    ref = O.rotate(vb, M)
    assert np.abs(got - ref).max() < 2e-5


def test_symmetry_average(built_lib, cuda):
    from emclarity_b200 import api
    v = smooth_volume((48, 48, 48), 14)
    M = api.define_matrix([10, 20, 30], "forward")
    sym = [api.define_matrix([0, 0, k * 120.0], "inv") for k in range(3)]
    ip = api.Interpolator(torch.from_numpy(v).cuda())
    got = ip.interp3d(M, (0.5, 0, -1), "forward", symmetry=sym).cpu().numpy()
    ref = O.rotate(v, M, (0.5, 0, -1), "forward", symmetry=sym)
    assert np.abs(got - ref).max() < 2e-5
