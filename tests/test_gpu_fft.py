"""Hand-written R2C / C2R transforms (mexFFT replacement) against the FP64 oracle and numpy."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [(64, 64, 64), (96, 96, 96), (128, 128, 128), (16, 24, 32), (48, 12, 8),
                                   (256, 64, 48), (8, 8, 512), (3, 6, 384), (64, 64, 2), (1, 1, 512), (1, 96, 192),
                                   (80, 84, 90), (108, 112, 120), (126, 144, 160), (162, 168, 180),
                                   (16, 416, 486), (8, 504, 400), (12, 378, 270)])
def test_r2c_c2r_against_oracle(built_lib, cuda, shape):
    from emclarity_b200 import api
    rng = np.random.default_rng(sum(shape))
    x = rng.standard_normal(shape).astype(np.float32)
    shp = tuple(s for s in shape)
    ft = api.FourierTransformer(shp)
    X = ft.fwd_fft(torch.from_numpy(x).cuda())
    ref = np.fft.rfftn(x.astype(np.float64)) if len(shp) == 3 else None
    if ref is None:
        ref = np.fft.rfftn(x.astype(np.float64))
    got = X.cpu().numpy().astype(np.complex128)
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() <= 2e-6 * scale
    if shape[0] > 1 and shape[1] > 1:
        assert np.abs(O.rfftn(x) - ref).max() <= 1e-10 * scale
    y = ft.inv_fft(X).cpu().numpy() / x.size
    assert np.abs(y - x).max() <= 2e-5 * np.abs(x).max()


def test_c2r_leaves_input_untouched(built_lib, cuda):
    from emclarity_b200 import api
    x = torch.randn(32, 32, 32, device="cuda")
    ft = api.FourierTransformer((32, 32, 32))
    X = ft.fwd_fft(x)
    keep = X.clone()
    ft.inv_fft(X)
    torch.cuda.synchronize()
    assert torch.equal(X, keep)


def test_batched_plan(built_lib, cuda):
    from emclarity_b200 import api
    x = torch.randn(5, 24, 32, 48, device="cuda")
    ft = api.FourierTransformer((24, 32, 48), batch=5)
    X = ft.fwd_fft(x).cpu().numpy()
    ref = np.fft.rfftn(x.cpu().numpy().astype(np.float64), axes=(1, 2, 3))
    assert np.abs(X - ref).max() <= 2e-6 * np.abs(ref).max()


def test_matches_cufft_comparator(built_lib, cuda):
    """cuFFT (through torch) as a comparator only."""
    from emclarity_b200 import api
    x = torch.randn(64, 64, 64, device="cuda")
    X = api.FourierTransformer((64, 64, 64)).fwd_fft(x)
    Y = torch.fft.rfftn(x)
    assert (X - Y).abs().max().item() <= 2e-6 * Y.abs().max().item()
