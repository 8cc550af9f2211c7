"""Generates tests/golden/ref_mex.npz from the reference's own MEX kernels.

The reference MEX sources (mexFiles/mexXform3d.cu, mexFiles/mexCTF.cu + utils/ctf.cu,
mexFiles/mexFFT.cu) are compiled by `make -C oracle ref` against the in-repo MEX stand-in into
oracle/_ref/ (this needs the reference source tree; the built libraries travel with the repo).
This script runs them on a GPU with seeded inputs and stores inputs and outputs, so that the
CPU oracle can be checked against the reference itself without a GPU:

    python tests/golden/make_ref_fixtures.py        (on a machine with a CUDA GPU)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def smooth_volume(shape, seed):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(shape)
    V = np.fft.rfftn(v)
    kz = np.fft.fftfreq(shape[0])[:, None, None]
    ky = np.fft.fftfreq(shape[1])[None, :, None]
    kx = np.fft.rfftfreq(shape[2])[None, None, :]
    V *= np.exp(-(kx ** 2 + ky ** 2 + kz ** 2) / (2 * 0.1 ** 2))
    v = np.fft.irfftn(V, s=shape, axes=(0, 1, 2))
    return (v / np.abs(v).max()).astype(np.float32)


def main():
    import torch

    import mexcall
    from oracle import oracle as O

    out = {}
    # ---- mexXform3d: texture trilinear, border addressing
    xf = mexcall.reference("mexXform3d")
    shapes = [(24, 24, 24), (20, 22, 25)]
    cases = [([20.0, 35.0, -50.0], (1.5, -0.75, 2.0), True), ([-70.0, 10.0, 130.0], (0.0, 0.0, 0.0), False),
             ([0.0, 90.0, 0.0], (-2.0, 1.0, 0.5), False), ([45.0, 0.0, 0.0], (0.25, 0.5, -0.25), True)]
    k = 0
    for si, shape in enumerate(shapes):
        vol = smooth_volume(shape, 100 + si)
        out["xform_vol_%d" % si] = vol
        for ang, sh, fwd in cases:
            R = O.define_matrix(ang, "forward" if fwd else "inv").astype(np.float32)
            size = np.array([shape[2], shape[1], shape[0]], dtype=np.uint64)
            res, tex, arr = xf(3, size, torch.from_numpy(vol).cuda(), R, np.asarray(sh, np.float32),
                               np.array(fwd))
            xf(0, tex, arr)
            out["xform_%d_R" % k] = R
            out["xform_%d_shift" % k] = np.asarray(sh, np.float32)
            out["xform_%d_fwd" % k] = np.array(fwd)
            out["xform_%d_vol" % k] = np.array(si)
            out["xform_%d_out" % k] = res.cpu().numpy()
            k += 1
    out["xform_n"] = np.array(k)
    # ---- mexCTF
    ctf = mexcall.reference("mexCTF")
    params = [(64, 64, 2.17, 0.01968697, 2.7, 26000.0, 24000.0, 35.0, 0.085, True, False, None),
              (96, 80, 2.5, 0.019687, 2.7, 25000.0, 25000.0, 0.0, 0.07, True, True, None),
              (48, 48, 1.8, 0.025079, 2.0, 15000.0, 13000.0, -60.0, 0.1, False, False, True),
              (64, 96, 3.0, 0.019687, 2.7, 40000.0, 38000.0, 100.0, 0.07, False, True, False)]
    for i, (nx, ny, pix, wl, cs, d1, d2, ast, ac, half, sq, centred) in enumerate(params):
        args = [np.array(half), np.array(sq), np.int32(nx), np.int32(ny), np.float32(pix), np.float32(wl),
                np.float32(cs), np.float32(d1), np.float32(d2), np.float32(ast), np.float32(ac)]
        if centred is not None:
            args.append(np.array(centred))
        (res,) = ctf(1, *args)
        out["ctf_%d_params" % i] = np.array([nx, ny, pix, wl, cs, d1, d2, ast, ac, half, sq,
                                             -1 if centred is None else centred], dtype=np.float64)
        out["ctf_%d_out" % i] = res.cpu().numpy()
    out["ctf_n"] = np.array(len(params))
    # ---- mexFFT (cuFFT)
    fft = mexcall.reference("mexFFT")
    for i, shape in enumerate([(16, 20, 24), (12, 18, 9)]):
        x = np.random.default_rng(200 + i).standard_normal(shape).astype(np.float32)
        inv_trim = np.int32(1 if shape[2] % 2 else 2)
        X, pf, pi = fft(3, torch.from_numpy(x).cuda(), inv_trim)
        X_saved = X.cpu().numpy()  # cufftExecC2R may overwrite its input
        (y,) = fft(1, X, inv_trim, pf, pi)
        fft(0, torch.zeros(1, device="cuda"), inv_trim, pf, pi)
        out["fft_%d_in" % i] = x
        out["fft_%d_fwd" % i] = X_saved
        out["fft_%d_fwd_ok" % i] = np.array(True)
        out["fft_%d_inv" % i] = y.cpu().numpy()
    out["fft_n"] = np.array(2)
    path = os.path.join(HERE, "ref_mex.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
