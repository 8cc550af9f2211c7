"""Second CPU arm of the baseline: the per-orientation search sequence in single precision with numpy
and scipy.fft (pocketfft), parallel over orientations in spawned worker processes.

TEST / BENCH INFRASTRUCTURE ONLY: timed by bench.py beside the C port (oracle/emc_oracle.c compiled
as liboracle_f32.so) so that the CPU baseline is the faster of two independent implementations;
checked against the FP64 oracle by tests/test_oracle.py.  The product never imports it.

Per orientation, as oracle.search (BH_alignRaw3d_v2.m:1287-1330 with the normalised map of
BH_multi_xcf_Translational_2.m:35-38 and the masked argmax of BH_multi_xcf_Translational.m:33-42):
  r = mask .* I(M (p - c - t) + c)          the C port's interpn-linear gather (orc_rotate)
  R = wref .* rfftn(r), R(0) = 0, R .*= wdgMask
  map = irfftn(refWdg .* P .* conj(R)) * numel / sqrt(sum|R|^2 sum|refWdg .* P|^2)
  peak = first maximum over the spherical window (MATLAB's column-major order of the fftshifted map)
Workers are started with the 'spawn' method, so the pool is safe after CUDA was initialised.
"""
import multiprocessing as mp
import os

import numpy as np

_S = {}


def _init(ref, P, mask, wref, ref_wdg, wdg_mask, shift, radius, interp):
    from oracle import oracle as O
    n = ref.shape[0]
    h = n // 2 + 1
    c = n // 2
    pw = np.asarray(P, np.complex64) * (1 if ref_wdg is None else np.asarray(ref_wdg, np.float32))
    ep = _herm_energy(pw.astype(np.complex128))
    # one weight on the reference spectrum: wref .* wdgMask, with R(0) = 0 folded in
    w = np.ones((n, n, h), np.float32)
    if wref is not None:
        w *= wref
    if wdg_mask is not None:
        w *= wdg_mask
    w[0, 0, 0] = 0
    win = np.array([(sx, sy, sz) for sz in range(-c, n - c) for sy in range(-c, n - c) for sx in range(-c, n - c)
                    if sx * sx + sy * sy + sz * sz <= radius * radius])
    _S.update(O=O, ref=np.ascontiguousarray(ref, np.float32), mask=mask, w=w, shift=shift, interp=interp, n=n,
              pw=np.ascontiguousarray(pw), ep=ep, win=win, idx=(win[:, 2] % n, win[:, 1] % n, win[:, 0] % n))
    O.lib("f32")


def _herm_energy(R):
    """sum |R|^2 over the full spectrum from the half spectrum R (x planes 0 and n/2 counted once)."""
    e = 2.0 * np.vdot(R, R).real
    return float(e - np.vdot(R[..., 0].copy(), R[..., 0].copy()).real - np.vdot(R[..., -1].copy(), R[..., -1].copy()).real)


def _one(M):
    import scipy.fft as sfft
    S = _S
    n = S["n"]
    r = S["O"].rotate(S["ref"], np.asarray(M, np.float64).T, S["shift"], "forward", interp=S["interp"],
                      precision="f32")
    if S["mask"] is not None:
        r *= S["mask"]
    R = sfft.rfftn(r, workers=1)
    R *= S["w"]
    er = _herm_energy(R)
    np.conjugate(R, out=R)
    R *= S["pw"]
    mp_ = sfft.irfftn(R, s=(n, n, n), workers=1)  # scipy scales by 1 / numel
    v = mp_[S["idx"]].astype(np.float64) * (n ** 3 / np.sqrt(er * S["ep"]))
    k = int(np.argmax(v))
    return float(v[k]), S["win"][k]


def _batch(mats):
    return [_one(M) for M in mats]


class Pool:
    """A spawned worker pool holding one particle's search operands; ``search(matrices)`` returns
    (cc, peak) per matrix like oracle.search."""

    def __init__(self, ref, P, mask=None, wref=None, ref_wdg=None, wdg_mask=None, shift=(0, 0, 0), radius=7,
                 interp=0, processes=None):
        from oracle import oracle as O
        O.lib("f32")  # built once here, not raced by the workers
        self.processes = processes or os.cpu_count() or 1
        f32 = lambda a: None if a is None else np.ascontiguousarray(a, np.float32)  # noqa: E731
        args = (np.ascontiguousarray(ref, np.float32), np.ascontiguousarray(P, np.complex64), f32(mask), f32(wref),
                f32(ref_wdg), f32(wdg_mask), tuple(float(v) for v in shift), int(radius), int(interp))
        os.environ.setdefault("OMP_NUM_THREADS", "1")
        self.pool = mp.get_context("spawn").Pool(self.processes, initializer=_init, initargs=args)

    def search(self, matrices):
        mats = [np.asarray(M, np.float64) for M in matrices]
        per = max(1, len(mats) // (2 * self.processes))
        chunks = [mats[i:i + per] for i in range(0, len(mats), per)]
        out = [r for part in self.pool.map(_batch, chunks) for r in part]
        return np.array([o[0] for o in out]), np.array([o[1] for o in out], dtype=np.int32)

    def close(self):
        self.pool.terminate()
        self.pool.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
