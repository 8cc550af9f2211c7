"""Strict parity checks of search results against the FP64 oracle (shared by the GPU tests).

A GPU result may differ from the oracle's only at a near-tie, and every such difference is
checked, not counted:
  * CC values within RTOL relative (+ ATOL absolute) of the oracle's;
  * an integer peak that differs from the oracle's is accepted only when the oracle's own map,
    read at the GPU's peak, equals the oracle's maximum within that tolerance;
  * a best orientation that differs from the oracle's is accepted only when the oracle's CC at
    the GPU's orientation equals the oracle's best within that tolerance.
"""
import numpy as np

RTOL = 1e-4
ATOL = 1e-6


def tol(v):
    return RTOL * abs(v) + ATOL


def check_cc_and_peaks(cc_g, pk_g, cc_o, pk_o, oracle_map, what=""):
    """oracle_map(o) -> the oracle's fftshifted normalised map (n^3, z, y, x) of orientation o."""
    cc_g = np.asarray(cc_g, dtype=np.float64)
    err = np.abs(cc_g - cc_o)
    bad = err > RTOL * np.abs(cc_o) + ATOL
    assert not bad.any(), "%s CC off at %d orientations, max |dcc| %.3g (first %d)" % (
        what, bad.sum(), err.max(), int(np.argmax(bad)))
    mism = np.flatnonzero(np.any(np.asarray(pk_g) != np.asarray(pk_o), axis=1))
    for o in mism:
        m = oracle_map(int(o))
        c = m.shape[0] // 2
        x, y, z = (int(v) for v in pk_g[o])
        v = m[z + c, y + c, x + c]
        assert abs(v - cc_o[o]) <= tol(cc_o[o]), (
            "%s orientation %d: GPU peak %s scores %.7g in the oracle map, oracle peak %s scores %.7g"
            % (what, o, tuple(pk_g[o]), v, tuple(pk_o[o]), cc_o[o]))
    return len(mism)


def check_best(best_orient, cc_o, offset=0, what=""):
    """best_orient: the GPU's best orientation (global index); cc_o: the oracle's CCs of the slice
    that starts at global index `offset`."""
    b = int(np.argmax(cc_o))  # numpy argmax: first index wins ties, as sortrows(..., -6)
    g = int(best_orient) - offset
    if g != b:
        assert 0 <= g < len(cc_o), "%s best orientation %d outside the slice" % (what, best_orient)
        assert abs(cc_o[g] - cc_o[b]) <= tol(cc_o[b]), (
            "%s best orientation %d (oracle CC %.7g) differs from the oracle's %d (%.7g)"
            % (what, g + offset, cc_o[g], b + offset, cc_o[b]))
    return g == b
