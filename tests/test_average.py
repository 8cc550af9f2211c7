"""Subtomogram averaging: symmetry operators and the FP64 restatement (CPU)."""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sym_O.npz")


def _as_set(mats):
    return sorted(tuple(np.round(m, 6).ravel()) for m in mats)


def test_octahedral_operators_match_reference_table(built_lib):
    """The 24 generated cube rotations are exactly the reference's literal table (as a set)."""
    from emclarity_b200 import api
    ref = np.load(GOLDEN)["O"]
    assert _as_set(api.symmetry_matrices("O")) == _as_set(ref)
    assert _as_set(O.symmetry_matrices_np("O")) == _as_set(ref)
    assert np.allclose(api.symmetry_matrices("O")[0], np.eye(3))


@pytest.mark.parametrize("sym", ["C1", "C2", "C5", "D3", "D6"])
def test_cyclic_operators_match_restatement(built_lib, sym):
    from emclarity_b200 import api
    a = api.symmetry_matrices(sym)
    b = O.symmetry_matrices_np(sym)
    assert a.shape == b.shape == (int(sym[1:]), 3, 3)
    assert np.allclose(a, b, atol=1e-14)
    # proper rotations about z
    assert np.allclose(np.linalg.det(a), 1.0) and np.allclose(a[:, 2, 2], 1.0)


def test_bad_symmetry_is_rejected(built_lib):
    from emclarity_b200 import EmcError, api
    for s in ["C0", "Cx", "T", "I", "D"]:
        with pytest.raises(EmcError):
            api.symmetry_matrices(s)


def test_average_restatement_identity_case():
    """One particle, identity rotation, no shift: the average is the normalised, masked particle."""
    rng = np.random.default_rng(3)
    n = 16
    p = rng.standard_normal((n, n, n))
    m = np.clip(rng.uniform(-0.2, 1.0, (n, n, n)), 0, None)
    res, kept = O.average_np([p], m, [np.eye(3)], [1])
    B = m > 0.01
    r = p - p[B].mean()
    r = r / np.sqrt(np.mean(r[B] ** 2)) * m
    assert kept[0] and res[1][2] == 1 and res[2][2] == 0
    assert np.allclose(res[1][0], r, atol=1e-12)
    assert np.isnan(res[2][0]).all()


def test_average_restatement_symmetry_is_invariant():
    """A C4-symmetrised average of a particle and of its 90-degree rotated copy are equal."""
    rng = np.random.default_rng(4)
    n = 16
    p = rng.standard_normal((n, n, n))
    m = np.ones((n, n, n))
    syms = O.symmetry_matrices_np("C4")
    r90 = O.define_matrix_np([0.0, 0.0, 90.0], "forward")
    a, _ = O.average_np([p], m, [np.eye(3)], [1], symmetry=syms)
    b, _ = O.average_np([p], m, [r90], [1], symmetry=syms)
    assert np.allclose(a[1][0], b[1][0], atol=1e-9)


def test_moving_average_restatement_basics():
    """Constant volumes stay constant (the weights sum to one, symmetric borders)."""
    v = np.full((12, 14, 16), 3.5)
    assert np.allclose(O.moving_average_np(v, 7), 3.5)
    assert np.allclose(O.moving_average_np(v, 6), 3.5)
