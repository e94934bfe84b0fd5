"""compute_diis (pscf/purif.c:491-641) through the C ABI against the oracle's
restatement, step by step.

The library keeps the DIIS bookkeeping on the device (slot of each
iteration, bordered matrix, Gauss-Jordan solve); the oracle keeps it on the
host and inverts the bordered matrix with LAPACK, as the reference does.
Each case feeds both the same seeded sequence of (D, F) pairs for 14
iterations, so the history fills its 10 slots and then replaces the
largest-error vector.
"""
import numpy as np
import pytest

from conftest import golden_xyz, load_golden

import gtfock_b200 as gb
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def _sequence(g, steps, seed):
    rng = np.random.default_rng(seed)
    n = int(g["nbf"])
    out = []
    for k in range(steps):
        a = 0.05 * 0.7 ** k
        dD = rng.standard_normal((n, n)) * a
        dF = rng.standard_normal((n, n)) * a
        out.append((g["D"] + 0.5 * (dD + dD.T), g["F"] + 0.5 * (dF + dF.T)))
    return out


@pytest.mark.parametrize("case", ["h2o_ccpvdz", "w8_631g"])
def test_diis_matches_oracle(case, tmp_path):
    g = load_golden(case)
    gbs, xyz = golden_xyz(g, tmp_path)
    b = gb.BasisSet(gbs, xyz)
    pr = gb.Purif(b)
    pr.set_sx(g["S"], g["X"])
    state = None
    for it, (D, F) in enumerate(_sequence(g, 14, 5)):
        Fg = pr.diis(None, D, F, it)
        Fo, _, state = po.diis_step_timed(g["X"], g["S"], D, F, it, state)
        assert np.isfinite(Fg).all()
        assert np.abs(Fg - Fo).max() < 1e-9 * max(1.0, np.abs(Fo).max()), (case, it)
    pr.close()


def test_diis_singular_system_keeps_f(tmp_path):
    """Two identical error vectors make the bordered matrix singular (the
    reference's LAPACK inverse would give non-finite coefficients): the step
    keeps this iteration's F, transformed (X F X^T), unextrapolated."""
    g = load_golden("h2o_ccpvdz")
    gbs, xyz = golden_xyz(g, tmp_path)
    b = gb.BasisSet(gbs, xyz)
    pr = gb.Purif(b)
    pr.set_sx(g["S"], g["X"])
    seq = _sequence(g, 2, 9)
    for it, (D, F) in enumerate(seq):
        pr.diis(None, D, F, it)
    D, F = seq[1]
    X = g["X"]
    pr.diis(None, D, F, 2)            # first stored error vector
    out = pr.diis(None, D, F, 3)      # the same one again: singular system
    assert np.isfinite(out).all()
    assert np.abs(out - X @ F.T @ X.T).max() < 1e-10
    pr.close()
