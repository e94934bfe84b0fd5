"""Non-symmetric densities (PFock_create with symm = 0), through the C ABI.

The engine forms F = 2 J[D] - K[D] exactly for a general D (symmetric part
through the usual build, antisymmetric part through the exchange terms only).
Fixtures (tests/golden/nosymm/, made by tests/golden/make_nosymm.py) hold a
seeded non-symmetric D and that F from the oracle's full ERI tensor; the
formula itself reproduces the reference's symmetric-density F to 1e-14.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_xyz, load_golden

import gtfock_b200 as gb

pytestmark = pytest.mark.gpu

F_TOL = 1e-10
CASES = ["h2o_631g", "h2o_ccpvdz"]


def _ns(case):
    return dict(np.load(os.path.join(GOLDEN, "nosymm", case + ".npz")))


@pytest.mark.parametrize("case", CASES)
def test_nosymm_matches_exact(case, tmp_path):
    g = load_golden(case)
    ns = _ns(case)
    gbs, xyz = golden_xyz(g, tmp_path)
    b = gb.BasisSet(gbs, xyz)
    pf = gb.PFock(b, tolscr=float(g["tol"]), symm=0)
    F = pf.compute_fock(ns["D_ns"])
    assert np.abs(F - ns["F_ns"]).max() < F_TOL
    assert np.abs(F - F.T).max() > 1e-3          # the result is not symmetric
    # a symmetric D gives the symm = 1 result
    F2 = pf.compute_fock(g["D"])
    assert np.abs(F2 - g["F"]).max() < F_TOL
    pf.close()
