"""Non-symmetric densities (PFock_create with symm = 0), through the C ABI.

By default the engine returns the reference's own symm = 0 result
(pfock/pfock.c:1704-1718): (F[D] + F[D^T]^T) / 2 of its unique-quartet
digestion, which for a non-symmetric D depends on the orientation of the
shell-pair lists.  Mode "exact" returns F = 2 J[D] - K[D].  Fixtures
(tests/golden/nosymm/, made by tests/golden/make_nosymm.py) hold a seeded
non-symmetric D, the reference build's output for it (F_ns_ref) and, for the
cases small enough for the oracle's full ERI tensor, the exact F (F_ns) and
the oracle's restatement of the reference's digestion (F_ns_port).
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_xyz, load_golden

import gtfock_b200 as gb

pytestmark = pytest.mark.gpu

F_TOL = 1e-10
CASES = ["h2o_631g", "h2o_ccpvdz", "ch4_ccpvdz", "c4h10_ccpvdz"]


def _ns(case):
    return dict(np.load(os.path.join(GOLDEN, "nosymm", case + ".npz")))


@pytest.mark.parametrize("case", CASES)
def test_nosymm_matches_reference(case, tmp_path):
    g = load_golden(case)
    ns = _ns(case)
    gbs, xyz = golden_xyz(g, tmp_path)
    b = gb.BasisSet(gbs, xyz)
    pf = gb.PFock(b, tolscr=float(g["tol"]), symm=0)
    F = pf.compute_fock(ns["D_ns"])
    assert np.abs(F - ns["F_ns_ref"]).max() < F_TOL
    if "F_ns_port" in ns:
        assert np.abs(F - ns["F_ns_port"]).max() < F_TOL
    assert np.abs(F - F.T).max() > 1e-3          # the result is not symmetric
    # a symmetric D gives the symm = 1 result
    F2 = pf.compute_fock(g["D"])
    assert np.abs(F2 - g["F"]).max() < F_TOL
    pf.close()


@pytest.mark.parametrize("case", [c for c in CASES if c != "c4h10_ccpvdz"])
def test_nosymm_exact(case, tmp_path):
    g = load_golden(case)
    ns = _ns(case)
    gbs, xyz = golden_xyz(g, tmp_path)
    b = gb.BasisSet(gbs, xyz)
    pf = gb.PFock(b, tolscr=float(g["tol"]), symm=0)
    pf.set_nosymm_mode("exact")
    F = pf.compute_fock(ns["D_ns"])
    assert np.abs(F - ns["F_ns"]).max() < F_TOL
    F2 = pf.compute_fock(g["D"])
    assert np.abs(F2 - g["F"]).max() < F_TOL
    # and back to the reference's result on the same engine
    pf.set_nosymm_mode("reference")
    F3 = pf.compute_fock(ns["D_ns"])
    assert np.abs(F3 - ns["F_ns_ref"]).max() < F_TOL
    pf.close()


def test_nosymm_mode_needs_symm0(tmp_path):
    g = load_golden("h2o_631g")
    gbs, xyz = golden_xyz(g, tmp_path)
    b = gb.BasisSet(gbs, xyz)
    pf = gb.PFock(b, tolscr=float(g["tol"]), symm=1)
    with pytest.raises(gb.GtfError):
        pf.set_nosymm_mode("exact")
    pf.close()


@pytest.mark.parametrize("symm", [1, 0])
def test_two_density_matrices(symm, tmp_path):
    """max_numdmat = 2 (pfock/pfock.c:1039-1055): one computeFock builds F
    for both densities, each read back by its index."""
    case = "h2o_ccpvdz"
    g = load_golden(case)
    ns = _ns(case)
    gbs, xyz = golden_xyz(g, tmp_path)
    b = gb.BasisSet(gbs, xyz)
    pf = gb.PFock(b, tolscr=float(g["tol"]), max_numdmat=2, symm=symm)
    D1, F1 = (ns["D_ns"], ns["F_ns_ref"]) if symm == 0 else (2.0 * g["D"], 2.0 * g["F"])
    pf.put_density(g["D"], 0)
    pf.put_density(D1, 1)
    pf.commit()
    pf.compute()
    assert np.abs(pf.get_mat(gb.MAT_F, 0) - g["F"]).max() < F_TOL
    assert np.abs(pf.get_mat(gb.MAT_F, 1) - F1).max() < 2 * F_TOL
    pf.close()
