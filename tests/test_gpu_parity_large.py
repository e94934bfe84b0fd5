"""GPU parity at the benchmark sizes: C54H18 / cc-pVDZ (846 functions),
(H2O)64 / 6-31G (832) and C96H24 / cc-pVDZ (1464), through the C-ABI.

Each fixture (tests/golden/large/, made by tests/golden/make_large.py from
the CPU oracle and, where marked ref_pinned, checked against the reference's
own pfock sources compiled here) holds the screening list, the quartet
counters and F for a seeded density.  Bars, as for the small fixtures: the
CSR pair list and usq / uitl bit-exact (pfock/screening.c:15-180,
pfock/fock_task.c:121-219), F elementwise within 1e-10 Ha."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_xyz, large_density, unpack_upper

import gtfock_b200 as gb

pytestmark = pytest.mark.gpu

F_TOL = 1e-10
LARGE = os.path.join(GOLDEN, "large")
CASES = sorted(f[:-4] for f in os.listdir(LARGE) if f.endswith(".npz")) if os.path.isdir(LARGE) else []


def _load(case):
    return dict(np.load(os.path.join(LARGE, case + ".npz"), allow_pickle=False))


def test_fixtures_present():
    assert {"c54h18_ccpvdz", "w64_631g"} <= set(CASES), CASES


@pytest.fixture(scope="module", params=CASES)
def built(request, tmp_path_factory):
    """One engine per case and one FP64 build of the fixture's density."""
    case = request.param
    g = _load(case)
    gbs, xyz = golden_xyz(g, tmp_path_factory.mktemp(case))
    b = gb.BasisSet(gbs, xyz)
    assert b.nbf == int(g["nbf"])
    pf = gb.PFock(b, tolscr=float(g["tol"]))
    D = large_density(b.nbf, int(g["density_seed"]))
    F = pf.compute_fock(D)
    yield case, g, pf, D, F
    pf.close()


def test_screening_bitexact(built):
    case, g, pf, _, _ = built
    sp, si, sr, sv, mx = pf.screening()
    assert np.array_equal(sp, g["shellptr"]), case
    assert np.array_equal(si, g["shellid"]), case
    assert np.array_equal(sr, g["shellrid"]), case
    assert np.array_equal(np.sign(sv), np.sign(g["shellvalue"])), case
    assert np.allclose(sv, g["shellvalue"], rtol=1e-11, atol=0), case
    assert abs(mx - float(g["maxvalue"])) <= 1e-11 * abs(float(g["maxvalue"]))


def test_quartet_counts_exact(built):
    case, g, pf, _, _ = built
    c = pf.counts()
    assert c["usq"] == float(g["usq"]), (case, c["usq"], float(g["usq"]))
    assert c["uitl"] == float(g["uitl"]), (case, c["uitl"], float(g["uitl"]))


def test_fock_matches_oracle(built):
    case, g, pf, D, F = built
    n = int(g["nbf"])
    F_ref = unpack_upper(g["F_upper"], n)
    err = float(np.abs(F - F_ref).max())
    assert err < F_TOL, "%s: max|dF| = %.3e" % (case, err)
    assert np.abs(F - F.T).max() < 1e-12


def test_fock_repeatable_and_linear(built):
    """A second build of the same density agrees to the atomics' rounding, and
    F[2D] = 2 F[D] (the build is linear in D)."""
    case, g, pf, D, F = built
    F2 = pf.compute_fock(2.0 * D)
    assert np.abs(F2 - 2.0 * F).max() < 2 * F_TOL, case
