"""Mixed precision: quartets whose Schwarz bound sqrt(v1 v2) falls below a
cutoff are evaluated in FP32 (Rys roots, 2-D integrals, primitive sum), the
rest in FP64; D, the J/K digestion and every accumulation into F stay FP64.

Checked through the C ABI against the FP64 oracle fixtures:
  * cutoff 0 sends no quartet to FP32 and reproduces the FP64 F (1e-10 Ha);
  * a cutoff above every bound sends all of them, and F stays within FP32
    rounding of the oracle (a wrong FP32 kernel would be off by O(1));
  * over the cutoff sweep 1e-4 .. 1e-8 the FP32 share shrinks monotonically
    and max|dF| stays below the cutoff itself (each FP32 integral is below
    the cutoff in magnitude and carries a relative error near 1e-7);
  * the SCF energy with cutoff 1e-6 is within 1e-6 Ha of the FP64 energy.
"""
import numpy as np
import pytest

from conftest import golden_xyz, load_golden

import gtfock_b200 as gb

pytestmark = pytest.mark.gpu

F_TOL = 1e-10
CUTOFFS = [1e-4, 1e-5, 1e-6, 1e-7, 1e-8]


def _engine(case, tmp_path):
    g = load_golden(case)
    gbs, xyz = golden_xyz(g, tmp_path)
    b = gb.BasisSet(gbs, xyz)
    pf = gb.PFock(b, tolscr=float(g["tol"]))
    return g, b, pf


@pytest.mark.parametrize("case", ["w8_631g", "c4h10_ccpvdz"])
def test_zero_cutoff_is_fp64(case, tmp_path):
    g, b, pf = _engine(case, tmp_path)
    pf.set_precision(1, 0.0)
    nq32, nq = pf.precision_stats()
    assert nq32 == 0 and nq == float(g["usq"])
    err = np.abs(pf.compute_fock(g["D"]) - g["F"]).max()
    assert err < F_TOL, err
    pf.close()


@pytest.mark.parametrize("case", ["w8_631g", "c4h10_ccpvdz"])
def test_all_fp32(case, tmp_path):
    g, b, pf = _engine(case, tmp_path)
    pf.set_precision(1, 1e30)
    nq32, nq = pf.precision_stats()
    assert nq32 == nq == float(g["usq"])
    err = np.abs(pf.compute_fock(g["D"]) - g["F"]).max()
    assert 1e-12 < err < 2e-3, err
    # back to FP64: the task lists are rebuilt and F is exact again
    pf.set_precision(0, 0.0)
    assert pf.precision_stats()[0] == 0
    err = np.abs(pf.compute_fock(g["D"]) - g["F"]).max()
    assert err < F_TOL, err
    pf.close()


@pytest.mark.parametrize("case", ["w8_631g", "c4h10_ccpvdz"])
def test_cutoff_sweep(case, tmp_path):
    g, b, pf = _engine(case, tmp_path)
    prev = None
    for cut in CUTOFFS:
        pf.set_precision(1, cut)
        nq32, nq = pf.precision_stats()
        assert 0 < nq32 < nq
        if prev is not None:
            assert nq32 <= prev
        prev = nq32
        err = np.abs(pf.compute_fock(g["D"]) - g["F"]).max()
        print("%s cutoff %.0e: FP32 share %.3f, max|dF| %.3e" % (case, cut, nq32 / nq, err))
        assert err < cut, (cut, err)
    pf.close()


def test_scf_energy_mixed(tmp_path):
    g = load_golden("w8_631g")
    gbs, xyz = golden_xyz(g, tmp_path)
    s = gb.SCFSolver(gbs, xyz, tolscr=float(g["tol"]))
    n = len(g["energies"])
    e64, _ = s.solve(niters=n)
    assert abs(e64[-1] - g["energies"][-1]) < 1e-9
    # both runs to convergence, then compare the converged energies
    s.set_options(precision=0, etol=1e-9)
    e64, _ = s.solve(niters=40)
    s.set_options(precision=1, fp32_cutoff=1e-6, etol=1e-9)
    e32, _ = s.solve(niters=40)
    assert len(e64) < 40 and len(e32) < 40
    print("FP64 %.10f (%d it)  mixed 1e-6 %.10f (%d it)" % (e64[-1], len(e64), e32[-1], len(e32)))
    assert abs(e32[-1] - e64[-1]) < 1e-6, (e32[-1], e64[-1])
    s.close()


@pytest.mark.parametrize("case", ["w8_631g", "c4h10_ccpvdz"])
def test_bf16_split_purification(case, tmp_path):
    """Purification with split-BF16 tensor-core products followed by FP64
    steps: the converged SCF energy within 1e-6 Ha of the FP64 purification,
    with both precisions of the ERIs, and an idempotent final density."""
    g = load_golden(case)
    gbs, xyz = golden_xyz(g, tmp_path)
    s = gb.SCFSolver(gbs, xyz, tolscr=float(g["tol"]))
    s.set_options(precision=0, etol=1e-9)
    e64, _ = s.solve(niters=40)
    s.set_purification(1)
    e16, _ = s.solve(niters=40)
    nb, n64 = s.purification_iters()
    assert nb > 0 and n64 > 0
    assert len(e64) < 40 and len(e16) < 40
    assert abs(e16[-1] - e64[-1]) < 1e-6, (e16[-1], e64[-1])
    s.set_options(precision=1, fp32_cutoff=1e-6, etol=1e-9)
    em, _ = s.solve(niters=40)
    assert abs(em[-1] - e64[-1]) < 1e-6, (em[-1], e64[-1])
    b = gb.BasisSet(gbs, xyz)
    pf = gb.PFock(b, tolscr=float(g["tol"]))
    S, _, _ = pf.one_electron()
    D = s.density()
    assert np.linalg.norm(D @ S @ D - D) < 1e-8
    assert abs(np.trace(D @ S) - b.nocc) < 1e-8
    print("%s: FP64 %.10f, bf16-split purification %.10f (%d bf16 + %d fp64 steps)" %
          (case, e64[-1], e16[-1], nb, n64))
    pf.close()
    s.close()
