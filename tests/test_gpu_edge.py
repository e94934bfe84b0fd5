"""Edge cases of the CUDA Fock path against the live oracle (small sizes),
and size-independent properties at the largest size of the benchmarks.

* one atom (every shell pair on one centre: A - B = 0, all HRR shifts zero);
* H2 / STO-3G: s shells only, a single class pair;
* two fragments 60 A apart: most shell pairs and whole ket ranges screened;
* an indefinite density with large elements (signs the SCF never produces);
* C96H24 / cc-pVDZ (1464 functions): F symmetric, linear in D, the shard
  parts summing to the whole build, FP32 quartets within their cutoff."""
import numpy as np
import pytest

from conftest import golden_xyz, load_golden

import gtfock_b200 as gb
from gtfock_b200 import molecules as mol
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

F_TOL = 1e-10


def _sym(n, seed, scale=0.1):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n)) * scale
    return A + A.T


def _compare(atoms, basis, tmp_path, D=None, tol=1e-10, seed=0):
    """Screening lists and counters bit-exact, then max |F - F_oracle|."""
    gbs = mol.basis_file(basis)
    xyz = mol.write_xyz(atoms, str(tmp_path / "m.xyz"))
    b = gb.BasisSet(gbs, xyz)
    pf = gb.PFock(b, tolscr=tol)
    ob = po.Basis(gbs, xyz)
    if D is None:
        D = _sym(b.nbf, seed)
    scr = po.screening(ob, tol)
    sp, si, sr, sv, mx = pf.screening()
    assert np.array_equal(sp, scr[0]) and np.array_equal(si, scr[1]) and np.array_equal(sr, scr[2])
    F_ref, usq, uitl = po.fock_build(ob, tol, D, scr=scr)
    c = pf.counts()
    assert c["usq"] == usq and c["uitl"] == uitl
    F = pf.compute_fock(D)
    err = np.abs(F - F_ref).max()
    pf.close()
    return err, usq


def test_single_atom(tmp_path):
    err, usq = _compare([("O", 0.0, 0.0, 0.0)], "cc-pvdz", tmp_path, seed=1)
    assert usq > 0 and err < F_TOL, err


def test_h2_s_shells_only(tmp_path):
    err, usq = _compare([("H", 0.0, 0.0, 0.0), ("H", 0.0, 0.0, 0.74)], "sto-3g", tmp_path, seed=2)
    assert usq > 0 and err < F_TOL, err


def test_far_fragments(tmp_path):
    w = mol.water_cluster(1, 3)
    far = [(s, x + 60.0, y, z) for s, x, y, z in w]
    err, usq = _compare(w + far, "6-31g", tmp_path, seed=3)
    assert err < F_TOL, err
    # each fragment's own quartets plus the cross-fragment Coulomb quartets
    # (aa|bb), whose Schwarz bounds do not decay with the distance
    err1, usq1 = _compare(w, "6-31g", tmp_path, seed=3)
    assert 2 * usq1 <= usq


def test_indefinite_density(tmp_path):
    atoms = mol.alkane(2)
    gbs = mol.basis_file("cc-pvdz")
    xyz = mol.write_xyz(atoms, str(tmp_path / "e.xyz"))
    n = gb.BasisSet(gbs, xyz).nbf
    D = _sym(n, 4, scale=3.0)
    err, _ = _compare(atoms, "cc-pvdz", tmp_path, D=D)
    assert err < F_TOL * 30, err   # |D| ~ 10 here: the bar scales with the density


def test_largest_size_properties(tmp_path):
    xyz = mol.write_xyz(mol.graphene_flake(3), str(tmp_path / "c96h24.xyz"))
    b = gb.BasisSet(mol.basis_file("cc-pvdz"), xyz)
    assert b.nbf == 1464
    pf = gb.PFock(b, tolscr=1e-10)
    D1 = _sym(b.nbf, 5, scale=0.02)
    D2 = np.eye(b.nbf) * 0.3
    F1 = pf.compute_fock(D1)
    F2 = pf.compute_fock(D2)
    F12 = pf.compute_fock(D1 + 2.0 * D2)
    scale = np.abs(F12).max()
    assert np.abs(F1 - F1.T).max() < 1e-13 * max(1.0, np.abs(F1).max())
    assert np.abs(F12 - (F1 + 2.0 * F2)).max() < 1e-12 * scale
    parts = []
    for r in range(3):
        pf.set_shard(r, 3)
        parts.append(pf.compute_fock(D2))
    pf.set_shard(0, 1)
    assert np.abs(sum(parts) - F2).max() < 1e-12 * np.abs(F2).max()
    pf.set_precision(1, 1e-6)
    F2m = pf.compute_fock(D2)
    nq32, nq = pf.precision_stats()
    assert nq32 > 0.3 * nq
    # FP32 quartets have Schwarz bounds below 1e-6; their rounding moves F
    # by far less than 1e-6 per element
    assert np.abs(F2m - F2).max() < 1e-6
    pf.close()


def test_primitive_quartets_after_screening(tmp_path):
    """The count of primitive quartets the kernels evaluate (after the
    |K_ab K_cd| < 1e-17 cut) is at most the model's count before it, for
    every class, and smaller in total on C12H26 / cc-pVDZ, whose contracted
    s shells have tight, small-coefficient primitives; for water / STO-3G
    the (ss|ss) count is the product of the pairs' primitive counts less
    the few cut quartets."""
    g = load_golden("h2o_sto3g")
    gbs, xyz = golden_xyz(g, tmp_path)
    pf = gb.PFock(gb.BasisSet(gbs, xyz), tolscr=1e-10)
    before = pf.class_work()
    after = pf.class_work_screened()
    for (fb, qb), (fa, qa) in zip(before, after):
        assert 0.5 * qb <= qa <= qb
    pf.close()
    g = load_golden("c12h26_ccpvdz")
    gbs, xyz = golden_xyz(g, tmp_path)
    pf = gb.PFock(gb.BasisSet(gbs, xyz), tolscr=1e-10)
    before = pf.class_work()
    after = pf.class_work_screened()
    for (fb, qb), (fa, qa) in zip(before, after):
        assert 0 <= qa <= qb and fa <= fb * (1 + 1e-12)
    assert sum(q for _, q in after) < sum(q for _, q in before)
    assert sum(q for _, q in after) > 0.1 * sum(q for _, q in before)
    pf.close()


def test_short_stride_rejected(tmp_path):
    """A row stride shorter than the block (the rows would overlap) is an
    argument error in PFock_getMat and PFock_putDenMat, before any copy."""
    import ctypes
    L = gb.load()
    g = load_golden("h2o_631g")
    gbs, xyz = golden_xyz(g, tmp_path)
    b = gb.BasisSet(gbs, xyz)
    pf = gb.PFock(b, tolscr=1e-10)
    n = b.nbf
    buf = np.zeros((n, n))
    ptr = buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    INVALID = 3
    assert L.PFock_getMat(pf.h, gb.MAT_F, 0, 0, n - 1, 0, n - 1, n - 1, ptr) == INVALID
    assert L.PFock_getMat(pf.h, gb.MAT_F, 0, 0, n - 1, 2, 5, 3, ptr) == INVALID
    assert L.PFock_getMat(pf.h, gb.MAT_F, 0, 0, n - 1, 2, 5, 4, ptr) == 0
    assert L.PFock_putDenMat(0, n - 1, 0, n - 1, n - 1, ptr, 0, pf.h) == INVALID
    F = pf.compute_fock(g["D"])
    assert np.abs(F - g["F"]).max() < 1e-10
    pf.close()
