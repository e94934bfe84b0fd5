"""CInt one-electron pair integrals (pfock/one_electron.c:14-25 callers of
CInt_computePairOvl / CInt_computePairCoreH) through the C ABI against the
oracle fixtures, and the one-electron matrices' symmetry.

CInt_createOED evaluates S, T and V of the whole basis on the device once;
each pair call returns the (A, B) block column-major, as the reference's
OED buffers hold it.  Assembling every block must give the fixtures' S and
H = T + V within 1e-10, and Kin + Pot must equal CoreH exactly.
"""
import ctypes

import numpy as np
import pytest

from conftest import golden_cases, golden_xyz, load_golden

import gtfock_b200 as gb

pytestmark = pytest.mark.gpu

TOL = 1e-10
CASES = [c for c in golden_cases() if "S" in load_golden(c)]

_vp = ctypes.c_void_p
_dpp = ctypes.POINTER(ctypes.POINTER(ctypes.c_double))
_ip = ctypes.POINTER(ctypes.c_int)


def _lib():
    L = gb.load()
    L.CInt_createOED.argtypes = [_vp, ctypes.POINTER(_vp)]
    L.CInt_createOED.restype = ctypes.c_int
    L.CInt_destroyOED.argtypes = [_vp]
    L.CInt_destroyOED.restype = ctypes.c_int
    for n in ("CInt_computePairOvl", "CInt_computePairKin", "CInt_computePairPot", "CInt_computePairCoreH"):
        f = getattr(L, n)
        f.argtypes = [_vp, _vp, ctypes.c_int, ctypes.c_int, _dpp, _ip]
        f.restype = ctypes.c_int
    return L


def _assemble(L, fn, b, oed):
    ns = L.CInt_getNumShells(b.h)
    nbf = L.CInt_getNumFuncs(b.h)
    start = [L.CInt_getFuncStartInd(b.h, s) for s in range(ns)] + [nbf]
    M = np.full((nbf, nbf), np.nan)
    ptr = ctypes.POINTER(ctypes.c_double)()
    n = ctypes.c_int()
    for A in range(ns):
        for B in range(ns):
            assert fn(b.h, oed, A, B, ctypes.byref(ptr), ctypes.byref(n)) == 0
            nr, nc = start[A + 1] - start[A], start[B + 1] - start[B]
            assert n.value == nr * nc
            blk = np.ctypeslib.as_array(ptr, shape=(nr * nc,)).reshape(nc, nr).T
            M[start[A]:start[A + 1], start[B]:start[B + 1]] = blk
    return M


@pytest.mark.parametrize("case", CASES)
def test_pair_blocks_match_oracle(case, tmp_path):
    g = load_golden(case)
    gbs, xyz = golden_xyz(g, tmp_path)
    b = gb.BasisSet(gbs, xyz)
    L = _lib()
    oed = _vp()
    assert L.CInt_createOED(b.h, ctypes.byref(oed)) == 0
    try:
        S = _assemble(L, L.CInt_computePairOvl, b, oed)
        H = _assemble(L, L.CInt_computePairCoreH, b, oed)
        T = _assemble(L, L.CInt_computePairKin, b, oed)
        V = _assemble(L, L.CInt_computePairPot, b, oed)
        # a shell index out of range is an argument error
        ptr = ctypes.POINTER(ctypes.c_double)()
        n = ctypes.c_int()
        ns = L.CInt_getNumShells(b.h)
        assert L.CInt_computePairOvl(b.h, oed, ns, 0, ctypes.byref(ptr), ctypes.byref(n)) != 0
    finally:
        L.CInt_destroyOED(oed)
    assert np.isfinite(S).all() and np.isfinite(H).all()
    assert np.abs(S - g["S"]).max() < TOL
    assert np.abs(H - g["H"]).max() < TOL
    assert np.array_equal(T + V, H)
    # kinetic energy matrix is positive definite; the potential is negative
    assert np.linalg.eigvalsh(0.5 * (T + T.T)).min() > 0.0
    assert np.trace(V) < 0.0


@pytest.mark.parametrize("case", CASES)
def test_one_electron_matrices_symmetric(case, tmp_path):
    """Each unordered shell pair is evaluated once and written with its
    transpose, so S and H come out exactly symmetric (and X, their
    eigen-decomposition's product, to rounding)."""
    g = load_golden(case)
    gbs, xyz = golden_xyz(g, tmp_path)
    b = gb.BasisSet(gbs, xyz)
    pf = gb.PFock(b, tolscr=float(g["tol"]))
    S, X, H = pf.one_electron()
    pf.close()
    assert np.array_equal(S, S.T)
    assert np.array_equal(H, H.T)
    assert np.abs(X - X.T).max() < 1e-12
    assert np.abs(np.diag(S) - 1.0).max() < 1e-12   # normalised basis functions


@pytest.mark.parametrize("pure", [True, False])
def test_one_electron_d_shells_against_oracle(pure, tmp_path):
    """C2H6 / cc-pVDZ with spherical and with Cartesian d shells (5 or 6
    functions each; every class pair ss..dd present): S, H and X against the
    oracle's CPU restatement (pfock/one_electron.c:28-119)."""
    import os
    from gtfock_b200 import molecules as mol
    from oracle import pyoracle as po
    text = open(mol.basis_file("cc-pvdz")).read()
    gbs = os.path.join(str(tmp_path), "cc-pvdz.gbs")
    with open(gbs, "w") as f:
        f.write(text if pure else text.replace("spherical", "cartesian", 1))
    xyz = mol.write_xyz(mol.alkane(2), os.path.join(str(tmp_path), "c2h6.xyz"))
    b = gb.BasisSet(gbs, xyz)
    assert b.nbf == (2 * 14 + 6 * 5 if pure else 2 * 15 + 6 * 5)
    pf = gb.PFock(b, tolscr=1e-10)
    S, X, H = pf.one_electron()
    pf.close()
    So, Ho, Xo = po.one_electron(po.Basis(gbs, xyz))
    assert np.abs(S - So).max() < TOL
    assert np.abs(H - Ho).max() < TOL
    assert np.abs(X - Xo).max() < 1e-9
