"""CPU checks of the oracle (oracle/): known answers, integral identities, and
the pin of the restatement to the reference's own compiled sources."""
import math
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, golden_cases, golden_xyz, load_golden
from oracle import pyoracle as po

BOHR = 0.529177210903


def _crawford_h2o(tmp_path):
    from gtfock_b200 import molecules as mol
    g = [("O", 0.0, -0.143225816552, 0.0), ("H", 1.638036840407, 1.136548822547, 0.0),
         ("H", -1.638036840407, 1.136548822547, 0.0)]
    atoms = [(s, x * BOHR, y * BOHR, z * BOHR) for s, x, y, z in g]
    return mol.write_xyz(atoms, str(tmp_path / "h2o.xyz"))


def test_known_answer_h2o_sto3g(tmp_path):
    """RHF/STO-3G water at the geometry of the Crawford-group SCF programming
    project: E_nuc = 8.002367061810450, E_SCF = -74.942079928192 Hartree."""
    from gtfock_b200 import molecules as mol
    b = po.Basis(mol.basis_file("sto-3g"), _crawford_h2o(tmp_path))
    assert abs(b.enuc - 8.002367061810450) < 1e-10
    e, _, _ = po.scf(b, 1e-11, 30)
    assert abs(e[-1] - (-74.942079928192)) < 1e-9


def test_ss_closed_form(tmp_path):
    """(ss|ss) of two contracted s shells against the closed form
    2 pi^(5/2) / (p q sqrt(p+q)) K_ab K_cd F0(T)."""
    from gtfock_b200 import molecules as mol
    xyz = mol.write_xyz([("H", 0.0, 0.0, 0.0), ("H", 0.0, 0.0, 0.74)], str(tmp_path / "h2.xyz"))
    b = po.Basis(mol.basis_file("sto-3g"), xyz)
    ints = po.shell_quartet(b, 0, 1, 1, 0)
    # STO-3G H exponents / coefficients (primitive-normalised here)
    al = np.array([3.42525091, 0.62391373, 0.16885540])
    d = np.array([0.15432897, 0.53532814, 0.44463454])
    c = d * (2 * al / math.pi) ** 0.75
    s = sum(c[i] * c[j] * (math.pi / (al[i] + al[j])) ** 1.5 for i in range(3) for j in range(3))
    c = c / math.sqrt(s)
    A = np.zeros(3)
    B = np.array([0.0, 0.0, 0.74 / BOHR])

    def F0(T):
        return 1.0 if T < 1e-14 else 0.5 * math.sqrt(math.pi / T) * math.erf(math.sqrt(T))
    centres = [A, B, B, A]
    total = 0.0
    for i in range(3):
        for j in range(3):
            for k in range(3):
                for l in range(3):
                    a, bb, cc, dd = al[i], al[j], al[k], al[l]
                    p, q = a + bb, cc + dd
                    P = (a * centres[0] + bb * centres[1]) / p
                    Q = (cc * centres[2] + dd * centres[3]) / q
                    Kab = math.exp(-a * bb / p * np.sum((centres[0] - centres[1]) ** 2))
                    Kcd = math.exp(-cc * dd / q * np.sum((centres[2] - centres[3]) ** 2))
                    T = p * q / (p + q) * np.sum((P - Q) ** 2)
                    total += c[i] * c[j] * c[k] * c[l] * 2 * math.pi ** 2.5 / (p * q * math.sqrt(p + q)) \
                        * Kab * Kcd * F0(T)
    assert abs(ints[0, 0, 0, 0] - total) < 1e-13


def test_eri_permutational_symmetry_and_schwarz(tmp_path):
    g = load_golden("c4h10_ccpvdz")
    gbs, xyz = golden_xyz(g, tmp_path)
    b = po.Basis(gbs, xyz)
    rng = np.random.default_rng(3)
    for _ in range(25):
        A, B, C, D = (int(x) for x in rng.integers(0, b.nshells, 4))
        I = po.shell_quartet(b, A, B, C, D)
        assert np.allclose(I, po.shell_quartet(b, B, A, C, D).transpose(1, 0, 2, 3), atol=1e-14)
        assert np.allclose(I, po.shell_quartet(b, C, D, A, B).transpose(2, 3, 0, 1), atol=1e-14)
        assert np.allclose(I, po.shell_quartet(b, A, B, D, C).transpose(0, 1, 3, 2), atol=1e-14)
        ab = po.shell_quartet(b, A, B, A, B)
        cd = po.shell_quartet(b, C, D, C, D)
        dab = np.einsum("ijij->ij", ab)
        dcd = np.einsum("ijij->ij", cd)
        bound = np.sqrt(np.abs(dab)[:, :, None, None] * np.abs(dcd)[None, None, :, :])
        assert np.all(np.abs(I) <= bound * (1 + 1e-12) + 1e-15)


def test_rotation_invariance_ccpvdz(tmp_path):
    """The SCF energy with spherical d functions is invariant under a rigid
    rotation of the molecule (checks the d normalisation and transform)."""
    from gtfock_b200 import molecules as mol
    atoms = mol.alkane(1)
    th = 0.7
    R = np.array([[math.cos(th), -math.sin(th), 0], [math.sin(th), math.cos(th), 0], [0, 0, 1]])
    R = R @ np.array([[1, 0, 0], [0, math.cos(1.1), -math.sin(1.1)], [0, math.sin(1.1), math.cos(1.1)]])
    rot = [(s,) + tuple(R @ np.array([x, y, z]) + np.array([0.3, -1.2, 2.0])) for s, x, y, z in atoms]
    e1 = po.scf(po.Basis(mol.basis_file("cc-pvdz"), mol.write_xyz(atoms, str(tmp_path / "a.xyz"))),
                1e-12, 15)[0][-1]
    e2 = po.scf(po.Basis(mol.basis_file("cc-pvdz"), mol.write_xyz(rot, str(tmp_path / "b.xyz"))),
                1e-12, 15)[0][-1]
    assert abs(e1 - e2) < 1e-9


@pytest.mark.parametrize("case", [c for c in golden_cases() if c != "c12h26_ccpvdz"])
def test_oracle_reproduces_golden(case, tmp_path):
    """The oracle regenerates its own fixture: identical screening lists and
    counters, F to 1e-12."""
    g = load_golden(case)
    gbs, xyz = golden_xyz(g, tmp_path)
    b = po.Basis(gbs, xyz)
    tol = float(g["tol"])
    scr = po.screening(b, tol)
    assert np.array_equal(scr[0], g["shellptr"])
    assert np.array_equal(scr[1], g["shellid"])
    assert np.array_equal(scr[2], g["shellrid"])
    assert np.array_equal(scr[3], g["shellvalue"])
    F, usq, uitl = po.fock_build(b, tol, g["D"], scr=scr)
    assert usq == float(g["usq"]) and uitl == float(g["uitl"])
    assert np.abs(F - g["F"]).max() < 1e-12


def test_fixtures_pinned_to_reference_build():
    """Every committed fixture was cross-checked, when it was generated,
    against the reference's own pfock sources compiled by oracle/ref/Makefile."""
    for case in golden_cases():
        g = load_golden(case)
        assert int(g["ref_pinned"]) == 1, case
        assert float(g["ref_max_dF"]) < 1e-11, case


def test_large_fixtures_pinned_to_reference_build():
    """The benchmark-size fixtures (C54H18, (H2O)64, C96H24) carry the
    reference build's F for the same density and lists (tests/golden/make_large.py)."""
    d = os.path.join(GOLDEN, "large")
    names = sorted(f[:-4] for f in os.listdir(d) if f.endswith(".npz"))
    assert names == ["c54h18_ccpvdz", "c96h24_ccpvdz", "w64_631g"]
    for n in names:
        g = np.load(os.path.join(d, n + ".npz"))
        assert int(g["ref_pinned"]) == 1, n
        assert float(g["ref_max_dF"]) < 1e-11, n


REF_PROBE = os.path.join(ROOT, "oracle", "_ref", "ref_probe")


@pytest.mark.skipif(not os.path.exists(REF_PROBE), reason="reference sources not compiled here")
def test_restatement_matches_reference_build(tmp_path):
    """oracle/fock_oracle.c against the reference's pfock/*.c on the same
    engine: bit-identical screening list and counters, F to 1e-12."""
    import sys
    sys.path.insert(0, GOLDEN)
    import make_golden
    g = load_golden("w8_631g")
    gbs, xyz = golden_xyz(g, tmp_path)
    b = po.Basis(gbs, xyz)
    D = make_golden.test_density(b.nbf, seed=11)
    ref = make_golden.ref_probe(gbs, xyz, float(g["tol"]), D)
    scr = po.screening(b, float(g["tol"]))
    F, usq, uitl = po.fock_build(b, float(g["tol"]), D, scr=scr)
    assert np.array_equal(ref["shellptr"], scr[0])
    assert np.array_equal(ref["shellid"], scr[1])
    assert np.array_equal(ref["shellvalue"], scr[3])
    assert ref["usq"] == usq and ref["uitl"] == uitl
    assert np.abs(ref["F"] - F).max() < 1e-12


def test_nosymm_fixtures_pinned():
    """The non-symmetric fixtures: the exact formula reproduced the symmetric
    fixture (reference-pinned) when they were generated, and the oracle's
    restatement of the reference's symm = 0 digestion equals the reference
    build's own output."""
    d = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "nosymm")
    for f in sorted(os.listdir(d)):
        z = np.load(os.path.join(d, f))
        n = z["D_ns"].shape[0]
        assert np.abs(z["D_ns"] - z["D_ns"].T).max() > 1e-3
        assert z["F_ns_ref"].shape == (n, n)
        if "F_ns" in z:
            assert float(z["sym_check"]) < 1e-9
            assert z["F_ns"].shape == (n, n)
            assert np.abs(z["F_ns_port"] - z["F_ns_ref"]).max() < 1e-12
            # the reference's symm = 0 result is not 2 J[D] - K[D]
            assert np.abs(z["F_ns"] - z["F_ns_ref"]).max() > 1e-2


def test_nosymm_restatement_live(tmp_path):
    """pyoracle.fock_nosymm_reference, run now, against the reference build's
    symm = 0 output stored in the fixture (H2O / 6-31G)."""
    g = load_golden("h2o_631g")
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "nosymm", "h2o_631g.npz"))
    gbs, xyz = golden_xyz(g, tmp_path)
    b = po.Basis(gbs, xyz)
    F = po.fock_nosymm_reference(b, float(g["tol"]), po.eri_tensor(b), z["D_ns"])
    assert np.abs(F - z["F_ns_ref"]).max() < 1e-12


def test_rys_table_accuracy():
    """The FP64 Rys table of the CUDA kernels (csrc/cuda/rys_table.h) against
    the 60-digit Gauss rule recomputed by its generator, at a few T per root
    count (both ends of the interval range, interior points, interval
    midpoints and edges)."""
    import re
    from gtfock_b200 import gen_rys_table as G
    hdr = open(os.path.join(ROOT, "gtfock_b200", "csrc", "cuda", "rys_table.h")).read()
    hl = [float(x) for x in re.search(r"#define RYS_H_LIST (.*)", hdr).group(1).split(",")]
    dl = [int(x) for x in re.search(r"#define RYS_DEG_LIST (.*)", hdr).group(1).split(",")]
    offs = [int(x) for x in re.search(r"#define RYS_OFF_LIST (.*)", hdr).group(1).split(",")]
    body = hdr[hdr.index("RYS_TABLE[RYS_TABLE_LEN] = {") + 28:]
    body = body[:body.index("};")]
    tab = np.array([float(x) for x in body.replace("\n", " ").split(",") if x.strip()])
    worst = 0.0
    for n in range(1, 6):
        h, deg = hl[n], dl[n]
        for T in (0.0, 0.3 * h, 2.6, 11.0 + 0.5 * h, 23.7, G.TMAX[n] - 1e-3):
            k = int(T / h)
            s = T - (k * h + 0.5 * h)
            c = tab[offs[n] + k * (deg + 1) * 2 * n:][:(deg + 1) * 2 * n].reshape(deg + 1, 2 * n)
            vals = np.polynomial.polynomial.polyval(s, c)   # c[j][f]: coefficient j of function f
            u, w = G.gauss_rule(T, n)
            ref = np.array([float(x) for x in list(u) + list(w)])
            worst = max(worst, float(np.max(np.abs(vals - ref) / np.abs(ref))))
    assert worst < 2e-15, worst
