"""Generate the golden fixtures under tests/golden/ from the CPU oracle.

For each case (molecule + basis + Schwarz threshold) it stores, in one .npz:
  * the reference-format screening list (shellptr, shellid, shellrid,
    shellvalue, maxvalue) of pfock/screening.c:15-180;
  * usq / uitl of one Fock build (pfock/fock_task.c:195-196);
  * a test density D and F = PFock_getMat(F) for it;
  * S, H_core, X for the small cases;
  * the SCF energies of pscf/scf.c's loop (10 iterations).
When the reference's own sources have been compiled (oracle/_ref/ref_probe,
built by oracle/ref/Makefile), the probe's screening list, counters and F
for the same density are checked against the oracle before anything is
written, so every fixture is pinned to the reference's code path.

Run:  python tests/golden/make_golden.py [case ...]
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gtfock_b200 import molecules as mol  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

BOHR = 0.529177210903
CRAWFORD_H2O_BOHR = [("O", 0.0, -0.143225816552, 0.0),
                     ("H", 1.638036840407, 1.136548822547, 0.0),
                     ("H", -1.638036840407, 1.136548822547, 0.0)]


def h2o_atoms():
    return [(s, x * BOHR, y * BOHR, z * BOHR) for s, x, y, z in CRAWFORD_H2O_BOHR]


# name: (atoms builder, basis, tol, store one-electron matrices, scf iterations)
CASES = {
    "h2o_sto3g": (h2o_atoms, "sto-3g", 1e-10, True, 20),
    "h2o_631g": (h2o_atoms, "6-31g", 1e-10, True, 15),
    "h2o_ccpvdz": (h2o_atoms, "cc-pvdz", 1e-10, True, 15),
    "ch4_ccpvdz": (lambda: mol.alkane(1), "cc-pvdz", 1e-10, True, 12),
    "c4h10_ccpvdz": (lambda: mol.alkane(4), "cc-pvdz", 1e-10, True, 10),
    "benzene_ccpvdz": (lambda: mol.graphene_flake(0), "cc-pvdz", 1e-10, True, 10),
    "w8_631g": (lambda: mol.water_cluster(8, 2024), "6-31g", 1e-10, True, 10),
    "c12h26_ccpvdz": (lambda: mol.alkane(12), "cc-pvdz", 1e-10, False, 10),
}


def test_density(n, seed=7):
    """A symmetric density-like matrix: the SCF density is used where
    available; this fallback is a seeded symmetric matrix with decaying
    off-diagonal elements."""
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n)) * 0.05
    idx = np.arange(n)
    A *= np.exp(-np.abs(idx[:, None] - idx[None, :]) / 20.0)
    return 0.5 * (A + A.T) + np.eye(n) * 0.3


def ref_probe(gbs, xyz, tol, D):
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_probe")
    if not os.path.exists(exe):
        return None
    with tempfile.TemporaryDirectory() as td:
        dpath = os.path.join(td, "D.bin")
        D.astype(np.float64).tofile(dpath)
        out = os.path.join(td, "out")
        subprocess.run([exe, gbs, xyz, "%.17g" % tol, "4", dpath, out], check=True,
                       stdout=subprocess.DEVNULL)
        raw = open(out + ".screen", "rb").read()
        ns, nnz = np.frombuffer(raw[:8], np.int32)
        maxv = np.frombuffer(raw[8:16], np.float64)[0]
        o = 16
        sp = np.frombuffer(raw[o:o + 4 * (ns + 1)], np.int32); o += 4 * (ns + 1)
        si = np.frombuffer(raw[o:o + 4 * nnz], np.int32); o += 4 * nnz
        sr = np.frombuffer(raw[o:o + 4 * nnz], np.int32); o += 4 * nnz
        sv = np.frombuffer(raw[o:o + 8 * nnz], np.float64)
        raw = open(out + ".fock", "rb").read()
        nbf = np.frombuffer(raw[:4], np.int32)[0]
        usq, uitl = np.frombuffer(raw[4:20], np.float64)
        F = np.frombuffer(raw[20:], np.float64).reshape(nbf, nbf)
        return dict(shellptr=sp, shellid=si, shellrid=sr, shellvalue=sv, maxvalue=maxv,
                    usq=usq, uitl=uitl, F=F)


def make(name):
    build, basis, tol, onee, niters = CASES[name]
    atoms = build()
    gbs = mol.basis_file(basis)
    with tempfile.TemporaryDirectory() as td:
        xyz = mol.write_xyz(atoms, os.path.join(td, name + ".xyz"), name)
        b = po.Basis(gbs, xyz)
        scr = po.screening(b, tol)
        energies, F_last, D_last = po.scf(b, tol, niters)
        D = D_last if np.abs(D_last).sum() > 0 else test_density(b.nbf)
        F, usq, uitl = po.fock_build(b, tol, D, scr=scr)
        out = dict(atoms_sym=np.array([a[0] for a in atoms]),
                   atoms_xyz=np.array([a[1:] for a in atoms], dtype=np.float64),
                   basis=np.array(basis), tol=np.array(tol),
                   nbf=np.array(b.nbf), nshells=np.array(b.nshells), nocc=np.array(b.nocc),
                   enuc=np.array(b.enuc),
                   shellptr=scr[0], shellid=scr[1], shellrid=scr[2], shellvalue=scr[3],
                   maxvalue=np.array(scr[4]), usq=np.array(usq), uitl=np.array(uitl),
                   D=D, F=F, energies=energies)
        if onee:
            S, H, X = po.one_electron(b)
            out.update(S=S, H=H, X=X)
        ref = ref_probe(gbs, xyz, tol, D)
        if ref is not None:
            for k in ("shellptr", "shellid", "shellrid"):
                assert np.array_equal(ref[k], out[k]), (name, k)
            assert np.array_equal(ref["shellvalue"], out["shellvalue"]), name
            assert ref["maxvalue"] == out["maxvalue"], name
            assert ref["usq"] == usq and ref["uitl"] == uitl, (name, ref["usq"], usq)
            err = np.abs(ref["F"] - F).max()
            assert err < 1e-11, (name, err)
            out["ref_pinned"] = np.array(1)
            out["ref_max_dF"] = np.array(err)
            print("%s: pinned to the reference build (max |dF| %.2e)" % (name, err))
        else:
            out["ref_pinned"] = np.array(0)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print("%s: nbf %d nshells %d nnz %d usq %.0f E %.10f" %
              (name, b.nbf, b.nshells, len(scr[1]), usq, energies[-1]))


if __name__ == "__main__":
    names = sys.argv[1:] or list(CASES)
    for n in names:
        make(n)
