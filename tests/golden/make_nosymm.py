"""Fixtures for non-symmetric densities (PFock_create with symm = 0).

For each case: a seeded non-symmetric density D_ns and, from the oracle's
full ERI tensor,
  F_ns:      the exact F = 2 J[D] - K[D], J_ab = sum_cd (ab|cd) D_cd and
             K_ab = sum_cd (ac|bd) D_cd (the same formula reproduces the
             reference's symmetric-density F, checked against the case's main
             fixture before writing);
  F_ns_port: the reference's symm = 0 result restated
             (pyoracle.fock_nosymm_reference): its unique-quartet digestion
             with a non-symmetric D depends on the orientation of the pair
             lists, so it is not 2 J[D] - K[D].
When the reference's own sources have been compiled (oracle/_ref/ref_probe),
its symm = 0 output for the same D is stored as F_ns_ref and the
restatement is checked against it before writing.  The cases of REF_ONLY are
too large for the full ERI tensor: they hold D_ns and the reference's own
F_ns_ref only.

Run:  python tests/golden/make_nosymm.py
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from gtfock_b200 import molecules as mol  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

CASES = ["h2o_631g", "h2o_ccpvdz", "ch4_ccpvdz"]
REF_ONLY = ["c4h10_ccpvdz"]


def fock_exact(eri, D):
    J = np.einsum("abcd,cd->ab", eri, D)
    K = np.einsum("acbd,cd->ab", eri, D)
    return 2.0 * J - K


def ref_nosymm(gbs, xyz, tol, D):
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_probe")
    if not os.path.exists(exe):
        return None
    n = D.shape[0]
    with tempfile.TemporaryDirectory() as td:
        dp = os.path.join(td, "D.bin")
        D.astype(np.float64).tofile(dp)
        out = os.path.join(td, "o")
        subprocess.run([exe, gbs, xyz, "%.17g" % tol, "4", dp, out, "0"], check=True, stdout=subprocess.DEVNULL)
        raw = open(out + ".fock", "rb").read()
        return np.frombuffer(raw[20:], np.float64).reshape(n, n).copy()


def seeded_density(g):
    rng = np.random.default_rng(11)
    n = int(g["nbf"])
    return g["D"] + 0.05 * rng.standard_normal((n, n))


def make_ref_only(name):
    g = dict(np.load(os.path.join(HERE, name + ".npz")))
    atoms = [(str(s),) + tuple(float(v) for v in x) for s, x in zip(g["atoms_sym"], g["atoms_xyz"])]
    gbs = mol.basis_file(str(g["basis"]))
    with tempfile.TemporaryDirectory() as td:
        xyz = mol.write_xyz(atoms, os.path.join(td, name + ".xyz"), name)
        Dns = seeded_density(g)
        ref = ref_nosymm(gbs, xyz, float(g["tol"]), Dns)
        if ref is None:
            raise SystemExit("%s needs the reference build (oracle/_ref/ref_probe)" % name)
        np.savez_compressed(os.path.join(HERE, "nosymm", name + ".npz"), D_ns=Dns, F_ns_ref=ref)
        print("%s: reference nosymm output stored" % name)


def make(name):
    g = dict(np.load(os.path.join(HERE, name + ".npz")))
    atoms = [(str(s),) + tuple(float(v) for v in x) for s, x in zip(g["atoms_sym"], g["atoms_xyz"])]
    gbs = mol.basis_file(str(g["basis"]))
    with tempfile.TemporaryDirectory() as td:
        xyz = mol.write_xyz(atoms, os.path.join(td, name + ".xyz"), name)
        b = po.Basis(gbs, xyz)
        eri = po.eri_tensor(b)
        err_sym = np.abs(fock_exact(eri, g["D"]) - g["F"]).max()
        assert err_sym < 1e-9, (name, err_sym)   # screening at tol drops < 1e-10 per integral
        Dns = seeded_density(g)
        out = dict(D_ns=Dns, F_ns=fock_exact(eri, Dns), sym_check=np.array(err_sym))
        out["F_ns_port"] = po.fock_nosymm_reference(b, float(g["tol"]), eri, Dns)
        ref = ref_nosymm(gbs, xyz, float(g["tol"]), Dns)
        if ref is not None:
            out["F_ns_ref"] = ref
            out["ref_minus_exact"] = np.array(np.abs(ref - out["F_ns"]).max())
            out["ref_minus_port"] = np.array(np.abs(ref - out["F_ns_port"]).max())
            assert float(out["ref_minus_port"]) < 1e-12, (name, float(out["ref_minus_port"]))
        np.savez_compressed(os.path.join(HERE, "nosymm", name + ".npz"), **out)
        print("%s: symmetric check %.2e, reference nosymm - exact %.3e, - restatement %.3e" %
              (name, err_sym, float(out.get("ref_minus_exact", np.nan)),
               float(out.get("ref_minus_port", np.nan))))


if __name__ == "__main__":
    for c in sys.argv[1:] or CASES + REF_ONLY:
        (make_ref_only if c in REF_ONLY else make)(c)
