"""Fixtures for non-symmetric densities (PFock_create with symm = 0).

For each case: a seeded non-symmetric density D_ns and the exact
F = 2 J[D] - K[D] with J_ab = sum_cd (ab|cd) D_cd and K_ab = sum_cd (ac|bd) D_cd,
from the oracle's full ERI tensor.  The same formula reproduces the
reference's symmetric-density F (checked against the case's main fixture
before writing).  When the reference's own sources have been compiled
(oracle/_ref/ref_probe), the reference's symm = 0 output for the same D is
stored too (F_ns_ref): its unique-quartet digestion with a non-symmetric D
depends on the orientation in which each quartet is enumerated, so it is
not 2 J[D] - K[D]; the difference is recorded, not used as a bar.

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
import make_golden as mg  # noqa: E402

CASES = ["h2o_631g", "h2o_ccpvdz"]


def eri_tensor(b):
    n, ns = b.nbf, b.nshells
    eri = np.zeros((n, n, n, n))
    for A in range(ns):
        for B in range(ns):
            for C in range(ns):
                for D in range(ns):
                    fa, fb, fc, fd = [b.func_start(s) for s in (A, B, C, D)]
                    da, db, dc, dd = [b.shell_dim(s) for s in (A, B, C, D)]
                    try:
                        blk = po.shell_quartet(b, A, B, C, D)
                    except ValueError:   # screened out inside the engine: zero block
                        continue
                    eri[fa:fa + da, fb:fb + db, fc:fc + dc, fd:fd + dd] = blk
    return eri


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


def make(name):
    g = dict(np.load(os.path.join(HERE, name + ".npz")))
    atoms = [(str(s),) + tuple(float(v) for v in x) for s, x in zip(g["atoms_sym"], g["atoms_xyz"])]
    gbs = mol.basis_file(str(g["basis"]))
    with tempfile.TemporaryDirectory() as td:
        xyz = mol.write_xyz(atoms, os.path.join(td, name + ".xyz"), name)
        b = po.Basis(gbs, xyz)
        eri = eri_tensor(b)
        err_sym = np.abs(fock_exact(eri, g["D"]) - g["F"]).max()
        assert err_sym < 1e-9, (name, err_sym)   # screening at tol drops < 1e-10 per integral
        rng = np.random.default_rng(11)
        n = b.nbf
        Dns = g["D"] + 0.05 * rng.standard_normal((n, n))
        out = dict(D_ns=Dns, F_ns=fock_exact(eri, Dns), sym_check=np.array(err_sym))
        ref = ref_nosymm(gbs, xyz, float(g["tol"]), Dns)
        if ref is not None:
            out["F_ns_ref"] = ref
            out["ref_minus_exact"] = np.array(np.abs(ref - out["F_ns"]).max())
        np.savez_compressed(os.path.join(HERE, "nosymm", name + ".npz"), **out)
        print("%s: symmetric check %.2e, reference nosymm - exact %.3e" %
              (name, err_sym, float(out.get("ref_minus_exact", np.nan))))


if __name__ == "__main__":
    for c in sys.argv[1:] or CASES:
        make(c)
