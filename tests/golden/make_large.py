"""Generate the large-molecule parity fixtures under tests/golden/large/.

These are the benchmark's own molecules at full size:
  * c54h18_ccpvdz  -- graphene flake C54H18 / cc-pVDZ, 846 functions;
  * w64_631g       -- (H2O)64, seed 2024, 6-31G, 832 functions;
  * c96h24_ccpvdz  -- graphene flake C96H24 / cc-pVDZ, 1464 functions.

Each .npz holds what the GPU path must reproduce for one Fock build:
  * the reference-format screening list (shellptr, shellid, shellrid,
    shellvalue, maxvalue) of pfock/screening.c:15-180;
  * the quartet counters usq / uitl of pfock/fock_task.c:195-196;
  * F = PFock_getMat(F) (pfock/pfock.c:1134-1188) for the density
    large_density(nbf, seed) of tests/conftest.py, stored as its upper
    triangle (F is symmetric after pfock/pfock.c:1719-1726).  The density
    is not stored: the test regenerates it from the seed (numpy's PCG64
    stream is the same on every machine).

The oracle (oracle/fock_oracle.c + oracle/cint_oracle.c) computes all of it.
When the reference's own sources have been compiled (oracle/_ref/ref_probe,
built by oracle/ref/Makefile) and --pin is given, the probe's screening list,
counters and F for the same density are compared with the oracle's and the
fixture records ref_pinned = 1 and the largest |dF|.

Run:  python tests/golden/make_large.py [--pin | --pin-existing] [--threads N] [case ...]
"""
import argparse
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from gtfock_b200 import molecules as mol  # noqa: E402
from oracle import pyoracle as po  # noqa: E402
from make_golden import ref_probe  # noqa: E402

sys.path.insert(0, os.path.dirname(HERE))
from conftest import large_density as density  # noqa: E402

OUT = os.path.join(HERE, "large")

# name: (atoms builder, basis, Schwarz threshold, density seed)
CASES = {
    "c54h18_ccpvdz": (lambda: mol.graphene_flake(2), "cc-pvdz", 1e-10, 11),
    "w64_631g": (lambda: mol.water_cluster(64, 2024), "6-31g", 1e-10, 12),
    "c96h24_ccpvdz": (lambda: mol.graphene_flake(3), "cc-pvdz", 1e-10, 13),
}


def upper(F):
    return F[np.triu_indices(F.shape[0])]


def make(name, pin, nthreads):
    build, basis, tol, seed = CASES[name]
    atoms = build()
    gbs = mol.basis_file(basis)
    os.makedirs(OUT, exist_ok=True)
    with tempfile.TemporaryDirectory() as td:
        xyz = mol.write_xyz(atoms, os.path.join(td, name + ".xyz"), name)
        b = po.Basis(gbs, xyz)
        t0 = time.time()
        scr = po.screening(b, tol, nthreads)
        D = density(b.nbf, seed)
        F, usq, uitl = po.fock_build(b, tol, D, scr=scr, nthreads=nthreads)
        t1 = time.time()
        asym = float(np.abs(F - F.T).max())
        out = dict(atoms_sym=np.array([a[0] for a in atoms]),
                   atoms_xyz=np.array([a[1:] for a in atoms], dtype=np.float64),
                   basis=np.array(basis), tol=np.array(tol), density_seed=np.array(seed),
                   nbf=np.array(b.nbf), nshells=np.array(b.nshells),
                   shellptr=scr[0].astype(np.int32), shellid=scr[1].astype(np.int32),
                   shellrid=scr[2].astype(np.int32), shellvalue=scr[3],
                   maxvalue=np.array(scr[4]), usq=np.array(usq), uitl=np.array(uitl),
                   F_upper=upper(F), oracle_seconds=np.array(t1 - t0),
                   oracle_threads=np.array(nthreads), ref_pinned=np.array(0))
        print("%s: nbf %d nshells %d nnz %d usq %.0f uitl %.0f |F-F^T| %.1e (%.0f s)"
              % (name, b.nbf, b.nshells, len(scr[1]), usq, uitl, asym, t1 - t0), flush=True)
        if pin:
            t0 = time.time()
            ref = ref_probe(gbs, xyz, tol, D)
            if ref is None:
                raise RuntimeError("oracle/_ref/ref_probe is not built (make -C oracle/ref)")
            for k in ("shellptr", "shellid", "shellrid"):
                assert np.array_equal(ref[k], out[k]), (name, k)
            assert np.array_equal(ref["shellvalue"], out["shellvalue"]), name
            assert ref["maxvalue"] == out["maxvalue"], name
            assert ref["usq"] == usq and ref["uitl"] == uitl, (name, ref["usq"], usq)
            err = float(np.abs(ref["F"] - F).max())
            assert err < 1e-11, (name, err)
            out["ref_pinned"] = np.array(1)
            out["ref_max_dF"] = np.array(err)
            out["ref_seconds"] = np.array(time.time() - t0)
            print("%s: pinned to the reference build (max |dF| %.2e, %.0f s)"
                  % (name, err, time.time() - t0), flush=True)
        np.savez_compressed(os.path.join(OUT, name + ".npz"), **out)


def pin_existing(name):
    """Check an existing fixture against oracle/_ref/ref_probe (the
    reference's own sources) without recomputing the oracle's F."""
    path = os.path.join(OUT, name + ".npz")
    out = dict(np.load(path, allow_pickle=False))
    atoms = [(str(sy),) + tuple(float(v) for v in x) for sy, x in zip(out["atoms_sym"], out["atoms_xyz"])]
    gbs = mol.basis_file(str(out["basis"]))
    tol = float(out["tol"])
    n = int(out["nbf"])
    F = np.zeros((n, n))
    iu = np.triu_indices(n)
    F[iu] = out["F_upper"]
    F.T[iu] = out["F_upper"]
    with tempfile.TemporaryDirectory() as td:
        xyz = mol.write_xyz(atoms, os.path.join(td, name + ".xyz"), name)
        t0 = time.time()
        ref = ref_probe(gbs, xyz, tol, density(n, int(out["density_seed"])))
        if ref is None:
            raise RuntimeError("oracle/_ref/ref_probe is not built (make -C oracle/ref)")
        for k in ("shellptr", "shellid", "shellrid"):
            assert np.array_equal(ref[k], out[k]), (name, k)
        assert np.array_equal(ref["shellvalue"], out["shellvalue"]), name
        assert ref["maxvalue"] == float(out["maxvalue"]), name
        assert ref["usq"] == float(out["usq"]) and ref["uitl"] == float(out["uitl"]), name
        err = float(np.abs(ref["F"] - F).max())
        assert err < 1e-11, (name, err)
        out["ref_pinned"] = np.array(1)
        out["ref_max_dF"] = np.array(err)
        out["ref_seconds"] = np.array(time.time() - t0)
        print("%s: pinned to the reference build (max |dF| %.2e, %.0f s)" % (name, err, time.time() - t0),
              flush=True)
    np.savez_compressed(path, **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("cases", nargs="*")
    ap.add_argument("--pin", action="store_true", help="check against oracle/_ref/ref_probe")
    ap.add_argument("--pin-existing", action="store_true",
                    help="pin the stored fixtures to oracle/_ref/ref_probe without recomputing them")
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    a = ap.parse_args()
    for n in a.cases or list(CASES):
        if a.pin_existing:
            pin_existing(n)
        else:
            make(n, a.pin, a.threads)


if __name__ == "__main__":
    main()
