"""Seeded request streams for the batched and served SCF workloads.

* batched(count, seed): `count` independent molecules, each a water cluster
  of 2-24 molecules (built as water_cluster) or an all-trans alkane C2-C16
  (built as alkane), with STO-3G or 6-31G chosen per molecule; 14 to ~200
  basis functions.
* served(count, seed, rate): a Poisson arrival stream (exponential gaps of
  mean 1/rate seconds) whose sizes are log-uniform over 20-1500 basis
  functions: water clusters of 2-110 molecules in 6-31G or alkanes C4-C40 in
  cc-pVDZ, whichever family has a member nearest the drawn size.

Every item is (name, atoms, basis name); served() adds the arrival time.
"""
import math

import numpy as np

from . import molecules as mol

# basis functions per unit (6-31G water: O 9 + 2 H x 2; cc-pVDZ CnH2n+2:
# C 14, H 5; STO-3G water: O 5 + 2 H x 1; STO-3G / 6-31G alkane: C 5 / 9, H 1 / 2)
_NBF = {
    ("water", "sto-3g"): lambda n: 7 * n,
    ("water", "6-31g"): lambda n: 13 * n,
    ("alkane", "sto-3g"): lambda n: 5 * n + (2 * n + 2),
    ("alkane", "6-31g"): lambda n: 9 * n + 2 * (2 * n + 2),
    ("alkane", "cc-pvdz"): lambda n: 14 * n + 5 * (2 * n + 2),
}


def nbf(kind, n, basis):
    """Basis-function count of a generated molecule."""
    return _NBF[(kind, basis)](n)


def build(kind, n, seed):
    if kind == "water":
        return mol.water_cluster(n, seed)
    return mol.alkane(n)


def batched(count=256, seed=2024):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        basis = "sto-3g" if rng.random() < 0.5 else "6-31g"
        if rng.random() < 0.5:
            kind, n = "water", int(rng.integers(2, 25))
        else:
            kind, n = "alkane", int(rng.integers(2, 17))
        s = int(rng.integers(1 << 30))
        name = "%s%d_%s_%d" % (kind, n, basis, i)
        out.append((name, build(kind, n, s), basis, nbf(kind, n, basis)))
    return out


def served(count=64, seed=7, rate=2.0, lo=20, hi=1500):
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        target = math.exp(rng.uniform(math.log(lo), math.log(hi)))
        nw = int(min(110, max(2, round(target / 13.0))))
        na = int(min(40, max(4, round((target - 10.0) / 24.0))))
        ew = abs(nbf("water", nw, "6-31g") - target)
        ea = abs(nbf("alkane", na, "cc-pvdz") - target)
        s = int(rng.integers(1 << 30))
        if ew <= ea:
            kind, n, basis = "water", nw, "6-31g"
        else:
            kind, n, basis = "alkane", na, "cc-pvdz"
        name = "%s%d_%s_%d" % (kind, n, basis, i)
        out.append((t, name, build(kind, n, s), basis, nbf(kind, n, basis)))
    return out
