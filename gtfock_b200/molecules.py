"""Deterministic synthetic molecules for the benchmark workloads.

* alkane(n): all-trans CnH(2n+2), C-C 1.54 A, C-H 1.09 A, tetrahedral angles,
  zig-zag carbon backbone in the xy-plane.
* graphene_flake(k): planar H-terminated hexagonal flake with k rings of
  hexagons around a central one (k=2: C54H18, k=3: C96H24), C-C 1.42 A,
  C-H 1.09 A.
* water_cluster(n, seed): n rigid H2O (O-H 0.9572 A, H-O-H 104.52 deg) with
  uniformly random orientations, O uniformly in a cube sized for 1.0 g/cm^3,
  rejection at O-O < 2.5 A.

Atoms are (symbol, x, y, z) in Angstrom; write_xyz() produces the .xyz text
CInt_loadBasisSet reads.
"""
import math
import os

import numpy as np

TETRA = math.acos(-1.0 / 3.0)   # 109.47 deg

DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


def basis_file(name):
    """Path of a bundled basis set: 'sto-3g', '6-31g' or 'cc-pvdz'."""
    path = os.path.join(DATA_DIR, name.lower() + ".gbs")
    if not os.path.exists(path):
        raise FileNotFoundError(path)
    return path


def alkane(n, rcc=1.54, rch=1.09):
    """All-trans CnH(2n+2) with the carbon zig-zag in the xy-plane.

    Carbon i sits at (i dx, (i mod 2) dy, 0).  Each carbon has two in-plane
    bonds (to its backbone neighbours, or to H where a chain end continues
    the zig-zag) and two out-of-plane C-H bonds -b cos(t/2) +- z sin(t/2),
    b the in-plane bisector and t the tetrahedral angle."""
    if n < 1:
        raise ValueError("n >= 1")
    half = TETRA / 2.0
    dx = rcc * math.sin(half)
    dy = rcc * math.cos(half)

    def site(i):
        return np.array([i * dx, (i % 2) * dy, 0.0])

    atoms = [("C",) + tuple(site(i)) for i in range(n)]
    hyd = []
    for i in range(n):
        c = site(i)
        for j in (i - 1, i + 1):
            if j < 0 or j >= n:       # chain end: H along the continued zig-zag
                d = (site(j) - c) / rcc
                hyd.append(c + rch * d)
        b = (site(i - 1) + site(i + 1) - 2 * c)
        b /= np.linalg.norm(b)
        for sz in (+1.0, -1.0):
            d = -b * math.cos(half) + np.array([0.0, 0.0, sz * math.sin(half)])
            hyd.append(c + rch * d)
    atoms += [("H",) + tuple(h) for h in hyd]
    return atoms


def graphene_flake(k, rcc=1.42, rch=1.09):
    """Hexagonal flake with 3k(k+1)+1 rings: C_{6(k+1)^2} H_{6(k+1)}."""
    # ring centres: triangular lattice (spacing sqrt(3) rcc) in axial
    # coordinates, hexagonal distance <= k from the central ring
    centres = []
    b1 = np.array([1.5 * rcc, math.sqrt(3) / 2 * rcc])
    b2 = np.array([0.0, math.sqrt(3) * rcc])
    for q in range(-k, k + 1):
        for r in range(-k, k + 1):
            s = -q - r
            if max(abs(q), abs(r), abs(s)) <= k:
                centres.append(q * b1 + r * b2)
    verts = {}
    for c in centres:
        for m in range(6):
            ang = math.pi / 3.0 * m
            v = c + rcc * np.array([math.cos(ang), math.sin(ang)])
            key = (round(v[0], 6), round(v[1], 6))
            verts[key] = v
    cs = sorted(verts.values(), key=lambda v: (round(v[1], 6), round(v[0], 6)))
    cs = np.array(cs)
    atoms = [("C", x, y, 0.0) for x, y in cs]
    for idx, v in enumerate(cs):
        d = np.linalg.norm(cs - v, axis=1)
        nbrs = np.where((d > 0.1) & (d < rcc * 1.1))[0]
        if len(nbrs) == 2:
            out = 2 * v - cs[nbrs[0]] - cs[nbrs[1]]
            out /= np.linalg.norm(out)
            h = v + rch * out
            atoms.append(("H", h[0], h[1], 0.0))
    return atoms


def _random_rotation(rng):
    # uniform random unit quaternion (Shoemake)
    u1, u2, u3 = rng.random(3)
    q = np.array([math.sqrt(1 - u1) * math.sin(2 * math.pi * u2),
                  math.sqrt(1 - u1) * math.cos(2 * math.pi * u2),
                  math.sqrt(u1) * math.sin(2 * math.pi * u3),
                  math.sqrt(u1) * math.cos(2 * math.pi * u3)])
    x, y, z, w = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def water_cluster(n, seed, roh=0.9572, angle_deg=104.52, density=1.0, min_oo=2.5):
    """n rigid waters in a cube at `density` g/cm^3, seeded."""
    rng = np.random.default_rng(seed)
    mass = n * 18.015 / 6.02214076e23                       # g
    side = (mass / density) ** (1.0 / 3.0) * 1e8            # cm -> Angstrom
    th = math.radians(angle_deg) / 2.0
    local = np.array([[0.0, 0.0, 0.0],
                      [roh * math.sin(th), 0.0, roh * math.cos(th)],
                      [-roh * math.sin(th), 0.0, roh * math.cos(th)]])
    oxy = []
    tries = 0
    while len(oxy) < n:
        tries += 1
        if tries > 1000000:
            raise RuntimeError("could not place %d waters" % n)
        p = rng.random(3) * side
        if all(np.linalg.norm(p - o) >= min_oo for o in oxy):
            oxy.append(p)
    atoms = []
    for o in oxy:
        R = _random_rotation(rng)
        xyz = local @ R.T + o
        atoms.append(("O",) + tuple(xyz[0]))
        atoms.append(("H",) + tuple(xyz[1]))
        atoms.append(("H",) + tuple(xyz[2]))
    return atoms


def write_xyz(atoms, path, title="gtfock-b200"):
    with open(path, "w") as f:
        f.write("%d\n%s\n" % (len(atoms), title))
        for s, x, y, z in atoms:
            f.write("%-2s %22.16f %22.16f %22.16f\n" % (s, x, y, z))
    return path


def formula(atoms):
    from collections import Counter
    c = Counter(a[0] for a in atoms)
    return "".join("%s%d" % (k, c[k]) for k in sorted(c))
