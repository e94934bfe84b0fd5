"""CPU tests of the product's host side: basis parsing, molecule generators,
C-ABI exports and argument checking (no GPU calls)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT

import gtfock_b200 as gb
from gtfock_b200 import molecules as mol

INCLUDE = os.path.join(ROOT, "include")


def _basis(atoms, basis, tmp_path, name="m"):
    xyz = mol.write_xyz(atoms, str(tmp_path / (name + ".xyz")))
    return gb.BasisSet(mol.basis_file(basis), xyz)


@pytest.mark.parametrize("atoms,basis,natoms,nshells,nbf,nocc", [
    (lambda: mol.alkane(12), "cc-pvdz", 38, 150, 298, 49),
    (lambda: mol.graphene_flake(2), "cc-pvdz", 72, 378, 846, 171),
    (lambda: mol.graphene_flake(3), "cc-pvdz", 120, 648, 1464, 300),
    (lambda: mol.water_cluster(64, 1234), "6-31g", 192, 576, 832, 320),
])
def test_workload_sizes(atoms, basis, natoms, nshells, nbf, nocc, tmp_path):
    """Atom, shell and function counts of the benchmark molecules match the
    sizes GTFock's own data files encode (e.g. graphene_72_378_846.xyz)."""
    b = _basis(atoms(), basis, tmp_path)
    assert (b.natoms, b.nshells, b.nbf, b.nocc) == (natoms, nshells, nbf, nocc)


def test_xyz_two_atoms_on_one_line(tmp_path):
    """The parser reads records as a token stream, as needed for
    data/graphene/graphene_120_648_1464.xyz:77 where two atoms share a line."""
    p = tmp_path / "two.xyz"
    p.write_text("3\n\nO 0.0 0.0 0.0\nH 0.0 0.757 0.586H 0.0 -0.757 0.586\n")
    b = gb.BasisSet(mol.basis_file("sto-3g"), str(p))
    assert (b.natoms, b.nshells, b.nbf) == (3, 5, 7)


def test_fortran_exponents_and_sp_shells(tmp_path):
    """'D' exponents and SP shells (split into S then P) in a .gbs file."""
    gbs = tmp_path / "t.gbs"
    gbs.write_text("cartesian\n\nH     0\nS   2   1.00\n  0.1D+01  0.5D0\n  0.2D00 0.6\n****\n"
                   "O     0\nSP   1   1.00\n  0.3D+00  1.0  1.0\n****\n")
    xyz = mol.write_xyz([("O", 0, 0, 0), ("H", 0, 0, 1.0)], str(tmp_path / "oh.xyz"))
    b = gb.BasisSet(str(gbs), xyz)
    assert (b.nshells, b.nbf) == (3, 5)


def test_pack_unpack_roundtrip(tmp_path):
    L = gb.load()
    b = _basis(mol.alkane(3), "cc-pvdz", tmp_path)
    buf = ctypes.c_void_p()
    size = ctypes.c_int()
    assert L.CInt_packBasisSet(b.h, ctypes.byref(buf), ctypes.byref(size)) == 0
    h2 = ctypes.c_void_p()
    L.CInt_createBasisSet(ctypes.byref(h2))
    assert L.CInt_unpackBasisSet(h2, buf) == 0
    assert L.CInt_getNumFuncs(h2) == b.nbf
    assert L.CInt_getNumShells(h2) == b.nshells
    assert abs(L.CInt_getNucEnergy(h2) - b.enuc) < 1e-12
    for s in range(b.nshells):
        assert L.CInt_getFuncStartInd(h2, s) == L.CInt_getFuncStartInd(b.h, s)
    L.CInt_destroyBasisSet(h2)


def _declared_functions():
    names = set()
    headers = [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    headers.append(os.path.join(INCLUDE, "mpi_stub", "mpi.h"))
    for h in headers:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"#define[^\n]*(\\\n[^\n]*)*", "", text)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(([^;{}]*)\)\s*;", text):
            name = m.group(1)
            if name in ("if", "while", "for", "switch", "return", "sizeof"):
                continue
            names.add(name)
    return names


def test_library_exports_every_declared_symbol():
    L = gb.load()
    names = _declared_functions()
    assert len(names) > 60
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing


def test_molecule_geometries():
    for n in (2, 5, 12):
        a = mol.alkane(n)
        X = np.array([x[1:] for x in a])
        d = np.linalg.norm(X[:, None] - X[None], axis=2)
        np.fill_diagonal(d, 9)
        assert abs(d.min() - 1.09) < 1e-9
        assert mol.formula(a) == "C%dH%d" % (n, 2 * n + 2)
    for k, f in ((2, "C54H18"), (3, "C96H24")):
        a = mol.graphene_flake(k)
        assert mol.formula(a) == f
        X = np.array([x[1:] for x in a])
        C = X[[i for i, x in enumerate(a) if x[0] == "C"]]
        dc = np.linalg.norm(C[:, None] - C[None], axis=2)
        np.fill_diagonal(dc, 9)
        assert abs(dc.min() - 1.42) < 1e-9
    w = mol.water_cluster(24, 99)
    O = np.array([x[1:] for x in w if x[0] == "O"])
    do = np.linalg.norm(O[:, None] - O[None], axis=2)
    np.fill_diagonal(do, 9)
    assert do.min() >= 2.5
    assert mol.water_cluster(24, 99) == w


def _gpu_present():
    try:
        return gb.device_info()[0] > 0
    except Exception:
        return False


def test_pfock_create_argument_checks(tmp_path):
    """Invalid arguments are rejected before any device work
    (pfock/pfock.c:841-862 semantics; nprow*npcol must be 1 on one GPU)."""
    L = gb.load()
    b = _basis(mol.alkane(1), "sto-3g", tmp_path)
    h = ctypes.c_void_p()
    INVALID = 3
    assert L.PFock_create(b.h, 2, 1, 4, 1e-10, 1, 1, ctypes.byref(h)) == INVALID
    assert L.PFock_create(b.h, 1, 1, 4, -1.0, 1, 1, ctypes.byref(h)) == INVALID
    assert L.PFock_create(b.h, 1, 1, 4, 1e-10, 0, 1, ctypes.byref(h)) == INVALID
    # symm = 0 (non-symmetric densities) is accepted; it is exercised on the GPU


@pytest.mark.skipif(_gpu_present(), reason="checks the no-device error path")
def test_pfock_create_without_device_fails_cleanly(tmp_path):
    L = gb.load()
    b = _basis(mol.alkane(1), "sto-3g", tmp_path)
    h = ctypes.c_void_p()
    assert L.PFock_create(b.h, 1, 1, 4, 1e-10, 1, 1, ctypes.byref(h)) == 1  # INIT_FAILED
    assert gb.device_info()[0] == 0


def test_tune_table_save_load(tmp_path):
    """The launch-shape table: entries round-trip through the text file, a
    file from another device model or a damaged one is refused and leaves
    the table as it was."""
    L = gb.load()
    gb.tune_clear()
    L.gtf_tune_put(0, 1, 0, 0, 3.0e5, 5, 2, 1.25)
    L.gtf_tune_put(1, 4, 4, 1, 9.0e3, 2, 4, 0.5)
    L.gtf_tune_put(2, -1, -1, 0, 2.0e9, 3, 0, 7.0)
    before = gb.tune_entries()
    assert len(before) == 3
    fock = [e for e in before if e["kind"] == "fock"][0]
    assert (fock["X"], fock["Y"], fock["ctas_per_sm"], fock["claim"], fock["bucket"]) == (1, 0, 5, 2, 18)
    prod = [e for e in before if e["kind"] == "products"][0]
    assert prod["shape"] == gb.GEMM_SHAPES[3] and prod["bucket"] == 30
    path = str(tmp_path / "tune.txt")
    gb.tune_save(path)
    gb.tune_clear()
    assert gb.tune_entries() == []
    gb.tune_load(path)
    assert gb.tune_entries() == before
    # same bucket: a lookup for another size in [2^18, 2^19) finds the entry
    a, b = ctypes.c_int(), ctypes.c_int()
    assert L.gtf_tune_get(0, 1, 0, 0, 4.0e5, ctypes.byref(a), ctypes.byref(b)) == 1
    assert (a.value, b.value) == (5, 2)
    assert L.gtf_tune_get(0, 1, 0, 0, 6.0e5, ctypes.byref(a), ctypes.byref(b)) == 0
    lines = open(path).read().splitlines()
    other = str(tmp_path / "other.txt")
    with open(other, "w") as f:
        f.write("gtfock_b200-tune 1 Some_Other_GPU_sm_90\n" + "\n".join(lines[1:]) + "\n")
    gb.tune_clear()
    with pytest.raises(gb.GtfError):
        gb.tune_load(other)
    bad = str(tmp_path / "bad.txt")
    with open(bad, "w") as f:
        f.write(lines[0] + "\n0 1 0 0 18 5\n")
    with pytest.raises(gb.GtfError):
        gb.tune_load(bad)
    assert gb.tune_entries() == []
    with pytest.raises(gb.GtfError):
        gb.tune_load(str(tmp_path / "missing.txt"))
    gb.tune_clear()


def test_admission_by_footprint():
    """HBM-footprint admission (gtfock_b200/serve.py): a request fits when its
    footprint fits the budget left and the device's free memory less the
    reserve; released jobs give their bytes back."""
    from gtfock_b200.serve import Admission, footprint_bytes
    free = [10 << 30]
    a = Admission(budget=None, reserve=1 << 30, free_fn=lambda: free[0])
    assert a.budget == 9 << 30
    assert a.fits(9 << 30) and not a.fits((9 << 30) + 1)
    a.hold("x", 6 << 30)
    free[0] -= 6 << 30
    assert a.used == 6 << 30
    assert a.fits(3 << 30)
    assert not a.fits((3 << 30) + 1)          # budget left
    free[0] = 2 << 30                          # another process took memory
    assert not a.fits(2 << 30)                 # free memory less the reserve
    assert a.fits(1 << 30)
    a.release("x")
    a.release("x")                             # idempotent
    assert a.used == 0
    b = Admission(budget=5 << 30, reserve=0, free_fn=lambda: 100 << 30)
    assert b.budget == 5 << 30 and not b.fits((5 << 30) + 1)
    # the estimate grows with the basis and with incremental builds
    assert footprint_bytes(800) > footprint_bytes(400) > 0
    assert footprint_bytes(800, incremental=True) > footprint_bytes(800)
