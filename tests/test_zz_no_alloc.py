"""The allocation-free Fock build (gtf_pfock_compute_noalloc) against the
regular one.

gtf_pfock_compute_noalloc serves callers that may not allocate device memory
while they run -- for example a host whose own pool allocator owns the GPU's
memory, or a real-time loop that cannot wait on the driver's allocator.  It
keeps its scratch in a static device array instead.  This test calls it
through the C ABI twice in a row (the shared scratch must be cleared between
calls) and compares each result with the regular device-resident build
(gtf_pfock_compute_dev) at the F tolerance of the parity tests.  It also
checks the cases around it: a basis just under the array's size limit, a
mixed-precision engine, Cartesian d shells, and the refusals (a basis above
the limit, a sharded engine).

The file is named to run last in a pytest session.
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import golden_xyz, load_golden

import gtfock_b200 as gb
from gtfock_b200 import molecules as mol

pytestmark = pytest.mark.gpu

F_TOL = 1e-10
_vp = ctypes.c_void_p


def _cudart():
    rt = ctypes.CDLL("/usr/local/cuda/lib64/libcudart.so")
    rt.cudaMalloc.argtypes = [ctypes.POINTER(_vp), ctypes.c_size_t]
    rt.cudaFree.argtypes = [_vp]
    rt.cudaMemcpy.argtypes = [_vp, _vp, ctypes.c_size_t, ctypes.c_int]
    rt.cudaDeviceSynchronize.argtypes = []
    return rt


class _DevBuf:
    """Test-side device buffer (the caller owns input and output memory)."""

    def __init__(self, rt, nbytes):
        self.rt = rt
        self.p = _vp()
        assert rt.cudaMalloc(ctypes.byref(self.p), nbytes) == 0
        self.n = nbytes

    def put(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert self.rt.cudaMemcpy(self.p, a.ctypes.data_as(_vp), self.n, 1) == 0

    def get(self, shape):
        out = np.zeros(shape)
        assert self.rt.cudaMemcpy(out.ctypes.data_as(_vp), self.p, self.n, 2) == 0
        return out

    def free(self):
        self.rt.cudaFree(self.p)


def _bind(L):
    L.gtf_pfock_compute_noalloc.argtypes = [_vp, _vp, _vp]
    L.gtf_pfock_compute_noalloc.restype = ctypes.c_int
    L.gtf_pfock_compute_dev.argtypes = [_vp, _vp, ctypes.POINTER(_vp)]
    L.gtf_pfock_compute_dev.restype = ctypes.c_int


def test_noalloc_matches_regular_build_twice(tmp_path):
    L = gb.load()
    _bind(L)
    rt = _cudart()
    g = load_golden("c4h10_ccpvdz")
    gbs, xyz = golden_xyz(g, tmp_path)
    b = gb.BasisSet(gbs, xyz)
    pf = gb.PFock(b, tolscr=float(g["tol"]))
    n = b.nbf
    nbytes = 8 * n * n
    dD, dF = _DevBuf(rt, nbytes), _DevBuf(rt, nbytes)
    try:
        for D in (g["D"], 0.5 * g["D"] + 0.01 * np.eye(n)):
            dD.put(D)
            # regular device-resident build
            fptr = _vp()
            assert L.gtf_pfock_compute_dev(pf.h, dD.p, ctypes.byref(fptr)) == 0
            F_ref = np.zeros((n, n))
            assert rt.cudaMemcpy(F_ref.ctypes.data_as(_vp), fptr, nbytes, 2) == 0
            # allocation-free build, twice in a row on the same input
            for _ in range(2):
                assert L.gtf_pfock_compute_noalloc(pf.h, dD.p, dF.p) == 0
                F = dF.get((n, n))
                assert np.abs(F - F_ref).max() < F_TOL
        # the first density is the fixture's: the result is the oracle's F too
        dD.put(g["D"])
        assert L.gtf_pfock_compute_noalloc(pf.h, dD.p, dF.p) == 0
        assert np.abs(dF.get((n, n)) - g["F"]).max() < F_TOL
    finally:
        dD.free()
        dF.free()
        pf.close()


def _compare_builds(L, rt, pf, n, densities):
    """gtf_pfock_compute_noalloc against gtf_pfock_compute_dev on each density,
    twice in a row; returns the last allocation-free F."""
    nbytes = 8 * n * n
    dD, dF = _DevBuf(rt, nbytes), _DevBuf(rt, nbytes)
    F = None
    try:
        for D in densities:
            dD.put(D)
            fptr = _vp()
            assert L.gtf_pfock_compute_dev(pf.h, dD.p, ctypes.byref(fptr)) == 0
            F_ref = np.zeros((n, n))
            assert rt.cudaMemcpy(F_ref.ctypes.data_as(_vp), fptr, nbytes, 2) == 0
            for _ in range(2):
                assert L.gtf_pfock_compute_noalloc(pf.h, dD.p, dF.p) == 0
                F = dF.get((n, n))
                assert np.abs(F - F_ref).max() < F_TOL
    finally:
        dD.free()
        dF.free()
    return F


def _density(n, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n)) * 0.05
    return 0.5 * (A + A.T) + 0.3 * np.eye(n)


def test_noalloc_near_size_limit(tmp_path):
    """(H2O)15 / cc-pVDZ: 375 Cartesian functions, just under the 384 limit,
    so the static array is used up to its last rows."""
    L = gb.load()
    _bind(L)
    rt = _cudart()
    xyz = mol.write_xyz(mol.water_cluster(15, 5), os.path.join(str(tmp_path), "w15.xyz"))
    b = gb.BasisSet(mol.basis_file("cc-pvdz"), xyz)
    pf = gb.PFock(b, tolscr=1e-10)
    try:
        n = b.nbf
        assert n == 360
        _compare_builds(L, rt, pf, n, [_density(n, 1), _density(n, 2)])
    finally:
        pf.close()


def test_noalloc_mixed_precision_engine(tmp_path):
    """An engine with FP32 quartets below a Schwarz bound of 1e-6: the
    allocation-free build runs the same FP64 and FP32 launches."""
    L = gb.load()
    _bind(L)
    rt = _cudart()
    g = load_golden("c4h10_ccpvdz")
    gbs, xyz = golden_xyz(g, tmp_path)
    b = gb.BasisSet(gbs, xyz)
    pf = gb.PFock(b, tolscr=float(g["tol"]))
    try:
        pf.set_precision(1, 1e-6)
        n32, nq = pf.precision_stats()
        assert 0 < n32 < nq
        F = _compare_builds(L, rt, pf, b.nbf, [g["D"]])
        assert np.abs(F - g["F"]).max() < 1e-6
    finally:
        pf.close()


def test_noalloc_cartesian_basis(tmp_path):
    """cc-pVDZ with Cartesian d shells (6 functions each): the density is used
    as given, without the spherical transform; checked against the regular
    build and the CPU oracle."""
    from oracle import pyoracle as po
    L = gb.load()
    _bind(L)
    rt = _cudart()
    text = open(mol.basis_file("cc-pvdz")).read()
    assert text.lstrip().lower().startswith("spherical")
    gbs = os.path.join(str(tmp_path), "cc-pvdz-cart.gbs")
    with open(gbs, "w") as f:
        f.write(text.replace("spherical", "cartesian", 1))
    xyz = mol.write_xyz(mol.alkane(2), os.path.join(str(tmp_path), "c2h6.xyz"))
    b = gb.BasisSet(gbs, xyz)
    pf = gb.PFock(b, tolscr=1e-10)
    try:
        n = b.nbf
        assert n == 2 * 15 + 6 * 5
        D = _density(n, 3)
        F = _compare_builds(L, rt, pf, n, [D])
        F_or, _, _ = po.fock_build(po.Basis(gbs, xyz), 1e-10, D)
        assert np.abs(F - F_or).max() < F_TOL
    finally:
        pf.close()


def test_noalloc_rejects_sharded_engine(tmp_path):
    """A sharded engine builds only its shard's part of F; the allocation-free
    entry point promises the whole F and refuses it."""
    L = gb.load()
    _bind(L)
    rt = _cudart()
    g = load_golden("h2o_ccpvdz")
    gbs, xyz = golden_xyz(g, tmp_path)
    b = gb.BasisSet(gbs, xyz)
    pf = gb.PFock(b, tolscr=1e-10)
    n = b.nbf
    dD, dF = _DevBuf(rt, 8 * n * n), _DevBuf(rt, 8 * n * n)
    try:
        dD.put(g["D"])
        pf.set_shard(0, 2)
        assert L.gtf_pfock_compute_noalloc(pf.h, dD.p, dF.p) == 3   # PFOCK_STATUS_INVALID_VALUE
        pf.set_shard(0, 1)
        assert L.gtf_pfock_compute_noalloc(pf.h, dD.p, dF.p) == 0
        assert np.abs(dF.get((n, n)) - g["F"]).max() < F_TOL
    finally:
        dD.free()
        dF.free()
        pf.close()


def test_noalloc_rejects_basis_above_limit(tmp_path):
    L = gb.load()
    _bind(L)
    rt = _cudart()
    xyz = mol.write_xyz(mol.graphene_flake(2), os.path.join(str(tmp_path), "c54h18.xyz"))
    b = gb.BasisSet(mol.basis_file("cc-pvdz"), xyz)   # 900 Cartesian functions
    pf = gb.PFock(b, tolscr=1e-10)
    n = b.nbf
    dD, dF = _DevBuf(rt, 8 * n * n), _DevBuf(rt, 8 * n * n)
    try:
        assert L.gtf_pfock_compute_noalloc(pf.h, dD.p, dF.p) == 3   # PFOCK_STATUS_INVALID_VALUE
    finally:
        dD.free()
        dF.free()
        pf.close()
