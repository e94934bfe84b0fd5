"""ctypes bindings of the CPU checker library (oracle/liboracle.so).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the gtfock_b200 package.  Each wrapper
names the reference function its C counterpart restates (see oracle/oracle.h).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build():
    """Compile liboracle.so with oracle/Makefile (gcc only, no GPU)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        vp, ip, dp, i, d = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), \
            ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_double
        L.CInt_createBasisSet.argtypes = [ctypes.POINTER(vp)]
        L.CInt_loadBasisSet.argtypes = [vp, ctypes.c_char_p, ctypes.c_char_p]
        L.CInt_destroyBasisSet.argtypes = [vp]
        for name in ("CInt_getNumShells", "CInt_getNumFuncs", "CInt_getNumAtoms",
                     "CInt_getNumOccOrb", "CInt_getMaxShellDim"):
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = i
        L.CInt_getNucEnergy.argtypes = [vp]
        L.CInt_getNucEnergy.restype = d
        L.CInt_getShellDim.argtypes = [vp, i]
        L.CInt_getFuncStartInd.argtypes = [vp, i]
        L.CInt_createERD.argtypes = [vp, ctypes.POINTER(vp), i]
        L.CInt_destroyERD.argtypes = [vp]
        L.CInt_computeShellQuartet.argtypes = [vp, vp, i, i, i, i, i,
                                               ctypes.POINTER(dp), ip]
        L.CInt_createOED.argtypes = [vp, ctypes.POINTER(vp)]
        L.CInt_destroyOED.argtypes = [vp]
        for name in ("CInt_computePairOvl", "CInt_computePairKin",
                     "CInt_computePairPot", "CInt_computePairCoreH"):
            getattr(L, name).argtypes = [vp, vp, i, i, ctypes.POINTER(dp), ip]
        L.or_screening.argtypes = [vp, d, i, ctypes.POINTER(ip), ctypes.POINTER(ip),
                                   ctypes.POINTER(ip), ctypes.POINTER(dp), ip, dp]
        L.or_fock_build.argtypes = [vp, d, i, ip, ip, ip, dp, dp, dp, dp, dp]
        L.or_fock_build_sample.argtypes = [vp, d, i, ip, ip, ip, dp, dp, dp, i, i, dp, dp]
        L.or_fock_build_shard.argtypes = [vp, d, i, ip, ip, ip, dp, dp, dp, i, i, i, dp, dp]
        L.or_fock_build_range.argtypes = [vp, d, i, ip, ip, ip, dp, dp, dp, i, i, dp, dp]
        L.or_fock_pair_cost.argtypes = [vp, d, i, ip, ip, ip, dp, dp]
        L.or_diis_create.argtypes = [i]
        L.or_diis_create.restype = vp
        L.or_diis_destroy.argtypes = [vp]
        L.or_diis_step.argtypes = [vp, dp, dp, dp, dp, i]
        L.or_one_electron.argtypes = [vp, dp, dp, dp]
        L.or_purification.argtypes = [i, i, dp, dp, dp]
        L.or_scf.argtypes = [vp, d, i, i, dp, dp, dp]
        L.or_free.argtypes = [vp]
        L.or_set_blas_threads.argtypes = [i]
        _LIB = L
    return _LIB


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


class Basis:
    """A CInt basis set loaded by the product's parser (basis.c) into the
    checker library."""

    def __init__(self, gbs, xyz):
        L = lib()
        self.h = ctypes.c_void_p()
        L.CInt_createBasisSet(ctypes.byref(self.h))
        st = L.CInt_loadBasisSet(self.h, gbs.encode(), xyz.encode())
        if st != 0:
            raise RuntimeError("CInt_loadBasisSet failed (%d) for %s / %s" % (st, gbs, xyz))
        self.nbf = L.CInt_getNumFuncs(self.h)
        self.nshells = L.CInt_getNumShells(self.h)
        self.natoms = L.CInt_getNumAtoms(self.h)
        self.nocc = L.CInt_getNumOccOrb(self.h)
        self.enuc = L.CInt_getNucEnergy(self.h)

    def __del__(self):
        try:
            lib().CInt_destroyBasisSet(self.h)
        except Exception:
            pass

    def shell_dim(self, s):
        return lib().CInt_getShellDim(self.h, s)

    def func_start(self, s):
        return lib().CInt_getFuncStartInd(self.h, s)


def shell_quartet(basis, A, B, C, D):
    """(AB|CD) block from the oracle engine, shape (dA,dB,dC,dD)."""
    L = lib()
    erd = ctypes.c_void_p()
    L.CInt_createERD(basis.h, ctypes.byref(erd), 1)
    ptr = ctypes.POINTER(ctypes.c_double)()
    n = ctypes.c_int()
    L.CInt_computeShellQuartet(basis.h, erd, 0, A, B, C, D, ctypes.byref(ptr), ctypes.byref(n))
    dims = [basis.shell_dim(s) for s in (A, B, C, D)]
    out = np.ctypeslib.as_array(ptr, shape=(n.value,)).copy()
    L.CInt_destroyERD(erd)
    # first index fastest -> reshape in Fortran order
    return out.reshape(dims, order="F")


def screening(basis, tol, nthreads=os.cpu_count()):
    """pfock/screening.c:15-180 -> (shellptr, shellid, shellrid, shellvalue, maxvalue)."""
    L = lib()
    sp, si, sr = (ctypes.POINTER(ctypes.c_int)() for _ in range(3))
    sv = ctypes.POINTER(ctypes.c_double)()
    nnz = ctypes.c_int()
    mx = ctypes.c_double()
    st = L.or_screening(basis.h, tol, nthreads, ctypes.byref(sp), ctypes.byref(si),
                        ctypes.byref(sr), ctypes.byref(sv), ctypes.byref(nnz), ctypes.byref(mx))
    if st != 0:
        raise RuntimeError("or_screening failed")
    n = nnz.value
    res = (np.ctypeslib.as_array(sp, shape=(basis.nshells + 1,)).copy(),
           np.ctypeslib.as_array(si, shape=(max(n, 1),))[:n].copy(),
           np.ctypeslib.as_array(sr, shape=(max(n, 1),))[:n].copy(),
           np.ctypeslib.as_array(sv, shape=(max(n, 1),))[:n].copy(),
           mx.value)
    for p in (sp, si, sr, sv):
        L.or_free(ctypes.cast(p, ctypes.c_void_p))
    return res


def fock_build(basis, tol, D, scr=None, nthreads=os.cpu_count()):
    """PFock_computeFock + getMat(F) restated: returns (F = 2J - K, usq, uitl)."""
    L = lib()
    if scr is None:
        scr = screening(basis, tol, nthreads)
    shellptr, shellid, shellrid, shellvalue, _ = scr
    D = np.ascontiguousarray(D, dtype=np.float64)
    F = np.zeros_like(D)
    usq = ctypes.c_double()
    uitl = ctypes.c_double()
    sid = np.ascontiguousarray(shellid, dtype=np.int32)
    srid = np.ascontiguousarray(shellrid, dtype=np.int32)
    sval = np.ascontiguousarray(shellvalue, dtype=np.float64)
    sptr = np.ascontiguousarray(shellptr, dtype=np.int32)
    if sid.size == 0:
        sid = np.zeros(1, np.int32); srid = np.zeros(1, np.int32); sval = np.zeros(1)
    st = L.or_fock_build(basis.h, tol, nthreads, _ip(sptr), _ip(sid), _ip(srid), _dp(sval),
                         _dp(D), _dp(F), ctypes.byref(usq), ctypes.byref(uitl))
    if st != 0:
        raise RuntimeError("or_fock_build failed")
    return F, usq.value, uitl.value


def fock_build_sample(basis, tol, D, stride, count_only=False, scr=None, nthreads=os.cpu_count()):
    """Every stride-th MN pair of one Fock build: (usq, uitl, seconds)."""
    import time
    L = lib()
    if scr is None:
        scr = screening(basis, tol, nthreads)
    shellptr, shellid, shellrid, shellvalue, _ = scr
    D = np.ascontiguousarray(D, dtype=np.float64)
    F = np.zeros_like(D)
    usq = ctypes.c_double()
    uitl = ctypes.c_double()
    sid = np.ascontiguousarray(shellid, dtype=np.int32)
    srid = np.ascontiguousarray(shellrid, dtype=np.int32)
    sval = np.ascontiguousarray(shellvalue, dtype=np.float64)
    sptr = np.ascontiguousarray(shellptr, dtype=np.int32)
    t0 = time.perf_counter()
    st = L.or_fock_build_sample(basis.h, tol, nthreads, _ip(sptr), _ip(sid), _ip(srid), _dp(sval),
                                _dp(D), _dp(F), stride, 1 if count_only else 0,
                                ctypes.byref(usq), ctypes.byref(uitl))
    dt = time.perf_counter() - t0
    if st != 0:
        raise RuntimeError("or_fock_build_sample failed")
    return usq.value, uitl.value, dt


def fock_build_shard(basis, tol, D, nshards, shard, scr=None, nthreads=os.cpu_count()):
    """Shard `shard` of an `nshards`-way split of one Fock build (every
    nshards-th MN pair from `shard`): its part of F.  The parts sum to F."""
    L = lib()
    if scr is None:
        scr = screening(basis, tol, nthreads)
    shellptr, shellid, shellrid, shellvalue, _ = scr
    D = np.ascontiguousarray(D, dtype=np.float64)
    F = np.zeros_like(D)
    usq = ctypes.c_double()
    uitl = ctypes.c_double()
    st = L.or_fock_build_shard(basis.h, tol, nthreads, _ip(np.ascontiguousarray(shellptr, dtype=np.int32)),
                               _ip(np.ascontiguousarray(shellid, dtype=np.int32)),
                               _ip(np.ascontiguousarray(shellrid, dtype=np.int32)),
                               _dp(np.ascontiguousarray(shellvalue, dtype=np.float64)), _dp(D), _dp(F),
                               nshards, shard, 0, ctypes.byref(usq), ctypes.byref(uitl))
    if st != 0:
        raise RuntimeError("or_fock_build_shard failed")
    return F


def diis_step_timed(X, S, D, F, it, state=None):
    """One DIIS step (pscf/purif.c:491-641) on the CPU; returns (F_out, seconds, state)."""
    import time
    L = lib()
    n = X.shape[0]
    if state is None:
        state = L.or_diis_create(n)
    F = np.ascontiguousarray(F, dtype=np.float64).copy()
    t0 = time.perf_counter()
    L.or_diis_step(state, _dp(np.ascontiguousarray(X)), _dp(np.ascontiguousarray(S)),
                   _dp(np.ascontiguousarray(D)), _dp(F), it)
    return F, time.perf_counter() - t0, state


def one_electron(basis):
    """(S, H, X) as PFock_createOvlMat / PFock_createCoreHMat produce them."""
    n = basis.nbf
    S = np.zeros((n, n)); H = np.zeros((n, n)); X = np.zeros((n, n))
    lib().or_one_electron(basis.h, _dp(S), _dp(H), _dp(X))
    return S, H, X


def purification(nobtls, X, F_orth):
    n = X.shape[0]
    D = np.zeros((n, n))
    it = lib().or_purification(n, nobtls, _dp(np.ascontiguousarray(X)),
                               _dp(np.ascontiguousarray(F_orth)), _dp(D))
    return D, it


def scf(basis, tol, niters, nthreads=os.cpu_count()):
    """pscf/scf.c main loop restated; returns (energies, F_last, D_last)."""
    n = basis.nbf
    e = np.zeros(niters)
    F = np.zeros((n, n))
    D = np.zeros((n, n))
    it = lib().or_scf(basis.h, tol, niters, nthreads, _dp(e), _dp(F), _dp(D))
    if it < 0:
        raise RuntimeError("or_scf failed")
    return e[:it], F, D


def _csr(basis, tol, scr, nthreads):
    if scr is None:
        scr = screening(basis, tol, nthreads)
    shellptr, shellid, shellrid, shellvalue, _ = scr
    return (np.ascontiguousarray(shellptr, dtype=np.int32), np.ascontiguousarray(shellid, dtype=np.int32),
            np.ascontiguousarray(shellrid, dtype=np.int32), np.ascontiguousarray(shellvalue, dtype=np.float64))


def pair_cost(basis, tol, scr=None, nthreads=os.cpu_count()):
    """Integrals of the screened quartets of every MN pair of the build (the
    pair's share of uitl), in the CSR order; no integrals evaluated."""
    sptr, sid, srid, sval = _csr(basis, tol, scr, nthreads)
    cost = np.zeros(max(sid.size, 1))
    if lib().or_fock_pair_cost(basis.h, tol, nthreads, _ip(sptr), _ip(sid), _ip(srid), _dp(sval), _dp(cost)) != 0:
        raise RuntimeError("or_fock_pair_cost failed")
    return cost[:sid.size]


def fock_build_range(basis, tol, D, lo, hi, scr=None, nthreads=os.cpu_count()):
    """The part of F from the MN pairs lo <= i < hi (CSR order); the parts of a
    partition of [0, nnz) sum to F."""
    sptr, sid, srid, sval = _csr(basis, tol, scr, nthreads)
    D = np.ascontiguousarray(D, dtype=np.float64)
    F = np.zeros_like(D)
    usq, uitl = ctypes.c_double(), ctypes.c_double()
    if lib().or_fock_build_range(basis.h, tol, nthreads, _ip(sptr), _ip(sid), _ip(srid), _dp(sval), _dp(D), _dp(F),
                                 int(lo), int(hi), ctypes.byref(usq), ctypes.byref(uitl)) != 0:
        raise RuntimeError("or_fock_build_range failed")
    return F


def eri_tensor(basis):
    """Full (ab|cd) tensor from the oracle engine, for small bases only."""
    n, ns = basis.nbf, basis.nshells
    eri = np.zeros((n, n, n, n))
    for A in range(ns):
        for B in range(ns):
            for C in range(ns):
                for D in range(ns):
                    fa, fb, fc, fd = [basis.func_start(s) for s in (A, B, C, D)]
                    da, db, dc, dd = [basis.shell_dim(s) for s in (A, B, C, D)]
                    try:
                        blk = shell_quartet(basis, A, B, C, D)
                    except ValueError:   # screened out inside the engine: zero block
                        continue
                    eri[fa:fa + da, fb:fb + db, fc:fc + dc, fd:fd + dd] = blk
    return eri


def fock_nosymm_reference(basis, tol, eri, D, scr=None):
    """The reference's symm = 0 Fock matrix for a (non-symmetric) D, restated
    in numpy for small bases: G[X] is fock_task's digestion of every unique
    quartet over the screened pair lists, in the orientation the lists give
    its bra and ket (pfock/fock_task.c:121-219, update_F at
    pfock/fock_task.c:29-117, J and K terms into one F as with __SCF__), and
    the result is (G[D] + G[D^T]^T) / 2 (PFock_commitDenMats transposes D,
    pfock/pfock.c:1113-1121; the correction step pfock/pfock.c:1704-1718)."""
    if scr is None:
        scr = screening(basis, tol)
    shellptr, shellid, shellrid, shellvalue, _ = scr
    ns, n = basis.nshells, basis.nbf
    fs = [basis.func_start(s) for s in range(ns)]
    dm = [basis.shell_dim(s) for s in range(ns)]

    def sl(s):
        return slice(fs[s], fs[s] + dm[s])

    tol2 = tol * tol

    def G(Dm):
        X = np.zeros((n, n))
        pairs = range(int(shellptr[0]), int(shellptr[ns]))
        for i in pairs:
            M, N, v1 = int(shellrid[i]), int(shellid[i]), float(shellvalue[i])
            f1 = 1 if v1 < 0.0 else 0
            for j in pairs:
                P, Q, v2 = int(shellrid[j]), int(shellid[j]), float(shellvalue[j])
                if (M > P and (M + P) % 2 == 1) or (M < P and (M + P) % 2 == 0):
                    continue
                if M == P and ((N > Q and (N + Q) % 2 == 1) or (N < Q and (N + Q) % 2 == 0)):
                    continue
                if abs(v1 * v2) < tol2:
                    continue
                f2 = 1 if v2 < 0.0 else 0
                f3 = 0 if (M == P and N == Q) else 1
                f4, f5, f6 = f1 & f2, f1 & f3, f2 & f3
                f7 = f4 & f3
                I = eri[sl(M), sl(N), sl(P), sl(Q)]
                X[sl(M), sl(N)] += 2.0 * (1 + f1 + f2 + f4) * np.einsum("mnpq,pq->mn", I, Dm[sl(P), sl(Q)])
                X[sl(P), sl(Q)] += 2.0 * (f3 + f5 + f6 + f7) * np.einsum("mnpq,mn->pq", I, Dm[sl(M), sl(N)])
                X[sl(M), sl(P)] -= (1 + f3) * np.einsum("mnpq,nq->mp", I, Dm[sl(N), sl(Q)])
                X[sl(N), sl(P)] -= (f1 + f5) * np.einsum("mnpq,mq->np", I, Dm[sl(M), sl(Q)])
                X[sl(M), sl(Q)] -= (f2 + f6) * np.einsum("mnpq,np->mq", I, Dm[sl(N), sl(P)])
                X[sl(N), sl(Q)] -= (f4 + f7) * np.einsum("mnpq,mp->nq", I, Dm[sl(M), sl(P)])
        return X

    D = np.asarray(D, dtype=np.float64)
    return 0.5 * (G(D) + G(np.ascontiguousarray(D.T)).T)
