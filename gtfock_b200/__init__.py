"""gtfock_b200 -- GTFock's Fock-build and purification hot path on one B200.

The product is the C-ABI library gtfock_b200/lib/libgtfock_b200.so (PFock,
purif and CInt APIs, see include/*.h).  This module binds it with ctypes for
tests, benchmarks and Python callers; it performs no computation itself and
fails loudly when the library (or a CUDA device, for compute calls) is
missing.

    import gtfock_b200 as gb
    basis = gb.BasisSet(gb.basis_file("cc-pvdz"), "mol.xyz")
    pf = gb.PFock(basis, tolscr=1e-10)
    pf.put_density(D); F = pf.compute_fock()
"""
import ctypes
import os

import numpy as np

from .molecules import basis_file  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libgtfock_b200.so")
SCF_BIN = os.path.join(_HERE, "lib", "scf")

MAT_D, MAT_F, MAT_J, MAT_K = 0, 1, 2, 3

_lib = None

_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double
_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)
_cp = ctypes.c_char_p


class GtfError(RuntimeError):
    pass


def _sig(L, name, args, res=ctypes.c_int):
    f = getattr(L, name)
    f.argtypes = args
    f.restype = res


def load():
    """Load libgtfock_b200.so (raises GtfError when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise GtfError("libgtfock_b200.so not built (%s); run __graft_entry__.build() "
                       "or make -C gtfock_b200" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    _sig(L, "CInt_createBasisSet", [ctypes.POINTER(_vp)])
    _sig(L, "CInt_destroyBasisSet", [_vp])
    _sig(L, "CInt_loadBasisSet", [_vp, _cp, _cp])
    for n in ("CInt_getNumShells", "CInt_getNumFuncs", "CInt_getNumAtoms",
              "CInt_getNumOccOrb", "CInt_getMaxShellDim", "CInt_getTotalCharge",
              "CInt_getNneutral"):
        _sig(L, n, [_vp])
    _sig(L, "CInt_getNucEnergy", [_vp], _d)
    _sig(L, "CInt_getShellDim", [_vp, _i])
    _sig(L, "CInt_getFuncStartInd", [_vp, _i])
    _sig(L, "CInt_packBasisSet", [_vp, ctypes.POINTER(_vp), _ip])
    _sig(L, "CInt_unpackBasisSet", [_vp, _vp])
    _sig(L, "PFock_create", [_vp, _i, _i, _i, _d, _i, _i, ctypes.POINTER(_vp)])
    _sig(L, "PFock_destroy", [_vp])
    _sig(L, "PFock_setNumDenMat", [_i, _vp])
    _sig(L, "PFock_putDenMat", [_i, _i, _i, _i, _i, _dp, _i, _vp])
    _sig(L, "PFock_fillDenMat", [_d, _i, _vp])
    _sig(L, "PFock_commitDenMats", [_vp])
    _sig(L, "PFock_sync", [_vp])
    _sig(L, "PFock_getMat", [_vp, _i, _i, _i, _i, _i, _i, _i, _dp])
    _sig(L, "PFock_computeFock", [_vp, _vp])
    _sig(L, "PFock_createOvlMat", [_vp, _vp])
    _sig(L, "PFock_destroyOvlMat", [_vp])
    _sig(L, "PFock_getOvlMat", [_vp, _i, _i, _i, _i, _i, _dp])
    _sig(L, "PFock_getOvlMat2", [_vp, _i, _i, _i, _i, _i, _dp])
    _sig(L, "PFock_createCoreHMat", [_vp, _vp])
    _sig(L, "PFock_destroyCoreHMat", [_vp])
    _sig(L, "PFock_getCoreHMat", [_vp, _i, _i, _i, _i, _i, _dp])
    _sig(L, "PFock_getMemorySize", [_vp, _dp])
    _sig(L, "PFock_getStatistics", [_vp])
    _sig(L, "create_purif", [_vp, _i, _i, _i], _vp)
    _sig(L, "destroy_purif", [_vp], None)
    _sig(L, "compute_purification", [_vp, _dp, _dp])
    _sig(L, "compute_diis", [_vp, _vp, _dp, _dp, _i], None)
    _sig(L, "gtf_pfock_counts", [_vp, _ip, _dp, _dp, _dp])
    _sig(L, "gtf_pfock_screening", [_vp, _ip, _ip, _ip, _dp])
    _sig(L, "gtf_pfock_timing", [_vp, _dp, _dp, _dp])
    _sig(L, "gtf_pfock_set_precision", [_vp, _i, _d])
    _sig(L, "gtf_pfock_set_nosymm_mode", [_vp, _i])
    _sig(L, "gtf_pfock_precision_stats", [_vp, _dp, _dp])
    _sig(L, "gtf_pfock_class_stats", [_vp, _ip, _ip, _dp, _dp])
    _sig(L, "gtf_pfock_class_work", [_vp, _dp, _dp])
    _sig(L, "gtf_scf_run", [_cp, _cp, _d, _i, _i, _dp, _dp])
    _sig(L, "gtf_scf_create", [_cp, _cp, _d], _vp)
    _sig(L, "gtf_scf_solve", [_vp, _i, _i, _dp, _dp])
    _sig(L, "gtf_scf_nbf", [_vp])
    _sig(L, "gtf_scf_set_options", [_vp, _i, _d, _d])
    _sig(L, "gtf_scf_get_density", [_vp, _dp])
    _sig(L, "gtf_scf_set_purification", [_vp, _i])
    _sig(L, "gtf_scf_purification_iters", [_vp, _ip, _ip])
    _sig(L, "gtf_scf_destroy", [_vp], None)
    _sig(L, "gtf_launch_count", [], ctypes.c_ulonglong)
    _sig(L, "gtf_batch_create", [_i], _vp)
    _sig(L, "gtf_batch_add", [_vp, _cp, _cp, _d, _i, _d, _i, _d])
    _sig(L, "gtf_batch_prepare", [_vp, _cp, _cp, _d, _i, _d, ctypes.POINTER(_vp)])
    _sig(L, "gtf_batch_attach", [_vp, _vp, _i, _d])
    _sig(L, "gtf_batch_job_free", [_vp], None)
    _sig(L, "gtf_batch_step", [_vp])
    _sig(L, "gtf_batch_run", [_vp])
    _sig(L, "gtf_batch_result", [_vp, _i, _dp, _ip, _ip])
    _sig(L, "gtf_batch_density", [_vp, _i, _dp])
    _sig(L, "gtf_batch_remove", [_vp, _i])
    _sig(L, "gtf_batch_info", [_vp, _ip, _ip, _dp, _dp, ctypes.POINTER(ctypes.c_size_t)])
    _sig(L, "gtf_batch_job_bytes", [_i], ctypes.c_size_t)
    _sig(L, "gtf_batch_stats", [_vp, _dp, _i])
    _sig(L, "gtf_batch_destroy", [_vp], None)
    _sig(L, "gtf_pfock_autotune", [_vp, _i])
    _sig(L, "gtf_pfock_set_shard", [_vp, _i, _i])
    _sig(L, "gtf_shard_range", [ctypes.c_longlong, _i, _i, ctypes.POINTER(ctypes.c_longlong),
                                ctypes.POINTER(ctypes.c_longlong)], None)
    _sig(L, "gtf_pfock_compute_dev", [_vp, _vp, ctypes.POINTER(_vp)])
    _sig(L, "gtf_batch_autotune", [_vp, _i])
    _sig(L, "gtf_tune_save", [_cp])
    _sig(L, "gtf_tune_load", [_cp])
    _sig(L, "gtf_tune_clear", [], None)
    _sig(L, "gtf_tune_put", [_i, _i, _i, _i, _d, _i, _i, _d], None)
    _sig(L, "gtf_tune_get", [_i, _i, _i, _i, _d, _ip, _ip])
    _sig(L, "gtf_tune_entries", [_ip, _i])
    _sig(L, "gtf_fp64_peak", [_dp])
    _sig(L, "gtf_device_info", [_ip, _ip])
    _sig(L, "gtf_pfock_set_incremental", [_vp, _i, _d, _i])
    _sig(L, "gtf_pfock_incremental_stats", [_vp, _dp, _dp, _dp])
    _sig(L, "gtf_scf_set_incremental", [_vp, _i, _d, _i])
    _sig(L, "gtf_batch_set_incremental", [_vp, _i, _d, _i])
    _sig(L, "gtf_batch_job_device_bytes", [_vp, _i], ctypes.c_size_t)
    _sig(L, "gtf_batch_job_stats", [_vp, _i, _dp, _i])
    _sig(L, "gtf_device_memory", [ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)])
    _sig(L, "gtf_set_device", [_i])
    _sig(L, "gtf_device_trim", [ctypes.c_size_t])
    _sig(L, "gtf_get_device", [_ip])
    _sig(L, "gtf_debug_fail_alloc", [_i], None)
    _sig(L, "gtf_debug_live_allocs", [], ctypes.c_longlong)
    _sig(L, "gtf_pfock_compute_noalloc", [_vp, _vp, _vp])
    _sig(L, "gtf_shard_split", [_dp, ctypes.c_longlong, _i, _i, ctypes.POINTER(ctypes.c_longlong),
                                ctypes.POINTER(ctypes.c_longlong)], None)
    _sig(L, "gtf_pfock_shard_work", [_vp, _dp])
    _sig(L, "gtf_pfock_class_work_screened", [_vp, _dp, _dp])
    _lib = L
    return L


def device_info():
    """(number of CUDA devices, compute capability of device 0 as 10*major+minor)."""
    L = load()
    n = ctypes.c_int()
    cc = ctypes.c_int()
    L.gtf_device_info(ctypes.byref(n), ctypes.byref(cc))
    return n.value, cc.value


def set_device(dev):
    """Device of the calling thread for the library's later calls (one
    process per GPU; a new thread starts on device 0 and selects again)."""
    if load().gtf_set_device(int(dev)) != 0:
        raise GtfError("gtf_set_device(%d) failed" % dev)


def device_trim(keep=0):
    """Return the library's cached pool blocks on the current device to the
    driver, down to `keep` bytes (waits for the device)."""
    if load().gtf_device_trim(int(keep)) != 0:
        raise GtfError("gtf_device_trim failed")


def get_device():
    d = ctypes.c_int()
    if load().gtf_get_device(ctypes.byref(d)) != 0:
        raise GtfError("gtf_get_device failed")
    return d.value


def device_memory():
    """(free bytes, total bytes) of the current CUDA device."""
    fr, to = ctypes.c_size_t(), ctypes.c_size_t()
    if load().gtf_device_memory(ctypes.byref(fr), ctypes.byref(to)) != 0:
        raise GtfError("gtf_device_memory failed (no CUDA device?)")
    return fr.value, to.value


def _dptr(a):
    return a.ctypes.data_as(_dp)


def _iptr(a):
    return a.ctypes.data_as(_ip)


class BasisSet:
    """CInt_createBasisSet + CInt_loadBasisSet (libcint/include/CInt.h:45-80)."""

    def __init__(self, gbs, xyz):
        L = load()
        self.h = _vp()
        L.CInt_createBasisSet(ctypes.byref(self.h))
        st = L.CInt_loadBasisSet(self.h, gbs.encode(), xyz.encode())
        if st != 0:
            L.CInt_destroyBasisSet(self.h)
            self.h = None
            raise GtfError("CInt_loadBasisSet failed (status %d): %s, %s" % (st, gbs, xyz))
        self.gbs, self.xyz = gbs, xyz
        self.nbf = L.CInt_getNumFuncs(self.h)
        self.nshells = L.CInt_getNumShells(self.h)
        self.natoms = L.CInt_getNumAtoms(self.h)
        self.nocc = L.CInt_getNumOccOrb(self.h)
        self.enuc = L.CInt_getNucEnergy(self.h)

    def close(self):
        if getattr(self, "h", None) is not None and _lib is not None:
            _lib.CInt_destroyBasisSet(self.h)
            self.h = None

    __del__ = close


class PFock:
    """The PFock engine (pfock/pfock.h:241-565) on the GPU."""

    def __init__(self, basis, tolscr=1e-10, max_numdmat=1, symm=1, nprow=1, npcol=1, ntasks=4):
        L = load()
        self.basis = basis
        self.h = _vp()
        st = L.PFock_create(basis.h, nprow, npcol, ntasks, tolscr, max_numdmat, symm,
                            ctypes.byref(self.h))
        if st != 0:
            self.h = None
            raise GtfError("PFock_create failed (status %d)" % st)
        self.nbf = basis.nbf
        L.PFock_setNumDenMat(max_numdmat, self.h)

    def close(self):
        if getattr(self, "h", None) is not None and _lib is not None:
            _lib.PFock_destroy(self.h)
            self.h = None

    __del__ = close

    def _check(self, st, what):
        if st != 0:
            raise GtfError("%s failed (status %d)" % (what, st))

    def put_density(self, D, index=0):
        D = np.ascontiguousarray(D, dtype=np.float64)
        n = self.nbf
        self._check(load().PFock_putDenMat(0, n - 1, 0, n - 1, n, _dptr(D), index, self.h),
                    "PFock_putDenMat")

    def commit(self):
        self._check(load().PFock_commitDenMats(self.h), "PFock_commitDenMats")

    def compute(self):
        self._check(load().PFock_computeFock(self.basis.h, self.h), "PFock_computeFock")

    def get_mat(self, mtype=MAT_F, index=0):
        n = self.nbf
        out = np.zeros((n, n))
        self._check(load().PFock_getMat(self.h, mtype, index, 0, n - 1, 0, n - 1, n, _dptr(out)),
                    "PFock_getMat")
        return out

    def compute_fock(self, D):
        """putDenMat + commitDenMats + computeFock + getMat(F), as pscf/scf.c:106-127."""
        self.put_density(D)
        self.commit()
        self.compute()
        return self.get_mat(MAT_F)

    def counts(self):
        L = load()
        nnz = ctypes.c_int()
        mx, usq, uitl = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        L.gtf_pfock_counts(self.h, ctypes.byref(nnz), ctypes.byref(mx), ctypes.byref(usq),
                           ctypes.byref(uitl))
        return {"nnz": nnz.value, "maxvalue": mx.value, "usq": usq.value, "uitl": uitl.value}

    def screening(self):
        c = self.counts()
        nnz = c["nnz"]
        sp = np.zeros(self.basis.nshells + 1, np.int32)
        si = np.zeros(max(nnz, 1), np.int32)
        sr = np.zeros(max(nnz, 1), np.int32)
        sv = np.zeros(max(nnz, 1))
        self._check(load().gtf_pfock_screening(self.h, _iptr(sp), _iptr(si), _iptr(sr), _dptr(sv)),
                    "gtf_pfock_screening")
        return sp, si[:nnz], sr[:nnz], sv[:nnz], c["maxvalue"]

    def timing(self):
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        load().gtf_pfock_timing(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return {"ms_total": a.value, "ms_eri": b.value, "eri_flops": c.value}

    def class_stats(self):
        """[(bra class, ket class, ms, quartets)] of the last build."""
        X = np.zeros(32, np.int32)
        Y = np.zeros(32, np.int32)
        ms = np.zeros(32)
        nq = np.zeros(32)
        n = load().gtf_pfock_class_stats(self.h, _iptr(X), _iptr(Y), _dptr(ms), _dptr(nq))
        return [(int(X[i]), int(Y[i]), float(ms[i]), float(nq[i])) for i in range(n)]

    def class_work(self):
        """[(Rys-model FLOPs, primitive quartets)] per class pair, same order."""
        fl = np.zeros(32)
        npq = np.zeros(32)
        n = load().gtf_pfock_class_work(self.h, _dptr(fl), _dptr(npq))
        if n < 0:
            raise GtfError("gtf_pfock_class_work failed (%d)" % n)
        return [(float(fl[i]), float(npq[i])) for i in range(n)]

    def class_work_screened(self):
        """[(Rys-model FLOPs, primitive quartets)] per class pair after
        primitive screening (what the kernels evaluate), same order."""
        f = np.zeros(21)
        q = np.zeros(21)
        n = load().gtf_pfock_class_work_screened(self.h, _dptr(f), _dptr(q))
        if n < 0:
            raise GtfError("gtf_pfock_class_work_screened failed (%d)" % n)
        return list(zip(f[:n], q[:n]))

    NOSYMM_MODES = {"reference": 1, "exact": 2}

    def set_nosymm_mode(self, mode):
        """Engines created with symm=0: "reference" (default) returns the
        reference's own symm = 0 result, (F[D] + F[D^T]^T) / 2 of its
        unique-quartet digestion; "exact" returns F = 2 J[D] - K[D]."""
        self._check(load().gtf_pfock_set_nosymm_mode(self.h, self.NOSYMM_MODES[mode]),
                    "gtf_pfock_set_nosymm_mode")

    def set_precision(self, mode, fp32_cutoff=0.0):
        """mode 0: FP64; mode 1: FP32 for quartets with Schwarz bound < fp32_cutoff."""
        self._check(load().gtf_pfock_set_precision(self.h, mode, fp32_cutoff),
                    "gtf_pfock_set_precision")

    def set_incremental(self, on=True, tau=0.0, period=8):
        """Incremental builds: F_k = F_k-1 + G[D_k - D_k-1], quartets of the
        change dropped below Schwarz bound x max|dD| < tau (tau <= 0: the
        Schwarz threshold), a full build every `period` builds."""
        self._check(load().gtf_pfock_set_incremental(self.h, 1 if on else 0, tau, period),
                    "gtf_pfock_set_incremental")

    def incremental_stats(self):
        """(FP64 quartets, FP32 quartets, max|dD|) of the last incremental build."""
        a, b, c = np.zeros(1), np.zeros(1), np.zeros(1)
        self._check(load().gtf_pfock_incremental_stats(self.h, _dptr(a), _dptr(b), _dptr(c)),
                    "gtf_pfock_incremental_stats")
        return float(a[0]), float(b[0]), float(c[0])

    def set_shard(self, shard, nshards):
        """Builds of this engine compute shard `shard` of `nshards` of every
        class launch's quartet units (their F is that shard's part)."""
        self._check(load().gtf_pfock_set_shard(self.h, shard, nshards), "gtf_pfock_set_shard")

    def shard_work(self):
        """Model FLOPs of this engine's shard of a build (whole build if unsharded)."""
        w = np.zeros(1)
        self._check(load().gtf_pfock_shard_work(self.h, _dptr(w)), "gtf_pfock_shard_work")
        return float(w[0])

    def compute_dev(self, d_ptr):
        """Fock build from a device density (pointer to nbf x nbf FP64);
        returns the device pointer of F (library memory, valid until the
        next build)."""
        out = _vp()
        self._check(load().gtf_pfock_compute_dev(self.h, _vp(d_ptr), ctypes.byref(out)), "gtf_pfock_compute_dev")
        return out.value

    def autotune(self, reps=2):
        """Time candidate launch shapes of every Fock launch on the density last
        put and record the fastest in the process-wide tuning table."""
        self._check(load().gtf_pfock_autotune(self.h, reps), "gtf_pfock_autotune")

    def precision_stats(self):
        """(quartets evaluated in FP32, all quartets) under the current mode."""
        a = np.zeros(1)
        b = np.zeros(1)
        self._check(load().gtf_pfock_precision_stats(self.h, _dptr(a), _dptr(b)),
                    "gtf_pfock_precision_stats")
        return float(a[0]), float(b[0])

    def one_electron(self):
        """(S, X, H) as PFock_createOvlMat/getOvlMat/getOvlMat2/createCoreHMat produce them."""
        L = load()
        n = self.nbf
        S, X, H = np.zeros((n, n)), np.zeros((n, n)), np.zeros((n, n))
        self._check(L.PFock_createOvlMat(self.h, self.basis.h), "PFock_createOvlMat")
        L.PFock_getOvlMat(self.h, 0, n - 1, 0, n - 1, n, _dptr(S))
        L.PFock_getOvlMat2(self.h, 0, n - 1, 0, n - 1, n, _dptr(X))
        L.PFock_destroyOvlMat(self.h)
        self._check(L.PFock_createCoreHMat(self.h, self.basis.h), "PFock_createCoreHMat")
        L.PFock_getCoreHMat(self.h, 0, n - 1, 0, n - 1, n, _dptr(H))
        L.PFock_destroyCoreHMat(self.h)
        return S, X, H


class Purif:
    """create_purif / compute_diis / compute_purification (pscf/purif.h:78-86)."""

    def __init__(self, basis):
        L = load()
        self.basis = basis
        self.h = L.create_purif(basis.h, 1, 1, 1)
        if not self.h:
            raise GtfError("create_purif failed")
        self.n = basis.nbf
        # purif_t field offsets: S_block and X_block pointers (see include/purif.h)
        self._struct = ctypes.cast(self.h, ctypes.POINTER(_PurifT)).contents

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.destroy_purif(self.h)
            self.h = None

    __del__ = close

    def _block(self, name):
        ptr = getattr(self._struct, name)
        return np.ctypeslib.as_array(ptr, shape=(self.n, self.n))

    def set_sx(self, S, X):
        self._block("S_block")[:] = S
        self._block("X_block")[:] = X

    def diis(self, pfock, D, F, it):
        D = np.ascontiguousarray(D, dtype=np.float64)
        F = np.ascontiguousarray(F, dtype=np.float64).copy()
        load().compute_diis(pfock.h if pfock else None, self.h, _dptr(D), _dptr(F), it)
        return F

    def purify(self, F_orth):
        F = np.ascontiguousarray(F_orth, dtype=np.float64).copy()
        D = np.zeros((self.n, self.n))
        it = load().compute_purification(self.h, _dptr(F), _dptr(D))
        if it < 0:
            raise GtfError("compute_purification failed")
        return D, it


class _PurifT(ctypes.Structure):
    _fields_ = [("runpurif", ctypes.c_int), ("rundgemm", ctypes.c_int), ("nbf", ctypes.c_int),
                ("nobtls", ctypes.c_int), ("np_purif", ctypes.c_int), ("nprow_purif", ctypes.c_int),
                ("npcol_purif", ctypes.c_int), ("npgrd_purif", ctypes.c_int),
                ("srow_purif", ctypes.c_int), ("scol_purif", ctypes.c_int),
                ("nrows_purif", ctypes.c_int), ("ncols_purif", ctypes.c_int),
                ("meshsize", ctypes.c_int), ("ldx", ctypes.c_int),
                ("H_block", _dp), ("X_block", _dp), ("S_block", _dp), ("F_block", _dp),
                ("D_block", _dp)]


def _timings(t):
    return {"fock_s": t[0], "diis_s": t[1], "purif_s": t[2], "total_s": t[3],
            "h2d_bytes": t[4], "d2h_bytes": t[5], "launches": int(t[6])}


def scf_run(gbs, xyz, tolscr=1e-10, niters=10, device_resident=False):
    """Native SCF loop of pscf/scf.c on the GPU (gtf_scf_run: set-up, solve,
    tear-down): returns (energies per iteration, timings dict)."""
    L = load()
    e = np.zeros(niters)
    t = np.zeros(8)
    it = L.gtf_scf_run(gbs.encode(), xyz.encode(), tolscr, niters, 1 if device_resident else 0,
                       _dptr(e), _dptr(t))
    if it < 0:
        raise GtfError("gtf_scf_run failed (%d)" % it)
    return e[:it], _timings(t)


class SCFSolver:
    """Set up once (gtf_scf_create), then solve repeatedly (gtf_scf_solve)."""

    def __init__(self, gbs, xyz, tolscr=1e-10):
        L = load()
        self.h = L.gtf_scf_create(gbs.encode(), xyz.encode(), tolscr)
        if not self.h:
            raise GtfError("gtf_scf_create failed")
        self.nbf = L.gtf_scf_nbf(self.h)

    def solve(self, niters=10, device_resident=True):
        e = np.zeros(niters)
        t = np.zeros(8)
        it = load().gtf_scf_solve(self.h, niters, 1 if device_resident else 0, _dptr(e), _dptr(t))
        if it < 0:
            raise GtfError("gtf_scf_solve failed (%d)" % it)
        return e[:it], _timings(t)

    def set_options(self, precision=0, fp32_cutoff=0.0, etol=1e-11):
        """precision 0: FP64 ERIs; 1: FP32 for quartets with Schwarz bound <
        fp32_cutoff.  The solve stops when |E_k - E_k-1| < etol."""
        r = load().gtf_scf_set_options(self.h, precision, fp32_cutoff, etol)
        if r != 0:
            raise GtfError("gtf_scf_set_options failed (%d)" % r)

    def set_incremental(self, on=True, tau=0.0, period=8):
        """Incremental Fock builds for this solver (see PFock.set_incremental);
        every solve starts with a full build."""
        r = load().gtf_scf_set_incremental(self.h, 1 if on else 0, tau, period)
        if r != 0:
            raise GtfError("gtf_scf_set_incremental failed (%d)" % r)

    def set_purification(self, mode):
        """0: FP64 products; 1: split-BF16 tensor-core products, FP64 finish."""
        r = load().gtf_scf_set_purification(self.h, mode)
        if r != 0:
            raise GtfError("gtf_scf_set_purification failed (%d)" % r)

    def purification_iters(self):
        """(split-BF16, FP64) iterations of the last purification."""
        a, b = ctypes.c_int(), ctypes.c_int()
        load().gtf_scf_purification_iters(self.h, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def density(self):
        """Density of the last solve (half density, AO basis)."""
        D = np.zeros((self.nbf, self.nbf))
        if load().gtf_scf_get_density(self.h, _dptr(D)) != 0:
            raise GtfError("gtf_scf_get_density failed")
        return D

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.gtf_scf_destroy(self.h)
            self.h = None

    __del__ = close


class Batch:
    """Many SCF jobs iterated in lock-step on one GPU (gtf_batch_*).

    add() sets a job up in a free slot and returns the slot; step() runs one
    SCF iteration of every running job and returns how many still run;
    result(slot) gives (energies, done).  Jobs may be added and removed
    between steps (continuous batching)."""

    def __init__(self, capacity):
        self.h = load().gtf_batch_create(capacity)
        if not self.h:
            raise GtfError("gtf_batch_create failed")
        self.capacity = capacity
        self.max_iters = {}

    def set_incremental(self, on=True, tau=0.0, period=8):
        """Incremental Fock builds for every job (set before the first add)."""
        r = load().gtf_batch_set_incremental(self.h, 1 if on else 0, tau, period)
        if r != 0:
            raise GtfError("gtf_batch_set_incremental failed (%d)" % r)

    def job_stats(self, slot):
        """(basis functions, SCF iterations, purification iterations of the
        last step, purification iterations in all) of the job in `slot`."""
        out = np.zeros(4)
        n = load().gtf_batch_job_stats(self.h, slot, _dptr(out), 4)
        return tuple(int(x) for x in out[:n])

    def job_device_bytes(self, slot):
        """Device bytes a job holds (its batch buffers and its Fock engine)."""
        return int(load().gtf_batch_job_device_bytes(self.h, slot))

    def add(self, gbs, xyz, tolscr=1e-10, precision=0, fp32_cutoff=0.0, max_iters=30, etol=1e-11):
        slot = load().gtf_batch_add(self.h, gbs.encode(), xyz.encode(), tolscr, precision, fp32_cutoff,
                                    max_iters, etol)
        if slot < 0:
            raise GtfError("gtf_batch_add failed (%d)" % slot)
        self.max_iters[slot] = max_iters
        return slot

    def prepare(self, gbs, xyz, tolscr=1e-10, precision=0, fp32_cutoff=0.0):
        """The part of add() that touches no state of the batch (basis,
        engine, S, H_core, X): may run while another thread steps the batch.
        Returns a job handle for attach()."""
        job = _vp()
        r = load().gtf_batch_prepare(self.h, gbs.encode(), xyz.encode(), tolscr, precision, fp32_cutoff,
                                     ctypes.byref(job))
        if r != 0:
            raise GtfError("gtf_batch_prepare failed (%d)" % r)
        return job

    def attach(self, job, max_iters=30, etol=1e-11):
        """Put a prepared job in a free slot (not while the batch steps);
        consumes the job.  Returns the slot."""
        slot = load().gtf_batch_attach(self.h, job, max_iters, etol)
        if slot < 0:
            raise GtfError("gtf_batch_attach failed (%d)" % slot)
        self.max_iters[slot] = max_iters
        return slot

    @staticmethod
    def release(job):
        """Release a prepared job that will not be attached."""
        load().gtf_batch_job_free(job)

    def step(self):
        r = load().gtf_batch_step(self.h)
        if r < 0:
            raise GtfError("gtf_batch_step failed (%d)" % r)
        return r

    def run(self):
        r = load().gtf_batch_run(self.h)
        if r < 0:
            raise GtfError("gtf_batch_run failed (%d)" % r)

    def result(self, slot):
        e = np.zeros(self.max_iters[slot])
        n = ctypes.c_int()
        done = ctypes.c_int()
        r = load().gtf_batch_result(self.h, slot, _dptr(e), ctypes.byref(n), ctypes.byref(done))
        if r != 0:
            raise GtfError("gtf_batch_result failed (%d)" % r)
        return e[:n.value].copy(), bool(done.value)

    def density(self, slot, nbf):
        D = np.zeros((nbf, nbf))
        if load().gtf_batch_density(self.h, slot, _dptr(D)) != 0:
            raise GtfError("gtf_batch_density failed")
        return D

    def remove(self, slot):
        if load().gtf_batch_remove(self.h, slot) != 0:
            raise GtfError("gtf_batch_remove failed")
        self.max_iters.pop(slot, None)

    def info(self):
        r, u = ctypes.c_int(), ctypes.c_int()
        mf, mr = ctypes.c_double(), ctypes.c_double()
        by = ctypes.c_size_t()
        load().gtf_batch_info(self.h, ctypes.byref(r), ctypes.byref(u), ctypes.byref(mf), ctypes.byref(mr),
                              ctypes.byref(by))
        st = np.zeros(6)
        load().gtf_batch_stats(self.h, _dptr(st), 6)
        return {"running": r.value, "used": u.value, "ms_fock": mf.value, "ms_rest": mr.value,
                "device_bytes": by.value, "ms_energy": st[1], "ms_diis": st[2], "ms_purification": st[3],
                "purification_steps": st[4], "steps": st[5]}

    def autotune(self, reps=2):
        """Tune the Fock launch shapes and the product tile shape for the jobs
        now in the batch (between steps)."""
        r = load().gtf_batch_autotune(self.h, reps)
        if r != 0:
            raise GtfError("gtf_batch_autotune failed (%d)" % r)

    @staticmethod
    def job_bytes(nbf):
        return int(load().gtf_batch_job_bytes(nbf))

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.gtf_batch_destroy(self.h)
            self.h = None

    __del__ = close


TUNE_KINDS = {0: "fock", 1: "fock-batch", 2: "products"}
GEMM_SHAPES = {0: "64x64 (4x4)", 1: "32x32 (2x2)", 2: "32x64 (2x4)", 3: "128x64 (8x4)"}


def tune_entries():
    """The process-wide tuning table as a list of dicts."""
    L = load()
    n = L.gtf_tune_entries(None, 0)
    rows = np.zeros(8 * max(n, 1), dtype=np.int32)
    n = L.gtf_tune_entries(rows.ctypes.data_as(_ip), n)
    out = []
    for r in rows[:8 * n].reshape(n, 8):
        kind = int(r[0])
        e = {"kind": TUNE_KINDS.get(kind, kind), "X": int(r[1]), "Y": int(r[2]), "part": int(r[3]),
             "bucket": int(r[4]), "ms": r[7] / 1000.0}
        if kind == 2:
            e["shape"] = GEMM_SHAPES.get(int(r[5]), int(r[5]))
        else:
            e["ctas_per_sm"] = int(r[5])
            e["claim"] = int(r[6])
        out.append(e)
    return out


def tune_save(path):
    if load().gtf_tune_save(path.encode()) != 0:
        raise GtfError("gtf_tune_save(%s) failed" % path)


def tune_load(path):
    """Merge a saved tuning table; raises GtfError for a missing file or one
    written on another device model."""
    r = load().gtf_tune_load(path.encode())
    if r != 0:
        raise GtfError("gtf_tune_load(%s) failed (%d)" % (path, r))


def tune_clear():
    load().gtf_tune_clear()


def launch_count():
    return int(load().gtf_launch_count())


def fp64_peak_gflops():
    g = ctypes.c_double()
    if load().gtf_fp64_peak(ctypes.byref(g)) != 0:
        raise GtfError("gtf_fp64_peak failed")
    return g.value
