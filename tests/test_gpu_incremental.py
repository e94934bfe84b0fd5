"""Incremental Fock builds (gtf_pfock_set_incremental) on the GPU.

F is linear in D, so F[D_k] = F[D_k-1] + G[D_k - D_k-1].  The engine builds
only the change, with its task lists rebuilt on the device for thresholds
scaled by max |D_k - D_k-1|.  Checked here:
  * with a vanishing drop threshold the quartet set is the plain build's, so a
    chain of incremental builds equals the plain build of the last density to
    the atomics' rounding (and the first build of a chain is a full one);
  * with the default threshold (the Schwarz threshold) the chain stays within
    a small bound of the plain build;
  * SCF energies with incremental builds (FP64, and FP32 quartets below the
    cutoff) agree with the plain FP64 path; batched jobs too;
  * after incremental builds, a plain build (allocation-free entry point,
    switching incremental off) uses the full task lists again."""
import numpy as np
import pytest

from conftest import golden_xyz, load_golden

import gtfock_b200 as gb

pytestmark = pytest.mark.gpu


def _chain(D0, n, k, scale, seed):
    """k densities, each a small symmetric change of the previous one."""
    rng = np.random.default_rng(seed)
    out = [D0]
    for _ in range(k - 1):
        E = rng.standard_normal((n, n)) * scale
        out.append(out[-1] + 0.5 * (E + E.T))
        scale *= 0.3
    return out


@pytest.mark.parametrize("case", ["c4h10_ccpvdz", "w8_631g"])
def test_chain_exact_without_drop(case, tmp_path):
    g = load_golden(case)
    gbs, xyz = golden_xyz(g, tmp_path)
    b = gb.BasisSet(gbs, xyz)
    plain = gb.PFock(b, tolscr=float(g["tol"]))
    inc = gb.PFock(b, tolscr=float(g["tol"]))
    try:
        inc.set_incremental(True, tau=1e-300, period=100)
        Ds = _chain(g["D"], b.nbf, 5, 1e-2, 1)
        for k, D in enumerate(Ds):
            F_inc = inc.compute_fock(D)
            F_ref = plain.compute_fock(D)
            assert np.abs(F_inc - F_ref).max() < 1e-11, (case, k)
            n64, n32, dmax = inc.incremental_stats()
            if k == 0:
                assert dmax == 0.0                  # the first build is a full one
                assert n64 + n32 == plain.counts()["usq"]
            else:
                assert dmax > 0.0
        # the full build of the fixture density is the oracle's F
        inc.set_incremental(True, tau=1e-300, period=100)
        assert np.abs(inc.compute_fock(g["D"]) - g["F"]).max() < 1e-10
    finally:
        plain.close()
        inc.close()


def test_chain_default_threshold_close(tmp_path):
    g = load_golden("c12h26_ccpvdz")
    gbs, xyz = golden_xyz(g, tmp_path)
    b = gb.BasisSet(gbs, xyz)
    plain = gb.PFock(b, tolscr=float(g["tol"]))
    inc = gb.PFock(b, tolscr=float(g["tol"]))
    try:
        inc.set_incremental(True, period=100)
        Ds = _chain(g["D"], b.nbf, 6, 1e-3, 2)
        usq = plain.counts()["usq"]
        for k, D in enumerate(Ds):
            F_inc = inc.compute_fock(D)
            F_ref = plain.compute_fock(D)
            n64, n32, dmax = inc.incremental_stats()
            assert np.abs(F_inc - F_ref).max() < 1e-8, k
            if k > 0:
                assert n64 + n32 < usq      # the change needs fewer quartets
    finally:
        plain.close()
        inc.close()


def test_mixed_incremental_uses_fp32_for_small_changes(tmp_path):
    g = load_golden("c4h10_ccpvdz")
    gbs, xyz = golden_xyz(g, tmp_path)
    b = gb.BasisSet(gbs, xyz)
    pf = gb.PFock(b, tolscr=1e-10)
    plain = gb.PFock(b, tolscr=1e-10)
    try:
        pf.set_precision(1, 1e-6)
        pf.set_incremental(True, period=100)
        Ds = _chain(g["D"], b.nbf, 3, 1e-4, 3)
        for k, D in enumerate(Ds):
            F = pf.compute_fock(D)
            n64, n32, dmax = pf.incremental_stats()
            assert np.abs(F - plain.compute_fock(D)).max() < 1e-6, k
        assert n32 > n64      # a change of 1e-5 leaves most quartets to FP32
    finally:
        pf.close()
        plain.close()


@pytest.mark.parametrize("case,prec", [("w8_631g", 0), ("c4h10_ccpvdz", 0), ("w8_631g", 1)])
def test_scf_energy_matches_plain(case, prec, tmp_path):
    g = load_golden(case)
    gbs, xyz = golden_xyz(g, tmp_path)
    ref = gb.SCFSolver(gbs, xyz, tolscr=1e-10)
    s = gb.SCFSolver(gbs, xyz, tolscr=1e-10)
    try:
        ref.set_options(precision=0, etol=1e-10)
        e_ref, _ = ref.solve(niters=40)
        # the dropped contributions (each below the Schwarz threshold) leave
        # ~1e-9 Ha of noise between iterations: converge to 1e-8
        s.set_options(precision=prec, fp32_cutoff=1e-6, etol=1e-8)
        s.set_incremental(True, period=8)
        e, _ = s.solve(niters=40)
        assert len(e_ref) < 40 and len(e) < 40, "not converged"
        tol = 1e-7 if prec == 0 else 1e-6
        assert abs(e[-1] - e_ref[-1]) < tol, (case, prec, e[-1] - e_ref[-1])
        # a second solve restarts the sum and gives the same energy
        e2, _ = s.solve(niters=40)
        assert abs(e2[-1] - e[-1]) < tol
    finally:
        ref.close()
        s.close()


def test_batch_incremental_matches_plain_batch(tmp_path):
    cases = ["h2o_631g", "w8_631g", "c4h10_ccpvdz"]
    files = [golden_xyz(load_golden(c), tmp_path) for c in cases]
    res = []
    for incr in (False, True):
        bt = gb.Batch(4)
        if incr:
            bt.set_incremental(True, period=8)
        slots = [bt.add(gbs, x, max_iters=40, etol=1e-10 if not incr else 1e-8) for gbs, x in files]
        bt.run()
        res.append([bt.result(s)[0] for s in slots])
        bt.close()
    for e_plain, e_inc in zip(*res):
        assert len(e_plain) < 40 and len(e_inc) < 40
        assert abs(e_plain[-1] - e_inc[-1]) < 1e-7


def test_plain_build_after_incremental(tmp_path):
    """The incremental builds overwrite the task-list arrays; a plain build
    afterwards (incremental off, or the allocation-free entry point) must see
    the full lists again."""
    g = load_golden("c4h10_ccpvdz")
    gbs, xyz = golden_xyz(g, tmp_path)
    b = gb.BasisSet(gbs, xyz)
    pf = gb.PFock(b, tolscr=float(g["tol"]))
    try:
        pf.set_incremental(True, period=100)
        for D in _chain(g["D"], b.nbf, 3, 1e-4, 4):
            pf.compute_fock(D)
        pf.set_incremental(False)
        assert np.abs(pf.compute_fock(g["D"]) - g["F"]).max() < 1e-10
    finally:
        pf.close()
