"""Failure paths on the GPU, made on the host (no device fault is involved).

* An injected device-allocation failure during PFock_create (the test hook
  gtf_debug_fail_alloc makes the n-th allocation fail as an out-of-memory
  cudaMalloc would) returns PFOCK_STATUS_ALLOC_FAILED
  (pfock/pfock.h:188-202), leaves no device allocation behind, and the next
  engine works: every allocation point of the set-up is tried.
* A request withdrawn from the batched engine between steps frees its slot;
  the other jobs finish exactly as they do without it."""
import ctypes

import numpy as np
import pytest

from conftest import golden_xyz, load_golden

import gtfock_b200 as gb
from gtfock_b200 import molecules as mol

pytestmark = pytest.mark.gpu

ALLOC_FAILED = 2


def test_create_alloc_failure_releases_everything(tmp_path):
    L = gb.load()
    g = load_golden("c4h10_ccpvdz")
    gbs, xyz = golden_xyz(g, tmp_path)
    b = gb.BasisSet(gbs, xyz)
    h = ctypes.c_void_p()
    # one good engine first: lazy module loading and pools settle
    assert L.PFock_create(b.h, 1, 1, 4, 1e-10, 1, 1, ctypes.byref(h)) == 0
    L.PFock_destroy(h)
    live0 = L.gtf_debug_live_allocs()
    free0 = gb.device_memory()[0]
    failures = 0
    n = 1
    while True:
        L.gtf_debug_fail_alloc(n)
        h = ctypes.c_void_p()
        st = L.PFock_create(b.h, 1, 1, 4, 1e-10, 1, 1, ctypes.byref(h))
        L.gtf_debug_fail_alloc(0)
        if st == 0:
            L.PFock_destroy(h)
            break                    # n is past the set-up's last allocation
        assert st == ALLOC_FAILED, (n, st)
        assert L.gtf_debug_live_allocs() == live0, "allocation %d: leaked" % n
        failures += 1
        n += 1
        assert n < 1000
    assert failures > 20             # every allocation point was exercised
    assert L.gtf_debug_live_allocs() == live0
    assert abs(gb.device_memory()[0] - free0) <= 64 << 20
    # the library still works after the failures
    pf = gb.PFock(b, tolscr=float(g["tol"]))
    assert np.abs(pf.compute_fock(g["D"]) - g["F"]).max() < 1e-10
    pf.close()


def test_batch_cancel_frees_slot(tmp_path):
    mols = [mol.water_cluster(3, 21), mol.alkane(3), mol.water_cluster(4, 22)]
    xyzs = [mol.write_xyz(a, str(tmp_path / ("m%d.xyz" % k))) for k, a in enumerate(mols)]
    gbs = mol.basis_file("6-31g")
    alone = []
    for x in (xyzs[0], xyzs[2]):
        bt = gb.Batch(1)
        s = bt.add(gbs, x, max_iters=30, etol=1e-10)
        bt.run()
        alone.append(bt.result(s)[0])
        bt.close()
    bt = gb.Batch(3)
    try:
        slots = [bt.add(gbs, x, max_iters=30, etol=1e-10) for x in xyzs]
        bt.step()
        bt.step()
        assert bt.info()["used"] == 3
        bt.remove(slots[1])          # withdrawn between steps
        assert bt.info()["used"] == 2
        bt.run()
        for s, e_ref in zip((slots[0], slots[2]), alone):
            e, done = bt.result(s)
            assert done
            assert len(e) == len(e_ref)
            assert np.abs(e - e_ref).max() < 1e-9
        # the freed slot takes a new job
        s_new = bt.add(gbs, xyzs[1], max_iters=30, etol=1e-10)
        assert s_new == slots[1]
    finally:
        bt.close()
