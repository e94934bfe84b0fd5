"""Sharded Fock builds (one molecule over several ranks), host side.

* The library's split functions (gtf_shard_range, gtf_shard_split) tile
  each range in order, and the weighted split balances the work.
* World-size-2 gloo ranks partition the build with the library's weighted
  split (gtfock_b200.shard.shard_split -- the function a sharded engine
  applies to each launch's bras), each build its part with the oracle on the
  CPU, and all-reduce through gtfock_b200.shard.allreduce_fock: the sum is
  the whole Fock matrix.  (Unmeasured on hardware: runs on 2+ GPUs are not
  available here.)"""
import os
import socket

import numpy as np
import pytest

from conftest import ROOT


def test_shard_ranges_partition():
    from gtfock_b200.shard import shard_range
    for nunits in (0, 1, 7, 31, 32, 1000, 123457):
        for n in (1, 2, 3, 4, 8):
            rs = [shard_range(nunits, r, n) for r in range(n)]
            assert rs[0][0] == 0 and rs[-1][1] == nunits
            for (a, b), (c, d) in zip(rs, rs[1:]):
                assert b == c
            sizes = [b - a for a, b in rs]
            assert max(sizes) - min(sizes) <= 1


def test_weighted_split_tiles_and_balances():
    from gtfock_b200.shard import shard_split
    rng = np.random.default_rng(3)
    for n_items in (0, 1, 5, 100, 4000):
        w = rng.exponential(1.0, n_items) ** 3          # heavy-tailed work, as d vs s classes
        if n_items > 10:
            w[::17] = 0.0                               # empty items
        for n in (1, 2, 3, 5, 8):
            rs = [shard_split(w, r, n) for r in range(n)]
            assert rs[0][0] == 0 and rs[-1][1] == n_items
            for (a, b), (c, d) in zip(rs, rs[1:]):
                assert a <= b == c <= d
            if n_items >= 100:
                parts = [w[a:b].sum() for a, b in rs]
                assert max(parts) - min(parts) <= 2 * w.max() + 1e-12
    # equal weights: shard sizes differ by at most one item
    for n in (2, 3, 7):
        sizes = [b - a for a, b in (shard_split(np.ones(100), r, n) for r in range(n))]
        assert max(sizes) - min(sizes) <= 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, gbs, xyz, out):
    import torch.distributed as dist
    from oracle import pyoracle as po
    from gtfock_b200.shard import allreduce_fock
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from gtfock_b200.shard import shard_split
        b = po.Basis(gbs, xyz)
        D = np.load(out + ".D.npy")
        scr = po.screening(b, 1e-10, 2)
        cost = po.pair_cost(b, 1e-10, scr=scr, nthreads=2)
        lo, hi = shard_split(cost, rank, world)
        np.save(out + ".range%d.npy" % rank, np.array([lo, hi, cost[lo:hi].sum(), cost.sum()]))
        F = po.fock_build_range(b, 1e-10, D, lo, hi, scr=scr, nthreads=2)
        np.save(out + ".part%d.npy" % rank, F)
        allreduce_fock(F)
        if rank == 0:
            np.save(out + ".sum.npy", F)
    finally:
        dist.destroy_process_group()


def test_gloo_ranks_sum_to_whole_fock(tmp_path):
    import multiprocessing as mp
    from oracle import pyoracle as po
    from gtfock_b200 import molecules as mol
    gbs = mol.basis_file("6-31g")
    xyz = mol.write_xyz(mol.water_cluster(4, 3), str(tmp_path / "w4.xyz"))
    b = po.Basis(gbs, xyz)
    rng = np.random.default_rng(5)
    A = rng.standard_normal((b.nbf, b.nbf)) * 0.1
    D = A + A.T
    out = str(tmp_path / "shard")
    np.save(out + ".D.npy", D)
    F_whole, _, _ = po.fock_build(b, 1e-10, D, nthreads=2)
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, gbs, xyz, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    parts = [np.load(out + ".part%d.npy" % r) for r in range(2)]
    # the all-reduce left each rank's buffer summed; the saved parts are pre-reduce copies
    assert np.max(np.abs(parts[0])) > 0 and np.max(np.abs(parts[1])) > 0
    F_sum = np.load(out + ".sum.npy")
    assert np.max(np.abs(F_sum - F_whole)) < 1e-12
    # the two ranges tile the MN pairs and carry about half the work each
    r0, r1 = (np.load(out + ".range%d.npy" % r) for r in range(2))
    assert r0[0] == 0 and r0[1] == r1[0] and r1[1] > r1[0]
    assert abs(r0[2] - r1[2]) <= 0.1 * r0[3]
