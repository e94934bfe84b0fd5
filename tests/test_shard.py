"""Sharded Fock builds (one molecule over several ranks), host side: the unit
ranges of the shards partition each launch, and world-size-2 gloo ranks that
each build one shard (oracle, CPU) and all-reduce through
gtfock_b200.shard.allreduce_fock reproduce the whole Fock matrix."""
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
        b = po.Basis(gbs, xyz)
        D = np.load(out + ".D.npy")
        F = po.fock_build_shard(b, 1e-10, D, world, rank, nthreads=2)
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
