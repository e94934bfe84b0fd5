"""Sharded Fock builds on the GPU: the parts of n shards built by the CUDA
kernels sum to the whole F (FP64 and mixed precision), the shards' work is
balanced by the weighted split, the NCCL path of ShardedFock (device F
all-reduced in place) gives the whole F on a one-rank group (the only NCCL
group a one-GPU run can form), and two processes sharing the GPU, each
building its shard and summing over gloo, both hold the whole F."""
import os
import socket

import numpy as np
import pytest

import gtfock_b200 as gb
from gtfock_b200 import molecules as mol
from conftest import golden_xyz, load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nshards", [2, 3, 5])
def test_shard_parts_sum_to_whole(tmp_path, nshards):
    xyz = mol.write_xyz(mol.alkane(4), str(tmp_path / "c4.xyz"))
    b = gb.BasisSet(mol.basis_file("cc-pvdz"), xyz)
    pf = gb.PFock(b, tolscr=1e-10)
    rng = np.random.default_rng(nshards)
    A = rng.standard_normal((b.nbf, b.nbf)) * 0.05
    D = A + A.T
    for prec in (0, 1):
        pf.set_shard(0, 1)
        pf.set_precision(prec, 1e-6)
        F = pf.compute_fock(D)
        parts = []
        for r in range(nshards):
            pf.set_shard(r, nshards)
            parts.append(pf.compute_fock(D))
        assert all(np.max(np.abs(p)) > 0 for p in parts)
        assert np.max(np.abs(sum(parts) - F)) < 1e-11
    pf.close()


def test_shard_against_oracle_fixture(tmp_path):
    g = load_golden("c4h10_ccpvdz")
    gbs, xyz = golden_xyz("c4h10_ccpvdz", tmp_path)
    b = gb.BasisSet(gbs, xyz)
    pf = gb.PFock(b, tolscr=float(g["tol"]))
    parts = []
    for r in range(4):
        pf.set_shard(r, 4)
        parts.append(pf.compute_fock(g["D"]))
    assert np.max(np.abs(sum(parts) - g["F"])) < 1e-10
    pf.close()


def test_shards_balanced_by_work(tmp_path):
    """The shards of a launch are split by the work model, so their model
    FLOPs sum to the whole build's and are within a few percent of each
    other (a split by unit counts leaves d-heavy and s-heavy ranges)."""
    xyz = mol.write_xyz(mol.alkane(12), str(tmp_path / "c12.xyz"))
    b = gb.BasisSet(mol.basis_file("cc-pvdz"), xyz)
    pf = gb.PFock(b, tolscr=1e-10)
    whole = pf.shard_work()
    for n in (2, 4):
        work = []
        for r in range(n):
            pf.set_shard(r, n)
            work.append(pf.shard_work())
        assert abs(sum(work) - whole) < 1e-6 * whole
        assert max(work) / min(work) < 1.05, work
    pf.close()


def test_set_shard_rejects_bad_arguments(tmp_path):
    xyz = mol.write_xyz(mol.alkane(2), str(tmp_path / "c2.xyz"))
    b = gb.BasisSet(mol.basis_file("sto-3g"), xyz)
    pf = gb.PFock(b, tolscr=1e-10)
    for r, n in ((2, 2), (-1, 3), (0, -1)):
        with pytest.raises(gb.GtfError):
            pf.set_shard(r, n)
    pf.close()


def test_sharded_fock_nccl_one_rank(tmp_path):
    import torch
    import torch.distributed as dist
    from gtfock_b200.shard import ShardedFock
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0, world_size=1)
    try:
        xyz = mol.write_xyz(mol.water_cluster(5, 9), str(tmp_path / "w5.xyz"))
        b = gb.BasisSet(mol.basis_file("6-31g"), xyz)
        ref = gb.PFock(b, tolscr=1e-10)
        D = np.eye(b.nbf) * 0.2
        F = ref.compute_fock(D)
        ref.close()
        sf = ShardedFock(b, tolscr=1e-10)
        Fd = sf.compute_fock_dev(torch.from_numpy(D).cuda())
        torch.cuda.synchronize()
        assert np.max(np.abs(Fd.cpu().numpy() - F)) < 1e-11
        Fh = sf.compute_fock(D)
        assert np.max(np.abs(Fh - F)) < 1e-11
        sf.close()
    finally:
        dist.destroy_process_group()


def _shard_rank(rank, world, port, gbs, xyz, tol, D_path, out):
    import torch
    import torch.distributed as dist
    import gtfock_b200 as gb_
    from gtfock_b200.shard import ShardedFock
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        b = gb_.BasisSet(gbs, xyz)
        D = np.load(D_path)
        sf = ShardedFock(b, tolscr=tol)
        Fh = sf.compute_fock(D)                               # host F, gloo all-reduce
        Fd = sf.compute_fock_dev(torch.from_numpy(D).cuda())  # device F, gloo all-reduce
        torch.cuda.synchronize()
        np.save(out + ".h%d.npy" % rank, Fh)
        np.save(out + ".d%d.npy" % rank, Fd.cpu().numpy())
        np.save(out + ".w%d.npy" % rank, np.array([sf.pf.shard_work()]))
        sf.close()
    finally:
        dist.destroy_process_group()


def test_sharded_fock_two_processes(tmp_path):
    """Two processes, each building one shard of every class launch with the
    library's split and summing F over a gloo group: both hold the pinned
    C4H10 / cc-pVDZ F.  With one GPU both processes share it (they wait on
    one another only on the host); a node with a GPU per rank runs the same
    code with NCCL for the device F."""
    import multiprocessing as mp
    g = load_golden("c4h10_ccpvdz")
    gbs, xyz = golden_xyz(g, tmp_path)
    D_path = str(tmp_path / "D.npy")
    np.save(D_path, g["D"])
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "sf")
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_shard_rank, args=(r, 2, port, gbs, xyz, float(g["tol"]), D_path, out))
             for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    for r in range(2):
        assert np.abs(np.load(out + ".h%d.npy" % r) - g["F"]).max() < 1e-10
        assert np.abs(np.load(out + ".d%d.npy" % r) - g["F"]).max() < 1e-10
    w0, w1 = (float(np.load(out + ".w%d.npy" % r)[0]) for r in range(2))
    assert abs(w0 - w1) <= 0.1 * (w0 + w1)
