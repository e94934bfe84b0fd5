"""Serving one stream (or one batch of molecules) on several GPUs, host side.

Each GPU has its own process and server; serve.route assigns every request
to a rank from the stream alone (no exchange on the data path), and
serve.gather_finished brings the finished requests together for the
statistics.  World-size-2 gloo ranks check that each keeps exactly the share
the others expect and that the gathered results are the union.  (Unmeasured
on hardware: runs on 2+ GPUs are not available here.)
"""
import os
import socket

import numpy as np

from gtfock_b200 import serve, workloads


def _stream(count=32, seed=7, rate=4.0):
    return [serve.Request(n, a, b, t, nb) for t, n, a, b, nb in workloads.served(count, seed, rate)]


def test_route_is_deterministic_and_spreads_the_work():
    reqs = _stream()
    for n in (1, 2, 3, 4, 8):
        a = serve.route(reqs, n)
        assert a == serve.route(list(reqs), n)
        assert set(a) <= set(range(n)) and len(a) == len(reqs)
        if n == 1:
            assert set(a) == {0}
            continue
        load = np.zeros(n)
        for r, k in zip(reqs, a):
            load[k] += serve.est_seconds(r.nbf)
        # list scheduling: no rank carries more than the average plus the largest request
        big = max(serve.est_seconds(r.nbf) for r in reqs)
        assert load.max() <= load.sum() / n + big + 1e-9
    # the two largest requests of the stream go to different GPUs
    a = serve.route(reqs, 2)
    top = sorted(range(len(reqs)), key=lambda i: -reqs[i].nbf)[:2]
    assert a[top[0]] != a[top[1]]


def test_split_jobs_balances_a_batch():
    nbfs = [it[3] for it in workloads.batched(256, 2024)]
    for n in (1, 2, 4, 8):
        a = serve.split_jobs(nbfs, n)
        assert a == serve.split_jobs(nbfs, n)
        load = np.zeros(n)
        for nb, k in zip(nbfs, a):
            load[k] += serve.est_seconds(nb)
        assert load.max() <= load.sum() / n + max(serve.est_seconds(x) for x in nbfs) + 1e-9
        assert all((np.array(a) == k).sum() > 0 for k in range(n))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        reqs = _stream()
        owner = serve.route(reqs, world)
        mine = [r for r, k in zip(reqs, owner) if k == rank]
        # stand-in for run_stream: finish each request of this rank's share
        for r in mine:
            r.admitted = r.arrival + 0.1
            r.finished = r.arrival + 1.0 + 1e-4 * r.nbf
            r.energies = np.array([-1.0 * rank, -float(r.nbf)])
        got = serve.gather_finished(mine)
        np.save(out + ".r%d.npy" % rank,
                np.array([(r.name, r.nbf, r.arrival, r.finished, r.energies[-1]) for r in got], dtype=object),
                allow_pickle=True)
    finally:
        dist.destroy_process_group()


def test_gloo_ranks_gather_the_whole_stream(tmp_path):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    port = _free_port()
    out = str(tmp_path / "serve")
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    reqs = _stream()
    want = {r.name: (r.nbf, r.arrival) for r in reqs}
    for rank in range(2):
        got = np.load(out + ".r%d.npy" % rank, allow_pickle=True)
        assert sorted(g[0] for g in got) == sorted(want)
        for name, nbf, arrival, finished, e_last in got:
            assert nbf == want[name][0] and arrival == want[name][1]
            assert e_last == -float(nbf)
    stats = serve.latency_stats([_req(g) for g in np.load(out + ".r0.npy", allow_pickle=True)])
    assert stats["solves_per_s"] > 0


def _req(g):
    name, nbf, arrival, finished, _ = g
    q = serve.Request(name, None, None, arrival, nbf)
    q.finished = finished
    return q
