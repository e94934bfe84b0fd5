"""Seeded workload streams (CPU): sizes, ranges and determinism."""
import os

import numpy as np

import gtfock_b200 as gb
from gtfock_b200 import molecules as mol
from gtfock_b200 import serve, workloads


def test_batched_stream(tmp_path):
    a = workloads.batched(256, 2024)
    b = workloads.batched(256, 2024)
    assert [x[0] for x in a] == [x[0] for x in b]
    sizes = [x[3] for x in a]
    assert min(sizes) >= 14 and max(sizes) <= 320
    assert {x[2] for x in a} == {"sto-3g", "6-31g"}
    for name, atoms, basis, n in a[:16]:
        xyz = mol.write_xyz(atoms, os.path.join(str(tmp_path), name + ".xyz"))
        assert gb.BasisSet(mol.basis_file(basis), xyz).nbf == n


def test_served_stream(tmp_path):
    s = workloads.served(64, 7, 2.0)
    t = [x[0] for x in s]
    assert all(t[i] < t[i + 1] for i in range(len(t) - 1))
    sizes = np.array([x[4] for x in s])
    assert sizes.min() >= 20 and sizes.max() <= 1500
    # log-uniform: both halves of the log range are populated
    mid = np.sqrt(20 * 1500)
    assert (sizes < mid).sum() > 10 and (sizes > mid).sum() > 10
    for t0, name, atoms, basis, n in s[:8]:
        xyz = mol.write_xyz(atoms, os.path.join(str(tmp_path), name + ".xyz"))
        assert gb.BasisSet(mol.basis_file(basis), xyz).nbf == n


def test_latency_stats():
    rs = []
    for k in range(10):
        r = serve.Request("r%d" % k, [], "sto-3g", arrival=float(k))
        r.finished = k + 1.0 + 0.1 * k
        rs.append(r)
    st = serve.latency_stats(rs)
    assert abs(st["p50_s"] - 1.45) < 1e-9
    assert st["makespan_s"] == rs[-1].finished
