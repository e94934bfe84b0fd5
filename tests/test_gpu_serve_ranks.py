"""A served stream over two ranks (processes), through bench.py's served
workload launched by torch.distributed.run: each rank serves the requests
serve.route gives it and the statistics gather all of them.

With one GPU both ranks share it (they wait on one another only on the
host, through gloo); the path is the one a node with a GPU per rank takes.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_served_stream_on_two_ranks():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--workload", "served", "--count", "8", "--rate", "8"]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stderr[-3000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1                       # rank 0 alone prints
    d = json.loads(lines[0])
    assert d["n_gpus"] == 2
    assert d["requests_served"] == 8
    assert d["iterations_served"] > 0 and d["iterations_fp64"] > 0
    # every request of the stream was served once, on one of the ranks
    assert d["served_mixed"]["solves_per_s"] > 0 and d["sequential_fp64"]["solves_per_s"] > 0
    assert d["converged_within_1e-6"] == d["converged_requests"]
    assert d["converged_requests"] >= 1
