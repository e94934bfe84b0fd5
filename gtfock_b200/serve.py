"""SCF serving loop over the batched engine (continuous batching).

A request is an SCF job (geometry + basis name).  The server keeps up to
`slots` jobs resident on the device and advances all of them together, one
SCF iteration per step (gtf_batch_step); a job leaves when its energy has
converged (|E_k - E_k-1| < etol) or after max_iters iterations, and a waiting
request is admitted as soon as a slot is free and its estimated device
footprint fits the memory budget.  Requests that arrive while others are on
the GPU therefore join the running batch between two steps, and their
iterations overlap with those of the jobs already running.

run_stream() replays an arrival stream against the wall clock and returns,
per request, its arrival, admission and completion times and its energies.
run_sequential() serves the same stream one job at a time on the plain
single-job GPU path (gtf_scf_*), FIFO, for comparison.
"""
import os
import tempfile
import time

import numpy as np

from . import Batch, SCFSolver
from . import molecules as mol


class Request:
    def __init__(self, name, atoms, basis, arrival=0.0, nbf=None):
        self.name = name
        self.atoms = atoms
        self.basis = basis
        self.arrival = arrival
        self.nbf = nbf
        self.xyz = None
        self.admitted = None
        self.finished = None
        self.energies = None
        self.slot = None


def footprint_bytes(nbf):
    """Device bytes of one job: batch buffers plus the Fock engine's matrices
    (D, F, J, K, S, X, H, Cartesian scratch) and pair data (bounded by 64 nbf^2
    doubles for the bases used here)."""
    return Batch.job_bytes(nbf) + 8 * 64 * nbf * nbf


class SCFServer:
    def __init__(self, slots=64, mem_budget=64 << 30, precision=1, fp32_cutoff=1e-6, max_iters=30,
                 etol=1e-6, tolscr=1e-10):
        self.batch = Batch(slots)
        self.slots = slots
        self.mem_budget = mem_budget
        self.kw = dict(tolscr=tolscr, precision=precision, fp32_cutoff=fp32_cutoff, max_iters=max_iters,
                       etol=etol)
        self.live = {}
        self.mem_used = 0
        self.tmp = tempfile.mkdtemp(prefix="gtf_serve_")

    def _xyz(self, r):
        if r.xyz is None:
            r.xyz = mol.write_xyz(r.atoms, os.path.join(self.tmp, r.name + ".xyz"), r.name)
        return r.xyz

    def can_admit(self, r):
        need = footprint_bytes(r.nbf or 1)
        return len(self.live) < self.slots and self.mem_used + need <= self.mem_budget

    def admit(self, r, now):
        r.slot = self.batch.add(mol.basis_file(r.basis), self._xyz(r), **self.kw)
        r.admitted = now
        self.live[r.slot] = r
        self.mem_used += footprint_bytes(r.nbf or 1)

    def step(self, now_fn):
        """One SCF iteration of every live job; returns the requests that finished."""
        if not self.live:
            return []
        self.batch.step()
        done = []
        for s in list(self.live):
            e, fin = self.batch.result(s)
            if fin:
                r = self.live.pop(s)
                r.energies = e
                r.finished = now_fn()
                self.batch.remove(s)
                self.mem_used -= footprint_bytes(r.nbf or 1)
                done.append(r)
        return done

    def close(self):
        self.batch.close()


def run_stream(requests, server):
    """Replay `requests` (sorted by arrival, seconds from start) against the
    wall clock through `server`; returns the finished requests."""
    pending = sorted(requests, key=lambda r: r.arrival)
    for r in pending:
        server._xyz(r)
    t0 = time.perf_counter()
    now = lambda: time.perf_counter() - t0  # noqa: E731
    finished = []
    waiting = []
    while pending or waiting or server.live:
        t = now()
        while pending and pending[0].arrival <= t:
            waiting.append(pending.pop(0))
        while waiting and server.can_admit(waiting[0]):
            server.admit(waiting.pop(0), now())
        if server.live:
            finished += server.step(now)
        elif pending:
            time.sleep(max(0.0, min(0.01, pending[0].arrival - now())))
        elif waiting:
            raise RuntimeError("request %s does not fit the server" % waiting[0].name)
    return finished


def run_sequential(requests, max_iters=30, etol=1e-6, tolscr=1e-10):
    """The same stream on the plain FP64 single-job GPU path, FIFO: each job's
    service time (set-up + solve) is measured alone; its completion time is
    max(arrival, previous completion) + service."""
    tmp = tempfile.mkdtemp(prefix="gtf_seq_")
    clock = 0.0
    out = []
    for r in sorted(requests, key=lambda q: q.arrival):
        xyz = r.xyz or mol.write_xyz(r.atoms, os.path.join(tmp, r.name + ".xyz"), r.name)
        t1 = time.perf_counter()
        s = SCFSolver(mol.basis_file(r.basis), xyz, tolscr=tolscr)
        s.set_options(precision=0, etol=etol)
        e, _ = s.solve(niters=max_iters)
        s.close()
        service = time.perf_counter() - t1
        start = max(clock, r.arrival)
        clock = start + service
        q = Request(r.name, r.atoms, r.basis, r.arrival, r.nbf)
        q.admitted = start
        q.finished = clock
        q.energies = e
        out.append(q)
    return out


def latency_stats(done):
    lat = np.array([r.finished - r.arrival for r in done])
    span = max(r.finished for r in done) - min(r.arrival for r in done)
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "solves_per_s": len(done) / span, "makespan_s": span}
