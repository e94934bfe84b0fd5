"""SCF serving loop over the batched engine (continuous batching).

A request is an SCF job (geometry + basis name).  The server keeps up to
`slots` jobs per size lane resident on the device and advances the jobs of a
lane together, one SCF iteration per step (gtf_batch_step); a job leaves when
its energy has converged (|E_k - E_k-1| < etol) or after max_iters
iterations, and a waiting request is admitted as soon as a slot of its lane
is free and its estimated device footprint fits the memory budget.  Requests that arrive while others are on
the GPU therefore join the running batch between two steps, and their
iterations overlap with those of the jobs already running.

run_stream() replays an arrival stream against the wall clock and returns,
per request, its arrival, admission and completion times and its energies.
run_sequential() serves the same stream one job at a time on the
single-job GPU path (gtf_scf_*), FIFO -- by default the plain FP64 path, for
comparison.

Admission is by HBM footprint (Admission): the estimated bytes of a waiting
request must fit the budget left by the jobs on the device, each counted at
its measured size, and the device's free memory at that moment.

Several GPUs serve one stream with one process (and one server) each and no
exchange between them: route() assigns every request to a rank from the
stream alone, so each process keeps its own share; split_jobs() does the
same for a fixed set of molecules; gather_finished() brings the finished
requests to every rank for the statistics.
"""
import os
import tempfile
import threading
import time

import numpy as np

from . import BasisSet, Batch, SCFSolver, device_memory, device_trim, set_device
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
        self.cancelled = False


def footprint_bytes(nbf, incremental=False):
    """Estimated device bytes of one job before it is set up: batch buffers
    plus the Fock engine's matrices (D, F, J, K, S, X, H, Cartesian scratch),
    pair data and task lists (bounded by 64 nbf^2 doubles for the bases used
    here), plus the previous density and the density change of incremental
    builds.  Once a job runs, the server holds its measured bytes instead."""
    return Batch.job_bytes(nbf) + 8 * (64 + (3 if incremental else 0)) * nbf * nbf


class Admission:
    """HBM-footprint admission.

    A request is admitted when its footprint fits the budget left (what the
    admitted jobs hold counted against `budget`) and, at that moment, the
    device's free memory less `reserve` (room for the set-up's temporaries).
    The budget defaults to the device's free memory when the server starts,
    less the reserve.  `free_fn` returns the device's free bytes (default:
    cudaMemGetInfo through gtf_device_memory)."""

    def __init__(self, budget=None, reserve=2 << 30, free_fn=None):
        self.free_fn = free_fn or (lambda: device_memory()[0])
        self.reserve = int(reserve)
        self.budget = int(self.free_fn() - self.reserve) if budget is None else int(budget)
        self.held = {}

    @property
    def used(self):
        return sum(self.held.values())

    def fits(self, nbytes):
        return self.used + nbytes <= self.budget and nbytes + self.reserve <= self.free_fn()

    def hold(self, key, nbytes):
        self.held[key] = int(nbytes)

    def release(self, key):
        self.held.pop(key, None)


class _Lane:
    def __init__(self, max_nbf, slots):
        self.max_nbf = max_nbf
        self.batch = Batch(slots)
        self.slots = slots
        self.live = {}
        self.ms = None          # moving average of a step's wall time
        # serialises this lane's batch calls (admission from the serving
        # thread, steps from the lane's own thread in concurrent mode)
        self.lock = threading.Lock()

    def fits(self, nbf):
        return self.max_nbf is None or nbf <= self.max_nbf


class SCFServer:
    """Continuous-batching SCF server.

    Requests are routed by size into lanes (default: up to 400 functions, and
    the rest), each a batch stepped in lock-step.  Steps of the lanes share
    the GPU: when several lanes have live jobs, the small-molecule lane runs
    until its step time adds up to `share` times the large lane's step, then
    the large lane takes one step -- so small jobs are not held to the pace of
    a 1000-function molecule, while the large ones keep progressing."""

    def __init__(self, slots=64, mem_budget=None, precision=1, fp32_cutoff=1e-4, max_iters=30,
                 etol=1e-6, tolscr=1e-10, lanes=((400, None), (None, None)), share=0.5,
                 incremental=False, incr_tau=0.0, incr_period=8, reserve=2 << 30, free_fn=None,
                 concurrent=False, device=None):
        # device: the GPU of this server (one process per GPU); the batches
        # are created on it, and the lane threads select it when they start
        self.device = device
        if device is not None:
            set_device(device)
        self.admission = Admission(mem_budget, reserve, free_fn)
        self._mu = threading.Lock()   # admission state
        # concurrent: run_stream steps every lane from a thread of its own,
        # so the lanes' launches (each batch has its own CUDA stream) overlap
        # on the GPU instead of taking turns
        self.concurrent = bool(concurrent)
        self.lanes = [_Lane(m, n if n else slots) for m, n in lanes]
        self.incremental = bool(incremental)
        if self.incremental:
            for ln in self.lanes:
                ln.batch.set_incremental(True, incr_tau, incr_period)
        self.share = share
        self.kw = dict(tolscr=tolscr, precision=precision, fp32_cutoff=fp32_cutoff, max_iters=max_iters,
                       etol=etol)
        self.credit = 0.0
        self.tmp = tempfile.mkdtemp(prefix="gtf_serve_")
        # host-side time accounting: job set-up (Batch.add), removal, and
        # the steps of each lane, in seconds
        self.stats = {"adds": 0, "add_s": 0.0, "prepare_s": 0.0, "attach_s": 0.0, "removes": 0, "remove_s": 0.0,
                      "steps": [0] * len(self.lanes), "step_s": [0.0] * len(self.lanes)}

    @property
    def mem_used(self):
        return self.admission.used

    @property
    def live(self):
        return {(k, s): r for k, ln in enumerate(self.lanes) for s, r in list(ln.live.items())}

    def has_live(self):
        return any(len(ln.live) for ln in self.lanes)

    def _xyz(self, r):
        if r.xyz is None:
            r.xyz = mol.write_xyz(r.atoms, os.path.join(self.tmp, r.name + ".xyz"), r.name)
        return r.xyz

    def _nbf(self, r):
        """The request's basis size (from its basis and geometry when not given)."""
        if r.nbf is None:
            b = BasisSet(mol.basis_file(r.basis), self._xyz(r))
            r.nbf = b.nbf
        return r.nbf

    def _lane(self, r):
        for ln in self.lanes:
            if ln.fits(self._nbf(r)):
                return ln
        return self.lanes[-1]

    def footprint(self, r):
        return footprint_bytes(self._nbf(r), self.incremental)

    def can_admit(self, r):
        ln = self._lane(r)
        with self._mu:
            return len(ln.live) < ln.slots and self.admission.fits(self.footprint(r))

    def admit(self, r, now):
        ln = self._lane(r)
        kw = self.kw
        # the set-up runs while the lane keeps stepping; only the attach
        # (batch buffers, slot) waits for the lane between two steps
        t0 = time.perf_counter()
        job = ln.batch.prepare(mol.basis_file(r.basis), self._xyz(r), tolscr=kw["tolscr"],
                               precision=kw["precision"], fp32_cutoff=kw["fp32_cutoff"])
        t1 = time.perf_counter()
        with ln.lock:
            t2 = time.perf_counter()
            r.slot = ln.batch.attach(job, max_iters=kw["max_iters"], etol=kw["etol"])
            self.stats["prepare_s"] += t1 - t0
            self.stats["attach_s"] += time.perf_counter() - t2
            self.stats["add_s"] += time.perf_counter() - t0
            self.stats["adds"] += 1
            r.admitted = now
            ln.live[r.slot] = r
            nbytes = ln.batch.job_device_bytes(r.slot)
        # the job's measured device bytes replace the estimate
        with self._mu:
            self.admission.hold(id(r), nbytes)

    def cancel(self, r):
        """Withdraw a live request between steps: its slot and memory are
        freed; the other jobs continue unaffected."""
        for ln in self.lanes:
            with ln.lock:
                if ln.live.get(r.slot) is r:
                    ln.live.pop(r.slot)
                    ln.batch.remove(r.slot)
                    with self._mu:
                        self.admission.release(id(r))
                    r.cancelled = True
                    return True
        return False

    def _pick(self):
        busy = [ln for ln in self.lanes if ln.live]
        if len(busy) <= 1:
            return busy[0] if busy else None
        small, large = busy[0], busy[-1]
        if large.ms is None or self.credit < self.share * large.ms:
            return small
        return large

    def step(self, now_fn):
        """One SCF iteration of every live job of one lane (the lanes take
        turns); returns the requests that finished."""
        ln = self._pick()
        if ln is None:
            return []
        busy = [x for x in self.lanes if x.live]   # before this step's jobs leave
        t0 = time.perf_counter()
        done = self.step_lane(ln, now_fn)
        dt = (time.perf_counter() - t0) * 1e3
        ln.ms = dt if ln.ms is None else 0.7 * ln.ms + 0.3 * dt
        if ln is busy[-1] and len(busy) > 1:
            self.credit = 0.0
        else:
            self.credit += dt
        return done

    def step_lane(self, ln, now_fn):
        """One SCF iteration of every live job of lane `ln`."""
        done = []
        with ln.lock:
            if not ln.live:
                return done
            k = self.lanes.index(ln)
            t0 = time.perf_counter()
            ln.batch.step()
            self.stats["step_s"][k] += time.perf_counter() - t0
            self.stats["steps"][k] += 1
            for s in list(ln.live):
                e, fin = ln.batch.result(s)
                if fin:
                    r = ln.live.pop(s)
                    r.energies = e
                    r.finished = now_fn()
                    t1 = time.perf_counter()
                    ln.batch.remove(s)
                    self.stats["remove_s"] += time.perf_counter() - t1
                    self.stats["removes"] += 1
                    with self._mu:
                        self.admission.release(id(r))
                    done.append(r)
        return done

    def close(self):
        for ln in self.lanes:
            ln.batch.close()
        device_trim(0)   # the jobs' cached device memory back to the driver


def run_stream(requests, server):
    """Replay `requests` (sorted by arrival, seconds from start) against the
    wall clock through `server`; returns the finished requests."""
    if server.concurrent:
        return _run_stream_concurrent(requests, server)
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
        # admit, in arrival order, every waiting request whose lane has room
        # (a full lane does not hold back requests for the other lanes)
        for r in list(waiting):
            if server.can_admit(r):
                waiting.remove(r)
                server.admit(r, now())
        if server.live:
            finished += server.step(now)
        elif pending:
            time.sleep(max(0.0, min(0.01, pending[0].arrival - now())))
        elif waiting:
            raise RuntimeError("request %s (%d functions, %.2f GB estimated) does not fit the device memory "
                               "budget of %.2f GB" % (waiting[0].name, waiting[0].nbf or 0,
                                                      server.footprint(waiting[0]) / 1e9,
                                                      server.admission.budget / 1e9))
    return finished


def _run_stream_concurrent(requests, server):
    """run_stream with one stepping thread per lane: the serving thread
    admits arriving requests; each lane's thread steps its batch while it has
    live jobs.  The library's calls release the GIL, so the lanes' CUDA
    streams run at the same time."""
    pending = sorted(requests, key=lambda r: r.arrival)
    for r in pending:
        server._xyz(r)
        server._nbf(r)
    t0 = time.perf_counter()
    now = lambda: time.perf_counter() - t0  # noqa: E731
    finished = []
    fin_mu = threading.Lock()
    stop = threading.Event()
    errors = []

    def lane_loop(ln):
        try:
            if server.device is not None:
                set_device(server.device)   # a new thread starts on device 0
            while not stop.is_set():
                if ln.live:
                    done = server.step_lane(ln, now)
                    if done:
                        with fin_mu:
                            finished.extend(done)
                else:
                    time.sleep(0.0005)
        except Exception as e:  # surfaced by the serving thread
            errors.append(e)
            stop.set()

    threads = [threading.Thread(target=lane_loop, args=(ln,), daemon=True) for ln in server.lanes]
    for th in threads:
        th.start()
    waiting = []
    try:
        while (pending or waiting or server.has_live()) and not errors:
            t = now()
            while pending and pending[0].arrival <= t:
                waiting.append(pending.pop(0))
            for r in list(waiting):
                if server.can_admit(r):
                    waiting.remove(r)
                    server.admit(r, now())
            if waiting and not pending and not server.has_live():
                raise RuntimeError("request %s (%d functions, %.2f GB estimated) does not fit the device "
                                   "memory budget of %.2f GB" % (waiting[0].name, waiting[0].nbf or 0,
                                                                 server.footprint(waiting[0]) / 1e9,
                                                                 server.admission.budget / 1e9))
            time.sleep(0.0005)
    finally:
        stop.set()
        for th in threads:
            th.join()
    if errors:
        raise errors[0]
    return finished


def run_sequential(requests, max_iters=30, etol=1e-6, tolscr=1e-10, precision=0, fp32_cutoff=0.0,
                   incremental=False, incr_tau=0.0, incr_period=8):
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
        s.set_options(precision=precision, fp32_cutoff=fp32_cutoff, etol=etol)
        if incremental:
            s.set_incremental(True, incr_tau, incr_period)
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


def est_seconds(nbf):
    """Rough service time of one request on one B200, in seconds: set-up plus
    20-30 SCF iterations whose Fock builds grow about as nbf^3 over 20-1500
    functions (1430 functions: about 5 s)."""
    return 0.05 + 1.7e-9 * float(nbf) ** 3


def route(requests, nranks):
    """Rank (0 .. nranks-1) of each request when `nranks` GPUs serve one
    stream, one process each: in arrival order, a request goes to the rank
    whose estimated backlog clears first (list scheduling on est_seconds;
    among ranks already idle, the one idle longest, then the lower rank).
    The assignment depends on the stream alone, so every process computes
    the same one and keeps its own share."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    out = [0] * len(requests)
    if nranks == 1:
        return out
    free = [0.0] * nranks
    order = sorted(range(len(requests)), key=lambda i: (requests[i].arrival, requests[i].name))
    for i in order:
        r = requests[i]
        if r.nbf is None:
            raise ValueError("route needs the basis size of request %s" % r.name)
        k = min(range(nranks), key=lambda j: (max(free[j], r.arrival), free[j], j))
        free[k] = max(free[k], r.arrival) + est_seconds(r.nbf)
        out[i] = k
    return out


def split_jobs(nbfs, nranks):
    """Rank of each molecule of a fixed batch over `nranks` GPUs: the
    costliest first, each to the least-loaded rank (est_seconds; ties to the
    lower rank)."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    load = [0.0] * nranks
    out = [0] * len(nbfs)
    for i in sorted(range(len(nbfs)), key=lambda i: (-nbfs[i], i)):
        k = min(range(nranks), key=lambda j: (load[j], j))
        load[k] += est_seconds(nbfs[i])
        out[i] = k
    return out


def gather_finished(done, group=None):
    """The finished requests of every rank, on every rank, as Request
    objects without geometry (name, basis size, arrival, admission and
    completion times, energies), through torch.distributed's object
    all-gather on `group` (the default group when None).  Each rank's times
    are seconds from its own start of the stream; the ranks start together
    after a barrier."""
    import torch.distributed as dist
    mine = [(r.name, r.nbf, r.arrival, r.admitted, r.finished,
             [float(e) for e in (r.energies if r.energies is not None else [])]) for r in done]
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, mine, group=group)
    out = []
    for part in parts:
        for name, nbf, arrival, admitted, finished, energies in part:
            q = Request(name, None, None, arrival, nbf)
            q.admitted, q.finished, q.energies = admitted, finished, np.array(energies)
            out.append(q)
    return out
