"""Benchmark: SCF solves/s of the Fock-build + purification path on one B200.

Workload (default): C54H18 hexagonal graphene flake (C-C 1.42 A, C-H 1.09 A),
cc-pVDZ (846 functions), Schwarz threshold 1e-10, 10 SCF iterations from the
core-Hamiltonian guess, all FP64.  One step = one SCF solve.

  value      SCF solves/s with the engine set up and D/F/S/X/H resident on the
             device (gtf_scf_solve, mode 1), CUDA-event timed on the engine's
             stream; max over ranks.
  e2e        SCF solves/s through the reference-facing C API with host
             buffers (gtf_scf_run, mode 0: basis load, PFock_create, one-
             electron set-up, and every iteration's putDenMat / getMat /
             compute_diis / compute_purification host<->device copies).
  roofline   the electron-repulsion kernels of one Fock build: Rys-model FLOPs
             (normalisation of the quartet work) / their CUDA-event time,
             against this device's FP64 FMA rate measured in-run by a probe
             kernel (no FP64 figure exists in MEASURED_PEAKS.json).
  cpu_baseline  the CPU restatement of the reference path (oracle/) on all
             host cores: a bounded sample of one Fock build (every k-th bra
             shell pair) scaled by the quartet-count ratio, plus one measured
             DIIS + purification step, extrapolated to the solve.

--impl reference prints the same metric for the reference's CPU path (the
oracle port, sampled as above), as the reference arm.
Multi-GPU: molecules are independent, so N GPUs run N replicas of the solve
(no collective); value = N solves / max-over-ranks time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

TOL = 1e-10
NITER = 10
MIXED_CUTOFF = 1e-6
# served and batched forms: FP32 quartets below a Schwarz bound of 1e-4
# (profiles/precision_sweep_w64.md: |dE| 6.8e-10 Ha at 1e-4 on (H2O)64)
SERVED_CUTOFF = 1e-4
# size lanes of the server: (largest basis of the lane, slots); None = no limit
LANES = {1: ((None, None),), 2: ((400, None), (None, None)), 3: ((400, None), (800, None), (None, None))}
INCR_PERIOD = 8          # incremental builds: a full build every 8 builds
# served form: quartets of the density change dropped below bound x max|dD| <
# 1e-9 (profiles/served_form_tau_sweep_w74.md: no measurable error added)
SERVED_TAU = 1e-9
SERVED_COUNT = 32        # requests of the served stream in the default run
# DRAM bytes (read + write) of all k_fock launches of one C54H18 build, from one
# ncu capture (profiles/fock_c54h18_dram_traffic.md); the kernels are FP64 bound
FOCK_BUILD_DRAM_BYTES = 648.2e6 + 84.9e6
METRIC = "SCF solves/s (C54H18 cc-pVDZ, 10 iterations, FP64)"
WORKLOAD = "C54H18 graphene flake / cc-pVDZ (846 bf), Schwarz 1e-10, 10 SCF iterations, FP64"


def _dist():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class _Ranks:
    """The ranks of a batched or served workload on several GPUs (one
    process each, launched by torch.distributed.run): each serves its own
    share of the molecules or requests, with no exchange on the data path;
    a gloo group carries the barriers and the gathers of the results.  On
    one GPU every method is a no-op."""

    def __init__(self):
        self.rank, self.world, self.local = _dist()
        self.dist = None
        self.device = None
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            import gtfock_b200 as gb
            # one rank per GPU; more ranks than GPUs share them in turn (the
            # ranks never wait on one another's kernels, only on the host)
            ndev = max(1, gb.device_info()[0])
            self.device = self.local % ndev
            gb.set_device(self.device)
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=1800))
            self.dist = dist

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def gather(self, obj):
        """Every rank's obj, in rank order (a one-element list on one GPU)."""
        if not self.dist:
            return [obj]
        parts = [None] * self.world
        self.dist.all_gather_object(parts, obj)
        return parts

    def close(self):
        if self.dist:
            self.dist.destroy_process_group()
            self.dist = None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons every 200 ms while running."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def make_workload(td):
    from gtfock_b200 import molecules as mol
    xyz = mol.write_xyz(mol.graphene_flake(2), os.path.join(td, "c54h18.xyz"), "C54H18")
    return mol.basis_file("cc-pvdz"), xyz


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def cpu_baseline(gbs, xyz, target_s=15.0):
    """Sampled CPU restatement of one SCF solve on all host cores."""
    import numpy as np
    from oracle import pyoracle as po
    cores = os.cpu_count()
    b = po.Basis(gbs, xyz)
    po.lib().or_set_blas_threads(cores)
    scr = po.screening(b, TOL, cores)
    D = np.eye(b.nbf) * 0.3
    usq_total, _, _ = po.fock_build_sample(b, TOL, D, 1, count_only=True, scr=scr, nthreads=cores)
    # calibrate the stride on small samples until one takes ~target_s
    stride = 4096
    usq_s, _, dt = po.fock_build_sample(b, TOL, D, stride, scr=scr, nthreads=cores)
    for _ in range(3):
        if dt >= 0.6 * target_s or stride == 1 or usq_s == 0:
            break
        stride = max(1, int(stride * dt / target_s)) if dt > 0.05 else max(1, stride // 8)
        usq_s, _, dt = po.fock_build_sample(b, TOL, D, stride, scr=scr, nthreads=cores)
    t_fock = dt * usq_total / usq_s
    # one DIIS step (iter > 1 form, 6 GEMMs) + one purification, full size
    S, H, X = po.one_electron(b)
    F = H.copy()
    state = None
    t_diis = 0.0
    for it in range(3):
        F2, t, state = po.diis_step_timed(X, S, D, F, it, state)
        t_diis = t
    t0 = time.perf_counter()
    _, pits = po.purification(b.nocc, X, F2)
    t_pur = time.perf_counter() - t0
    t_solve = NITER * (t_fock + t_diis + t_pur)
    return {
        "value": 1.0 / t_solve, "unit": "solves/s", "cores": cores, "kind": "port",
        "sample": "every %d-th bra shell pair of one C54H18/cc-pVDZ Fock build (%d of %d quartets, "
                  "%.1f s) scaled by the quartet ratio; DIIS + purification (%d iterations) timed "
                  "once at full size; x%d iterations" % (stride, usq_s, usq_total, dt, pits, NITER),
        "fock_build_s_est": t_fock, "diis_s": t_diis, "purif_s": t_pur,
    }


def reference_driver_c12h26(cores):
    """GTFock's own SCF driver (pscf/scf.c with pfock/*.c and pscf/purif.c,
    compiled unchanged by oracle/ref/Makefile into oracle/_ref/scf_ref) on
    C12H26 / cc-pVDZ, 10 iterations, on `cores` host threads: wall time of the
    whole run and its last energies.  None when the binary was not built."""
    from gtfock_b200 import molecules as mol
    exe = os.path.join(ROOT, "oracle", "_ref", "scf_ref")
    if not os.path.exists(exe):
        return None
    with tempfile.TemporaryDirectory() as td:
        xyz = mol.write_xyz(mol.alkane(12), os.path.join(td, "c12h26.xyz"))
        env = dict(os.environ, OMP_NUM_THREADS=str(cores))
        t0 = time.perf_counter()
        out = subprocess.run([exe, mol.basis_file("cc-pvdz"), xyz, "1", "1", "1", "4", str(NITER)], env=env,
                             capture_output=True, text=True, timeout=1200)
        dt = time.perf_counter() - t0
    es = [float(l.split()[1]) for l in out.stdout.splitlines() if l.strip().startswith("energy")]
    return {"workload": "C12H26 / cc-pVDZ (298 bf), 10 SCF iterations, FP64 (the driver's own Schwarz 1e-11)",
            "kind": "reference", "cores": cores, "rc": out.returncode, "solve_s": dt, "solves_per_s": 1.0 / dt,
            "energies_last": es[-3:]}


def run_reference(args):
    rank, world, _ = _dist()
    if rank != 0:
        return
    with tempfile.TemporaryDirectory() as td:
        gbs, xyz = make_workload(td)
        per = []
        walls = []
        for _ in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            per.append(cpu_baseline(gbs, xyz, target_s=4.0))
            walls.append(time.perf_counter() - t0)
        timed = per[args.warmup:]
        v = statistics.median([p["value"] for p in timed])
        cb = dict(timed[-1])
        cb["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            # a step is a bounded sample of the solve: its own wall time here,
            # the solve time it extrapolates to below
            "ms_per_step": 1000.0 * statistics.median(walls[args.warmup:]),
            "extrapolated_ms_per_solve": 1000.0 / v,
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "parallelism": "cpu (%d threads)" % cb["cores"]},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    line["cpu_baseline"]["estimate"] = ("value extrapolated from each step's sample (every k-th bra pair of one "
                                        "build, scaled by the quartet ratio, x10 iterations)")
    # one measured (not extrapolated) run of the reference's own driver on the
    # CPU-runnable configuration, for the ratio on a case both sides finish
    line["measured_c12h26"] = reference_driver_c12h26(os.cpu_count())
    print(json.dumps(line), flush=True)


def run(args):
    import numpy as np
    import gtfock_b200 as gb
    rank, world, local = _dist()
    pg = None
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
        pg = dist
    os.environ.setdefault("CUDA_VISIBLE_DEVICES", os.environ.get("CUDA_VISIBLE_DEVICES", ""))
    n, cc = gb.device_info()
    if n < 1:
        raise SystemExit("no CUDA device")
    with tempfile.TemporaryDirectory() as td:
        gbs, xyz = make_workload(td)
        solver = gb.SCFSolver(gbs, xyz, TOL)
        nbf = solver.nbf
        # warm-up solves (device-resident)
        for _ in range(args.warmup):
            e_warm, _ = solver.solve(NITER, device_resident=True)
        # timed region: value (device-resident)
        if pg:
            pg.barrier()
        l0 = gb.launch_count()
        with ClockSampler(local) as clk:
            t0 = time.perf_counter()
            energies = None
            fock_s = diis_s = pur_s = 0.0
            for _ in range(args.steps):
                energies, tm = solver.solve(NITER, device_resident=True)
                fock_s += tm["fock_s"]
                diis_s += tm["diis_s"]
                pur_s += tm["purif_s"]
            dt = time.perf_counter() - t0
        launches = gb.launch_count() - l0
        if pg:
            import torch
            t = torch.tensor([dt], device="cuda")
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            dt = float(t.item())
        clocks = clk.summary()
        # the same solves with FP32 quartets below a Schwarz bound of 1e-6
        solver.set_options(precision=1, fp32_cutoff=MIXED_CUTOFF, etol=1e-11)
        solver.solve(NITER, device_resident=True)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e_mixed, tm_m = solver.solve(NITER, device_resident=True)
        dt_mixed = time.perf_counter() - t0
        solver.set_options(precision=0, etol=1e-11)
        # one Fock build's ERI kernels for the roofline
        pf_basis = gb.BasisSet(gbs, xyz)
        pf = gb.PFock(pf_basis, tolscr=TOL)
        D = np.eye(nbf) * 0.3
        eri_ms = []
        for k in range(4):
            pf.compute_fock(D)
            if k:
                eri_ms.append(pf.timing()["ms_eri"])
        tm = pf.timing()
        counts = pf.counts()
        eri_flops = tm["eri_flops"]
        # the same model over the primitive quartets the kernels evaluate
        # (after primitive screening at |K_ab K_cd| < 1e-17)
        scr = pf.class_work_screened()
        eri_flops_scr = sum(w[0] for w in scr)
        primq_scr = sum(w[1] for w in scr)
        primq_all = sum(w[1] for w in pf.class_work())
        pf.close()
        solver.close()
        # e2e through the C API with host buffers (set-up included); the
        # median of at least 3 timed runs, since from the core-Hamiltonian
        # guess the purification step counts (and so the solve time) vary
        # from run to run
        e2e_times = []
        e2e_bytes = (0, 0)
        for k in range(1 + max(3, args.steps)):
            t1 = time.perf_counter()
            e_e2e, te = gb.scf_run(gbs, xyz, TOL, NITER, device_resident=False)
            if k:
                e2e_times.append(time.perf_counter() - t1)
            e2e_bytes = (te["h2d_bytes"], te["d2h_bytes"])
        fp64_peak = gb.fp64_peak_gflops()
    value = world * args.steps / dt
    eri_s = statistics.median(eri_ms) * 1e-3
    achieved = eri_flops / eri_s / 1e12
    peak = fp64_peak / 1e3
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1000.0,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (generated C54H18 geometry)",
        "config": {"workload": WORKLOAD, "nbf": nbf, "parallelism": "replicas x%d" % world,
                   "l2": "inputs resident; F/D working set (2 x 5.7 MB) stays in L2 by design",
                   "usq": counts["usq"], "uitl": counts["uitl"], "nnz_pairs": counts["nnz"]},
        "energy_last": float(energies[-1]) if energies is not None else None,
        "phase_s_per_solve": {"fock": fock_s / args.steps, "diis": diis_s / args.steps,
                              "purification": pur_s / args.steps},
        "e2e": {"value": 1.0 / statistics.median(e2e_times), "unit": "solves/s",
                "h2d_bytes_per_step": int(e2e_bytes[0]), "d2h_bytes_per_step": int(e2e_bytes[1])},
        "gpu_launches": int(launches),
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": FOCK_BUILD_DRAM_BYTES,
                     "traffic_unit": "bytes per build (ncu dram__bytes_read + write, profiles/)",
                     "kernel": "k_fock<*> (all class pairs of one Fock build)",
                     "peak_source": "FP64 FMA probe kernel measured in this run "
                                    "(MEASURED_PEAKS.json has no FP64 figure)",
                     "work": "Rys-model FLOPs per build %.4g, over every primitive quartet of every "
                             "screened quartet (before primitive screening)" % eri_flops,
                     "eri_ms_per_build": eri_s * 1e3,
                     "after_primitive_screening": {
                         "work_flops": eri_flops_scr, "primitive_quartets": primq_scr,
                         "primitive_quartets_before": primq_all,
                         "achieved": eri_flops_scr / eri_s / 1e12,
                         "frac": eri_flops_scr / eri_s / 1e12 / peak}},
        "clocks": clocks,
        "mixed_precision": {"value": world * args.steps / dt_mixed, "unit": "solves/s",
                            "fp32_cutoff": MIXED_CUTOFF,
                            "dE_last_vs_fp64": float(abs(e_mixed[-1] - energies[-1])),
                            "note": "FP32 ERIs for quartets with Schwarz bound below the cutoff; "
                                    "digestion and F accumulation FP64. The 10-iteration C54H18 SCF "
                                    "from the core-Hamiltonian guess is not converged and its iterates "
                                    "differ by ~0.05 Ha between two FP64 runs (atomic summation "
                                    "order), so dE_last_vs_fp64 measures that, not the FP32 error; "
                                    "converged energies agree within 1e-11 Ha (--workload precision)"},
    }
    if world == 1 and not args.quick:
        # the headline metric's own forms, measured in the same run: the
        # served stream and the batched workload, each against the plain FP64
        # GPU path on the same molecules, and the CPU-runnable C12H26 solve
        line["served"] = served_measure(SERVED_COUNT, 7, 4.0, SERVED_CUTOFF, 64, 2, True, repeats=3)
        line["batched"] = batched_measure(256, 2024, SERVED_CUTOFF, True, 64)
        line["c12h26"] = c12h26_measure(3, 5)
        sv, bt = line["served"], line["batched"]
        line["served_target"] = {
            "served_speedup_vs_fp64": sv["speedup_solves_per_s"],
            "served_p50_s": sv["served_mixed"]["p50_s"], "served_p99_s": sv["served_mixed"]["p99_s"],
            "fp64_p50_s": sv["sequential_fp64"]["p50_s"], "fp64_p99_s": sv["sequential_fp64"]["p99_s"],
            "served_max_dE_vs_fp64": sv["max_dE_served_vs_fp64"],
            "served_converged_within_1e-6": "%d of %d" % (sv["converged_within_1e-6"], sv["converged_requests"]),
            "batched_speedup_vs_fp64": bt["speedup_batched_mixed_incremental_vs_sequential_fp64"],
            "batched_max_dE_vs_fp64": bt["max_dE_mixed_incremental_vs_fp64"],
            "target": ">= 4x solves/s with every converged energy within 1e-6 Ha of FP64"}
    if rank == 0 and not args.no_cpu_baseline:
        with tempfile.TemporaryDirectory() as td2:
            g2, x2 = make_workload(td2)
            cb = cpu_baseline(g2, x2)
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        line["cpu_baseline"]["estimate"] = ("extrapolated from the sample: the time of every k-th bra pair "
                                            "scaled by the quartet ratio, x10 iterations")
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def profile_fock(args):
    """A few Fock builds of one molecule with per-class-pair kernel times (the
    small cases profiled with ncu): c12h26 (298 bf) or c54h18 (846 bf)."""
    import numpy as np
    import gtfock_b200 as gb
    from gtfock_b200 import molecules as mol
    atoms = {"c12h26": mol.alkane(12), "c54h18": mol.graphene_flake(2),
             "c96h24": mol.graphene_flake(3), "w64": mol.water_cluster(64, 2024)}[args.profile_fock]
    with tempfile.TemporaryDirectory() as td:
        xyz = mol.write_xyz(atoms, os.path.join(td, args.profile_fock + ".xyz"))
        b = gb.BasisSet(mol.basis_file("6-31g" if args.profile_fock == "w64" else "cc-pvdz"), xyz)
        pf = gb.PFock(b, tolscr=TOL)
        if args.fp32_cutoff is not None:
            pf.set_precision(1, args.fp32_cutoff)
        D = np.eye(b.nbf) * 0.3
        tune = None
        if args.autotune:
            pf.compute_fock(D)
            t0 = time.perf_counter()
            pf.autotune(2)
            tune = {"seconds": time.perf_counter() - t0, "entries": gb.tune_entries()}
        for _ in range(args.builds):
            pf.compute_fock(D)
        tm = pf.timing()
        nq32, nq = pf.precision_stats()
        out = {"molecule": args.profile_fock, "nbf": b.nbf, "counts": pf.counts(), "timing": tm, "autotune": tune,
               "fp32_cutoff": args.fp32_cutoff, "fp32_share": nq32 / nq if nq else 0.0,
               "classes": [{"bra": x, "ket": y, "ms": ms, "quartets": q, "gflop": w[0] / 1e9,
                            "primq": w[1], "tflops": w[0] / ms / 1e9 if ms > 0 else 0.0}
                           for (x, y, ms, q), w in zip(pf.class_stats(), pf.class_work()) if q > 0]}
        pf.close()
    print(json.dumps(out), flush=True)


def run_setup(args):
    """Set-up steps of one solve through the C API, in the order pscf/scf.c
    calls them (basis, PFock_create, createOvlMat, createCoreHMat,
    create_purif) and their tear-down, for C54H18 / cc-pVDZ and
    (H2O)16 / 6-31G: the median of `steps` repeats after `warmup`, ms."""
    import gtfock_b200 as gb
    from gtfock_b200 import molecules as mol
    L = gb.load()
    out = {"workload": "set-up of one solve through the C API", "unit": "ms (median)", "molecules": []}
    with tempfile.TemporaryDirectory() as td:
        for name, atoms, bas in (("C54H18 / cc-pVDZ", mol.graphene_flake(2), "cc-pvdz"),
                                 ("(H2O)16 / 6-31G", mol.water_cluster(16, 7), "6-31g")):
            xyz = mol.write_xyz(atoms, os.path.join(td, "m.xyz"))
            rows = {k: [] for k in ("basis", "PFock_create", "createOvlMat", "createCoreHMat", "create_purif",
                                    "work_model", "destroy")}
            nbf = 0
            for k in range(args.warmup + args.steps):
                t = [time.perf_counter()]
                b = gb.BasisSet(mol.basis_file(bas), xyz)
                t.append(time.perf_counter())
                pf = gb.PFock(b, tolscr=TOL)
                t.append(time.perf_counter())
                L.PFock_createOvlMat(pf.h, b.h)
                t.append(time.perf_counter())
                L.PFock_createCoreHMat(pf.h, b.h)
                t.append(time.perf_counter())
                pr = gb.Purif(b)
                t.append(time.perf_counter())
                pf.timing()
                t.append(time.perf_counter())
                nbf = b.nbf
                pr.close()
                pf.close()
                b.close()
                t.append(time.perf_counter())
                if k >= args.warmup:
                    for key, a, z in zip(rows, t[:-1], t[1:]):
                        rows[key].append(1e3 * (z - a))
            out["molecules"].append({"molecule": name, "nbf": nbf,
                                     **{k: round(statistics.median(v), 3) for k, v in rows.items()}})
    print(json.dumps(out), flush=True)


def run_c12h26(args):
    print(json.dumps(c12h26_measure(args.warmup, args.steps)), flush=True)


def c12h26_measure(warmup, steps):
    """10-iteration SCF of C12H26 / cc-pVDZ (298 bf), the CPU-runnable
    configuration the reference's own driver is timed on (--impl reference):
    resident solves (mean of `steps` after `warmup`) and the median of five
    end-to-end runs from the host files through the C API (after a garbage
    collection of the Python heap, so that none falls inside them)."""
    import gtfock_b200 as gb
    from gtfock_b200 import molecules as mol
    with tempfile.TemporaryDirectory() as td:
        xyz = mol.write_xyz(mol.alkane(12), os.path.join(td, "c12h26.xyz"))
        gbs = mol.basis_file("cc-pvdz")
        s = gb.SCFSolver(gbs, xyz, tolscr=TOL)
        s.set_options(precision=0, etol=0.0)
        for _ in range(warmup):
            s.solve(niters=NITER)
        t0 = time.perf_counter()
        for _ in range(steps):
            e, tm = s.solve(niters=NITER)
        dt = (time.perf_counter() - t0) / steps
        s.close()
        import gc
        gc.collect()
        e2e = []
        for _ in range(5):
            t0 = time.perf_counter()
            e2, _ = gb.scf_run(gbs, xyz, TOL, NITER, device_resident=False)
            e2e.append(time.perf_counter() - t0)
    return {"workload": "C12H26 / cc-pVDZ (298 bf), Schwarz 1e-10, 10 SCF iterations, FP64",
            "solve_s": dt, "solves_per_s": 1.0 / dt, "fock_s_per_solve": tm["fock_s"],
            "purif_s_per_solve": tm["purif_s"], "e2e_solve_s": statistics.median(e2e),
            "e2e_solves_per_s": 1.0 / statistics.median(e2e), "energies": [float(x) for x in e[-3:]],
            "energy_last_e2e": float(e2[-1])}


def run_batch_scaling(args):
    """Large molecules in one batch: the Fock time per step of 1, 2 and 3
    copies of C54H18 / cc-pVDZ and of (H2O)64 / 6-31G against one build of
    the molecule alone, with the default solo-launch rule and, with
    GTFOCK_SOLO_UNITS set very high, with every launch batched."""
    import numpy as np
    import gtfock_b200 as gb
    from gtfock_b200 import molecules as mol
    out = {"workload": "1-3 copies of C54H18 / cc-pVDZ (846 bf) and (H2O)64 / 6-31G (832 bf) per batch, "
                       "Fock ms per SCF step (2 steps after 1)"}
    with tempfile.TemporaryDirectory() as td:
        for name, atoms, basis in (("c54h18", mol.graphene_flake(2), "cc-pvdz"),
                                   ("w64", mol.water_cluster(64, 2024), "6-31g")):
            xyz = mol.write_xyz(atoms, os.path.join(td, name + ".xyz"))
            gbs = mol.basis_file(basis)
            b = gb.BasisSet(gbs, xyz)
            pf = gb.PFock(b, tolscr=TOL)
            D = np.eye(b.nbf) * 0.3
            for _ in range(3):
                pf.compute_fock(D)
            out[name + "_single_ms"] = pf.timing()["ms_eri"]
            pf.close()
            for rule, env in (("solo_rule", None), ("all_batched", "1000000000000000")):
                if env:
                    os.environ["GTFOCK_SOLO_UNITS"] = env
                for m in (2, 3):
                    bt = gb.Batch(m)
                    for _ in range(m):
                        bt.add(gbs, xyz, tolscr=TOL, max_iters=4, etol=0.0)
                    bt.step()
                    i0 = bt.info()
                    bt.step()
                    bt.step()
                    i1 = bt.info()
                    out["%s_x%d_%s_ms" % (name, m, rule)] = (i1["ms_fock"] - i0["ms_fock"]) / 2
                    bt.close()
                os.environ.pop("GTFOCK_SOLO_UNITS", None)
    print(json.dumps(out), flush=True)


def run_batched(args):
    """Batched workload (--workload batched): see batched_measure."""
    rk = _Ranks()
    out = batched_measure(args.count, args.seed, args.fp32_cutoff if args.fp32_cutoff is not None else SERVED_CUTOFF,
                          args.autotune, args.seq_sample, rk)
    if rk.rank == 0:
        print(json.dumps(out), flush=True)
    rk.close()


def batched_measure(count, seed, cut, autotune, seq_sample, rk=None):
    """Batched workload: `count` seeded molecules (water clusters of 2-24 and
    alkanes C2-C16, STO-3G or 6-31G), 15 SCF iterations each.  Solves/s of the
    batched engine in FP64, in mixed precision, and in mixed precision with
    incremental Fock builds, against the plain FP64 GPU path solving the same
    molecules one after another (set-up excluded in all; it is reported
    separately).  On several GPUs (rk) each rank batches its share of the
    molecules (serve.split_jobs) and solves/s is all molecules over the
    slowest rank's time; the ranks start each variant together."""
    import numpy as np
    import gtfock_b200 as gb
    from gtfock_b200 import molecules as mol, serve, workloads
    rk = rk or _Ranks()
    items = workloads.batched(count, seed)
    owner = serve.split_jobs([i[3] for i in items], rk.world)
    mine = [k for k in range(len(items)) if owner[k] == rk.rank]
    niter = 15
    out = {"metric": "SCF solves/s, batched (%d molecules, 15 iterations)" % count, "unit": "solves/s",
           "workload": "seeded water clusters 2-24 / alkanes C2-C16, STO-3G or 6-31G, %d-%d bf" %
           (min(i[3] for i in items), max(i[3] for i in items)), "seed": seed, "fp32_cutoff": cut,
           "n_gpus": rk.world}
    with tempfile.TemporaryDirectory() as td:
        files = [(mol.basis_file(items[k][2]), mol.write_xyz(items[k][1], os.path.join(td, items[k][0] + ".xyz"),
                                                              items[k][0])) for k in mine]
        res = {}
        for tag, prec, incr in (("batched_fp64", 0, False), ("batched_mixed", 1, False),
                                ("batched_mixed_incremental", 1, True)):
            b = gb.Batch(max(1, len(files)))
            if incr:
                b.set_incremental(True, 0.0, INCR_PERIOD)
            t0 = time.perf_counter()
            slots = [b.add(g, x, tolscr=TOL, precision=prec, fp32_cutoff=cut, max_iters=niter, etol=0.0)
                     for g, x in files]
            t1 = time.perf_counter()
            setup_s = t1 - t0
            tune_s = None
            if autotune and files:
                b.autotune(2)
                tune_s = time.perf_counter() - t1
            rk.barrier()
            t1 = time.perf_counter()
            l0 = gb.launch_count()
            if files:
                b.run()
            t2 = time.perf_counter()
            info = b.info()
            mine_e = {k: [float(x) for x in b.result(s)[0]] for k, s in zip(mine, slots)}
            stats = {"n": len(files), "solve_s": t2 - t1, "setup_s": setup_s, "autotune_s": tune_s,
                     "ms_fock": info["ms_fock"], "ms_energy": info["ms_energy"], "ms_diis": info["ms_diis"],
                     "ms_purification": info["ms_purification"],
                     "purification_steps": info["purification_steps"], "steps": info["steps"],
                     "launches": gb.launch_count() - l0}
            b.close()
            gb.device_trim(0)   # untimed: the jobs' cached device memory back to the driver
            parts = rk.gather((mine_e, stats))
            res[tag] = {}
            for e, _ in parts:
                res[tag].update({int(k): v for k, v in e.items()})
            solve_s = max(p[1]["solve_s"] for p in parts)
            out[tag] = dict(parts[0][1], solves_per_s=len(items) / solve_s, solve_s=solve_s)
            out[tag].pop("n")
            if rk.world > 1:
                out[tag]["per_rank"] = [p[1] for p in parts]
        # the plain FP64 GPU path, one molecule after another (each rank its
        # share's first molecules)
        nseq = min(len(files), -(-seq_sample // rk.world))
        tsolve = tset = 0.0
        eseq_mine = {}
        for k, (g, x) in zip(mine[:nseq], files[:nseq]):
            t0 = time.perf_counter()
            s = gb.SCFSolver(g, x, tolscr=TOL)
            s.set_options(precision=0, etol=0.0)
            t1 = time.perf_counter()
            e, _ = s.solve(niters=niter)
            t2 = time.perf_counter()
            s.close()
            tset += t1 - t0
            tsolve += t2 - t1
            eseq_mine[k] = [float(v) for v in e]
        parts = rk.gather((eseq_mine, nseq, tsolve, tset))
        eseq_d = {}
        for e, _, _, _ in parts:
            eseq_d.update(e)
        nseq = sum(p[1] for p in parts)
        out["sequential_fp64"] = {"solves_per_s": nseq / max(p[2] for p in parts), "molecules_timed": nseq,
                                  "setup_s_per_molecule": sum(p[3] for p in parts) / nseq}
        # molecules in the order of the global list, where the one-job path ran
        order = sorted(eseq_d)
        eseq = [np.array(eseq_d[k]) for k in order]
        res = {tag: [np.array(v[k]) for k in order] for tag, v in res.items()}
        nseq = len(order)
        # energies are compared on the molecules whose FP64 one-job run has
        # converged after the 15 iterations (|E_15 - E_14| < 1e-6 Ha); from the
        # core-Hamiltonian guess some clusters and chains do not, and their
        # last iterate is not a converged energy on either path
        conv = [k for k in range(nseq) if len(eseq[k]) >= 2 and np.isfinite(eseq[k][-1]) and
                abs(eseq[k][-1] - eseq[k][-2]) < 1e-6]
        d_seq = max([abs(eseq[k][-1] - res["batched_fp64"][k][-1]) for k in conv] or [0.0])
        d_mix = max([abs(res["batched_mixed"][k][-1] - eseq[k][-1]) for k in conv] or [0.0])
        d_inc = max([abs(res["batched_mixed_incremental"][k][-1] - eseq[k][-1]) for k in conv] or [0.0])
        out["converged_molecules"] = len(conv)
        out["max_dE_batched_vs_sequential"] = d_seq
        out["max_dE_mixed_vs_fp64"] = d_mix
        out["max_dE_mixed_incremental_vs_fp64"] = d_inc
        out["speedup_batched_mixed_vs_sequential_fp64"] = (out["batched_mixed"]["solves_per_s"] /
                                                           out["sequential_fp64"]["solves_per_s"])
        out["speedup_batched_mixed_incremental_vs_sequential_fp64"] = (
            out["batched_mixed_incremental"]["solves_per_s"] / out["sequential_fp64"]["solves_per_s"])
        if autotune:
            out["tuned"] = [e for e in gb.tune_entries() if e["kind"] != "fock"]
    return out


def run_served(args):
    """Served workload (--workload served): see served_measure."""
    rk = _Ranks()
    out = served_measure(args.count, args.seed, args.rate, args.fp32_cutoff if args.fp32_cutoff is not None
                         else SERVED_CUTOFF, args.slots, args.lanes, not args.no_incremental, not args.turns, rk=rk,
                         repeats=args.repeats)
    if rk.rank == 0:
        print(json.dumps(out), flush=True)
    rk.close()


def served_measure(count, seed, rate, cut, slots, lanes, incremental, concurrent=True, with_sequential=True,
                   rk=None, repeats=1):
    """Served workload: a seeded Poisson stream of SCF requests, sizes
    log-uniform over 20-1500 bf (water clusters in 6-31G, alkanes C4-C40 in
    cc-pVDZ), each iterated until |dE| < 1e-6 Ha (max 30 iterations).  The
    continuous-batching server (mixed precision, incremental Fock builds,
    HBM-footprint admission) against the same stream on the plain FP64 GPU
    path, one job at a time.  On several GPUs (rk) each rank serves the
    requests serve.route gives it, from a common start, and the statistics
    cover the requests of all ranks; the FP64 comparison runs the same shares
    one job at a time per rank.  The stream is replayed against the wall
    clock, so which requests share a batch step varies from run to run: with
    repeats > 1 the served form runs that many times and the run of median
    makespan gives the statistics (every run's energies are checked)."""
    import gtfock_b200  # noqa: F401
    from gtfock_b200 import serve, workloads
    rk = rk or _Ranks()
    items = workloads.served(count, seed, rate)

    def share():
        reqs_all = [serve.Request(n, a, b, t, nb) for t, n, a, b, nb in items]
        owner = serve.route(reqs_all, rk.world)
        return [r for r, k in zip(reqs_all, owner) if k == rk.rank]

    runs = []
    host = []
    for _ in range(max(1, repeats)):
        reqs = share()
        srv = serve.SCFServer(slots=slots, precision=1, fp32_cutoff=cut, max_iters=30, etol=1e-6, tolscr=TOL,
                              lanes=LANES[lanes],
                              incremental=incremental, incr_tau=SERVED_TAU, incr_period=INCR_PERIOD,
                              concurrent=concurrent,
                              device=rk.device if rk.world > 1 else None)
        rk.barrier()
        done = serve.run_stream(reqs, srv)
        budget = srv.admission.budget
        host.append(dict(srv.stats))
        srv.close()
        if rk.world > 1:
            done = serve.gather_finished(done)
        runs.append(done)
    spans = [serve.latency_stats(d)["makespan_s"] for d in runs]
    done = runs[sorted(range(len(runs)), key=lambda i: spans[i])[len(runs) // 2]]
    reqs = share()
    if not with_sequential:
        return {"served_mixed": serve.latency_stats(done), "energies": {r.name: float(r.energies[-1]) for r in done},
                "iterations": {r.name: len(r.energies) for r in done}}
    seq = serve.run_sequential(reqs, max_iters=30, etol=1e-6, tolscr=TOL)
    if rk.world > 1:
        seq = serve.gather_finished(seq)
    by = {r.name: r for r in seq}
    # compared where both runs converged (|dE| < 1e-6 Ha before 30 iterations)
    conv = [r for r in done if len(r.energies) < 30 and len(by[r.name].energies) < 30]
    dE = max([abs(r.energies[-1] - by[r.name].energies[-1]) for d in runs for r in d
              if len(r.energies) < 30 and len(by[r.name].energies) < 30] or [0.0])
    worst = max(conv, key=lambda r: abs(r.energies[-1] - by[r.name].energies[-1])) if conv else None
    within = sum(1 for r in conv if abs(r.energies[-1] - by[r.name].energies[-1]) <= 1e-6)
    out = {"metric": "SCF solves/s and p50/p99 time-to-converged-energy, served (%d requests)" % count,
           "workload": "Poisson rate %.2f/s, seed %d, %d-%d bf" % (rate, seed,
                                                                 min(i[4] for i in items), max(i[4] for i in items)),
           "served_form": "continuous batching%s, FP32 quartets below %g%s" % (
               ", size lanes stepped concurrently on their own streams" if concurrent else "",
               cut, ", incremental Fock builds (full every %d, change screened at %g)" % (INCR_PERIOD, SERVED_TAU)
               if incremental else ""),
           "fp32_cutoff": cut, "slots_per_lane": slots, "lanes": lanes, "n_gpus": rk.world,
           "hbm_budget_gb": budget / 1e9,
           "served_mixed": serve.latency_stats(done), "sequential_fp64": serve.latency_stats(seq),
           "max_dE_served_vs_fp64": dE, "converged_requests": len(conv),
           "converged_within_1e-6": within, "requests_served": len(done),
           "served_runs": {"solves_per_s": [serve.latency_stats(d)["solves_per_s"] for d in runs],
                           "host": host,
                           "note": "the stream replayed %d times; statistics of the run of median makespan, "
                                   "max_dE over all runs" % len(runs)},
           "iterations_served": sum(len(r.energies) for r in done),
           "iterations_fp64": sum(len(r.energies) for r in seq),
           "worst_request": None if worst is None else {
               "name": worst.name, "nbf": worst.nbf, "served_energies": [float(x) for x in worst.energies],
               "fp64_energies": [float(x) for x in by[worst.name].energies]}}
    out["speedup_solves_per_s"] = out["served_mixed"]["solves_per_s"] / out["sequential_fp64"]["solves_per_s"]
    return out


def run_served_tau(args):
    """Served-form screening sweep (--workload served-tau): the largest
    request below 1000 functions of the served stream (32 requests, seed 7,
    rate 4/s), solved to |dE| < 1e-6 Ha (30 iterations at most) on the plain
    FP64 path and in the served form (FP32 quartets below 1e-6, incremental
    builds, full every 8) with the quartets of the density change dropped
    below bound x max|dD| < tau for tau = the Schwarz threshold (the
    default), 1e-9, 1e-8, 1e-7: solve time (set-up excluded, one warm-up
    solve first) and |E - E_FP64|."""
    import gtfock_b200 as gb
    from gtfock_b200 import molecules as mol, workloads
    items = workloads.served(32, 7, 4.0)
    t, name, atoms, basis, nbf = max((i for i in items if i[4] < 1000), key=lambda i: i[4])
    rows = []
    with tempfile.TemporaryDirectory() as td:
        xyz = mol.write_xyz(atoms, os.path.join(td, name + ".xyz"), name)
        gbs = mol.basis_file(basis)
        for label, prec, tau in [("fp64", 0, None), ("served, tau 1e-10 (default)", 1, 0.0),
                                 ("served, tau 1e-9", 1, 1e-9), ("served, tau 1e-8", 1, 1e-8),
                                 ("served, tau 1e-7", 1, 1e-7)]:
            s = gb.SCFSolver(gbs, xyz, tolscr=TOL)
            s.set_options(precision=prec, fp32_cutoff=1e-6 if prec else 0.0, etol=1e-6)
            if tau is not None:
                s.set_incremental(True, tau, INCR_PERIOD)
            s.solve(niters=2)
            t0 = time.perf_counter()
            e, _ = s.solve(niters=30)
            dt = time.perf_counter() - t0
            s.close()
            rows.append({"form": label, "solve_s": dt, "iterations": len(e), "energy": float(e[-1])})
    for r in rows:
        r["dE_vs_fp64"] = abs(r["energy"] - rows[0]["energy"])
        r["speedup_vs_fp64"] = rows[0]["solve_s"] / r["solve_s"]
    print(json.dumps({"workload": "%s (%d bf) of the served stream" % (name, nbf), "rows": rows}), flush=True)


def run_precision(args):
    """Precision variant: (H2O)64 / 6-31G (832 bf, seed 2024), FP32 ERIs below
    a Schwarz-bound cutoff swept over 1e-4 .. 1e-8, against the FP64 path:
    max|dF| of one build at the converged FP64 density, |dE| of the converged
    SCF energy, ||D S D - D||_F and |tr(D S) - N_occ| of the final density."""
    import numpy as np
    import gtfock_b200 as gb
    from gtfock_b200 import molecules as mol
    with tempfile.TemporaryDirectory() as td:
        xyz = mol.write_xyz(mol.water_cluster(64, 2024), os.path.join(td, "w64.xyz"))
        gbs = mol.basis_file("6-31g")
        b = gb.BasisSet(gbs, xyz)
        pf = gb.PFock(b, tolscr=TOL)
        S, _, _ = pf.one_electron()
        s = gb.SCFSolver(gbs, xyz, tolscr=TOL)
        s.set_options(precision=0, etol=1e-10)
        t0 = time.perf_counter()
        e64, _ = s.solve(niters=60)
        t64 = time.perf_counter() - t0
        D64 = s.density()
        F64 = pf.compute_fock(D64)
        ms64 = pf.timing()["ms_eri"]
        rows = []
        for cut in (1e-4, 1e-5, 1e-6, 1e-7, 1e-8):
            pf.set_precision(1, cut)
            F = pf.compute_fock(D64)
            msc = pf.timing()["ms_eri"]
            nq32, nq = pf.precision_stats()
            s.set_options(precision=1, fp32_cutoff=cut, etol=1e-10)
            # FP64 purification products: these rows isolate the ERI precision
            # (mixed precision would otherwise select the split-BF16 products)
            s.set_purification(0)
            t0 = time.perf_counter()
            e, _ = s.solve(niters=60)
            tc = time.perf_counter() - t0
            D = s.density()
            rows.append({"fp32_cutoff": cut, "fp32_share": nq32 / nq, "max_dF": float(np.abs(F - F64).max()),
                         "dE": float(abs(e[-1] - e64[-1])), "idempotency_DSD_minus_D": float(
                             np.linalg.norm(D @ S @ D - D)), "trace_error": float(abs(np.trace(D @ S) - b.nocc)),
                         "fock_ms": msc, "scf_s": tc, "iterations": len(e)})
        # split-BF16 purification products on the tensor cores (FP64 finish),
        # with FP64 ERIs and with FP32 ERIs below 1e-6
        bf = []
        for prec, cut in ((0, 0.0), (1, 1e-6)):
            s.set_options(precision=prec, fp32_cutoff=cut, etol=1e-10)
            s.set_purification(1)
            t0 = time.perf_counter()
            e, tm = s.solve(niters=60)
            tc = time.perf_counter() - t0
            nb, n64 = s.purification_iters()
            D = s.density()
            bf.append({"eri": "fp64" if prec == 0 else "fp32 below %g" % cut, "dE": float(abs(e[-1] - e64[-1])),
                       "idempotency_DSD_minus_D": float(np.linalg.norm(D @ S @ D - D)),
                       "trace_error": float(abs(np.trace(D @ S) - b.nocc)), "scf_s": tc, "iterations": len(e),
                       "purification_s_per_solve": tm["purif_s"],
                       "last_purification_steps": {"bf16_split": nb, "fp64": n64}})
            s.set_purification(0)
        s.set_options(precision=0, etol=1e-10)
        s.solve(niters=60)
        nb0, n640 = s.purification_iters()
        pf.close()
        s.close()
    out = {"metric": "precision sweep, (H2O)64 / 6-31G (832 bf)", "fp64": {
        "energy": float(e64[-1]), "iterations": len(e64), "fock_ms": ms64, "scf_s": t64,
        "idempotency_DSD_minus_D": float(np.linalg.norm(D64 @ S @ D64 - D64)),
        "trace_error": float(abs(np.trace(D64 @ S) - b.nocc)),
        "last_purification_steps": {"fp64": n640}}, "mixed": rows, "bf16_split_purification": bf}
    print(json.dumps(out), flush=True)


def profile_purification(args):
    """Two SCF iterations of (H2O)64 / 6-31G with the split-BF16 purification
    (the small case profiled with ncu for the tensor-core products)."""
    import gtfock_b200 as gb
    from gtfock_b200 import molecules as mol
    with tempfile.TemporaryDirectory() as td:
        xyz = mol.write_xyz(mol.water_cluster(64, 2024), os.path.join(td, "w64.xyz"))
        s = gb.SCFSolver(mol.basis_file("6-31g"), xyz, tolscr=TOL)
        s.set_purification(1)
        e, tm = s.solve(niters=2)
        nb, n64 = s.purification_iters()
        s.close()
    print(json.dumps({"purification_s": tm["purif_s"], "bf16_split_steps": nb, "fp64_steps": n64,
                      "energies": [float(x) for x in e]}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gtfock_b200", choices=["gtfock_b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-fock", choices=["c12h26", "c54h18", "c96h24", "w64"], default=None)
    ap.add_argument("--builds", type=int, default=2)
    ap.add_argument("--autotune", action="store_true",
                    help="--profile-fock: tune the launch shapes before timing")
    ap.add_argument("--no-autotune", action="store_true",
                    help="--workload batched: keep the default launch shapes (tuned by default)")
    ap.add_argument("--profile-purif", action="store_true",
                    help="two SCF iterations of (H2O)64 with the split-BF16 purification (ncu case)")
    ap.add_argument("--fp32-cutoff", type=float, default=None,
                    help="with --profile-fock: FP32 for quartets with Schwarz bound below this")
    ap.add_argument("--workload", choices=["default", "batched", "served", "served-tau", "precision", "c12h26",
                                           "batch-scaling", "setup"], default="default",
                    help="batched / served / precision: the batched, served and precision-sweep workloads; "
                         "c12h26: the 10-iteration C12H26 solve timed beside the reference driver; "
                         "batch-scaling: large molecules in one batch against builds alone; "
                         "served-tau: screening of the density change swept on one served request; "
                         "setup: the C-API set-up steps of one solve, timed one by one")
    ap.add_argument("--count", type=int, default=None, help="molecules (batched) or requests (served)")
    ap.add_argument("--seed", type=int, default=None)
    ap.add_argument("--rate", type=float, default=2.0, help="served: Poisson arrival rate (1/s)")
    ap.add_argument("--slots", type=int, default=64, help="served: resident jobs per lane at most")
    ap.add_argument("--lanes", type=int, default=2, choices=[1, 2, 3],
                    help="served: size lanes (2: up to 400 functions, and the rest)")
    ap.add_argument("--seq-sample", type=int, default=256, help="batched: molecules timed on the one-job path")
    ap.add_argument("--no-incremental", action="store_true", help="served: plain (not incremental) Fock builds")
    ap.add_argument("--repeats", type=int, default=1,
                    help="served: replays of the stream by the server (statistics of the median one)")
    ap.add_argument("--turns", action="store_true",
                    help="served: the lanes take turns on one thread instead of stepping concurrently")
    ap.add_argument("--quick", action="store_true",
                    help="default workload only: leave out the served, batched and C12H26 blocks")
    args = ap.parse_args()
    if args.workload == "batched":
        args.autotune = not args.no_autotune
        args.count = args.count or 256
        args.seed = 2024 if args.seed is None else args.seed
        run_batched(args)
        return
    if args.workload == "served":
        args.count = args.count or 64
        args.seed = 7 if args.seed is None else args.seed
        run_served(args)
        return
    if args.workload == "precision":
        run_precision(args)
        return
    if args.workload == "served-tau":
        run_served_tau(args)
        return
    if args.workload == "c12h26":
        run_c12h26(args)
        return
    if args.workload == "batch-scaling":
        run_batch_scaling(args)
        return
    if args.workload == "setup":
        run_setup(args)
        return
    if args.profile_purif:
        profile_purification(args)
        return
    if args.profile_fock:
        profile_fock(args)
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run(args)


if __name__ == "__main__":
    main()
