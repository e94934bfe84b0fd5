/*
 * gtfock_b200.h -- entry points of libgtfock_b200 beyond GTFock's own API.
 *
 * The drop-in API is pfock.h / purif.h / CInt.h.  The functions below expose
 * what the reference keeps inside its PFock struct (screening lists,
 * counters), the device-resident forms used by the benchmark, and the native
 * SCF driver.  Plain C types only; 0 (or PFOCK_STATUS_SUCCESS) on success.
 */
#ifndef GTFOCK_B200_H
#define GTFOCK_B200_H

#include "CInt.h"
#include "pfock.h"
#include "purif.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Screening results of PFock_create: the reference's PFock fields nnz,
 * maxvalue (pfock/pfock.h:22-29) and the quartet counters usq / uitl that
 * PFock_getStatistics reports (pfock/fock_task.c:195-196). */
PFockStatus_t gtf_pfock_counts(PFock_t pfock, int *nnz, double *maxvalue,
                               double *usq, double *uitl);

/* Copy of the CSR shell-pair list (shellptr[nshells+1], shellid[nnz],
 * shellrid[nnz], shellvalue[nnz]) built as pfock/screening.c:110-175. */
PFockStatus_t gtf_pfock_screening(PFock_t pfock, int *shellptr, int *shellid,
                                  int *shellrid, double *shellvalue);

/* CUDA-event timings (ms) of the last PFock_computeFock: whole build and the
 * electron-repulsion kernels alone; Rys-model FLOPs of one build. */
PFockStatus_t gtf_pfock_timing(PFock_t pfock, double *ms_total, double *ms_eri,
                               double *eri_flops);

/* Per angular-class-pair statistics of the last build (21 pairs for s/p/d
 * shells): bra / ket pair classes (ss=0 ps=1 pp=2 ds=3 dp=4 dd=5), CUDA-event
 * ms of each class kernel and its quartet count.  Returns the pair count. */
int gtf_pfock_class_stats(PFock_t pfock, int *X, int *Y, double *ms, double *nquart);

/* Per class pair (same order): Rys-model FLOPs of one build and the number of
 * primitive quartets before primitive screening.  Returns the pair count. */
int gtf_pfock_class_work(PFock_t pfock, double *flops, double *nprimq);
/* The same after primitive screening: the primitive quartets the kernels
 * evaluate (their loops stop at |K_ab K_cd| < 1e-17) and the Rys-model FLOPs
 * of those.  Returns the pair count, or < 0 on error. */
int gtf_pfock_class_work_screened(PFock_t pfock, double *flops, double *nprimq);

/* Precision of the ERI kernels: 0 = FP64 (default), 1 = FP32 for quartets
 * whose Schwarz bound sqrt(v1 v2) is below fp32_cutoff (Rys roots, 2-D
 * integrals and the primitive sum in FP32; D, the J/K digestion and every
 * accumulation into F stay FP64).  Rebuilds the task lists. */
PFockStatus_t gtf_pfock_set_precision(PFock_t pfock, int mode, double fp32_cutoff);

/* Engines created with symm = 0 (non-symmetric densities):
 *   mode 1 (default): the reference's own result, (F[D] + F[D^T]^T) / 2 of
 *     its unique-quartet digestion (pfock/pfock.c:1704-1718), which for a
 *     non-symmetric D depends on the orientation of its shell-pair lists;
 *   mode 2: the exact F = 2 J[D] - K[D], J_ab = sum_cd (ab|cd) D_cd,
 *     K_ab = sum_cd (ac|bd) D_cd.
 * Both equal the symm = 1 result for a symmetric D.  Returns
 * PFOCK_STATUS_INVALID_VALUE on an engine created with symm = 1. */
PFockStatus_t gtf_pfock_set_nosymm_mode(PFock_t pfock, int mode);

/* One molecule over several GPUs (one process per GPU): with
 * gtf_pfock_set_shard(pf, r, n) every class launch of this engine's builds
 * covers shard r of n of its quartet units (the 2-D task decomposition of
 * pfock/pfock.c:22-154 becomes a split of each class's unit range), so
 * PFock_getMat / gtf_pfock_compute_dev return this rank's part of F; the
 * parts of the n ranks sum to the whole F (one all-reduce per build).
 * n <= 1 restores the whole build.  The split is contiguous and weighted:
 * each launch's bras are divided by gtf_shard_split on their work model
 * (primitive quartets x Rys-model FLOPs per primitive quartet, plus the
 * per-quartet contraction and digestion), so the shards get equal work.
 * gtf_shard_split: items [lo, hi) of shard r of nshards for n items of
 * weights w (contiguous, in order, each shard within one item's weight of
 * the mean).  gtf_shard_range: the same for equal weights (units [lo, hi)
 * of a launch of `nunits`).  gtf_pfock_shard_work: model FLOPs of this
 * engine's shard of a build (the whole build when not sharded). */
PFockStatus_t gtf_pfock_set_shard(PFock_t pfock, int shard, int nshards);
void gtf_shard_split(const double *w, long long n, int r, int nshards, long long *lo, long long *hi);
void gtf_shard_range(long long nunits, int r, int n, long long *lo, long long *hi);
PFockStatus_t gtf_pfock_shard_work(PFock_t pfock, double *work);

/* Launch-shape autotuning.  gtf_pfock_autotune times, for every class pair
 * and precision part of this engine's Fock build (on the density last put),
 * candidate shapes of the persistent kernels -- blocks per SM (the occupancy
 * limit, one less, half), and in batched launches also the quartets a warp
 * claims at once (32, 64, 128) -- and records the fastest in a process-wide table keyed by (single / batch,
 * class pair, part, floor(log2(units of work))); later builds of any engine
 * or batch of that size use it.  gtf_batch_autotune does the same for a
 * batch's Fock launches and picks the tile shape of its batched dense
 * products (64x64, 32x32, 32x64, 128x64 output tiles).  The table is saved /
 * merged from a text file whose first line names the device model; a file
 * from another model is refused.  gtf_tune_entries writes rows of 8 ints
 * (kind 0 single / 1 batch / 2 products, class X, class Y, part, size bucket,
 * blocks per SM or tile shape, claim, ms x 1000) and returns the count. */
PFockStatus_t gtf_pfock_autotune(PFock_t pfock, int reps);
int gtf_tune_save(const char *path);
int gtf_tune_load(const char *path);
void gtf_tune_clear(void);
int gtf_tune_entries(int *rows, int max_rows);

/* Incremental Fock builds (no counterpart in the reference, whose builds
 * always start from zero).  F is linear in D, so with on = 1 each build of
 * density 0 computes only the change: F_k = F_k-1 + G[D_k - D_k-1].  A
 * quartet of the change is dropped when its Schwarz bound times
 * dmax = max |D_k - D_k-1| is below tau (tau <= 0: the engine's Schwarz
 * threshold, so each dropped contribution is below what the plain build's
 * screening drops), and evaluated in FP32 (mixed precision mode) when that
 * product is below the FP32 cutoff.  The task lists are rebuilt on the device
 * for every build.  Every `period` builds (and the first after this call) is
 * a full one, which restarts the sum.  Symmetric densities on an unsharded
 * engine only; on = 0 returns to plain builds.
 * gtf_pfock_incremental_stats: quartets of the last build in FP64 and FP32,
 * and its dmax (0 for a full build). */
PFockStatus_t gtf_pfock_set_incremental(PFock_t pfock, int on, double tau, int period);
PFockStatus_t gtf_pfock_incremental_stats(PFock_t pfock, double *nquart_fp64, double *nquart_fp32,
                                          double *dmax);

/* Quartets evaluated in FP32 under the current mode, and all quartets. */
PFockStatus_t gtf_pfock_precision_stats(PFock_t pfock, double *nquart_fp32, double *nquart);

/* Device-resident Fock build for callers that keep D on the GPU: dev_D is a
 * device pointer to the nbf x nbf density; the result stays on the device
 * (returned through *dev_F, valid until the next build).  The engine reads
 * dev_D on its own stream, which is not ordered after the caller's streams:
 * the kernels or copies that write dev_D must have completed before the call
 * (synchronize the stream that produced it).  The call returns once F is
 * complete.  *dev_F is freed with the engine on the engine's own stream:
 * work of other streams that still reads or writes it must have completed
 * before PFock_destroy. */
PFockStatus_t gtf_pfock_compute_dev(PFock_t pfock, const double *dev_D,
                                    const double **dev_F);

/* Fock build that allocates nothing.  No counterpart in the reference.
 * For callers that may not allocate device memory while they run (a host
 * whose own pool allocator owns the GPU memory, a real-time loop that must
 * not wait on the driver's allocator, a plugin in a process that forbids
 * allocation after start-up).  Same inputs and result as
 * gtf_pfock_compute_dev: dev_D is the nbf x nbf density and dev_F receives
 * F = J + K, both device pointers owned by the caller.  The scratch lives in
 * one static device array of about 5.9 MB that every GPU loading the library
 * keeps until exit; bases above 384 Cartesian functions are rejected with
 * PFOCK_STATUS_INVALID_VALUE, and so are engines built with symm = 0 or
 * sharded with gtf_pfock_set_shard (this call returns the whole F).  All
 * calls on a GPU share that array: calls whose work overlaps on the GPU race
 * and must be ordered by the caller.  As for gtf_pfock_compute_dev, dev_D
 * must be complete on the device before the call, which returns once dev_F
 * holds F.  The first call on a device looks up the array's address; make it
 * before any stream capture.  The engine must have been created on the
 * current device. */
PFockStatus_t gtf_pfock_compute_noalloc(PFock_t pfock, const double *dev_D, double *dev_F);

/* Native SCF driver: the loop of pscf/scf.c:329-459 (Fock build, energy,
 * DIIS, purification) on one GPU for the molecule in xyzfile with basis
 * bsfile.  gtf_scf_create performs the set-up (basis, PFock_create with its
 * screening, create_purif, S / X / H_core) once; gtf_scf_solve runs one SCF
 * from the initial guess and may be called repeatedly.
 *   mode 0: host D/F buffers cross the C API every iteration (as scf.c);
 *   mode 1: D and F stay resident on the device.
 * energies[k] = total energy (incl. nuclear) of iteration k.  timings
 * (optional, 7 doubles): seconds in Fock builds, DIIS, purification, total;
 * host->device bytes, device->host bytes, library kernel launches.
 * Returns iterations run, or a negative value on error. */
typedef struct gtf_scf gtf_scf_t;
gtf_scf_t *gtf_scf_create(const char *bsfile, const char *xyzfile, double tolscr);
int gtf_scf_solve(gtf_scf_t *s, int niters, int mode, double *energies, double *timings);
int gtf_scf_nbf(gtf_scf_t *s);
/* ERI precision of the engine (as gtf_pfock_set_precision) and the energy
 * convergence tolerance: a solve stops once |E_k - E_k-1| < etol (default
 * 1e-11).  Mixed precision (prec_mode 1) also selects the split-BF16
 * purification products (gtf_scf_set_purification mode 1) unless a mode was
 * set explicitly.  0 on success. */
int gtf_scf_set_options(gtf_scf_t *s, int prec_mode, double fp32_cutoff, double etol);
/* Incremental Fock builds for this solver's engine (gtf_pfock_set_incremental);
 * every solve starts with a full build.  0 on success. */
int gtf_scf_set_incremental(gtf_scf_t *s, int on, double tau, int period);
/* Purification products: mode 0 FP64 (default); mode 1 split-BF16 products
 * on the tensor cores (each FP64 factor as a sum of two BF16 matrices, FP32
 * accumulation) until the idempotency error stops falling, then FP64 steps
 * to ||D - D^2||_F < 1e-11.  0 on success. */
int gtf_scf_set_purification(gtf_scf_t *s, int mode);
/* Iterations of the last purification: split-BF16 and FP64 steps. */
int gtf_scf_purification_iters(gtf_scf_t *s, int *bf16_iters, int *fp64_iters);
/* Copy of the density (half density, AO basis, nbf x nbf) left by the last
 * solve.  0 on success. */
int gtf_scf_get_density(gtf_scf_t *s, double *D);
void gtf_scf_destroy(gtf_scf_t *s);
/* create + solve + destroy; timings[3] covers the whole job */
int gtf_scf_run(const char *bsfile, const char *xyzfile, double tolscr,
                int niters, int mode, double *energies, double *timings);

/* Batched and served SCF: many molecules (jobs) of different sizes iterated
 * in lock-step on one GPU.  Each gtf_batch_step runs one SCF iteration of
 * every running job: one batched Fock build (one launch per class pair,
 * precision part and slice covering all jobs), the energy, DIIS and canonical
 * purification as launches that cover all jobs.  Jobs join (gtf_batch_add)
 * and leave (gtf_batch_remove) between steps, so a serving loop can admit a
 * request as soon as a slot and device memory are free.
 *   gtf_batch_create(capacity): at most `capacity` jobs at a time.
 *   gtf_batch_add: set-up of one job (basis, screening, S, X, H_core,
 *     initial guess) with its ERI precision (as gtf_pfock_set_precision;
 *     jobs above 640 functions in mixed precision also purify with the
 *     split-BF16 products), at most max_iters iterations, stopping once
 *     |E_k - E_k-1| < etol;
 *     returns the job's slot (>= 0) or a negative error (-2: no free slot).
 *   gtf_batch_step: returns the number of jobs still running, or < 0.
 *   gtf_batch_run: steps until every job is done.
 *   gtf_batch_result: energies (total, incl. nuclear) of the iterations run
 *     so far, their count, and whether the job is done.
 *   gtf_batch_density: the job's current density (AO basis, nbf x nbf).
 *   gtf_batch_info: running / used slots, accumulated ms of the Fock builds
 *     and of the rest of the steps, device bytes held by the jobs.
 *   gtf_batch_job_bytes: device bytes of a job's batch buffers for nbf
 *     functions (admission estimate; the Fock engine comes on top). */
typedef struct gtf_batch gtf_batch_t;
gtf_batch_t *gtf_batch_create(int capacity);
int gtf_batch_add(gtf_batch_t *b, const char *bsfile, const char *xyzfile, double tolscr, int prec_mode,
                  double fp32_cutoff, int max_iters, double etol);
/* gtf_batch_add in two parts, for a server that sets a job up on one host
 * thread while the batch steps on another: gtf_batch_prepare does the whole
 * set-up that touches no state of the batch (basis, engine, S, H_core, X, on
 * the engine's own stream; it reads only the batch's incremental setting,
 * fixed before the first job) and may overlap a gtf_batch_step of `b`;
 * gtf_batch_attach puts the job in a free slot (its batch buffers and initial
 * density) and must not overlap a step.  attach consumes the job, on success
 * and on error alike; gtf_batch_job_free releases one never attached.
 * Return codes as gtf_batch_add's (prepare: 0 on success). */
typedef struct gtf_batch_job gtf_batch_job_t;
int gtf_batch_prepare(gtf_batch_t *b, const char *bsfile, const char *xyzfile, double tolscr, int prec_mode,
                      double fp32_cutoff, gtf_batch_job_t **job);
int gtf_batch_attach(gtf_batch_t *b, gtf_batch_job_t *job, int max_iters, double etol);
void gtf_batch_job_free(gtf_batch_job_t *job);
int gtf_batch_step(gtf_batch_t *b);
int gtf_batch_run(gtf_batch_t *b);
int gtf_batch_result(gtf_batch_t *b, int slot, double *energies, int *niters, int *done);
int gtf_batch_density(gtf_batch_t *b, int slot, double *D);
int gtf_batch_remove(gtf_batch_t *b, int slot);
int gtf_batch_info(gtf_batch_t *b, int *nrunning, int *nused, double *ms_fock, double *ms_rest,
                   size_t *job_bytes);
size_t gtf_batch_job_bytes(int nbf);
/* Device bytes held by the job in `slot` (its batch buffers and its Fock
 * engine); 0 for an empty slot. */
size_t gtf_batch_job_device_bytes(gtf_batch_t *b, int slot);
/* Per-job statistics of the job in `slot`: [0] basis functions, [1] SCF
 * iterations run, [2] purification iterations of its last step, [3] its
 * purification iterations over all steps.  Writes min(n, 4) values and
 * returns that count (0 for an empty slot). */
int gtf_batch_job_stats(gtf_batch_t *b, int slot, double *out, int n);
/* Accumulated statistics of a batch: [0] ms of the Fock builds, [1] of the
 * energies, [2] of DIIS, [3] of purification, [4] purification steps of the
 * batched jobs, [5] batch steps.  Writes min(n, 6) values, returns that count. */
int gtf_batch_stats(gtf_batch_t *b, double *out, int n);
/* Incremental Fock builds (gtf_pfock_set_incremental) for every job of the
 * batch; set before the first gtf_batch_add or gtf_batch_prepare (-2 after a
 * job has joined).  0 on success. */
int gtf_batch_set_incremental(gtf_batch_t *b, int on, double tau, int period);
/* Tunes the batch's launch shapes for its current jobs (see
 * gtf_pfock_autotune); call between steps. */
int gtf_batch_autotune(gtf_batch_t *b, int reps);
void gtf_batch_destroy(gtf_batch_t *b);

/* Device of the calling host thread for the library's later calls on it
 * (cudaSetDevice; engines, batches and solvers stay on the device they were
 * created on).  One process per GPU selects its own device; a host thread
 * it starts selects again.  0 on success, negative for a device that does
 * not exist. */
int gtf_set_device(int dev);
int gtf_get_device(int *dev);

/* Free and total bytes of the current device (cudaMemGetInfo, plus the
 * blocks cached in the library's memory pool, which its next allocations
 * reuse); 0 on success. */
int gtf_device_memory(size_t *free_bytes, size_t *total_bytes);
/* The library takes device buffers from the device's stream-ordered memory
 * pool and keeps up to 16 GiB of freed blocks cached; gtf_device_trim waits
 * for the device and returns the cached blocks to the driver down to `keep`
 * bytes (a server calls it when it stops).  0 on success. */
int gtf_device_trim(size_t keep);

/* Test hook: the n-th device allocation of an engine's set-up from now on
 * fails as an out-of-memory cudaMalloc would (n <= 0 disarms), so that the
 * error paths of PFock_create can be checked for leaks. */
void gtf_debug_fail_alloc(int n);
/* Device allocations made through that hook's allocator (engine set-up and
 * engine buffers) that have not been freed yet. */
long long gtf_debug_live_allocs(void);

/* Number of this library's own kernel launches so far (all threads). */
unsigned long long gtf_launch_count(void);

/* Measured FP64 FMA throughput of device 0 in GFLOP/s (probe kernel). */
int gtf_fp64_peak(double *gflops);

/* Device and library identification for tests: number of CUDA devices seen
 * and the compute capability of device 0 (major*10+minor); -1 on error. */
int gtf_device_info(int *ndev, int *cc);

#ifdef __cplusplus
}
#endif

#endif
