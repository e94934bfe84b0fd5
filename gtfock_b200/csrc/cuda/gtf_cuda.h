/*
 * gtf_cuda.h -- C ABI between the host C library (pfock.c, purif.c) and the
 * CUDA modules (fock.cu, onee.cu, purif.cu).  Plain pointers and sizes only;
 * every function returns 0 on success or a negative gtf_err_t.
 */
#ifndef GTF_CUDA_H
#define GTF_CUDA_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    GTF_OK = 0,
    GTF_ERR_CUDA = -1,       /* a CUDA runtime / library call failed */
    GTF_ERR_ALLOC = -2,      /* device or host allocation failed */
    GTF_ERR_INVALID = -3,    /* bad argument */
    GTF_ERR_NODEVICE = -4,   /* no CUDA device visible */
    GTF_ERR_DEVICE_FLAG = -5,/* a kernel reported an error through its status word */
    GTF_ERR_IO = -6          /* a file could not be opened, read or written */
} gtf_err_t;

/* read-only view of a loaded basis (gtf_basis.h fields) */
typedef struct {
    int natoms, nshells, nbf, nbf_cart, nprims, pure;
    const int *Z;
    const double *xyz;       /* [3*natoms] bohr */
    const int *sh_atom, *sh_L, *sh_nprim, *sh_pstart;
    const int *f_start;      /* [nshells+1] */
    const int *fc_start;     /* [nshells+1] */
    const double *alpha, *coef;
} gtf_basis_view_t;

typedef struct gtf_fock_dev gtf_fock_dev_t;

/* precision of the electron-repulsion kernels */
typedef enum {
    GTF_PREC_FP64 = 0,       /* every quartet in FP64 */
    GTF_PREC_MIXED = 1       /* quartets with Schwarz bound below a cutoff in FP32 */
} gtf_prec_t;

int gtf_fock_create(const gtf_basis_view_t *b, double tolscr, int max_numdmat,
                    gtf_fock_dev_t **out);
void gtf_fock_destroy(gtf_fock_dev_t *f);
const char *gtf_last_error(void);

/* screening results (pfock/screening.c:15-180) */
int gtf_fock_screening_info(gtf_fock_dev_t *f, int *nnz, double *maxvalue,
                            double *usq, double *uitl);
int gtf_fock_get_csr(gtf_fock_dev_t *f, int *shellptr, int *shellid, int *shellrid,
                     double *shellvalue);

/* density matrices (spherical/AO basis, full nbf x nbf) */
int gtf_fock_fill_density(gtf_fock_dev_t *f, int index, double value);
int gtf_fock_put_density(gtf_fock_dev_t *f, int index, int r0, int r1, int c0, int c1,
                         int stride, const double *host);
int gtf_fock_put_density_dev(gtf_fock_dev_t *f, int index, const double *dev);

/* J/K build for densities [0, numdmat) */
int gtf_fock_compute(gtf_fock_dev_t *f, int numdmat);
/* type: 0 D, 1 F (= J + K), 2 J, 3 K, as PFockMatType_t */
int gtf_fock_get_mat(gtf_fock_dev_t *f, int type, int index, int r0, int r1, int c0, int c1,
                     int stride, double *host);
const double *gtf_fock_mat_dev(gtf_fock_dev_t *f, int type, int index);

/* Fock build with its scratch in a static device array (no allocation);
 * dev_D in, dev_F (= J + K) out, both device pointers of nbf x nbf */
int gtf_fock_compute_fixed(gtf_fock_dev_t *f, const double *dev_D, double *dev_F);

/* one-electron matrices on the device: 0 S, 1 X = S^-1/2, 2 H_core */
int gtf_fock_one_electron(gtf_fock_dev_t *f, int want_sx, int want_h);
int gtf_fock_get_onee(gtf_fock_dev_t *f, int which, int r0, int r1, int c0, int c1,
                      int stride, double *host);
const double *gtf_fock_onee_dev(gtf_fock_dev_t *f, int which);
void gtf_fock_release_onee(gtf_fock_dev_t *f, int which);

/* precision control and statistics */
int gtf_fock_set_precision(gtf_fock_dev_t *f, int prec, double fp32_cutoff);
/* incremental builds: F_k = F_k-1 + G[D_k - D_k-1], quartets of the change
 * screened against tau / max |D_k - D_k-1|, a full build every `period`
 * builds (density 0, symmetric, unsharded); statistics of the last build */
int gtf_fock_set_incremental(gtf_fock_dev_t *f, int on, double tau, int period);
int gtf_fock_incremental_stats(gtf_fock_dev_t *f, double *nq64, double *nq32, double *dmax);
/* non-symmetric densities (PFock_create with symm = 0): the reference's own
 * symm = 0 output, or F = 2 J[D] - K[D] exactly for a general D; off */
#define GTF_NOSYMM_OFF 0
#define GTF_NOSYMM_REFERENCE 1
#define GTF_NOSYMM_EXACT 2
int gtf_fock_set_nosymm(gtf_fock_dev_t *f, int mode);
int gtf_fock_last_timing(gtf_fock_dev_t *f, double *ms_total, double *ms_eri, double *ms_other);
int gtf_fock_eri_flops(gtf_fock_dev_t *f, double *flops);
/* batched Fock builds over many engines (molecules): one launch per class
 * pair, precision part and slice for the whole batch.  Each engine reads its
 * own density buffer (gtf_fock_mat_dev(f, 0, 0)) and fills its own F/J/K. */
typedef struct gtf_fock_batch gtf_fock_batch_t;
int gtf_fock_batch_create(gtf_fock_dev_t *const *engines, int M, void *stream, gtf_fock_batch_t **out);
int gtf_fock_batch_compute(gtf_fock_batch_t *b);
/* incremental batches: full[m] != 0 makes member m's next build a full one */
int gtf_fock_batch_set_full(gtf_fock_batch_t *b, const int *full);
void gtf_fock_batch_destroy(gtf_fock_batch_t *b);

/* sharded builds (one molecule over several GPUs): every class launch covers
 * shard r of n of its units; the F of the shards sum to the whole build */
int gtf_fock_set_shard(gtf_fock_dev_t *f, int shard, int nshards);
void gtf_shard_range(long long nunits, int r, int n, long long *lo, long long *hi);
void gtf_shard_split(const double *w, long long n, int r, int nshards, long long *lo, long long *hi);
int gtf_fock_shard_work(gtf_fock_dev_t *f, double *work);

/* launch-shape autotuning (process-wide table, see fock.cu): time candidate
 * shapes of every Fock launch of an engine / a batch on its current density
 * and record the fastest; the table can be saved and reloaded */
int gtf_fock_autotune(gtf_fock_dev_t *f, int reps);
int gtf_fock_batch_autotune(gtf_fock_batch_t *b, int reps);
int gtf_tune_get(int kind, int X, int Y, int part, double size, int *a, int *b);
void gtf_tune_put(int kind, int X, int Y, int part, double size, int a, int b, double ms);
void gtf_tune_clear(void);
int gtf_tune_entries(int *rows, int max_rows);
int gtf_tune_save(const char *path);
int gtf_tune_load(const char *path);
/* per class pair: Rys-model FLOPs and primitive quartets of one build */
int gtf_fock_class_work(gtf_fock_dev_t *f, double *flops, double *nprimq);
/* the same after primitive screening (primitive quartets the kernels evaluate) */
int gtf_fock_class_work_screened(gtf_fock_dev_t *f, double *flops, double *nprimq);
/* quartets evaluated in FP32 under the current precision mode, and all */
int gtf_fock_fp32_quartets(gtf_fock_dev_t *f, double *nq32, double *nq);
/* per angular class pair (21 of them for s/p/d): classes, ms of the last
 * build, quartet counts; returns the number of class pairs */
int gtf_fock_class_stats(gtf_fock_dev_t *f, int *X, int *Y, double *ms, double *nquart);
void *gtf_fock_stream(gtf_fock_dev_t *f);
size_t gtf_fock_device_bytes(gtf_fock_dev_t *f);

/* ---- split BF16 products on the tensor cores (purif_bf16.cu) ---- */
typedef struct gtf_bf16x3 gtf_bf16x3_t;
int gtf_bf16x3_create(int n, void *stream, gtf_bf16x3_t **out);
void gtf_bf16x3_destroy(gtf_bf16x3_t *g);
int gtf_bf16x3_abt(gtf_bf16x3_t *g, const double *A, const double *B, double *C, void *stream);

/* ---- purification / DIIS on the device (purif.cu) ---- */
typedef struct gtf_purif_dev gtf_purif_dev_t;
int gtf_purif_create(int nbf, int nocc, void *stream, gtf_purif_dev_t **out);
void gtf_purif_destroy(gtf_purif_dev_t *p);
int gtf_purif_set_sx(gtf_purif_dev_t *p, const double *S_host, const double *X_host);
int gtf_purif_set_sx_dev(gtf_purif_dev_t *p, const double *S_dev, const double *X_dev);
/* canonical purification of F (orthogonal basis); D_AO returned; iterations */
int gtf_purif_run(gtf_purif_dev_t *p, const double *F_host, double *D_host, int *iters);
int gtf_purif_run_dev(gtf_purif_dev_t *p, const double *F_dev, double *D_dev, int *iters);
/* 0: FP64 products (default); 1: split-BF16 tensor-core canonical steps until
 * ||D - D^2||_F < 1e-2 or it stops falling, then FP64 canonical steps to 1e-11 */
int gtf_purif_set_mode(gtf_purif_dev_t *p, int mode);
/* iterations of the last purification: split-BF16 and FP64 */
void gtf_purif_last_iters(gtf_purif_dev_t *p, int *bf16_iters, int *fp64_iters);
/* one DIIS step: F (AO, host or device) in, extrapolated orthogonal F out */
int gtf_diis_step(gtf_purif_dev_t *p, const double *D_host, double *F_host, int iter);
int gtf_diis_step_dev(gtf_purif_dev_t *p, const double *D_dev, double *F_dev, int iter);
void gtf_purif_reset(gtf_purif_dev_t *p);
int gtf_purif_stats(gtf_purif_dev_t *p, double *ms_gemm, double *ms_total, double *errnorm,
                    double *idem_err, double *tr_err);

/* page-locked host blocks from a process-wide free list (devmem.cu) */
void *gtf_pinned_alloc(size_t bytes);
void gtf_pinned_free(void *p);

/* bookkeeping (scf_dev.cu) */
void gtf_note_launches(int n);
unsigned long long gtf_launch_count(void);
int gtf_fp64_peak(double *gflops);

#ifdef __cplusplus
}
#endif

#endif
