/*
 * pfock.c -- the PFock API (pfock/pfock.h:241-565) on one B200.
 *
 * Host-side state and argument checking follow pfock/pfock.c; the compute
 * lives in cuda/fock.cu (screening, pair list, Fock build) and cuda/onee.cu
 * (S, H, X).  Messages use the reference's PFOCK_PRINTF convention
 * (pfock/config.h:16-29).
 */
#define _GNU_SOURCE
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "gtf_basis.h"
#include "cuda/gtf_cuda.h"
#include "gtfock_b200.h"
#include "pfock.h"

#define PFOCK_PRINTF(level, fmt, ...)                                               \
    do {                                                                            \
        if ((unsigned)(level) <= 2) {                                               \
            fprintf(stdout, "%s() line %d: " fmt, __FUNCTION__, __LINE__, ##__VA_ARGS__); \
            fflush(stdout);                                                         \
        }                                                                           \
    } while (0)

struct PFock {
    BasisSet_t basis;
    gtf_fock_dev_t *dev;
    int nbf, nshells, natoms;
    int nprow, npcol, ntasks;
    int max_numdmat, num_dmat;
    int nosymm;
    int committed;
    double tolscr;
    double mem_cpu;
    double *local_mirror;       /* PFock_getLocalMatPtr snapshot */
    double timepass;            /* seconds of the last PFock_computeFock */
};

static double wall(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static gtf_basis_view_t view_of(BasisSet_t b)
{
    gtf_basis_view_t v;
    v.natoms = b->natoms;
    v.nshells = b->nshells;
    v.nbf = b->nbf;
    v.nbf_cart = b->nbf_cart;
    v.nprims = b->nprims;
    v.pure = b->pure;
    v.Z = b->Z;
    v.xyz = b->xyz;
    v.sh_atom = b->sh_atom;
    v.sh_L = b->sh_L;
    v.sh_nprim = b->sh_nprim;
    v.sh_pstart = b->sh_pstart;
    v.f_start = b->f_start;
    v.fc_start = b->fc_start;
    v.alpha = b->alpha;
    v.coef = b->coef;
    return v;
}

static PFockStatus_t map_err(int e)
{
    switch (e) {
        case GTF_OK: return PFOCK_STATUS_SUCCESS;
        case GTF_ERR_ALLOC: return PFOCK_STATUS_ALLOC_FAILED;
        case GTF_ERR_INVALID: return PFOCK_STATUS_INVALID_VALUE;
        case GTF_ERR_NODEVICE: return PFOCK_STATUS_INIT_FAILED;
        default: return PFOCK_STATUS_EXECUTION_FAILED;
    }
}

PFockStatus_t PFock_create(BasisSet_t basis, int nprow, int npcol, int ntasks,
                           double tolscr, int max_numdmat, int symm, PFock_t *_pfock)
{
    if (_pfock == NULL || basis == NULL || basis->nshells <= 0) return PFOCK_STATUS_INVALID_VALUE;
    *_pfock = NULL;
    /* one GPU holds the whole problem: the process grid is 1 x 1
     * (pfock/pfock.c:841-849 checks nprow*npcol against the MPI size) */
    if (nprow != 1 || npcol != 1) {
        PFOCK_PRINTF(1, "Invalid nprow or npcol\n");
        return PFOCK_STATUS_INVALID_VALUE;
    }
    const char *env = getenv("GTFOCK_TOLSCR");
    if (env && *env) {
        double t = atof(env);
        if (t > 0.0) tolscr = t;
    }
    if (tolscr < 0.0) {
        PFOCK_PRINTF(1, "Invalid screening threshold\n");
        return PFOCK_STATUS_INVALID_VALUE;
    }
    if (max_numdmat <= 0) {
        PFOCK_PRINTF(1, "Invalid number of density matrices\n");
        return PFOCK_STATUS_INVALID_VALUE;
    }
    PFock_t pf = (PFock_t)calloc(1, sizeof(struct PFock));
    if (pf == NULL) {
        PFOCK_PRINTF(1, "Failed to allocate memory: %zu\n", sizeof(struct PFock));
        return PFOCK_STATUS_ALLOC_FAILED;
    }
    pf->basis = basis;
    pf->nbf = basis->nbf;
    pf->nshells = basis->nshells;
    pf->natoms = basis->natoms;
    pf->nprow = nprow;
    pf->npcol = npcol;
    pf->ntasks = ntasks;
    pf->max_numdmat = max_numdmat;
    pf->num_dmat = max_numdmat;
    pf->nosymm = 0;
    pf->tolscr = tolscr;
    gtf_basis_view_t v = view_of(basis);
    int e = gtf_fock_create(&v, tolscr, max_numdmat, &pf->dev);
    if (e != GTF_OK) {
        PFOCK_PRINTF(1, "device initialisation failed: %s\n", gtf_last_error());
        if (pf->dev) gtf_fock_destroy(pf->dev);
        free(pf);
        return map_err(e);
    }
    /* symm = 0 (pfock/pfock.c:828): densities may be non-symmetric.  The
     * engine returns what the reference returns, (F[D] + F[D^T]^T) / 2 with
     * its unique-quartet digestion (pfock/pfock.c:1704-1718);
     * gtf_pfock_set_nosymm_mode selects the exact F = 2 J[D] - K[D] instead.
     * For a symmetric D both are the symm = 1 result. */
    if (symm == 0) {
        e = gtf_fock_set_nosymm(pf->dev, GTF_NOSYMM_REFERENCE);
        if (e != GTF_OK) {
            gtf_fock_destroy(pf->dev);
            free(pf);
            return map_err(e);
        }
        pf->nosymm = 1;
    }
    pf->mem_cpu = sizeof(struct PFock) + (double)gtf_fock_device_bytes(pf->dev);
    *_pfock = pf;
    return PFOCK_STATUS_SUCCESS;
}

PFockStatus_t PFock_destroy(PFock_t pf)
{
    if (pf == NULL) return PFOCK_STATUS_INVALID_VALUE;
    gtf_fock_destroy(pf->dev);
    free(pf->local_mirror);
    free(pf);
    return PFOCK_STATUS_SUCCESS;
}

/* Note: like the reference (pfock/pfock.c:1041-1055) this returns
 * PFOCK_STATUS_EXECUTION_FAILED after setting the count successfully; callers
 * such as pscf/scf.c:333 ignore the status. */
PFockStatus_t PFock_setNumDenMat(int numdmat, PFock_t pf)
{
    if (pf->committed == 1) {
        PFOCK_PRINTF(1, "Can't change number of matrices after PFock_commitDenMats() is called.\n");
        return PFOCK_STATUS_EXECUTION_FAILED;
    }
    if (numdmat <= 0 || numdmat > pf->max_numdmat) {
        PFOCK_PRINTF(1, "Invalid number of density matrices\n");
        return PFOCK_STATUS_INVALID_VALUE;
    }
    pf->num_dmat = numdmat;
    return PFOCK_STATUS_EXECUTION_FAILED;
}

PFockStatus_t PFock_putDenMat(int rowstart, int rowend, int colstart, int colend,
                              int stride, double *dmat, int index, PFock_t pf)
{
    if (pf->committed == 1) {
        PFOCK_PRINTF(1, "Can't change density matrix after PFock_commitDenMats() is called.\n");
        return PFOCK_STATUS_EXECUTION_FAILED;
    }
    if (index < 0 || index >= pf->num_dmat) {
        PFOCK_PRINTF(1, "Invalid index\n");
        return PFOCK_STATUS_INVALID_VALUE;
    }
    if (dmat == NULL || stride < colend - colstart + 1) return PFOCK_STATUS_INVALID_VALUE;
    return map_err(gtf_fock_put_density(pf->dev, index, rowstart, rowend, colstart, colend, stride, dmat));
}

PFockStatus_t PFock_putDenMatGA(int ga, int index, PFock_t pf)
{
    (void)ga; (void)index; (void)pf;
    PFOCK_PRINTF(1, "Global Arrays are not used on one GPU\n");
    return PFOCK_STATUS_INVALID_VALUE;
}

PFockStatus_t PFock_fillDenMat(double value, int index, PFock_t pf)
{
    if (pf->committed == 1) {
        PFOCK_PRINTF(1, "Can't change density matrix after PFock_commitDenMats() is called.\n");
        return PFOCK_STATUS_EXECUTION_FAILED;
    }
    if (index < 0 || index >= pf->num_dmat) {
        PFOCK_PRINTF(1, "Invalid index\n");
        return PFOCK_STATUS_INVALID_VALUE;
    }
    return map_err(gtf_fock_fill_density(pf->dev, index, value));
}

PFockStatus_t PFock_commitDenMats(PFock_t pf)
{
    pf->committed = 1;
    return PFOCK_STATUS_SUCCESS;
}

PFockStatus_t PFock_sync(PFock_t pf)
{
    (void)pf;
    return PFOCK_STATUS_SUCCESS;
}

PFockStatus_t PFock_getMat(PFock_t pf, PFockMatType_t type, int index,
                           int rowstart, int rowend, int colstart, int colend,
                           int stride, double *mat)
{
    if (index < 0 || index >= pf->max_numdmat) {
        PFOCK_PRINTF(1, "Invalid index\n");
        return PFOCK_STATUS_INVALID_VALUE;
    }
    if ((int)type < 0 || (int)type > 3 || mat == NULL) return PFOCK_STATUS_INVALID_VALUE;
    return map_err(gtf_fock_get_mat(pf->dev, (int)type, index, rowstart, rowend, colstart, colend,
                                    stride, mat));
}

PFockStatus_t PFock_getMatGA(PFock_t pf, PFockMatType_t type, int index, int ga)
{
    (void)pf; (void)type; (void)index; (void)ga;
    PFOCK_PRINTF(1, "Global Arrays are not used on one GPU\n");
    return PFOCK_STATUS_INVALID_VALUE;
}

PFockStatus_t PFock_getLocalMatInds(PFock_t pf, int *rowstart, int *rowend,
                                    int *colstart, int *colend)
{
    /* the single process owns the whole matrix */
    *rowstart = 0;
    *rowend = pf->nbf - 1;
    *colstart = 0;
    *colend = pf->nbf - 1;
    return PFOCK_STATUS_SUCCESS;
}

/* Returns a host snapshot of the whole matrix (the local block of the only
 * process); writes to it do not reach the device copy. */
PFockStatus_t PFock_getLocalMatPtr(PFock_t pf, PFockMatType_t type, int index,
                                   int *rowstart, int *rowend, int *colstart, int *colend,
                                   int *stride, double **mat)
{
    if (index < 0 || index >= pf->max_numdmat) {
        PFOCK_PRINTF(1, "Invalid index\n");
        return PFOCK_STATUS_INVALID_VALUE;
    }
    if (pf->local_mirror == NULL) {
        pf->local_mirror = (double *)malloc(sizeof(double) * (size_t)pf->nbf * pf->nbf);
        if (pf->local_mirror == NULL) return PFOCK_STATUS_ALLOC_FAILED;
    }
    PFockStatus_t st = PFock_getMat(pf, type, index, 0, pf->nbf - 1, 0, pf->nbf - 1, pf->nbf,
                                    pf->local_mirror);
    if (st != PFOCK_STATUS_SUCCESS) return st;
    PFock_getLocalMatInds(pf, rowstart, rowend, colstart, colend);
    *stride = pf->nbf;
    *mat = pf->local_mirror;
    return PFOCK_STATUS_SUCCESS;
}

PFockStatus_t PFock_getMatGAHandle(PFock_t pf, PFockMatType_t type, int index, int *ga)
{
    (void)pf; (void)type; (void)index;
    if (ga) *ga = 0;
    return PFOCK_STATUS_INVALID_VALUE;
}

PFockStatus_t PFock_computeFock(BasisSet_t basis, PFock_t pf)
{
    (void)basis;
    const double t0 = wall();
    pf->committed = 0;
    int e = gtf_fock_compute(pf->dev, pf->num_dmat);
    if (e != GTF_OK) {
        PFOCK_PRINTF(1, "Fock build failed: %s\n", gtf_last_error());
        return map_err(e);
    }
    pf->timepass = wall() - t0;
    return PFOCK_STATUS_SUCCESS;
}

PFockStatus_t PFock_createCoreHMat(PFock_t pf, BasisSet_t basis)
{
    (void)basis;
    return map_err(gtf_fock_one_electron(pf->dev, 0, 1));
}

PFockStatus_t PFock_destroyCoreHMat(PFock_t pf)
{
    gtf_fock_release_onee(pf->dev, 2);
    return PFOCK_STATUS_SUCCESS;
}

PFockStatus_t PFock_getCoreHMat(PFock_t pf, int rowstart, int rowend, int colstart, int colend,
                                int stride, double *mat)
{
    return map_err(gtf_fock_get_onee(pf->dev, 2, rowstart, rowend, colstart, colend, stride, mat));
}

PFockStatus_t PFock_createOvlMat(PFock_t pf, BasisSet_t basis)
{
    (void)basis;
    return map_err(gtf_fock_one_electron(pf->dev, 1, 0));
}

PFockStatus_t PFock_destroyOvlMat(PFock_t pf)
{
    gtf_fock_release_onee(pf->dev, 0);
    gtf_fock_release_onee(pf->dev, 1);
    return PFOCK_STATUS_SUCCESS;
}

PFockStatus_t PFock_getOvlMat(PFock_t pf, int rowstart, int rowend, int colstart, int colend,
                              int stride, double *mat)
{
    return map_err(gtf_fock_get_onee(pf->dev, 0, rowstart, rowend, colstart, colend, stride, mat));
}

PFockStatus_t PFock_getOvlMat2(PFock_t pf, int rowstart, int rowend, int colstart, int colend,
                               int stride, double *mat)
{
    return map_err(gtf_fock_get_onee(pf->dev, 1, rowstart, rowend, colstart, colend, stride, mat));
}

PFockStatus_t PFock_getMemorySize(PFock_t pf, double *mem_cpu)
{
    /* bytes held by the engine: the host struct plus its device buffers */
    *mem_cpu = pf->mem_cpu;
    return PFOCK_STATUS_SUCCESS;
}

PFockStatus_t PFock_getStatistics(PFock_t pf)
{
    int nnz;
    double maxv, usq, uitl, ms_total, ms_eri, ms_other;
    gtf_fock_screening_info(pf->dev, &nnz, &maxv, &usq, &uitl);
    gtf_fock_last_timing(pf->dev, &ms_total, &ms_eri, &ms_other);
    /* total unique quartets before screening (pfock/pfock.c:1994-1995) */
    double tsq = pf->nshells;
    tsq = ((tsq + 1) * tsq / 2.0 + 1) * tsq * (tsq + 1) / 4.0;
    printf("    PFock Statistics:\n");
    printf("      average totaltime   = %.3g\n"
           "      average timegather  = %.3g\n"
           "      average timeinit    = %.3g\n"
           "      average timecomp    = %.3g\n"
           "      average timereduce  = %.3g\n"
           "      average timescatter = %.3g\n"
           "      comp/total = %.3g\n",
           ms_total * 1e-3, 0.0, ms_other * 1e-3, ms_eri * 1e-3, 0.0, 0.0,
           ms_total > 0 ? ms_eri / ms_total : 0.0);
    printf("      usq = %.4g (lb = %.3g)\n"
           "      uitl = %.4g (lb = %.3g)\n"
           "      nsq = %.4g (screening = %.3g)\n",
           usq, 1.0, uitl, 1.0, tsq, usq / tsq);
    printf("      load blance = %.3lf\n", 1.0);
    printf("      steals = %.3g (average = %.3g)\n"
           "      stealfrom = %.3g (average = %.3g)\n"
           "      GAcalls = %.3g\n"
           "      GAvolume %.3g MB\n",
           0.0, 0.0, 0.0, 0.0, 0.0, 0.0);
    return PFOCK_STATUS_SUCCESS;
}

/* ---------------- extensions (gtfock_b200.h) ---------------- */

PFockStatus_t gtf_pfock_counts(PFock_t pf, int *nnz, double *maxvalue, double *usq, double *uitl)
{
    return map_err(gtf_fock_screening_info(pf->dev, nnz, maxvalue, usq, uitl));
}

PFockStatus_t gtf_pfock_screening(PFock_t pf, int *shellptr, int *shellid, int *shellrid,
                                  double *shellvalue)
{
    return map_err(gtf_fock_get_csr(pf->dev, shellptr, shellid, shellrid, shellvalue));
}

PFockStatus_t gtf_pfock_timing(PFock_t pf, double *ms_total, double *ms_eri, double *eri_flops)
{
    gtf_fock_last_timing(pf->dev, ms_total, ms_eri, NULL);
    if (eri_flops) gtf_fock_eri_flops(pf->dev, eri_flops);
    return PFOCK_STATUS_SUCCESS;
}

int gtf_pfock_class_stats(PFock_t pf, int *X, int *Y, double *ms, double *nquart)
{
    return gtf_fock_class_stats(pf->dev, X, Y, ms, nquart);
}

int gtf_pfock_class_work(PFock_t pf, double *flops, double *nprimq)
{
    return gtf_fock_class_work(pf->dev, flops, nprimq);
}

PFockStatus_t gtf_pfock_set_precision(PFock_t pf, int mode, double fp32_cutoff)
{
    return map_err(gtf_fock_set_precision(pf->dev, mode, fp32_cutoff));
}

PFockStatus_t gtf_pfock_set_nosymm_mode(PFock_t pf, int mode)
{
    if (pf == NULL) return PFOCK_STATUS_INVALID_VALUE;
    if (!pf->nosymm || (mode != GTF_NOSYMM_REFERENCE && mode != GTF_NOSYMM_EXACT)) {
        PFOCK_PRINTF(1, "non-symmetric density mode: engine created with symm = 1, or mode not 1 or 2\n");
        return PFOCK_STATUS_INVALID_VALUE;
    }
    int e = gtf_fock_set_nosymm(pf->dev, mode);
    if (e != GTF_OK) PFOCK_PRINTF(1, "%s\n", gtf_last_error());
    return map_err(e);
}

PFockStatus_t gtf_pfock_set_shard(PFock_t pf, int shard, int nshards)
{
    if (pf == NULL) return PFOCK_STATUS_INVALID_VALUE;
    return map_err(gtf_fock_set_shard(pf->dev, shard, nshards));
}

PFockStatus_t gtf_pfock_autotune(PFock_t pf, int reps)
{
    if (pf == NULL) return PFOCK_STATUS_INVALID_VALUE;
    return map_err(gtf_fock_autotune(pf->dev, reps));
}

PFockStatus_t gtf_pfock_precision_stats(PFock_t pf, double *nquart_fp32, double *nquart)
{
    return map_err(gtf_fock_fp32_quartets(pf->dev, nquart_fp32, nquart));
}

PFockStatus_t gtf_pfock_compute_dev(PFock_t pf, const double *dev_D, const double **dev_F)
{
    int e = gtf_fock_put_density_dev(pf->dev, 0, dev_D);
    if (e == GTF_OK) e = gtf_fock_compute(pf->dev, 1);
    if (e != GTF_OK) return map_err(e);
    if (dev_F) *dev_F = gtf_fock_mat_dev(pf->dev, 1, 0);
    return PFOCK_STATUS_SUCCESS;
}

PFockStatus_t gtf_pfock_compute_noalloc(PFock_t pf, const double *dev_D, double *dev_F)
{
    if (pf == NULL) return PFOCK_STATUS_INVALID_VALUE;
    int e = gtf_fock_compute_fixed(pf->dev, dev_D, dev_F);
    if (e != GTF_OK) PFOCK_PRINTF(1, "%s\n", gtf_last_error());
    return map_err(e);
}

PFockStatus_t gtf_pfock_set_incremental(PFock_t pf, int on, double tau, int period)
{
    if (pf == NULL) return PFOCK_STATUS_INVALID_VALUE;
    int e = gtf_fock_set_incremental(pf->dev, on, tau, period);
    if (e != GTF_OK) PFOCK_PRINTF(1, "%s\n", gtf_last_error());
    return map_err(e);
}

PFockStatus_t gtf_pfock_incremental_stats(PFock_t pf, double *nquart_fp64, double *nquart_fp32, double *dmax)
{
    if (pf == NULL) return PFOCK_STATUS_INVALID_VALUE;
    return map_err(gtf_fock_incremental_stats(pf->dev, nquart_fp64, nquart_fp32, dmax));
}

int gtf_pfock_class_work_screened(PFock_t pf, double *flops, double *nprimq)
{
    if (pf == NULL) return -1;
    return gtf_fock_class_work_screened(pf->dev, flops, nprimq);
}

PFockStatus_t gtf_pfock_shard_work(PFock_t pf, double *work)
{
    if (pf == NULL) return PFOCK_STATUS_INVALID_VALUE;
    return map_err(gtf_fock_shard_work(pf->dev, work));
}

/* internal accessors for scf_driver.c */
gtf_fock_dev_t *gtf_pfock_device(PFock_t pf) { return pf->dev; }
