/*
 * scf_driver.c -- native SCF driver (gtfock_b200.h: gtf_scf_*).
 *
 * Runs the loop of pscf/scf.c:329-459 on one GPU: initial guess
 * (pscf/scf.c:34-76), Fock build, energy E = sum D (H + F)
 * (pscf/scf.c:80-102), DIIS, purification; stops early when
 * |E - E_prev| < 1e-11 (pscf/scf.c:373).
 *   mode 0: every matrix crosses the C API in host memory, as scf.c does;
 *   mode 1: D, F, S, X, H stay in device memory between the steps.
 * gtf_scf_create does the set-up of pscf/scf.c:298-314 and init_oedmat
 * (pscf/scf.c:131-185) once; gtf_scf_solve can then run many solves.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "cuda/gtf_cuda.h"
#include "gtfock_b200.h"

extern gtf_fock_dev_t *gtf_pfock_device(PFock_t pf);
extern int gtf_dev_malloc(void **p, size_t bytes);
extern void gtf_dev_free(void *p);
extern int gtf_dev_copy(void *dst, const void *src, size_t bytes, int kind, void *stream);
extern int gtf_dev_energy(double *F, const double *H, const double *D, int n, void *stream, double *energy);

struct gtf_scf {
    BasisSet_t basis;
    PFock_t pf;
    purif_t *pur;
    int n;
    double enuc;
    double *D0;          /* initial guess (host) */
    double *dD, *dF;     /* device-resident D and F (mode 1) */
    double etol;         /* stop when |E_k - E_k-1| < etol */
    int incr, incr_period;   /* incremental Fock builds (restarted by every solve) */
    int pur_mode_set;        /* purification mode chosen by gtf_scf_set_purification */
    double incr_tau;
    int last_mode;       /* where the last solve left D: 0 host, 1 device */
};

static double wall(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* initial guess of pscf/scf.c:34-76 (half density from the per-atom guess
 * blocks, scaled by R/2); also used by the batched driver */
int gtf_initial_density(BasisSet_t basis, double *D, int n)
{
    memset(D, 0, sizeof(double) * (size_t)n * n);
    double R = 1.0;
    int Nn = CInt_getNneutral(basis), Q = CInt_getTotalCharge(basis);
    if (Q != 0 && Nn != 0) R = (Nn - Q) / (double)Nn;
    for (int a = 0; a < CInt_getNumAtoms(basis); a++) {
        double *g;
        int sp, ep;
        CInt_getInitialGuess(basis, a, &g, &sp, &ep);
        const int ld = ep - sp + 1;
        for (int r = sp; r <= ep; r++)
            for (int c = sp; c <= ep; c++) D[(size_t)r * n + c] = g[(r - sp) * ld + (c - sp)];
    }
    for (size_t k = 0; k < (size_t)n * n; k++) D[k] *= R / 2.0;
    return 0;
}

void gtf_scf_destroy(gtf_scf_t *s)
{
    if (!s) return;
    gtf_dev_free(s->dD);
    gtf_dev_free(s->dF);
    if (s->pf) {
        PFock_destroyOvlMat(s->pf);
        PFock_destroyCoreHMat(s->pf);
    }
    if (s->pur) destroy_purif(s->pur);
    if (s->pf) PFock_destroy(s->pf);
    if (s->basis) CInt_destroyBasisSet(s->basis);
    free(s->D0);
    free(s);
}

gtf_scf_t *gtf_scf_create(const char *bsfile, const char *xyzfile, double tolscr)
{
    if (!bsfile || !xyzfile) return NULL;
    gtf_scf_t *s = (gtf_scf_t *)calloc(1, sizeof(gtf_scf_t));
    if (!s) return NULL;
    CInt_createBasisSet(&s->basis);
    if (CInt_loadBasisSet(s->basis, (char *)bsfile, (char *)xyzfile) != CINT_STATUS_SUCCESS) {
        gtf_scf_destroy(s);
        return NULL;
    }
    s->n = CInt_getNumFuncs(s->basis);
    s->enuc = CInt_getNucEnergy(s->basis);
    const int n = s->n;
    if (PFock_create(s->basis, 1, 1, 4, tolscr, 1, 1, &s->pf) != PFOCK_STATUS_SUCCESS) {
        s->pf = NULL;
        gtf_scf_destroy(s);
        return NULL;
    }
    s->pur = create_purif(s->basis, 1, 1, 1);
    s->D0 = (double *)malloc(sizeof(double) * (size_t)n * n);
    if (!s->pur || !s->D0 ||
        gtf_dev_malloc((void **)&s->dD, sizeof(double) * (size_t)n * n) ||
        gtf_dev_malloc((void **)&s->dF, sizeof(double) * (size_t)n * n)) {
        gtf_scf_destroy(s);
        return NULL;
    }
    /* init_oedmat, pscf/scf.c:131-185; the device copies are kept for mode 1 */
    PFock_createOvlMat(s->pf, s->basis);
    PFock_getOvlMat(s->pf, 0, n - 1, 0, n - 1, n, s->pur->S_block);
    PFock_getOvlMat2(s->pf, 0, n - 1, 0, n - 1, n, s->pur->X_block);
    PFock_createCoreHMat(s->pf, s->basis);
    PFock_getCoreHMat(s->pf, 0, n - 1, 0, n - 1, n, s->pur->H_block);
    PFock_setNumDenMat(1, s->pf);
    gtf_initial_density(s->basis, s->D0, n);
    s->etol = 1e-11;
    s->last_mode = 0;
    return s;
}

int gtf_scf_set_options(gtf_scf_t *s, int prec_mode, double fp32_cutoff, double etol)
{
    if (!s || !(etol >= 0.0)) return -1;
    if (gtf_pfock_set_precision(s->pf, prec_mode, fp32_cutoff) != PFOCK_STATUS_SUCCESS) return -2;
    s->etol = etol;
    /* mixed precision takes the split-BF16 tensor-core purification products
     * too, unless a mode was chosen explicitly */
    if (!s->pur_mode_set && gtf_purif_set_mode((gtf_purif_dev_t *)s->pur->dev, prec_mode == 1 ? 1 : 0) != GTF_OK)
        return -3;
    return 0;
}

int gtf_scf_set_incremental(gtf_scf_t *s, int on, double tau, int period)
{
    if (!s) return -1;
    if (gtf_pfock_set_incremental(s->pf, on, tau, period) != PFOCK_STATUS_SUCCESS) return -2;
    s->incr = on ? 1 : 0;
    s->incr_tau = tau;
    s->incr_period = period;
    return 0;
}

int gtf_scf_set_purification(gtf_scf_t *s, int mode)
{
    if (!s || !s->pur) return -1;
    s->pur_mode_set = 1;
    return gtf_purif_set_mode((gtf_purif_dev_t *)s->pur->dev, mode) == GTF_OK ? 0 : -2;
}

int gtf_scf_purification_iters(gtf_scf_t *s, int *bf16_iters, int *fp64_iters)
{
    if (!s || !s->pur) return -1;
    gtf_purif_last_iters((gtf_purif_dev_t *)s->pur->dev, bf16_iters, fp64_iters);
    return 0;
}

int gtf_scf_get_density(gtf_scf_t *s, double *D)
{
    if (!s || !D) return -1;
    const size_t mb = sizeof(double) * (size_t)s->n * s->n;
    if (s->last_mode == 1) {
        void *st = gtf_fock_stream(gtf_pfock_device(s->pf));
        return gtf_dev_copy(D, s->dD, mb, 1, st) == 0 ? 0 : -2;
    }
    memcpy(D, s->pur->D_block, mb);
    return 0;
}

int gtf_scf_nbf(gtf_scf_t *s) { return s ? s->n : -1; }

int gtf_scf_solve(gtf_scf_t *s, int niters, int mode, double *energies, double *timings)
{
    if (!s || niters <= 0 || (mode != 0 && mode != 1)) return -1;
    s->last_mode = mode;
    const int n = s->n;
    const size_t nn = (size_t)n * n, mb = sizeof(double) * nn;
    purif_t *pur = s->pur;
    gtf_purif_dev_t *pd = (gtf_purif_dev_t *)pur->dev;
    gtf_purif_reset(pd);
    pur->len_diis = 0;
    /* an incremental sum never carries over from the previous solve */
    if (s->incr && gtf_pfock_set_incremental(s->pf, 1, s->incr_tau, s->incr_period) != PFOCK_STATUS_SUCCESS)
        return -7;
    double t_fock = 0.0, t_diis = 0.0, t_pur = 0.0, h2d = 0.0, d2h = 0.0;
    const unsigned long long l0 = gtf_launch_count();
    const double t_start = wall();
    int iter, ret = 0;
    double e0 = -1.0;
    memcpy(pur->D_block, s->D0, mb);
    if (mode == 0) {
        if (!pur->sx_uploaded) {
            h2d += 2.0 * mb;   /* S and X read once by purif */
        }
        for (iter = 0; iter < niters; iter++) {
            double t1 = wall();
            PFock_putDenMat(0, n - 1, 0, n - 1, n, pur->D_block, 0, s->pf);
            PFock_commitDenMats(s->pf);
            if (PFock_computeFock(s->basis, s->pf) != PFOCK_STATUS_SUCCESS) { ret = -5; break; }
            PFock_getMat(s->pf, PFOCK_MAT_TYPE_F, 0, 0, n - 1, 0, n - 1, n, pur->F_block);
            h2d += mb;
            d2h += mb;
            double e = 0.0;
            for (size_t k = 0; k < nn; k++) {
                pur->F_block[k] += pur->H_block[k];
                e += pur->D_block[k] * (pur->H_block[k] + pur->F_block[k]);
            }
            double t2 = wall();
            t_fock += t2 - t1;
            if (energies) energies[iter] = e + s->enuc;
            if (iter > 0 && fabs(e - e0) < s->etol) {
                iter++;
                break;
            }
            e0 = e;
            t1 = wall();
            compute_diis(s->pf, pur, pur->D_block, pur->F_block, iter);
            h2d += 2.0 * mb;
            d2h += mb;
            t2 = wall();
            t_diis += t2 - t1;
            if (compute_purification(pur, pur->F_block, pur->D_block) < 0) { ret = -6; break; }
            h2d += mb;
            d2h += mb;
            t_pur += wall() - t2;
        }
    } else {
        gtf_fock_dev_t *fd = gtf_pfock_device(s->pf);
        void *st = gtf_fock_stream(fd);
        gtf_purif_set_sx_dev(pd, gtf_fock_onee_dev(fd, 0), gtf_fock_onee_dev(fd, 1));
        pur->sx_uploaded = 1;
        const double *dH = gtf_fock_onee_dev(fd, 2);
        gtf_dev_copy(s->dD, s->D0, mb, 0, st);
        h2d += mb;
        for (iter = 0; iter < niters; iter++) {
            double t1 = wall();
            const double *dFock = NULL;
            if (gtf_pfock_compute_dev(s->pf, s->dD, &dFock) != PFOCK_STATUS_SUCCESS) { ret = -5; break; }
            gtf_dev_copy(s->dF, dFock, mb, 2, st);
            double e = 0.0;
            gtf_dev_energy(s->dF, dH, s->dD, n, st, &e);
            double t2 = wall();
            t_fock += t2 - t1;
            if (energies) energies[iter] = e + s->enuc;
            if (iter > 0 && fabs(e - e0) < s->etol) {
                iter++;
                break;
            }
            e0 = e;
            t1 = wall();
            gtf_diis_step_dev(pd, s->dD, s->dF, iter);
            t2 = wall();
            t_diis += t2 - t1;
            int it = 0;
            if (gtf_purif_run_dev(pd, s->dF, s->dD, &it) != GTF_OK) { ret = -6; break; }
            t_pur += wall() - t2;
        }
    }
    if (timings) {
        timings[0] = t_fock;
        timings[1] = t_diis;
        timings[2] = t_pur;
        timings[3] = wall() - t_start;
        timings[4] = h2d;
        timings[5] = d2h;
        timings[6] = (double)(gtf_launch_count() - l0);
    }
    return ret < 0 ? ret : iter;
}

int gtf_scf_run(const char *bsfile, const char *xyzfile, double tolscr, int niters, int mode,
                double *energies, double *timings)
{
    if (!bsfile || !xyzfile || niters <= 0 || (mode != 0 && mode != 1)) return -1;
    const double t0 = wall();
    gtf_scf_t *s = gtf_scf_create(bsfile, xyzfile, tolscr);
    if (!s) return -3;
    double t[8] = {0};
    int it = gtf_scf_solve(s, niters, mode, energies, t);
    gtf_scf_destroy(s);
    if (timings) {
        for (int k = 0; k < 7; k++) timings[k] = t[k];
        timings[3] = wall() - t0;  /* whole job: set-up, solve, tear-down */
    }
    return it;
}
