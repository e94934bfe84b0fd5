/*
 * scf_driver.c -- native SCF driver (gtfock_b200.h: gtf_scf_run).
 *
 * Runs the loop of pscf/scf.c:329-459 on one GPU: initial guess
 * (pscf/scf.c:34-76), Fock build, energy E = sum D (H + F)
 * (pscf/scf.c:80-102), DIIS, purification; stops early when
 * |E - E_prev| < 1e-11 (pscf/scf.c:373).
 *   mode 0: every matrix crosses the C API in host memory, as scf.c does;
 *   mode 1: D, F, S, X, H stay in device memory between the steps.
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

static double wall(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static void initial_density(BasisSet_t basis, double *D, int n)
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
}

int gtf_scf_run(const char *bsfile, const char *xyzfile, double tolscr, int niters, int mode,
                double *energies, double *timings)
{
    if (!bsfile || !xyzfile || niters <= 0 || (mode != 0 && mode != 1)) return -1;
    BasisSet_t basis;
    CInt_createBasisSet(&basis);
    if (CInt_loadBasisSet(basis, (char *)bsfile, (char *)xyzfile) != CINT_STATUS_SUCCESS) {
        CInt_destroyBasisSet(basis);
        return -2;
    }
    const int n = CInt_getNumFuncs(basis);
    const size_t nn = (size_t)n * n;
    PFock_t pf;
    if (PFock_create(basis, 1, 1, 4, tolscr, 1, 1, &pf) != PFOCK_STATUS_SUCCESS) {
        CInt_destroyBasisSet(basis);
        return -3;
    }
    purif_t *pur = create_purif(basis, 1, 1, 1);
    if (!pur) {
        PFock_destroy(pf);
        CInt_destroyBasisSet(basis);
        return -4;
    }
    const double enuc = CInt_getNucEnergy(basis);
    double t_fock = 0.0, t_diis = 0.0, t_pur = 0.0;
    const double t_start = wall();
    int iter, ret = 0;
    double e0 = -1.0;
    PFock_createOvlMat(pf, basis);
    PFock_getOvlMat(pf, 0, n - 1, 0, n - 1, n, pur->S_block);
    PFock_getOvlMat2(pf, 0, n - 1, 0, n - 1, n, pur->X_block);
    PFock_createCoreHMat(pf, basis);
    PFock_getCoreHMat(pf, 0, n - 1, 0, n - 1, n, pur->H_block);
    PFock_setNumDenMat(1, pf);
    initial_density(basis, pur->D_block, n);
    if (mode == 0) {
        PFock_destroyOvlMat(pf);
        PFock_destroyCoreHMat(pf);
        for (iter = 0; iter < niters; iter++) {
            double t1 = wall();
            PFock_putDenMat(0, n - 1, 0, n - 1, n, pur->D_block, 0, pf);
            PFock_commitDenMats(pf);
            if (PFock_computeFock(basis, pf) != PFOCK_STATUS_SUCCESS) { ret = -5; break; }
            PFock_getMat(pf, PFOCK_MAT_TYPE_F, 0, 0, n - 1, 0, n - 1, n, pur->F_block);
            double e = 0.0;
            for (size_t k = 0; k < nn; k++) {
                pur->F_block[k] += pur->H_block[k];
                e += pur->D_block[k] * (pur->H_block[k] + pur->F_block[k]);
            }
            double t2 = wall();
            t_fock += t2 - t1;
            if (energies) energies[iter] = e + enuc;
            if (iter > 0 && fabs(e - e0) < 1e-11) {
                iter++;
                break;
            }
            e0 = e;
            t1 = wall();
            compute_diis(pf, pur, pur->D_block, pur->F_block, iter);
            t2 = wall();
            t_diis += t2 - t1;
            if (compute_purification(pur, pur->F_block, pur->D_block) < 0) { ret = -6; break; }
            t_pur += wall() - t2;
        }
    } else {
        gtf_fock_dev_t *fd = gtf_pfock_device(pf);
        void *st = gtf_fock_stream(fd);
        gtf_purif_dev_t *pd = (gtf_purif_dev_t *)pur->dev;
        double *dD = NULL, *dF = NULL;
        if (gtf_dev_malloc((void **)&dD, sizeof(double) * nn) || gtf_dev_malloc((void **)&dF, sizeof(double) * nn)) {
            ret = -7;
            iter = 0;
        } else {
            gtf_purif_set_sx_dev(pd, gtf_fock_onee_dev(fd, 0), gtf_fock_onee_dev(fd, 1));
            pur->sx_uploaded = 1;
            const double *dH = gtf_fock_onee_dev(fd, 2);
            gtf_dev_copy(dD, pur->D_block, sizeof(double) * nn, 0, st);
            for (iter = 0; iter < niters; iter++) {
                double t1 = wall();
                const double *dFock = NULL;
                if (gtf_pfock_compute_dev(pf, dD, &dFock) != PFOCK_STATUS_SUCCESS) { ret = -5; break; }
                gtf_dev_copy(dF, dFock, sizeof(double) * nn, 2, st);
                double e = 0.0;
                gtf_dev_energy(dF, dH, dD, n, st, &e);
                double t2 = wall();
                t_fock += t2 - t1;
                if (energies) energies[iter] = e + enuc;
                if (iter > 0 && fabs(e - e0) < 1e-11) {
                    iter++;
                    break;
                }
                e0 = e;
                t1 = wall();
                gtf_diis_step_dev(pd, dD, dF, iter);
                t2 = wall();
                t_diis += t2 - t1;
                int it = 0;
                if (gtf_purif_run_dev(pd, dF, dD, &it) != GTF_OK) { ret = -6; break; }
                t_pur += wall() - t2;
            }
        }
        gtf_dev_free(dD);
        gtf_dev_free(dF);
        PFock_destroyOvlMat(pf);
        PFock_destroyCoreHMat(pf);
    }
    if (timings) {
        timings[0] = t_fock;
        timings[1] = t_diis;
        timings[2] = t_pur;
        timings[3] = wall() - t_start;
    }
    destroy_purif(pur);
    PFock_destroy(pf);
    CInt_destroyBasisSet(basis);
    return ret < 0 ? ret : iter;
}
