/*
 * ref_probe.c -- drives the reference's own PFock engine (pfock/pfock.c,
 * compiled unchanged from the reference sources by oracle/ref/Makefile) on
 * one process and dumps what the tests compare the oracle against:
 *   <out>.screen : nshells, nnz, maxvalue, shellptr[nshells+1],
 *                  shellid[nnz], shellrid[nnz], shellvalue[nnz]
 *                  (pfock/screening.c:110-175)
 *   <out>.fock   : nbf, usq, uitl, F[nbf*nbf] = PFock_getMat(F) for the
 *                  density read from <D.bin> (nbf*nbf doubles, row-major)
 * Test infrastructure only.
 *
 * usage: ref_probe <basis.gbs> <mol.xyz> <tolscr> <ntasks> <D.bin> <out> [symm]
 * symm 0 runs the reference's non-symmetric-density path (PFock_create's
 * symm argument, pfock/pfock.c:828, 1117-1121, 1704-1718).
 */
#include <stdio.h>
#include <stdlib.h>

#include <mpi.h>
#include "pfock.h"
#include "CInt.h"

int main(int argc, char **argv)
{
    if (argc != 7 && argc != 8) {
        fprintf(stderr, "usage: %s basis xyz tolscr ntasks D.bin out [symm]\n", argv[0]);
        return 2;
    }
    const int symm = argc == 8 ? atoi(argv[7]) : 1;
    int provided;
    MPI_Init_thread(&argc, &argv, MPI_THREAD_MULTIPLE, &provided);
    BasisSet_t basis;
    CInt_createBasisSet(&basis);
    if (CInt_loadBasisSet(basis, argv[1], argv[2]) != CINT_STATUS_SUCCESS) return 3;
    double tol = atof(argv[3]);
    int ntasks = atoi(argv[4]);
    PFock_t pf;
    if (PFock_create(basis, 1, 1, ntasks, tol, 1, symm, &pf) != PFOCK_STATUS_SUCCESS) return 4;
    int nshells = pf->nshells, nnz = pf->nnz, nbf = pf->nbf;
    char path[2048];
    snprintf(path, sizeof(path), "%s.screen", argv[6]);
    FILE *fp = fopen(path, "wb");
    fwrite(&nshells, sizeof(int), 1, fp);
    fwrite(&nnz, sizeof(int), 1, fp);
    fwrite(&pf->maxvalue, sizeof(double), 1, fp);
    fwrite(pf->shellptr, sizeof(int), nshells + 1, fp);
    fwrite(pf->shellid, sizeof(int), nnz, fp);
    fwrite(pf->shellrid, sizeof(int), nnz, fp);
    fwrite(pf->shellvalue, sizeof(double), nnz, fp);
    fclose(fp);

    double *D = (double *)malloc(sizeof(double) * nbf * nbf);
    double *F = (double *)malloc(sizeof(double) * nbf * nbf);
    fp = fopen(argv[5], "rb");
    if (fp == NULL || fread(D, sizeof(double), (size_t)nbf * nbf, fp) != (size_t)nbf * nbf) return 5;
    fclose(fp);
    PFock_setNumDenMat(1, pf);
    PFock_putDenMat(0, nbf - 1, 0, nbf - 1, nbf, D, 0, pf);
    PFock_commitDenMats(pf);
    PFock_computeFock(basis, pf);
    PFock_getMat(pf, PFOCK_MAT_TYPE_F, 0, 0, nbf - 1, 0, nbf - 1, nbf, F);
    snprintf(path, sizeof(path), "%s.fock", argv[6]);
    fp = fopen(path, "wb");
    fwrite(&nbf, sizeof(int), 1, fp);
    fwrite(&pf->usq, sizeof(double), 1, fp);
    fwrite(&pf->uitl, sizeof(double), 1, fp);
    fwrite(F, sizeof(double), (size_t)nbf * nbf, fp);
    fclose(fp);
    PFock_destroy(pf);
    CInt_destroyBasisSet(basis);
    MPI_Finalize();
    return 0;
}
