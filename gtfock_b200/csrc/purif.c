/*
 * purif.c -- purification / DIIS API (pscf/purif.h:78-86) on one GPU.
 *
 * create_purif lays out the single "process" of the purification grid as the
 * whole matrix (pscf/purif.c:22-150 with nprow = npcol = npgrd = 1): host
 * blocks of nbf x nbf, ldx = nbf.  compute_diis and compute_purification
 * copy the host blocks to the device, run cuda/purif.cu and copy back, so
 * pscf/scf.c keeps reading and writing its host arrays unchanged.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "cuda/gtf_cuda.h"
#include "purif.h"

static double wall(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

purif_t *create_purif(BasisSet_t basis, int nprow_purif, int npcol_purif, int npgrd_purif)
{
    if (basis == NULL) return NULL;
    if (nprow_purif != 1 || npcol_purif != 1 || npgrd_purif != 1) {
        fprintf(stderr, "create_purif: one GPU runs a 1 x 1 x 1 purification grid\n");
        return NULL;
    }
    printf("Initializing purification ...\n");
    purif_t *p = (purif_t *)calloc(1, sizeof(purif_t));
    if (p == NULL) return NULL;
    const int n = CInt_getNumFuncs(basis);
    p->nbf = n;
    p->nobtls = CInt_getNumOccOrb(basis);
    p->nprow_purif = p->npcol_purif = p->npgrd_purif = 1;
    p->np_purif = 1;
    p->runpurif = 1;
    p->rundgemm = 1;
    p->srow_purif = 0;
    p->scol_purif = 0;
    p->nrows_purif = n;
    p->ncols_purif = n;
    p->ldx = n;
    p->meshsize = n * n;
    p->bmax_id = -1;
    const size_t bytes = sizeof(double) * (size_t)n * n;
    /* page-locked, so that every copy of a block to or from the device is a
     * direct DMA; plain heap memory if the pinned blocks cannot be had */
    double **blk[5] = {&p->H_block, &p->X_block, &p->S_block, &p->F_block, &p->D_block};
    p->host_pinned = 1;
    for (int k = 0; k < 5; k++) {
        *blk[k] = (double *)gtf_pinned_alloc(bytes);
        if (*blk[k] == NULL) {
            p->host_pinned = 0;
            break;
        }
        memset(*blk[k], 0, bytes);
    }
    if (!p->host_pinned) {
        for (int k = 0; k < 5; k++) {
            gtf_pinned_free(*blk[k]);
            *blk[k] = (double *)calloc(1, bytes);
        }
    }
    if (!p->H_block || !p->X_block || !p->S_block || !p->F_block || !p->D_block) {
        destroy_purif(p);
        return NULL;
    }
    gtf_purif_dev_t *dev = NULL;
    if (gtf_purif_create(n, p->nobtls, NULL, &dev) != GTF_OK) {
        fprintf(stderr, "create_purif: device initialisation failed\n");
        destroy_purif(p);
        return NULL;
    }
    p->dev = dev;
    printf("  GPU uses %.3f MB\n", (2.0 * MAX_DIIS + 10.0) * bytes / 1024.0 / 1024.0);
    printf("  Done\n");
    return p;
}

void destroy_purif(purif_t *p)
{
    if (p == NULL) return;
    if (p->dev) gtf_purif_destroy((gtf_purif_dev_t *)p->dev);
    double *blk[5] = {p->H_block, p->X_block, p->S_block, p->F_block, p->D_block};
    for (int k = 0; k < 5; k++) {
        if (p->host_pinned)
            gtf_pinned_free(blk[k]);
        else
            free(blk[k]);
    }
    free(p);
}

static int ensure_sx(purif_t *p)
{
    if (p->sx_uploaded) return 0;
    if (gtf_purif_set_sx((gtf_purif_dev_t *)p->dev, p->S_block, p->X_block) != GTF_OK) return -1;
    p->sx_uploaded = 1;
    return 0;
}

int compute_purification(purif_t *p, double *F_block, double *D_block)
{
    p->timedgemm = p->timepdgemm = p->timepass = p->timetr = 0.0;
    if (ensure_sx(p) != 0) return -1;
    const double t0 = wall();
    int it = 0;
    if (gtf_purif_run((gtf_purif_dev_t *)p->dev, F_block, D_block, &it) != GTF_OK) {
        fprintf(stderr, "compute_purification: device failure\n");
        return -1;
    }
    const double t1 = wall();
    p->timepass = t1 - t0;
    p->timepdgemm = t1 - t0;
    p->timedgemm = t1 - t0;
    p->last_iters = it;
    return it;
}

void compute_diis(PFock_t pfock, purif_t *p, double *D_block, double *F_block, int iter)
{
    (void)pfock;
    if (ensure_sx(p) != 0) return;
    if (gtf_diis_step((gtf_purif_dev_t *)p->dev, D_block, F_block, iter) != GTF_OK)
        fprintf(stderr, "compute_diis: device failure\n");
}
