/*
 * purif.h -- density purification and DIIS of gtfock-b200.
 *
 * Same entry points as GTFock's pscf/purif.h:78-86 and a purif_t carrying
 * every field pscf/scf.c reads or writes (runpurif, H/X/S/F/D_block,
 * nrows/ncols/srow/scol_purif, ldx, np_purif and the four timers), so scf.c
 * compiles unchanged.  On one GPU the purification "grid" is one process:
 * the blocks are the full nbf x nbf matrices (row-major, ldx = nbf), host
 * arrays that scf.c fills and reads; the GEMMs and element-wise steps run on
 * the device.  S_block and X_block are read once, by the first compute_diis
 * or compute_purification call (scf.c fills them before its SCF loop).
 */
#ifndef __PURIF_H__
#define __PURIF_H__

#include <mpi.h>

#include "CInt.h"
#include "pfock.h"

#define MAX_DIIS 10
#define LDBMAT 128

typedef struct _purif_t
{
    int runpurif;
    int rundgemm;
    int nbf;
    int nobtls;
    int np_purif;
    int nprow_purif;
    int npcol_purif;
    int npgrd_purif;
    int srow_purif;
    int scol_purif;
    int nrows_purif;
    int ncols_purif;
    int meshsize;
    int ldx;
    double *H_block;
    double *X_block;
    double *S_block;
    double *F_block;
    double *D_block;
    int len_diis;
    int bmax_id;
    double bmax;
    /* statistics (seconds) */
    double timedgemm;
    double timepdgemm;
    double timetr;
    double timepass;
    /* device state (gtfock_b200/csrc/cuda/purif.cu) */
    void *dev;
    int sx_uploaded;
    int last_iters;
    int host_pinned;   /* the five blocks are page-locked (copied by DMA) */
} purif_t;

#ifdef __cplusplus
extern "C" {
#endif

/* pscf/purif.h:78-79 */
purif_t *create_purif(BasisSet_t basis, int nprow_purif, int npcol_purif, int npgrd_purif);
/* pscf/purif.h:81 */
void destroy_purif(purif_t *purif);
/* pscf/purif.h:83 */
int compute_purification(purif_t *purif, double *F_block, double *D_block);
/* pscf/purif.h:85-86 */
void compute_diis(PFock_t pfock, purif_t *purif, double *D_block, double *F_block, int iter);

#ifdef __cplusplus
}
#endif

#endif /* __PURIF_H__ */
