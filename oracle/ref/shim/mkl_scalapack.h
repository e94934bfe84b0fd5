/* mkl_scalapack.h -- the ScaLAPACK/BLACS calls of pfock/one_electron.c:122-266
 * on a 1 x 1 process grid (pdsyevd becomes LAPACK dsyevd). */
#ifndef GTF_REF_MKL_SCALAPACK_H
#define GTF_REF_MKL_SCALAPACK_H
void Cblacs_pinfo(int *mypnum, int *nprocs);
void Cblacs_get(int ictxt, int what, int *val);
int Cblacs_gridinit(int *ictxt, char *order, int nprow, int npcol);
void Cblacs_gridinfo(int ictxt, int *nprow, int *npcol, int *myrow, int *mycol);
void Cblacs_gridexit(int ictxt);
int numroc_(int *n, int *nb, int *iproc, int *isrcproc, int *nprocs);
int indxl2g_(int *indxloc, int *nb, int *iproc, int *isrcproc, int *nprocs);
void descinit_(int *desc, int *m, int *n, int *mb, int *nb, int *irsrc, int *icsrc,
               int *ictxt, int *lld, int *info);
void pdsyevd(char *jobz, char *uplo, int *n, double *a, int *ia, int *ja, int *desca,
             double *w, double *z, int *iz, int *jz, int *descz, double *work,
             int *lwork, int *iwork, int *liwork, int *info);
#endif
