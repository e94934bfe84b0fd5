/*
 * pfock.h -- PFock engine API of gtfock-b200.
 *
 * Same functions, enums and argument meaning as GTFock's engine header
 * (pfock/pfock.h:188-565), so pscf/scf.c compiles against it unchanged.  The
 * engine is single-GPU: D and F live in device memory, the Fock build runs as
 * sm_100a kernels, and host buffers are copied at putDenMat / getMat.
 * PFock_t is opaque here (scf.c never dereferences it); the reference's GA
 * handles and MPI process grid have no meaning on one GPU, so PFock_create
 * accepts nprow = npcol = 1 only and the *GA functions report
 * PFOCK_STATUS_INVALID_VALUE.
 *
 * Environment overrides read by PFock_create:
 *   GTFOCK_TOLSCR   Schwarz threshold replacing the tolscr argument
 *                   (scf.c hard-codes 1e-11, pscf/scf.c:303)
 */
#ifndef __PFOCK_H__
#define __PFOCK_H__

#include "CInt.h"

struct PFock;
typedef struct PFock *PFock_t;

typedef enum
{
    PFOCK_STATUS_SUCCESS = 0,
    PFOCK_STATUS_INIT_FAILED = 1,
    PFOCK_STATUS_ALLOC_FAILED = 2,
    PFOCK_STATUS_INVALID_VALUE = 3,
    PFOCK_STATUS_EXECUTION_FAILED = 4,
    PFOCK_STATUS_INTERNAL_ERROR = 5
} PFockStatus_t;

typedef enum
{
    PFOCK_MAT_TYPE_D = 0,
    PFOCK_MAT_TYPE_F = 1,
    PFOCK_MAT_TYPE_J = 2,
    PFOCK_MAT_TYPE_K = 3
} PFockMatType_t;

#ifdef __cplusplus
extern "C" {
#endif

/* pfock/pfock.h:241-243 */
PFockStatus_t PFock_create(BasisSet_t basis, int nprow, int npcol, int ntasks,
                           double tolscr, int max_numdmat, int symm,
                           PFock_t *_pfock);
/* pfock/pfock.h:252 */
PFockStatus_t PFock_destroy(PFock_t pfock);
/* pfock/pfock.h:262 */
PFockStatus_t PFock_setNumDenMat(int numdmat, PFock_t pfock);
/* pfock/pfock.h:282-285 */
PFockStatus_t PFock_putDenMat(int rowstart, int rowend,
                              int colstart, int colend,
                              int stride, double *dmat,
                              int index, PFock_t pfock);
/* pfock/pfock.h:296 */
PFockStatus_t PFock_putDenMatGA(int ga, int index, PFock_t pfock);
/* pfock/pfock.h:307-308 */
PFockStatus_t PFock_fillDenMat(double value, int index, PFock_t pfock);
/* pfock/pfock.h:320 */
PFockStatus_t PFock_commitDenMats(PFock_t pfock);
/* pfock/pfock.h:329 */
PFockStatus_t PFock_sync(PFock_t pfock);
/* pfock/pfock.h:350-358 */
PFockStatus_t PFock_getMat(PFock_t pfock, PFockMatType_t type, int index,
                           int rowstart, int rowend, int colstart, int colend,
                           int stride, double *mat);
/* pfock/pfock.h:370-371 */
PFockStatus_t PFock_getMatGA(PFock_t pfock, PFockMatType_t type, int index, int ga);
/* pfock/pfock.h:386-390 */
PFockStatus_t PFock_getLocalMatInds(PFock_t pfock, int *rowstart, int *rowend,
                                    int *colstart, int *colend);
/* pfock/pfock.h:409-414 */
PFockStatus_t PFock_getLocalMatPtr(PFock_t pfock, PFockMatType_t type, int index,
                                   int *rowstart, int *rowend,
                                   int *colstart, int *colend,
                                   int *stride, double **mat);
/* pfock/pfock.h:426-428 */
PFockStatus_t PFock_getMatGAHandle(PFock_t pfock, PFockMatType_t type, int index, int *ga);
/* pfock/pfock.h:441-442 */
PFockStatus_t PFock_computeFock(BasisSet_t basis, PFock_t pfock);
/* pfock/pfock.h:455 */
PFockStatus_t PFock_createCoreHMat(PFock_t pfock, BasisSet_t basis);
/* pfock/pfock.h:466 */
PFockStatus_t PFock_destroyCoreHMat(PFock_t pfock);
/* pfock/pfock.h:483-485 */
PFockStatus_t PFock_getCoreHMat(PFock_t pfock, int rowstart, int rowend,
                                int colstart, int colend, int stride, double *mat);
/* pfock/pfock.h:497 */
PFockStatus_t PFock_createOvlMat(PFock_t pfock, BasisSet_t basis);
/* pfock/pfock.h:508 */
PFockStatus_t PFock_destroyOvlMat(PFock_t pfock);
/* pfock/pfock.h:525-527 */
PFockStatus_t PFock_getOvlMat(PFock_t pfock, int rowstart, int rowend,
                              int colstart, int colend, int stride, double *mat);
/* pfock/pfock.h:544-546 */
PFockStatus_t PFock_getOvlMat2(PFock_t pfock, int rowstart, int rowend,
                               int colstart, int colend, int stride, double *mat);
/* pfock/pfock.h:556 */
PFockStatus_t PFock_getMemorySize(PFock_t pfock, double *mem_cpu);
/* pfock/pfock.h:565 */
PFockStatus_t PFock_getStatistics(PFock_t pfock);

#ifdef __cplusplus
}
#endif

#endif /* __PFOCK_H__ */
