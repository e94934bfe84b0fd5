/*
 * CInt.h -- basis-set and integral interface of gtfock-b200.
 *
 * Same declarations as GTFock's integral layer (libcint/include/CInt.h:45-181),
 * so pscf/scf.c and pfock callers compile against it unchanged.  The basis-set
 * functions (load, pack/unpack, counts, start indices, initial guess, nuclear
 * energy) are implemented in C in gtfock_b200/csrc/basis.c.  The integral
 * functions (ERD/OED) are served on the GPU inside the PFock engine; the
 * per-quartet CInt_computeShellQuartet entry point exists only in the CPU
 * checker library under oracle/.
 *
 * Conventions (fixed here, because the reference's integral engine ships only
 * as a binary):
 *   - coordinates in .xyz files are Angstrom, converted with
 *     1 bohr = 0.529177210903 Angstrom (CODATA 2018);
 *   - each contracted shell is normalised so that its x^L Cartesian component
 *     has unit norm; the other Cartesian components share that factor;
 *   - Cartesian order within a shell is lexicographic (xx, xy, xz, yy, yz, zz);
 *   - spherical d functions are ordered m = -2..2:
 *       xy*sqrt3, yz*sqrt3, zz-(xx+yy)/2, xz*sqrt3, (xx-yy)*sqrt3/2;
 *   - integral blocks are returned with the first shell index fastest
 *     (I[iA + dA*(iB + dB*(iC + dC*iD))]), as pfock/fock_task.c:73-74 reads them.
 */
#ifndef __CINT_H__
#define __CINT_H__

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <unistd.h>

struct ERD;
struct OED;
struct BasisSet;

typedef struct OED *OED_t;
typedef struct ERD *ERD_t;
typedef struct BasisSet *BasisSet_t;

typedef enum
{
    CINT_STATUS_SUCCESS = 0,
    CINT_STATUS_NOT_INITIALIZED = 1,
    CINT_STATUS_ALLOC_FAILED = 2,
    CINT_STATUS_INVALID_VALUE = 3,
    CINT_STATUS_EXECUTION_FAILED = 4,
    CINT_STATUS_INTERNAL_ERROR = 5,
    CINT_STATUS_FILEIO_FAILED = 6,
    CINT_STATUS_OFFLOAD_ERROR = 7
} CIntStatus_t;

#ifdef __cplusplus
extern "C" {
#endif

/* ---- basis set (libcint/include/CInt.h:45-86,123-145) ---- */
CIntStatus_t CInt_createBasisSet(BasisSet_t *basis);
CIntStatus_t CInt_destroyBasisSet(BasisSet_t basis);
CIntStatus_t CInt_unpackBasisSet(BasisSet_t basis, void *buf);
CIntStatus_t CInt_importBasisSet(BasisSet_t basis,
                                 int natoms, int *Zs,
                                 double *X, double *Y, double *Z,
                                 int nprims, int nshells, int pure,
                                 int *shells_p_atom,
                                 int *prims_p_shell,
                                 int *L, double *cc, double *alpha);
CIntStatus_t CInt_loadBasisSet(BasisSet_t basis, char *bsfile, char *xyzfile);
CIntStatus_t CInt_packBasisSet(BasisSet_t basis, void **buf, int *bufsize);
int CInt_getNumShells(BasisSet_t basis);
int CInt_getNumFuncs(BasisSet_t basis);
int CInt_getNumAtoms(BasisSet_t basis);
int CInt_getMaxShellDim(BasisSet_t basis);
int CInt_getNumOccOrb(BasisSet_t basis);
int CInt_getFuncEndInd(BasisSet_t basis, int shellid);
int CInt_getAtomStartInd(BasisSet_t basis, int atomid);
void CInt_getShellxyz(BasisSet_t basis, int shellid,
                      double *x, double *y, double *z);
int CInt_getShellDim(BasisSet_t basis, int shellid);
int CInt_getFuncStartInd(BasisSet_t basis, int shellid);
void CInt_getInitialGuess(BasisSet_t basis, int atomid,
                          double **guess, int *spos, int *epos);
int CInt_getTotalCharge(BasisSet_t basis);
int CInt_getNneutral(BasisSet_t basis);
double CInt_getNucEnergy(BasisSet_t basis);

/* ---- one-electron integrals (libcint/include/CInt.h:90-121) ---- */
CIntStatus_t CInt_createOED(BasisSet_t basis, OED_t *oed);
CIntStatus_t CInt_destroyOED(OED_t oed);
CIntStatus_t CInt_computePairKin(BasisSet_t basis, OED_t oed, int A, int B,
                                 double **integrals, int *nints);
CIntStatus_t CInt_computePairOvl(BasisSet_t basis, OED_t oed, int A, int B,
                                 double **integrals, int *nints);
CIntStatus_t CInt_computePairPot(BasisSet_t basis, OED_t oed, int A, int B,
                                 double **integrals, int *nints);
CIntStatus_t CInt_computePairCoreH(BasisSet_t basis, OED_t oed, int A, int B,
                                   double **integrals, int *nints);

/* ---- two-electron integrals (libcint/include/CInt.h:152-181) ---- */
CIntStatus_t CInt_createERD(BasisSet_t basis, ERD_t *erd, int nthreads);
CIntStatus_t CInt_destroyERD(ERD_t erd);
CIntStatus_t CInt_computeShellQuartet(BasisSet_t basis, ERD_t erd, int tid,
                                      int A, int B, int C, int D,
                                      double **integrals, int *nints);
CIntStatus_t CInt_computeShellQuartets(BasisSet_t basis, ERD_t erd,
                                       uint32_t threadId,
                                       uint32_t shellIndixA,
                                       const uint32_t *shellIndicesB,
                                       uint32_t shellIndixC,
                                       const uint32_t *shellIndicesD,
                                       uint32_t shellIndicesCount,
                                       double **integrals,
                                       int *integralsCount);
void CInt_getMaxMemory(ERD_t erd, double *memsize);

#ifdef __cplusplus
}
#endif

#define CINT_ASSERT(condition) if (!(condition)) { \
    dprintf(2, "ASSERTION FAILED: %s in %s:%d\n", #condition, __FILE__, __LINE__); \
    fsync(2); \
    abort(); \
}

#endif /* __CINT_H__ */
