/*
 * oracle.h -- CPU restatement of GTFock's Fock-build and purification path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the oracle: tests/, the
 * __graft_entry__ smoke check and bench.py's CPU-baseline leg call it; the
 * product library (gtfock_b200/) never links, loads or calls it.
 *
 * Every function restates one reference function for a single process
 * (nprow = npcol = 1, full nbf x nbf matrices) and cites it.  Integrals come
 * from cint_oracle.c (FP64, Obara-Saika/Head-Gordon-Pople).
 */
#ifndef GTF_ORACLE_H
#define GTF_ORACLE_H

#include "CInt.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Schwarz screening, pfock/screening.c:15-180.  Arrays are malloc'ed and
 * owned by the caller (free with or_free).  Returns 0 on success. */
int or_screening(BasisSet_t basis, double tolscr, int nthreads,
                 int **shellptr, int **shellid, int **shellrid,
                 double **shellvalue, int *nnz, double *maxvalue);

/* Fock build, pfock/pfock.c:1274-1729 with pfock/fock_task.c:121-219 and
 * update_F (pfock/fock_task.c:29-117).  D is the full nbf x nbf row-major
 * (half) density; F receives 2J - K after symmetrisation, i.e. what
 * PFock_getMat(PFOCK_MAT_TYPE_F) returns (pfock/pfock.c:1134-1188).
 * usq/uitl are the reference's counters (pfock/fock_task.c:195-196). */
int or_fock_build(BasisSet_t basis, double tolscr, int nthreads,
                  const int *shellptr, const int *shellid, const int *shellrid,
                  const double *shellvalue,
                  const double *D, double *F, double *usq, double *uitl);

/* The same build restricted to every stride-th MN pair (count_only: count
 * quartets without computing them); the timed CPU baseline samples large
 * builds this way. */
int or_fock_build_sample(BasisSet_t basis, double tolscr, int nthreads,
                         const int *shellptr, const int *shellid, const int *shellrid,
                         const double *shellvalue, const double *D, double *F,
                         int stride, int count_only, double *usq, double *uitl);
int or_fock_build_shard(BasisSet_t basis, double tolscr, int nthreads,
                        const int *shellptr, const int *shellid, const int *shellrid,
                        const double *shellvalue, const double *D, double *F,
                        int stride, int offset, int count_only, double *usq_o, double *uitl_o);
int or_fock_build_range(BasisSet_t basis, double tolscr, int nthreads,
                        const int *shellptr, const int *shellid, const int *shellrid,
                        const double *shellvalue, const double *D, double *F, int lo, int hi,
                        double *usq_o, double *uitl_o);
int or_fock_pair_cost(BasisSet_t basis, double tolscr, int nthreads,
                      const int *shellptr, const int *shellid, const int *shellrid,
                      const double *shellvalue, double *cost);

/* S, H_core and X = U diag(1/sqrt(lambda)) U^T
 * (pfock/one_electron.c:28-119, pfock/pfock.c:1782-1867). */
int or_one_electron(BasisSet_t basis, double *S, double *H, double *X);

/* Canonical purification, pscf/purif.c:257-488; F_orth in, D_AO out.
 * Returns the iteration count. */
int or_purification(int nbf, int nobtls, const double *X,
                    const double *F_orth, double *D_out);

/* DIIS state and step, pscf/purif.c:491-641 (F_block updated in place to the
 * extrapolated orthogonal-basis F). */
typedef struct or_diis_s or_diis_t;
or_diis_t *or_diis_create(int nbf);
void or_diis_destroy(or_diis_t *d);
void or_diis_step(or_diis_t *d, const double *X, const double *S,
                  const double *D, double *F, int iter);

/* Whole SCF as pscf/scf.c:189-474 drives it (1 rank).  energies[niters]
 * receives the printed total energy (electronic + nuclear) per iteration;
 * returns the number of iterations run (early stop at |dE| < 1e-11). */
int or_scf(BasisSet_t basis, double tolscr, int niters, int nthreads,
           double *energies, double *F_last, double *D_last);

void or_free(void *p);
void or_set_blas_threads(int n);

#ifdef __cplusplus
}
#endif

#endif
