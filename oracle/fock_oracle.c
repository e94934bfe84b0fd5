/*
 * fock_oracle.c -- CPU restatement of GTFock's hot path for one process.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle; never linked by the product).
 * Restates, for nprow = npcol = np2 = 1 and full nbf x nbf matrices:
 *   schwartz_screening   pfock/screening.c:15-180
 *   fock_task + update_F pfock/fock_task.c:29-219
 *   F/K symmetrisation   pfock/pfock.c:1719-1726, getMat F = J + K
 *                        pfock/pfock.c:1161-1185
 *   S, H, X              pfock/one_electron.c:28-119, pfock/pfock.c:1782-1867
 *   purification         pscf/purif.c:257-488
 *   DIIS                 pscf/purif.c:491-641
 *   SCF driver loop      pscf/scf.c:34-127, 329-459
 * Dense linear algebra goes to the OpenBLAS build that ships with scipy
 * (scipy_-prefixed symbols), standing in for MKL.
 */
#include <float.h>
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#include "gtf_basis.h"
#include "oracle.h"

/* ---- BLAS/LAPACK from the scipy OpenBLAS (LP64) ---- */
enum { RowMajor = 101, NoTrans = 111, Trans = 112 };
extern void scipy_cblas_dgemm(int order, int ta, int tb, int m, int n, int k,
                              double alpha, const double *a, int lda,
                              const double *b, int ldb, double beta,
                              double *c, int ldc);
extern void scipy_dsyevd_(const char *jobz, const char *uplo, const int *n, double *a,
                          const int *lda, double *w, double *work, const int *lwork,
                          int *iwork, const int *liwork, int *info, size_t, size_t);
extern void scipy_dgetrf_(const int *m, const int *n, double *a, const int *lda,
                          int *ipiv, int *info);
extern void scipy_dgetri_(const int *n, double *a, const int *lda, const int *ipiv,
                          double *work, const int *lwork, int *info);
extern void scipy_openblas_set_num_threads(int);

void or_set_blas_threads(int n) { scipy_openblas_set_num_threads(n); }
void or_free(void *p) { free(p); }

/* C = A * B^T for square n x n row-major matrices: the single-rank result of
 * pdgemm3D_2 (pscf/pdgemm.c:164-238, cblas NoTrans/Trans at :222). */
static void gemm_abt(int n, const double *A, const double *B, double *C)
{
    scipy_cblas_dgemm(RowMajor, NoTrans, Trans, n, n, n, 1.0, A, n, B, n, 0.0, C, n);
}

/* C = A * B (pscf/pdgemm.c:141) */
static void gemm_ab(int n, const double *A, const double *B, double *C)
{
    scipy_cblas_dgemm(RowMajor, NoTrans, NoTrans, n, n, n, 1.0, A, n, B, n, 0.0, C, n);
}

/* ------------------------------------------------------------------------ */
/* screening                                                                 */
/* ------------------------------------------------------------------------ */

int or_screening(BasisSet_t basis, double tolscr, int nthreads,
                 int **shellptr_o, int **shellid_o, int **shellrid_o,
                 double **shellvalue_o, int *nnz_o, double *maxvalue_o)
{
    const int nshells = basis->nshells;
    ERD_t erd;
    if (CInt_createERD(basis, &erd, nthreads) != CINT_STATUS_SUCCESS) return -1;
    double *sq = (double *)malloc(sizeof(double) * nshells * nshells);
    if (!sq) return -1;
    double maxtmp = 0.0;
    /* pfock/screening.c:59-90: max |(mn|mn)| over the diagonal of (MN|MN) */
    #pragma omp parallel num_threads(nthreads) reduction(max:maxtmp)
    {
        int tid = omp_get_thread_num();
        #pragma omp for schedule(dynamic)
        for (int M = 0; M < nshells; M++) {
            int dimM = CInt_getShellDim(basis, M);
            for (int N = 0; N < nshells; N++) {
                int dimN = CInt_getShellDim(basis, N);
                int nints;
                double *ints;
                CInt_computeShellQuartet(basis, erd, tid, M, N, M, N, &ints, &nints);
                double mv = 0.0;
                if (nints != 0) {
                    for (int iM = 0; iM < dimM; iM++) {
                        for (int iN = 0; iN < dimN; iN++) {
                            int index = iM * (dimN * dimM * dimN + dimN) + iN * (dimM * dimN + 1);
                            if (mv < fabs(ints[index])) mv = fabs(ints[index]);
                        }
                    }
                }
                sq[M * nshells + N] = mv;
                if (mv > maxtmp) maxtmp = mv;
            }
        }
    }
    CInt_destroyERD(erd);
    /* pfock/screening.c:110-175: CSR list, parity rule, signed values */
    const double eta = tolscr * tolscr / maxtmp;
    int *shellptr = (int *)calloc(nshells + 1, sizeof(int));
    int nnz = 0;
    for (int M = 0; M < nshells; M++) {
        shellptr[M] = nnz;
        for (int N = 0; N < nshells; N++) {
            if (sq[M * nshells + N] > eta) {
                if ((M > N && (M + N) % 2 == 1) || (M < N && (M + N) % 2 == 0)) continue;
                nnz++;
            }
        }
        shellptr[M + 1] = nnz;
    }
    double *shellvalue = (double *)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
    int *shellid = (int *)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
    int *shellrid = (int *)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
    nnz = 0;
    for (int A = 0; A < nshells; A++) {
        shellptr[A] = nnz;
        for (int B = 0; B < nshells; B++) {
            double mv = sq[A * nshells + B];
            if (mv > eta) {
                if ((A > B && (A + B) % 2 == 1) || (A < B && (A + B) % 2 == 0)) continue;
                shellvalue[nnz] = (A == B) ? mv : -mv;
                shellid[nnz] = B;
                shellrid[nnz] = A;
                nnz++;
            }
        }
    }
    free(sq);
    *shellptr_o = shellptr;
    *shellid_o = shellid;
    *shellrid_o = shellrid;
    *shellvalue_o = shellvalue;
    *nnz_o = nnz;
    *maxvalue_o = maxtmp;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Fock build                                                                */
/* ------------------------------------------------------------------------ */

/* update_F (pfock/fock_task.c:29-117) on full row-major matrices (ld = nbf):
 * J receives the Coulomb-like terms, K the (negative) exchange terms. */
static void update_F_full(int nbf, const double *I, int dimM, int dimN, int dimP, int dimQ,
                          int fM, int fN, int fP, int fQ,
                          int flag1, int flag2, int flag3,
                          const double *D, double *J, double *K)
{
    const int flag4 = (flag1 == 1 && flag2 == 1) ? 1 : 0;
    const int flag5 = (flag1 == 1 && flag3 == 1) ? 1 : 0;
    const int flag6 = (flag2 == 1 && flag3 == 1) ? 1 : 0;
    const int flag7 = (flag4 == 1 && flag3 == 1) ? 1 : 0;
    for (int iN = 0; iN < dimN; iN++) {
        for (int iQ = 0; iQ < dimQ; iQ++) {
            double k_NQ = 0.0;
            for (int iM = 0; iM < dimM; iM++) {
                double j_MN = 0.0;
                double k_MQ = 0.0;
                for (int iP = 0; iP < dimP; iP++) {
                    const int m = fM + iM, n = fN + iN, p = fP + iP, q = fQ + iQ;
                    const double Iv = I[iM + dimM * (iN + dimN * (iP + dimP * iQ))];
                    j_MN += 2.0 * (1 + flag1 + flag2 + flag4) * D[p * nbf + q] * Iv;
                    J[p * nbf + q] += 2.0 * (flag3 + flag5 + flag6 + flag7) * D[m * nbf + n] * Iv;
                    K[m * nbf + p] -= (1 + flag3) * 1.0 * D[n * nbf + q] * Iv;
                    K[n * nbf + p] -= (flag1 + flag5) * 1.0 * D[m * nbf + q] * Iv;
                    k_MQ -= (flag2 + flag6) * 1.0 * D[n * nbf + p] * Iv;
                    k_NQ -= (flag4 + flag7) * 1.0 * D[m * nbf + p] * Iv;
                }
                J[(fM + iM) * nbf + fN + iN] += j_MN;
                K[(fM + iM) * nbf + fQ + iQ] += k_MQ;
            }
            K[(fN + iN) * nbf + fQ + iQ] += k_NQ;
        }
    }
}

/* One Fock build restricted to every `stride`-th MN pair of the task loop
 * (stride 1 = the whole build); count_only skips the integrals and the
 * digestion and only counts quartets.  Used for the timed CPU baseline on a
 * bounded sample of a large build. */
int or_fock_build_sample(BasisSet_t basis, double tolscr, int nthreads,
                         const int *shellptr, const int *shellid, const int *shellrid,
                         const double *shellvalue, const double *D, double *F,
                         int stride, int count_only, double *usq_o, double *uitl_o);

int or_fock_build(BasisSet_t basis, double tolscr, int nthreads,
                  const int *shellptr, const int *shellid, const int *shellrid,
                  const double *shellvalue,
                  const double *D, double *F, double *usq_o, double *uitl_o)
{
    return or_fock_build_sample(basis, tolscr, nthreads, shellptr, shellid, shellrid, shellvalue,
                                D, F, 1, 0, usq_o, uitl_o);
}

int or_fock_build_shard(BasisSet_t basis, double tolscr, int nthreads,
                        const int *shellptr, const int *shellid, const int *shellrid,
                        const double *shellvalue, const double *D, double *F,
                        int stride, int offset, int count_only, double *usq_o, double *uitl_o);

int or_fock_build_sample(BasisSet_t basis, double tolscr, int nthreads,
                         const int *shellptr, const int *shellid, const int *shellrid,
                         const double *shellvalue, const double *D, double *F,
                         int stride, int count_only, double *usq_o, double *uitl_o)
{
    return or_fock_build_shard(basis, tolscr, nthreads, shellptr, shellid, shellrid, shellvalue, D, F,
                               stride, 0, count_only, usq_o, uitl_o);
}

static int fock_build_sel(BasisSet_t basis, double tolscr, int nthreads, const int *shellptr,
                          const int *shellid, const int *shellrid, const double *shellvalue,
                          const double *D, double *F, int stride, int offset, int lo, int hi,
                          int count_only, double *usq_o, double *uitl_o, double *pair_cost);

/* The MN pairs i with (i - first) % stride == offset: with stride = n and
 * offset = r, shard r of an n-way split of the build (the shards' F sum to
 * the whole F, since the symmetrisation at the end is linear). */
int or_fock_build_shard(BasisSet_t basis, double tolscr, int nthreads,
                        const int *shellptr, const int *shellid, const int *shellrid,
                        const double *shellvalue, const double *D, double *F,
                        int stride, int offset, int count_only, double *usq_o, double *uitl_o)
{
    return fock_build_sel(basis, tolscr, nthreads, shellptr, shellid, shellrid, shellvalue, D, F, stride,
                          offset, 0, 1 << 30, count_only, usq_o, uitl_o, NULL);
}

/* The MN pairs lo <= i - first < hi: a contiguous shard of the build, as a
 * partition of the MN-pair range into ranks' slices produces. */
int or_fock_build_range(BasisSet_t basis, double tolscr, int nthreads,
                        const int *shellptr, const int *shellid, const int *shellrid,
                        const double *shellvalue, const double *D, double *F, int lo, int hi,
                        double *usq_o, double *uitl_o)
{
    return fock_build_sel(basis, tolscr, nthreads, shellptr, shellid, shellrid, shellvalue, D, F, 1, 0, lo,
                          hi, 0, usq_o, uitl_o, NULL);
}

/* Work of every MN pair of the build: the integrals of its screened quartets
 * (sum of dM dN dP dQ, the uitl counter of pfock/fock_task.c:195-196 per
 * pair), into cost[nnz]; no integrals are evaluated. */
int or_fock_pair_cost(BasisSet_t basis, double tolscr, int nthreads,
                      const int *shellptr, const int *shellid, const int *shellrid,
                      const double *shellvalue, double *cost)
{
    return fock_build_sel(basis, tolscr, nthreads, shellptr, shellid, shellrid, shellvalue, NULL, NULL, 1,
                          0, 0, 1 << 30, 1, NULL, NULL, cost);
}

static int fock_build_sel(BasisSet_t basis, double tolscr, int nthreads, const int *shellptr,
                          const int *shellid, const int *shellrid, const double *shellvalue,
                          const double *D, double *F, int stride, int offset, int lo, int hi,
                          int count_only, double *usq_o, double *uitl_o, double *pair_cost)
{
    if (stride < 1) stride = 1;
    if (offset < 0 || offset >= stride) return -1;
    if (!count_only && (!D || !F)) return -1;
    const int nbf = basis->nbf;
    const int nshells = basis->nshells;
    const double tolscr2 = tolscr * tolscr;
    const int *f_startind = basis->f_start;
    const size_t nn = (size_t)nbf * nbf;
    double *Jt = (double *)calloc(nn * nthreads, sizeof(double));
    double *Kt = (double *)calloc(nn * nthreads, sizeof(double));
    if (!Jt || !Kt) { free(Jt); free(Kt); return -1; }
    ERD_t erd;
    if (CInt_createERD(basis, &erd, nthreads) != CINT_STATUS_SUCCESS) { free(Jt); free(Kt); return -1; }
    const int startMN = shellptr[0], endMN = shellptr[nshells];
    double usq = 0.0, uitl = 0.0;
    /* pfock/fock_task.c:141-218 with the whole shell range as one task */
    #pragma omp parallel num_threads(nthreads) reduction(+:usq, uitl)
    {
        const int nt = omp_get_thread_num();
        double *J = Jt + nn * nt;
        double *K = Kt + nn * nt;
        #pragma omp for schedule(dynamic)
        for (int i = startMN; i < endMN; i++) {
            if ((i - startMN) % stride != offset) continue;
            if (i - startMN < lo || i - startMN >= hi) continue;
            double cost_i = 0.0;
            const int M = shellrid[i];
            const int N = shellid[i];
            const double value1 = shellvalue[i];
            const int dimM = f_startind[M + 1] - f_startind[M];
            const int dimN = f_startind[N + 1] - f_startind[N];
            const int flag1 = (value1 < 0.0) ? 1 : 0;
            for (int j = startMN; j < endMN; j++) {
                const int P = shellrid[j];
                const int Q = shellid[j];
                if ((M > P && (M + P) % 2 == 1) || (M < P && (M + P) % 2 == 0)) continue;
                if ((M == P) && ((N > Q && (N + Q) % 2 == 1) || (N < Q && (N + Q) % 2 == 0)))
                    continue;
                const double value2 = shellvalue[j];
                const int dimP = f_startind[P + 1] - f_startind[P];
                const int dimQ = f_startind[Q + 1] - f_startind[Q];
                const int flag3 = (M == P && Q == N) ? 0 : 1;
                const int flag2 = (value2 < 0.0) ? 1 : 0;
                if (fabs(value1 * value2) >= tolscr2) {
                    int nints;
                    double *ints;
                    usq += 1.0;
                    uitl += dimM * dimN * dimP * dimQ;
                    cost_i += dimM * dimN * dimP * dimQ;
                    if (count_only) continue;
                    CInt_computeShellQuartet(basis, erd, nt, M, N, P, Q, &ints, &nints);
                    if (nints != 0) {
                        update_F_full(nbf, ints, dimM, dimN, dimP, dimQ,
                                      f_startind[M], f_startind[N], f_startind[P], f_startind[Q],
                                      flag1, flag2, flag3, D, J, K);
                    }
                }
            }
            if (pair_cost) pair_cost[i - startMN] = cost_i;
        }
    }
    CInt_destroyERD(erd);
    if (count_only && !F) {
        free(Jt);
        free(Kt);
        if (usq_o) *usq_o = usq;
        if (uitl_o) *uitl_o = uitl;
        return 0;
    }
    /* reduce the per-thread copies (reduce_F, pfock/fock_task.c:257-324) */
    for (int t = 1; t < nthreads; t++) {
        for (size_t k = 0; k < nn; k++) {
            Jt[k] += Jt[nn * t + k];
            Kt[k] += Kt[nn * t + k];
        }
    }
    /* GA_Symmetrize of ga_F and ga_K, then getMat(F) = F + K */
    for (int r = 0; r < nbf; r++) {
        for (int c = 0; c < nbf; c++) {
            double js = 0.5 * (Jt[r * nbf + c] + Jt[c * nbf + r]);
            double ks = 0.5 * (Kt[r * nbf + c] + Kt[c * nbf + r]);
            F[r * nbf + c] = js + ks;
        }
    }
    free(Jt);
    free(Kt);
    if (usq_o) *usq_o = usq;
    if (uitl_o) *uitl_o = uitl;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* one-electron matrices                                                     */
/* ------------------------------------------------------------------------ */

int or_one_electron(BasisSet_t basis, double *S, double *H, double *X)
{
    const int nbf = basis->nbf, nsh = basis->nshells;
    OED_t oed;
    CInt_createOED(basis, &oed);
    /* matrix_block_write, pfock/one_electron.c:14-25: block[k + nrows*l] */
    for (int A = 0; A < nsh; A++) {
        for (int B = 0; B < nsh; B++) {
            int r0 = basis->f_start[A], c0 = basis->f_start[B];
            int nr = basis->f_start[A + 1] - r0, nc = basis->f_start[B + 1] - c0;
            double *ints;
            int n;
            if (S) {
                CInt_computePairOvl(basis, oed, A, B, &ints, &n);
                for (int k = 0; k < nr; k++)
                    for (int l = 0; l < nc; l++) S[(r0 + k) * nbf + c0 + l] = ints[k + nr * l];
            }
            if (H) {
                CInt_computePairCoreH(basis, oed, A, B, &ints, &n);
                for (int k = 0; k < nr; k++)
                    for (int l = 0; l < nc; l++) H[(r0 + k) * nbf + c0 + l] = ints[k + nr * l];
            }
        }
    }
    CInt_destroyOED(oed);
    if (X && S) {
        /* my_peig (pdsyevd) then X = (U diag(1/sqrt(lambda))) U^T */
        double *U = (double *)malloc(sizeof(double) * nbf * nbf);
        double *w = (double *)malloc(sizeof(double) * nbf);
        double *US = (double *)malloc(sizeof(double) * nbf * nbf);
        memcpy(U, S, sizeof(double) * nbf * nbf); /* symmetric: row/col major alike */
        int n = nbf, lwork = -1, liwork = -1, info = 0, iw;
        double wq;
        scipy_dsyevd_("V", "U", &n, U, &n, w, &wq, &lwork, &iw, &liwork, &info, 1, 1);
        lwork = (int)wq + 1;
        liwork = iw;
        double *work = (double *)malloc(sizeof(double) * lwork);
        int *iwork = (int *)malloc(sizeof(int) * liwork);
        scipy_dsyevd_("V", "U", &n, U, &n, w, work, &lwork, iwork, &liwork, &info, 1, 1);
        free(work);
        free(iwork);
        if (info != 0) { free(U); free(w); free(US); return -1; }
        /* column-major U: eigenvector k is U[k*nbf + i]; row-major Ut = U^T */
        for (int i = 0; i < nbf; i++)
            for (int k = 0; k < nbf; k++) US[i * nbf + k] = U[k * nbf + i] / sqrt(w[k]);
        /* X = US * U_rowmajor^T where U_rowmajor[i][k] = U[k*nbf+i] */
        double *Ur = (double *)malloc(sizeof(double) * nbf * nbf);
        for (int i = 0; i < nbf; i++)
            for (int k = 0; k < nbf; k++) Ur[i * nbf + k] = U[k * nbf + i];
        gemm_abt(nbf, US, Ur, X);
        free(Ur);
        free(U);
        free(w);
        free(US);
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* purification                                                              */
/* ------------------------------------------------------------------------ */

#define OR_MAX_PURF_ITERS 200

int or_purification(int nbf, int nobtls, const double *X, const double *F, double *D)
{
    const int n = nbf;
    const size_t nn = (size_t)n * n;
    double *D2 = (double *)malloc(sizeof(double) * nn);
    double *D3 = (double *)malloc(sizeof(double) * nn);
    /* Gershgorin bounds, pscf/purif.c:302-340 */
    double hmin = DBL_MAX, hmax = -DBL_MAX;
    for (int i = 0; i < n; i++) {
        double off = 0.0, dg = 0.0;
        for (int j = 0; j < n; j++) {
            off += fabs(F[i + j * n]);
            if (j == i) dg = F[i + j * n];
        }
        off = off - fabs(dg);
        double lo = dg - off, hi = dg + off;
        hmin = lo > hmin ? hmin : lo;
        hmax = hi < hmax ? hmax : hi;
    }
    double trF = 0.0;
    for (int i = 0; i < n; i++) trF += F[i * n + i];
    const double mu_bar = trF / (double)n;
    const double lambda = fmin((double)nobtls / (hmax - mu_bar),
                               (double)(n - nobtls) / (mu_bar - hmin));
    for (size_t i = 0; i < nn; i++) D[i] = F[i] * (-lambda / n);
    for (int i = 0; i < n; i++) D[i * n + i] += lambda * mu_bar / (double)n + (double)nobtls / n;
    int it;
    for (it = 0; it < OR_MAX_PURF_ITERS; it++) {
        gemm_abt(n, D, D, D2);    /* D2 = D D^T   (pscf/pdgemm.c:102) */
        gemm_ab(n, D, D2, D3);    /* D3 = D D2    (pscf/pdgemm.c:141) */
        double err = 0.0;
        for (size_t i = 0; i < nn; i++) err += (D[i] - D2[i]) * (D[i] - D2[i]);
        err = sqrt(err);
        double tr = 0.0, tr2 = 0.0;
        for (int i = 0; i < n; i++) {
            tr += D2[i * n + i] - D3[i * n + i];
            tr2 += D[i * n + i] - D2[i * n + i];
        }
        const double c = tr / tr2;
        if (c < 0.5) {
            for (size_t i = 0; i < nn; i++)
                D[i] = ((1.0 - 2.0 * c) * D[i] + (1.0 + c) * D2[i] - D3[i]) / (1.0 - c);
        } else {
            for (size_t i = 0; i < nn; i++) D[i] = ((1.0 + c) * D2[i] - D3[i]) / c;
        }
        if (err < 1e-11) break;
    }
    /* D_AO = X D X, pscf/purif.c:469-476 */
    gemm_abt(n, X, D, D2);
    gemm_abt(n, D2, X, D);
    free(D2);
    free(D3);
    return it;
}

/* ------------------------------------------------------------------------ */
/* DIIS                                                                      */
/* ------------------------------------------------------------------------ */

#define OR_MAX_DIIS 10
#define OR_LDBMAT 128

struct or_diis_s {
    int n;
    int len;
    int bmax_id;
    double bmax;
    double *vecs;   /* [MAX_DIIS][n*n] error vectors */
    double *Fvecs;  /* [MAX_DIIS][n*n] orthogonal-basis F */
    double *work;
    double b[OR_LDBMAT * OR_LDBMAT];
};

or_diis_t *or_diis_create(int n)
{
    or_diis_t *d = (or_diis_t *)calloc(1, sizeof(or_diis_t));
    d->n = n;
    d->vecs = (double *)calloc((size_t)OR_MAX_DIIS * n * n, sizeof(double));
    d->Fvecs = (double *)calloc((size_t)OR_MAX_DIIS * n * n, sizeof(double));
    d->work = (double *)calloc((size_t)n * n, sizeof(double));
    d->bmax = DBL_MIN;
    d->bmax_id = -1;
    for (int i = 0; i < OR_LDBMAT; i++)
        for (int j = 0; j < OR_LDBMAT; j++) d->b[i * OR_LDBMAT + j] = (i != j) ? -1.0 : 0.0;
    return d;
}

void or_diis_destroy(or_diis_t *d)
{
    if (!d) return;
    free(d->vecs);
    free(d->Fvecs);
    free(d->work);
    free(d);
}

void or_diis_step(or_diis_t *d, const double *X, const double *S,
                  const double *D, double *F, int iter)
{
    const int n = d->n;
    const size_t nn = (size_t)n * n;
    double *workm = d->work;
    double *cur_F = F;
    int cur_idx = 0;
    if (iter > 1) {
        if (d->len < OR_MAX_DIIS) {
            cur_idx = d->len;
            d->len++;
        } else {
            cur_idx = d->bmax_id;
        }
        double *cur = d->vecs + nn * cur_idx;
        cur_F = d->Fvecs + nn * cur_idx;
        gemm_abt(n, F, D, workm);      /* F D */
        gemm_abt(n, workm, S, cur);    /* F D S */
        memcpy(workm, cur, sizeof(double) * nn);  /* MPI_Sendrecv to itself */
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) cur[i * n + j] -= workm[j * n + i];
        gemm_abt(n, X, cur, workm);
        gemm_abt(n, workm, X, cur);
        for (int i = 0; i < d->len; i++) {
            const double *v2 = d->vecs + nn * i;
            double dot = 0.0;
            for (int j = 0; j < n; j++)
                for (int k = 0; k < n; k++) dot += cur[j * n + k] * v2[j * n + k];
            d->b[cur_idx * OR_LDBMAT + i] = dot;
        }
        d->bmax = -DBL_MAX;
        for (int i = 0; i < d->len; i++) {
            d->b[i * OR_LDBMAT + cur_idx] = d->b[cur_idx * OR_LDBMAT + i];
            if (d->bmax < d->b[i * OR_LDBMAT + i]) {
                d->bmax = d->b[i * OR_LDBMAT + i];
                d->bmax_id = i;
            }
        }
    }
    /* F = X F X */
    gemm_abt(n, X, F, workm);
    gemm_abt(n, workm, X, cur_F);
    if (iter > 1) {
        int sizeb = d->len + 1;
        double binv[OR_LDBMAT * OR_LDBMAT];
        int ipiv[OR_LDBMAT];
        memcpy(binv, d->b, sizeof(binv));
        /* The bordered DIIS matrix is symmetric, so the column-major LAPACK
         * inverse equals the row-major one of LAPACKE_dgetrf/dgetri. */
        int ld = OR_LDBMAT, info = 0, lwork = OR_LDBMAT * 4;
        double wk[OR_LDBMAT * 4];
        scipy_dgetrf_(&sizeb, &sizeb, binv, &ld, ipiv, &info);
        scipy_dgetri_(&sizeb, binv, &ld, ipiv, wk, &lwork, &info);
        double coeffs[OR_LDBMAT];
        for (int i = 0; i < sizeb; i++) coeffs[i] = -binv[i * OR_LDBMAT + sizeb - 1];
        memset(F, 0, sizeof(double) * nn);
        for (int i = 0; i < d->len; i++) {
            const double *Fv = d->Fvecs + nn * i;
            for (size_t j = 0; j < nn; j++) F[j] += coeffs[i] * Fv[j];
        }
    }
}

/* ------------------------------------------------------------------------ */
/* SCF driver                                                                */
/* ------------------------------------------------------------------------ */

int or_scf(BasisSet_t basis, double tolscr, int niters, int nthreads,
           double *energies, double *F_last, double *D_last)
{
    const int n = basis->nbf;
    const size_t nn = (size_t)n * n;
    int *shellptr, *shellid, *shellrid, nnz;
    double *shellvalue, maxv;
    if (or_screening(basis, tolscr, nthreads, &shellptr, &shellid, &shellrid,
                     &shellvalue, &nnz, &maxv) != 0) return -1;
    double *S = (double *)calloc(nn, sizeof(double));
    double *H = (double *)calloc(nn, sizeof(double));
    double *X = (double *)calloc(nn, sizeof(double));
    double *D = (double *)calloc(nn, sizeof(double));
    double *F = (double *)calloc(nn, sizeof(double));
    or_one_electron(basis, S, H, X);
    /* initial_guess, pscf/scf.c:34-76 */
    double R = 1.0;
    int Nn = CInt_getNneutral(basis), Q = CInt_getTotalCharge(basis);
    if (Q != 0 && Nn != 0) R = (Nn - Q) / (double)Nn;
    for (int a = 0; a < basis->natoms; a++) {
        double *g;
        int sp, ep;
        CInt_getInitialGuess(basis, a, &g, &sp, &ep);
        int ld = ep - sp + 1;
        for (int r = sp; r <= ep; r++)
            for (int c = sp; c <= ep; c++) D[r * n + c] = g[(r - sp) * ld + (c - sp)];
    }
    for (size_t k = 0; k < nn; k++) D[k] *= R / 2.0;
    const double enuc = CInt_getNucEnergy(basis);
    const int nocc = CInt_getNumOccOrb(basis);
    or_diis_t *diis = or_diis_create(n);
    double e0 = -1.0;
    int iter;
    for (iter = 0; iter < niters; iter++) {
        or_fock_build(basis, tolscr, nthreads, shellptr, shellid, shellrid, shellvalue,
                      D, F, NULL, NULL);
        /* compute_energy, pscf/scf.c:80-102 */
        double e = 0.0;
        for (size_t k = 0; k < nn; k++) {
            F[k] += H[k];
            e += D[k] * (H[k] + F[k]);
        }
        if (energies) energies[iter] = e + enuc;
        if (F_last) memcpy(F_last, F, sizeof(double) * nn);
        if (iter > 0 && fabs(e - e0) < 1e-11) {
            iter++;
            break;
        }
        e0 = e;
        or_diis_step(diis, X, S, D, F, iter);
        or_purification(n, nocc, X, F, D);
        if (D_last) memcpy(D_last, D, sizeof(double) * nn);
    }
    or_diis_destroy(diis);
    free(S); free(H); free(X); free(D); free(F);
    free(shellptr); free(shellid); free(shellrid); free(shellvalue);
    return iter;
}
