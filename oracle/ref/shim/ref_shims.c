/*
 * ref_shims.c -- single-process Global Arrays, MKL and ScaLAPACK stand-ins
 * for compiling the reference's own pfock/*.c and pscf/*.c with gcc
 * (oracle/ref/Makefile).  Test infrastructure only: nothing here is part of
 * the product library.
 *
 * Global arrays are local row-major 2-D arrays (the distribution of one
 * process owns everything); non-blocking operations complete immediately.
 * Dense linear algebra is the scipy OpenBLAS (scipy_-prefixed LP64 symbols).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ga.h"
#include "macdecls.h"
#include "mkl.h"
#include "mkl_scalapack.h"

void *gtf_ref_aligned_calloc(size_t size, size_t align)
{
    void *p = NULL;
    if (align < sizeof(void *)) align = sizeof(void *);
    if (posix_memalign(&p, align, size ? size : 1) != 0) return NULL;
    memset(p, 0, size);
    return p;
}

/* ---------------- Global Arrays ---------------- */

typedef struct {
    int used;
    int type;
    int dims[2];
    size_t esize;
    void *data;
} ga_t;

#define MAX_GA 4096
static ga_t g_ga[MAX_GA];

static ga_t *ga_get(int h)
{
    if (h <= 0 || h >= MAX_GA || !g_ga[h].used) {
        fprintf(stderr, "GA shim: invalid handle %d\n", h);
        abort();
    }
    return &g_ga[h];
}

void GA_Initialize(void) {}
void GA_Terminate(void) {}
int MA_init(int type, long stack, long heap) { (void)type; (void)stack; (void)heap; return 1; }
void GA_Sync(void) {}

static int ga_alloc(int type, int d0, int d1)
{
    for (int h = 1; h < MAX_GA; h++) {
        if (!g_ga[h].used) {
            ga_t *g = &g_ga[h];
            g->used = 1;
            g->type = type;
            g->dims[0] = d0;
            g->dims[1] = d1;
            g->esize = (type == C_INT) ? sizeof(int) : sizeof(double);
            g->data = calloc((size_t)d0 * d1, g->esize);
            if (g->data == NULL) { g->used = 0; return 0; }
            return h;
        }
    }
    return 0;
}

int NGA_Create_irreg(int type, int ndim, int dims[], char *name, int block[], int map[])
{
    (void)name; (void)block; (void)map;
    if (ndim == 1) return ga_alloc(type, 1, dims[0]);
    return ga_alloc(type, dims[0], dims[1]);
}

int GA_Duplicate(int g_a, char *name)
{
    (void)name;
    ga_t *a = ga_get(g_a);
    return ga_alloc(a->type, a->dims[0], a->dims[1]);
}

void GA_Destroy(int g_a)
{
    ga_t *a = ga_get(g_a);
    free(a->data);
    memset(a, 0, sizeof(*a));
}

void GA_Fill(int g_a, void *val)
{
    ga_t *a = ga_get(g_a);
    size_t n = (size_t)a->dims[0] * a->dims[1];
    if (a->type == C_INT) {
        int v = *(int *)val;
        for (size_t i = 0; i < n; i++) ((int *)a->data)[i] = v;
    } else {
        double v = *(double *)val;
        for (size_t i = 0; i < n; i++) ((double *)a->data)[i] = v;
    }
}

static void block_copy(ga_t *a, int lo[], int hi[], void *buf, int ld, int dir, double alpha)
{
    /* dir 0: buf -> ga (put), 1: ga -> buf (get), 2: ga += alpha*buf (acc) */
    const int ncol = a->dims[1];
    for (int r = lo[0]; r <= hi[0]; r++) {
        for (int c = lo[1]; c <= hi[1]; c++) {
            size_t gi = (size_t)r * ncol + c;
            size_t bi = (size_t)(r - lo[0]) * ld + (c - lo[1]);
            if (a->type == C_INT) {
                int *g = (int *)a->data, *b = (int *)buf;
                if (dir == 0) g[gi] = b[bi];
                else if (dir == 1) b[bi] = g[gi];
                else g[gi] += (int)(alpha * b[bi]);
            } else {
                double *g = (double *)a->data, *b = (double *)buf;
                if (dir == 0) g[gi] = b[bi];
                else if (dir == 1) b[bi] = g[gi];
                else g[gi] += alpha * b[bi];
            }
        }
    }
}

void NGA_Put(int g_a, int lo[], int hi[], void *buf, int ld[])
{
    block_copy(ga_get(g_a), lo, hi, buf, ld[0], 0, 0.0);
}

void NGA_Get(int g_a, int lo[], int hi[], void *buf, int ld[])
{
    block_copy(ga_get(g_a), lo, hi, buf, ld[0], 1, 0.0);
}

void NGA_Acc(int g_a, int lo[], int hi[], void *buf, int ld[], void *alpha)
{
    block_copy(ga_get(g_a), lo, hi, buf, ld[0], 2, *(double *)alpha);
}

void NGA_NbPut(int g_a, int lo[], int hi[], void *buf, int ld[], ga_nbhdl_t *h)
{
    NGA_Put(g_a, lo, hi, buf, ld);
    if (h) *h = 0;
}

void NGA_NbGet(int g_a, int lo[], int hi[], void *buf, int ld[], ga_nbhdl_t *h)
{
    NGA_Get(g_a, lo, hi, buf, ld);
    if (h) *h = 0;
}

void NGA_NbAcc(int g_a, int lo[], int hi[], void *buf, int ld[], void *alpha, ga_nbhdl_t *h)
{
    NGA_Acc(g_a, lo, hi, buf, ld, alpha);
    if (h) *h = 0;
}

int NGA_NbWait(ga_nbhdl_t *h) { (void)h; return 0; }

void NGA_Access(int g_a, int lo[], int hi[], void *ptr, int ld[])
{
    (void)hi;
    ga_t *a = ga_get(g_a);
    char *base = (char *)a->data + ((size_t)lo[0] * a->dims[1] + lo[1]) * a->esize;
    *(void **)ptr = base;
    ld[0] = a->dims[1];
}

void NGA_Release(int g_a, int lo[], int hi[]) { (void)g_a; (void)lo; (void)hi; }
void NGA_Release_update(int g_a, int lo[], int hi[]) { (void)g_a; (void)lo; (void)hi; }

long NGA_Read_inc(int g_a, int subscript[], long inc)
{
    ga_t *a = ga_get(g_a);
    size_t i = (size_t)subscript[0] * a->dims[1] + subscript[1];
    int *d = (int *)a->data;
    long old = d[i];
    d[i] += (int)inc;
    return old;
}

void NGA_Distribution(int g_a, int iproc, int lo[], int hi[])
{
    ga_t *a = ga_get(g_a);
    if (iproc != 0) {
        lo[0] = lo[1] = 0;
        hi[0] = hi[1] = -1;
        return;
    }
    lo[0] = 0;
    lo[1] = 0;
    hi[0] = a->dims[0] - 1;
    hi[1] = a->dims[1] - 1;
}

void GA_Copy(int g_a, int g_b)
{
    ga_t *a = ga_get(g_a), *b = ga_get(g_b);
    memcpy(b->data, a->data, (size_t)a->dims[0] * a->dims[1] * a->esize);
}

void GA_Add(void *alpha, int g_a, void *beta, int g_b, int g_c)
{
    ga_t *a = ga_get(g_a), *b = ga_get(g_b), *c = ga_get(g_c);
    double al = *(double *)alpha, be = *(double *)beta;
    size_t n = (size_t)a->dims[0] * a->dims[1];
    double *A = (double *)a->data, *B = (double *)b->data, *C = (double *)c->data;
    for (size_t i = 0; i < n; i++) C[i] = al * A[i] + be * B[i];
}

void GA_Transpose(int g_a, int g_b)
{
    ga_t *a = ga_get(g_a), *b = ga_get(g_b);
    int r = a->dims[0], c = a->dims[1];
    double *A = (double *)a->data, *B = (double *)b->data;
    for (int i = 0; i < r; i++)
        for (int j = 0; j < c; j++) B[(size_t)j * r + i] = A[(size_t)i * c + j];
}

void GA_Symmetrize(int g_a)
{
    ga_t *a = ga_get(g_a);
    int n = a->dims[0];
    double *A = (double *)a->data;
    for (int i = 0; i < n; i++) {
        for (int j = i + 1; j < n; j++) {
            double v = 0.5 * (A[(size_t)i * n + j] + A[(size_t)j * n + i]);
            A[(size_t)i * n + j] = v;
            A[(size_t)j * n + i] = v;
        }
    }
}

void GA_Dgemm(char ta, char tb, int m, int n, int k, double alpha,
              int g_a, int g_b, double beta, int g_c)
{
    ga_t *a = ga_get(g_a), *b = ga_get(g_b), *c = ga_get(g_c);
    CBLAS_TRANSPOSE TA = (ta == 'T' || ta == 't') ? CblasTrans : CblasNoTrans;
    CBLAS_TRANSPOSE TB = (tb == 'T' || tb == 't') ? CblasTrans : CblasNoTrans;
    cblas_dgemm(CblasRowMajor, TA, TB, m, n, k, alpha, (double *)a->data, a->dims[1],
                (double *)b->data, b->dims[1], beta, (double *)c->data, c->dims[1]);
}

/* ---------------- MKL -> OpenBLAS ---------------- */

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

void *mkl_malloc(size_t size, int align) { return gtf_ref_aligned_calloc(size, (size_t)align); }
void mkl_free(void *p) { free(p); }

void cblas_dgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                 int m, int n, int k, double alpha, const double *a, int lda,
                 const double *b, int ldb, double beta, double *c, int ldc)
{
    scipy_cblas_dgemm((int)layout, (int)ta, (int)tb, m, n, k, alpha, a, lda, b, ldb,
                      beta, c, ldc);
}

/* Row-major LU/inverse through the column-major LAPACK on the transpose. */
static void transpose_sq(double *a, int n, int lda)
{
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++) {
            double t = a[(size_t)i * lda + j];
            a[(size_t)i * lda + j] = a[(size_t)j * lda + i];
            a[(size_t)j * lda + i] = t;
        }
}

int LAPACKE_dgetrf(int layout, int m, int n, double *a, int lda, int *ipiv)
{
    int info = 0;
    if (layout == LAPACK_ROW_MAJOR) transpose_sq(a, n, lda);
    scipy_dgetrf_(&m, &n, a, &lda, ipiv, &info);
    if (layout == LAPACK_ROW_MAJOR) transpose_sq(a, n, lda);
    return info;
}

int LAPACKE_dgetri(int layout, int n, double *a, int lda, const int *ipiv)
{
    int info = 0;
    int lwork = 64 * (n > 1 ? n : 1);
    double *work = (double *)malloc(sizeof(double) * lwork);
    if (layout == LAPACK_ROW_MAJOR) transpose_sq(a, n, lda);
    scipy_dgetri_(&n, a, &lda, ipiv, work, &lwork, &info);
    if (layout == LAPACK_ROW_MAJOR) transpose_sq(a, n, lda);
    free(work);
    return info;
}

/* ---------------- ScaLAPACK / BLACS on a 1 x 1 grid ---------------- */

void Cblacs_pinfo(int *mypnum, int *nprocs) { *mypnum = 0; *nprocs = 1; }
void Cblacs_get(int ictxt, int what, int *val) { (void)ictxt; (void)what; *val = 0; }
int Cblacs_gridinit(int *ictxt, char *order, int nprow, int npcol)
{
    (void)order; (void)nprow; (void)npcol;
    *ictxt = 0;
    return 0;
}
void Cblacs_gridinfo(int ictxt, int *nprow, int *npcol, int *myrow, int *mycol)
{
    (void)ictxt;
    *nprow = 1; *npcol = 1; *myrow = 0; *mycol = 0;
}
void Cblacs_gridexit(int ictxt) { (void)ictxt; }

int numroc_(int *n, int *nb, int *iproc, int *isrcproc, int *nprocs)
{
    /* number of rows/cols of a block-cyclic distribution owned by iproc */
    int mydist = (*nprocs + *iproc - *isrcproc) % *nprocs;
    int nblocks = *n / *nb;
    int num = (nblocks / *nprocs) * *nb;
    int extrablks = nblocks % *nprocs;
    if (mydist < extrablks) num += *nb;
    else if (mydist == extrablks) num += *n % *nb;
    return num;
}

int indxl2g_(int *indxloc, int *nb, int *iproc, int *isrcproc, int *nprocs)
{
    return *nprocs * *nb * ((*indxloc - 1) / *nb) + (*indxloc - 1) % *nb +
           ((*nprocs + *iproc - *isrcproc) % *nprocs) * *nb + 1;
}

void descinit_(int *desc, int *m, int *n, int *mb, int *nb, int *irsrc, int *icsrc,
               int *ictxt, int *lld, int *info)
{
    desc[0] = 1; desc[1] = *ictxt; desc[2] = *m; desc[3] = *n; desc[4] = *mb;
    desc[5] = *nb; desc[6] = *irsrc; desc[7] = *icsrc; desc[8] = *lld;
    *info = 0;
}

void pdsyevd(char *jobz, char *uplo, int *n, double *a, int *ia, int *ja, int *desca,
             double *w, double *z, int *iz, int *jz, int *descz, double *work,
             int *lwork, int *iwork, int *liwork, int *info)
{
    (void)ia; (void)ja; (void)iz; (void)jz; (void)descz;
    const int N = *n;
    if (*lwork == -1 || *liwork == -1) {
        work[0] = 1.0 + 6.0 * N + 2.0 * N * N;
        iwork[0] = 3 + 5 * N;
        *info = 0;
        return;
    }
    int lda = desca[8];
    for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++) z[(size_t)j * N + i] = a[(size_t)j * lda + i];
    scipy_dsyevd_(jobz, uplo, n, z, n, w, work, lwork, iwork, liwork, info, 1, 1);
}
