/*
 * cint_dev.c -- the integral half of the CInt API (libcint/include/CInt.h:
 * 90-181) served by the GPU kernels.
 *
 * The Fock build never calls these (its quartets are evaluated inside the
 * Fock kernels); they exist for callers that ask for single integral blocks:
 *   CInt_computeShellQuartet: one quartet by the device Rys evaluator
 *     (cuda/eri_single.cu) in canonical orientation, then permuted to the
 *     requested (A B | C D) order and transformed to spherical d; layout
 *     I[iA + dA*(iB + dB*(iC + dC*iD))] as pfock/fock_task.c:73-74 reads it;
 *   CInt_computePair{Ovl,Kin,Pot,CoreH}: blocks of S, T, V computed once per
 *     OED object on the device for the whole basis; layout block[iA + dA*iB]
 *     (pfock/one_electron.c:14-25).
 * Calls on one ERD object are serialised by a mutex (one device stream).
 */
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include "cuda/gtf_cuda.h"
#include "gtf_basis.h"

extern int gtf_basis_dev_create(const gtf_basis_view_t *b, gtf_fock_dev_t **out);
extern int gtf_eri_single(gtf_fock_dev_t *f, const gtf_basis_view_t *b, int a, int bb, int c, int d,
                          double *dev_buf, double *out);
extern int gtf_onee_full(gtf_fock_dev_t *f, double *S, double *T, double *V);
extern int gtf_dev_malloc(void **p, size_t bytes);
extern void gtf_dev_free(void *p);

#define MAXC 6
#define MAXQ (MAXC * MAXC * MAXC * MAXC)

static const double k_s3 = 1.7320508075688772935;

static gtf_basis_view_t view_of(BasisSet_t b)
{
    gtf_basis_view_t v;
    v.natoms = b->natoms;
    v.nshells = b->nshells;
    v.nbf = b->nbf;
    v.nbf_cart = b->nbf_cart;
    v.nprims = b->nprims;
    v.pure = b->pure;
    v.Z = b->Z;
    v.xyz = b->xyz;
    v.sh_atom = b->sh_atom;
    v.sh_L = b->sh_L;
    v.sh_nprim = b->sh_nprim;
    v.sh_pstart = b->sh_pstart;
    v.f_start = b->f_start;
    v.fc_start = b->fc_start;
    v.alpha = b->alpha;
    v.coef = b->coef;
    return v;
}

struct ERD {
    gtf_fock_dev_t *dev;
    double *dbuf;
    int nthreads;
    double *out;   /* [nthreads][MAXQ] */
    pthread_mutex_t lock;
};

CIntStatus_t CInt_createERD(BasisSet_t basis, ERD_t *erd, int nthreads)
{
    if (basis == NULL || erd == NULL || nthreads <= 0) return CINT_STATUS_INVALID_VALUE;
    ERD_t e = (ERD_t)calloc(1, sizeof(struct ERD));
    if (e == NULL) return CINT_STATUS_ALLOC_FAILED;
    gtf_basis_view_t v = view_of(basis);
    if (gtf_basis_dev_create(&v, &e->dev) != GTF_OK ||
        gtf_dev_malloc((void **)&e->dbuf, sizeof(double) * 8192) != GTF_OK) {
        if (e->dev) gtf_fock_destroy(e->dev);
        free(e);
        return CINT_STATUS_NOT_INITIALIZED;
    }
    e->nthreads = nthreads;
    e->out = (double *)malloc(sizeof(double) * MAXQ * 3 * (size_t)nthreads);
    pthread_mutex_init(&e->lock, NULL);
    *erd = e;
    return CINT_STATUS_SUCCESS;
}

CIntStatus_t CInt_destroyERD(ERD_t erd)
{
    if (erd == NULL) return CINT_STATUS_INVALID_VALUE;
    gtf_dev_free(erd->dbuf);
    gtf_fock_destroy(erd->dev);
    pthread_mutex_destroy(&erd->lock);
    free(erd->out);
    free(erd);
    return CINT_STATUS_SUCCESS;
}

void CInt_getMaxMemory(ERD_t erd, double *memsize)
{
    *memsize = erd ? (double)sizeof(double) * MAXQ * 3 * erd->nthreads : 0.0;
}

static int cls_of(int la, int lb)
{
    if (la < lb) { int t = la; la = lb; lb = t; }
    return la * (la + 1) / 2 + lb;
}

static void sph_row(int m, double *c) /* spherical d row m over xx..zz */
{
    memset(c, 0, sizeof(double) * 6);
    switch (m) {
        case 0: c[1] = k_s3; break;
        case 1: c[4] = k_s3; break;
        case 2: c[0] = -0.5; c[3] = -0.5; c[5] = 1.0; break;
        case 3: c[2] = k_s3; break;
        case 4: c[0] = 0.5 * k_s3; c[3] = -0.5 * k_s3; break;
    }
}

/* transform index pos of a 4-index block (dims n[], first index fastest)
 * from 6 Cartesian to 5 spherical d components */
static void sph_index(const double *in, double *out, int n[4], int pos)
{
    int stride = 1, outer = 1;
    for (int k = 0; k < pos; k++) stride *= n[k];
    for (int k = pos + 1; k < 4; k++) outer *= n[k];
    for (int o = 0; o < outer; o++)
        for (int m = 0; m < 5; m++) {
            double c[6];
            sph_row(m, c);
            for (int s = 0; s < stride; s++) {
                double v = 0.0;
                for (int k = 0; k < 6; k++)
                    if (c[k] != 0.0) v += c[k] * in[s + stride * (k + 6 * o)];
                out[s + stride * (m + 5 * o)] = v;
            }
        }
    n[pos] = 5;
}

CIntStatus_t CInt_computeShellQuartet(BasisSet_t basis, ERD_t erd, int tid, int A, int B, int C, int D,
                                      double **integrals, int *nints)
{
    if (erd == NULL || tid < 0 || tid >= erd->nthreads) return CINT_STATUS_INVALID_VALUE;
    const int req[4] = {A, B, C, D};
    for (int k = 0; k < 4; k++)
        if (req[k] < 0 || req[k] >= basis->nshells) return CINT_STATUS_INVALID_VALUE;
    /* canonical order: L(a) >= L(b), L(c) >= L(d), class(ab) >= class(cd) */
    int pos[4] = {0, 1, 2, 3};   /* canonical slot k holds requested index pos[k] */
    if (basis->sh_L[A] < basis->sh_L[B]) { pos[0] = 1; pos[1] = 0; }
    if (basis->sh_L[C] < basis->sh_L[D]) { pos[2] = 3; pos[3] = 2; }
    if (cls_of(basis->sh_L[A], basis->sh_L[B]) < cls_of(basis->sh_L[C], basis->sh_L[D])) {
        int t0 = pos[0], t1 = pos[1];
        pos[0] = pos[2]; pos[1] = pos[3];
        pos[2] = t0; pos[3] = t1;
    }
    double *cart = erd->out + (size_t)tid * MAXQ * 3;
    double *tmp = cart + MAXQ, *res = cart + 2 * MAXQ;
    pthread_mutex_lock(&erd->lock);
    gtf_basis_view_t v = view_of(basis);
    int e = gtf_eri_single(erd->dev, &v, req[pos[0]], req[pos[1]], req[pos[2]], req[pos[3]], erd->dbuf, tmp);
    pthread_mutex_unlock(&erd->lock);
    if (e != GTF_OK) return CINT_STATUS_EXECUTION_FAILED;
    int nc[4], can_n[4];
    for (int k = 0; k < 4; k++) nc[k] = gtf_cart_dim(basis->sh_L[req[k]]);
    for (int k = 0; k < 4; k++) can_n[k] = nc[pos[k]];
    /* permute canonical -> requested order */
    int idx[4];
    for (idx[3] = 0; idx[3] < nc[3]; idx[3]++)
        for (idx[2] = 0; idx[2] < nc[2]; idx[2]++)
            for (idx[1] = 0; idx[1] < nc[1]; idx[1]++)
                for (idx[0] = 0; idx[0] < nc[0]; idx[0]++) {
                    int ci[4];
                    for (int k = 0; k < 4; k++) ci[k] = idx[pos[k]];
                    const int src = ci[0] + can_n[0] * (ci[1] + can_n[1] * (ci[2] + can_n[2] * ci[3]));
                    const int dst = idx[0] + nc[0] * (idx[1] + nc[1] * (idx[2] + nc[2] * idx[3]));
                    cart[dst] = tmp[src];
                }
    double *src = cart, *dst = tmp;
    int n[4] = {nc[0], nc[1], nc[2], nc[3]};
    if (basis->pure) {
        for (int k = 0; k < 4; k++) {
            if (basis->sh_L[req[k]] == 2) {
                sph_index(src, dst, n, k);
                double *t = src; src = dst; dst = t;
            }
        }
    }
    const int total = n[0] * n[1] * n[2] * n[3];
    memcpy(res, src, sizeof(double) * total);
    *integrals = res;
    *nints = total;
    return CINT_STATUS_SUCCESS;
}

CIntStatus_t CInt_computeShellQuartets(BasisSet_t basis, ERD_t erd, uint32_t threadId,
                                       uint32_t shellIndixA, const uint32_t *shellIndicesB,
                                       uint32_t shellIndixC, const uint32_t *shellIndicesD,
                                       uint32_t shellIndicesCount, double **integrals, int *integralsCount)
{
    static __thread double *buf = NULL;
    static __thread size_t cap = 0;
    size_t need = (size_t)shellIndicesCount * 625;
    if (need > cap) {
        free(buf);
        buf = (double *)malloc(sizeof(double) * (need ? need : 1));
        cap = buf ? need : 0;
        if (!buf) return CINT_STATUS_ALLOC_FAILED;
    }
    int off = 0;
    for (uint32_t k = 0; k < shellIndicesCount; k++) {
        double *ints;
        int n;
        CIntStatus_t st = CInt_computeShellQuartet(basis, erd, (int)threadId, (int)shellIndixA,
                                                   (int)shellIndicesB[k], (int)shellIndixC,
                                                   (int)shellIndicesD[k], &ints, &n);
        if (st != CINT_STATUS_SUCCESS) return st;
        memcpy(buf + off, ints, sizeof(double) * n);
        off += n;
    }
    *integrals = buf;
    *integralsCount = off;
    return CINT_STATUS_SUCCESS;
}

struct OED {
    int nbf;
    const int *f_start;
    double *S, *T, *V;
    double out[36];
};

CIntStatus_t CInt_createOED(BasisSet_t basis, OED_t *oed)
{
    if (basis == NULL || oed == NULL) return CINT_STATUS_INVALID_VALUE;
    OED_t o = (OED_t)calloc(1, sizeof(struct OED));
    if (o == NULL) return CINT_STATUS_ALLOC_FAILED;
    const size_t nn = (size_t)basis->nbf * basis->nbf;
    o->nbf = basis->nbf;
    o->f_start = basis->f_start;
    o->S = (double *)malloc(sizeof(double) * nn);
    o->T = (double *)malloc(sizeof(double) * nn);
    o->V = (double *)malloc(sizeof(double) * nn);
    gtf_basis_view_t v = view_of(basis);
    gtf_fock_dev_t *dev = NULL;
    int e = (o->S && o->T && o->V) ? gtf_basis_dev_create(&v, &dev) : GTF_ERR_ALLOC;
    if (e == GTF_OK) e = gtf_onee_full(dev, o->S, o->T, o->V);
    if (dev) gtf_fock_destroy(dev);
    if (e != GTF_OK) {
        free(o->S); free(o->T); free(o->V); free(o);
        return CINT_STATUS_NOT_INITIALIZED;
    }
    *oed = o;
    return CINT_STATUS_SUCCESS;
}

CIntStatus_t CInt_destroyOED(OED_t oed)
{
    if (oed == NULL) return CINT_STATUS_INVALID_VALUE;
    free(oed->S); free(oed->T); free(oed->V);
    free(oed);
    return CINT_STATUS_SUCCESS;
}

static CIntStatus_t pair_block(BasisSet_t basis, OED_t o, int A, int B, int which, double **I, int *n)
{
    if (A < 0 || B < 0 || A >= basis->nshells || B >= basis->nshells) return CINT_STATUS_INVALID_VALUE;
    const int r0 = basis->f_start[A], nr = basis->f_start[A + 1] - r0;
    const int c0 = basis->f_start[B], nc = basis->f_start[B + 1] - c0;
    for (int l = 0; l < nc; l++)
        for (int k = 0; k < nr; k++) {
            const size_t g = (size_t)(r0 + k) * o->nbf + c0 + l;
            double v = which == 0 ? o->S[g] : which == 1 ? o->T[g] : which == 2 ? o->V[g] : o->T[g] + o->V[g];
            o->out[k + nr * l] = v;
        }
    *I = o->out;
    *n = nr * nc;
    return CINT_STATUS_SUCCESS;
}

CIntStatus_t CInt_computePairOvl(BasisSet_t b, OED_t o, int A, int B, double **I, int *n)
{
    return pair_block(b, o, A, B, 0, I, n);
}

CIntStatus_t CInt_computePairKin(BasisSet_t b, OED_t o, int A, int B, double **I, int *n)
{
    return pair_block(b, o, A, B, 1, I, n);
}

CIntStatus_t CInt_computePairPot(BasisSet_t b, OED_t o, int A, int B, double **I, int *n)
{
    return pair_block(b, o, A, B, 2, I, n);
}

CIntStatus_t CInt_computePairCoreH(BasisSet_t b, OED_t o, int A, int B, double **I, int *n)
{
    return pair_block(b, o, A, B, 3, I, n);
}
