// eri_single.cu -- one contracted shell quartet on the device, for the
// per-quartet CInt entry points (CInt_computeShellQuartet,
// libcint/include/CInt.h:159-167) that callers outside the Fock build use.
// The quartet is evaluated in canonical orientation (L(a) >= L(b),
// L(c) >= L(d), bra class >= ket class) by the same Rys evaluator as the Fock
// kernels; the host side (cint_dev.c) permutes and applies the spherical
// transform.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>

#define GTF_MAX_PRIM_PAIRS 256

#include "gtf_cuda.h"
#include "gtf_dev.cuh"

// bra pair (a,b) and ket pair (c,d): records [0], [1]; primitive pairs in pp
template <int LA, int LB, int LC, int LD>
__global__ void k_single(const PairRec *__restrict__ pr, PrimPairs pp, double *__restrict__ out)
{
    constexpr int NQ = ncart(LA) * ncart(LB) * ncart(LC) * ncart(LD);
    PPStored src{pp};
    const PairRec pb = pr[0], pk = pr[1];
    double acc[NQ];
    for (int k = 0; k < NQ; k++) acc[k] = 0.0;
    eri_accumulate<LA, LB, LC, LD>(src, pb, src, pk, acc);
    for (int k = 0; k < NQ; k++) out[k] = acc[k];
}

static int launch_single(const PairRec *pr, PrimPairs pp, int la, int lb, int lc, int ld, double *out,
                         cudaStream_t st)
{
#define SQ(A, B, C, D)                                                    \
    if (la == A && lb == B && lc == C && ld == D) {                       \
        k_single<A, B, C, D><<<1, 1, 0, st>>>(pr, pp, out);               \
        return cudaGetLastError() == cudaSuccess ? GTF_OK : GTF_ERR_CUDA; \
    }
    SQ(0, 0, 0, 0)
    SQ(1, 0, 0, 0) SQ(1, 0, 1, 0)
    SQ(1, 1, 0, 0) SQ(1, 1, 1, 0) SQ(1, 1, 1, 1)
    SQ(2, 0, 0, 0) SQ(2, 0, 1, 0) SQ(2, 0, 1, 1) SQ(2, 0, 2, 0)
    SQ(2, 1, 0, 0) SQ(2, 1, 1, 0) SQ(2, 1, 1, 1) SQ(2, 1, 2, 0) SQ(2, 1, 2, 1)
    SQ(2, 2, 0, 0) SQ(2, 2, 1, 0) SQ(2, 2, 1, 1) SQ(2, 2, 2, 0) SQ(2, 2, 2, 1)
    SQ(2, 2, 2, 2)
#undef SQ
    return GTF_ERR_INVALID;
}

extern "C" void gtf_fock_basis_dev(gtf_fock_dev_t *f, const int **sh_L, const int **sh_nprim,
                                   const int **sh_pstart, const int **f_start, const int **fc_start,
                                   const double **sh_xyz, const double **alpha, const double **coef,
                                   const int **Z, const double **atom_xyz, int *nshells, int *natoms, int *nbf,
                                   int *pure);
extern "C" void *gtf_fock_stream(gtf_fock_dev_t *f);

// canonical-order Cartesian block of (a b | c d), first index fastest, into
// host `out` (<= 1296 doubles).  The caller passes the host basis so the pair
// data are formed here; dev_buf holds >= 8192 doubles of device scratch.
extern "C" int gtf_eri_single(gtf_fock_dev_t *f, const gtf_basis_view_t *b, int a, int bb, int c, int d,
                              double *dev_buf, double *out)
{
    const int sh[4] = {a, bb, c, d};
    for (int k = 0; k < 4; k++)
        if (sh[k] < 0 || sh[k] >= b->nshells) return GTF_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)gtf_fock_stream(f);
    PairRec pr[2];
    const int K0 = b->sh_nprim[a] * b->sh_nprim[bb], K1 = b->sh_nprim[c] * b->sh_nprim[d];
    const int npp = K0 + K1;
    double hpp[5 * 2 * GTF_MAX_PRIM_PAIRS];
    if (npp > 2 * GTF_MAX_PRIM_PAIRS) return GTF_ERR_INVALID;
    int off = 0;
    for (int k = 0; k < 2; k++) {
        const int x = sh[2 * k], y = sh[2 * k + 1];
        const double *A = b->xyz + 3 * b->sh_atom[x], *B = b->xyz + 3 * b->sh_atom[y];
        PairRec &r = pr[k];
        r.Ax = A[0]; r.Ay = A[1]; r.Az = A[2];
        r.ABx = A[0] - B[0]; r.ABy = A[1] - B[1]; r.ABz = A[2] - B[2];
        r.fa = r.fb = 0;
        r.off = off;
        r.n = b->sh_nprim[x] * b->sh_nprim[y];
        const double r2 = r.ABx * r.ABx + r.ABy * r.ABy + r.ABz * r.ABz;
        for (int i = 0; i < b->sh_nprim[x]; i++)
            for (int j = 0; j < b->sh_nprim[y]; j++) {
                const double al = b->alpha[b->sh_pstart[x] + i], be = b->alpha[b->sh_pstart[y] + j];
                const double p = al + be, ip = 1.0 / p;
                const int o = off + i * b->sh_nprim[y] + j;
                hpp[o] = p;
                hpp[npp + o] = (al * A[0] + be * B[0]) * ip;
                hpp[2 * npp + o] = (al * A[1] + be * B[1]) * ip;
                hpp[3 * npp + o] = (al * A[2] + be * B[2]) * ip;
                hpp[4 * npp + o] = GTF_PAIR_PREF * b->coef[b->sh_pstart[x] + i] * b->coef[b->sh_pstart[y] + j] *
                                   exp(-al * be * ip * r2) * ip;
            }
        off += r.n;
    }
    double *d_out = dev_buf;                       // 1296
    double *d_pp = dev_buf + 1296;                 // 5 * npp
    PairRec *d_pr = (PairRec *)(dev_buf + 1296 + 5 * 2 * GTF_MAX_PRIM_PAIRS);
    if (cudaMemcpyAsync(d_pp, hpp, sizeof(double) * 5 * npp, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(d_pr, pr, sizeof(pr), cudaMemcpyHostToDevice, st) != cudaSuccess)
        return GTF_ERR_CUDA;
    PrimPairs pp{d_pp, d_pp + npp, d_pp + 2 * npp, d_pp + 3 * npp, d_pp + 4 * npp};
    const int L[4] = {b->sh_L[a], b->sh_L[bb], b->sh_L[c], b->sh_L[d]};
    const int lr = launch_single(d_pr, pp, L[0], L[1], L[2], L[3], d_out, st);
    if (lr != GTF_OK) return lr;
    const int n = ncart(L[0]) * ncart(L[1]) * ncart(L[2]) * ncart(L[3]);
    if (cudaMemcpyAsync(out, d_out, sizeof(double) * n, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return GTF_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return GTF_ERR_CUDA;
    return GTF_OK;
}
