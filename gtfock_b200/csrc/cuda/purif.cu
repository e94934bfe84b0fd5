// purif.cu -- canonical density purification and Pulay DIIS on one GPU
// (pscf/purif.c:257-641; the 3-D pdgemm of pscf/pdgemm.c becomes one DGEMM).
//
// Purification (pscf/purif.c:301-476): Gershgorin bounds and tr F give the
// initial D; each iteration forms D2 = D D^T and D3 = D D2, reduces
// ||D - D2||_F, tr(D2 - D3) and tr(D - D2) deterministically (fixed block
// partials summed in order), updates D with the trace-conserving polynomial,
// and stops once ||D - D2||_F < 1e-11.  D_AO = X D X at the end.
// DIIS (pscf/purif.c:491-641): error X (F D S - S D F) X, dot products into
// the bordered B matrix, (m+1)^2 solve on the host, F = sum c_i F_i.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "devmem.cuh"
#include "diis_dev.cuh"
#include "gtf_cuda.h"

#define PUR_MAX_ITERS 200
#define PUR_MAX_DIIS GTF_MAX_DIIS
#define RED_BLOCKS 148
#define RED_THREADS 256

#define CKP(call)                                                                       \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            fprintf(stderr, "gtfock_b200 %s:%d %s\n", __FILE__, __LINE__, cudaGetErrorString(e_)); \
            return GTF_ERR_CUDA;                                                        \
        }                                                                               \
    } while (0)
#define CKB(call)                                                       \
    do {                                                                \
        if ((call) != CUBLAS_STATUS_SUCCESS) {                          \
            fprintf(stderr, "gtfock_b200 %s:%d cuBLAS failure\n", __FILE__, __LINE__); \
            return GTF_ERR_CUDA;                                        \
        }                                                               \
    } while (0)

extern "C" void gtf_note_launches(int n);

struct gtf_purif_dev {
    int n, nocc;
    cudaStream_t st;
    int own_st;               // the stream was created here
    cublasHandle_t blas;      // leased for the duration of one call (BlasLease)
    double *S, *X, *D, *D2, *D3, *F, *W, *W2;
    double *vecs, *Fvecs;
    double *part;     // [RED_BLOCKS * 16] block partials
    double *scal;     // device scalars
    double *h_scal;   // pinned mirror
    double *E;        // this iteration's DIIS error vector, before it enters its slot
    struct DiisState *ds;   // device: DIIS bookkeeping and coefficients
    int sx_set;
    cudaEvent_t e0, e1;
    double ms_gemm, ms_total, errnorm, idem, trerr;
    int mode;                 // 0 FP64, 1 split-BF16 then FP64
    gtf_bf16x3_t *bx;
    int it_bf16, it_fp64;
};

// row-major C = A B^T (pdgemm3D_2) and C = A B, via column-major cuBLAS
static int gemm_abt(gtf_purif_dev *p, const double *A, const double *B, double *C)
{
    const double one = 1.0, zero = 0.0;
    CKB(cublasDgemm(p->blas, CUBLAS_OP_T, CUBLAS_OP_N, p->n, p->n, p->n, &one, B, p->n, A, p->n, &zero, C, p->n));
    return GTF_OK;
}

static int gemm_ab(gtf_purif_dev *p, const double *A, const double *B, double *C)
{
    const double one = 1.0, zero = 0.0;
    CKB(cublasDgemm(p->blas, CUBLAS_OP_N, CUBLAS_OP_N, p->n, p->n, p->n, &one, B, p->n, A, p->n, &zero, C, p->n));
    return GTF_OK;
}

// per column i: Gershgorin interval [diag - off, diag + off], off = sum_j |F[j][i]| - |diag|
// (pscf/purif.c:309-322); block partials of min, max and the trace
__global__ void k_gersh(const double *__restrict__ F, int n, double *__restrict__ part)
{
    __shared__ double smin[RED_THREADS], smax[RED_THREADS], str[RED_THREADS];
    double lmin = DBL_MAX, lmax = -DBL_MAX, ltr = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double off = 0.0, dg = 0.0;
        for (int j = 0; j < n; j++) {
            const double v = F[(size_t)j * n + i];
            off += fabs(v);
            if (j == i) dg = v;
        }
        off -= fabs(dg);
        lmin = fmin(lmin, dg - off);
        lmax = fmax(lmax, dg + off);
        ltr += dg;
    }
    smin[threadIdx.x] = lmin;
    smax[threadIdx.x] = lmax;
    str[threadIdx.x] = ltr;
    __syncthreads();
    for (int s = RED_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + s]);
            smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + s]);
            str[threadIdx.x] += str[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x] = smin[0];
        part[3 * blockIdx.x + 1] = smax[0];
        part[3 * blockIdx.x + 2] = str[0];
    }
}

// scal[0] = -lambda/n, scal[1] = lambda mu_bar / n + nocc / n (pscf/purif.c:355-373)
__global__ void k_purif_init(const double *__restrict__ part, int nblk, int n, int nocc, double *scal)
{
    if (threadIdx.x != 0) return;
    double hmin = DBL_MAX, hmax = -DBL_MAX, trF = 0.0;
    for (int b = 0; b < nblk; b++) {
        hmin = fmin(hmin, part[3 * b]);
        hmax = fmax(hmax, part[3 * b + 1]);
        trF += part[3 * b + 2];
    }
    const double mu_bar = trF / (double)n;
    const double lambda = fmin((double)nocc / (hmax - mu_bar), (double)(n - nocc) / (mu_bar - hmin));
    scal[0] = -lambda / n;
    scal[1] = lambda * mu_bar / (double)n + (double)nocc / n;
    scal[2] = hmin;
    scal[3] = hmax;
    scal[4] = mu_bar;
    scal[5] = lambda;
}

__global__ void k_purif_d0(const double *__restrict__ F, double *__restrict__ D, int n, const double *scal)
{
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (size_t)n * n) return;
    double v = F[k] * scal[0];
    if (k / n == k % n) v += scal[1];
    D[k] = v;
}

// block partials of ||D - D2||^2, tr(D2 - D3), tr(D - D2)
__global__ void k_purif_stats(const double *__restrict__ D, const double *__restrict__ D2,
                              const double *__restrict__ D3, int n, double *__restrict__ part)
{
    __shared__ double s0[RED_THREADS], s1[RED_THREADS], s2[RED_THREADS];
    const size_t nn = (size_t)n * n;
    double e = 0.0, t = 0.0, t2 = 0.0;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += (size_t)gridDim.x * blockDim.x) {
        const double d = D[k] - D2[k];
        e += d * d;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const size_t k = (size_t)i * n + i;
        t += D2[k] - D3[k];
        t2 += D[k] - D2[k];
    }
    s0[threadIdx.x] = e;
    s1[threadIdx.x] = t;
    s2[threadIdx.x] = t2;
    __syncthreads();
    for (int s = RED_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            s0[threadIdx.x] += s0[threadIdx.x + s];
            s1[threadIdx.x] += s1[threadIdx.x + s];
            s2[threadIdx.x] += s2[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x] = s0[0];
        part[3 * blockIdx.x + 1] = s1[0];
        part[3 * blockIdx.x + 2] = s2[0];
    }
}

// scal[6] = errnorm, scal[7] = c = tr(D2-D3)/tr(D-D2) (pscf/purif.c:394-440).
// Where the reference would divide 0/0 (an exactly idempotent D) and write NaN
// into D, the iteration stops instead: errnorm is reported as 0 and the
// update below is skipped (c set to NaN).  It stops the same way when c is
// far outside [0, 1]: with every eigenvalue of D in [0, 1], c lies in [0, 1];
// far outside it the eigenvalues have left that interval and the cubic
// update diverges (in the reference, to Inf and NaN within a few steps).
// The loop's stop is kept on the device, so the host need not wait for every
// step: scal[8] != 0 once a step found ||D - D2||_F < 1e-11 (that step's
// update still applies, as in pscf/purif.c:394-455) or stopped as above;
// later steps then change nothing.  scal[9] counts the steps that ran.
// It also stops once the error, already below PURIF_FLOOR, has not fallen by
// 1% in PURIF_STALL steps (scal[10] the best error so far, 0 before the first
// step; scal[11] the steps since): rounding that holds the error just above
// the 1e-11 tolerance keeps the reference's loop running to its cap without
// changing D.  Above the floor the early steps of a purification can move
// the error by less than 1% for many steps, so no such stop applies there.
#define PURIF_C_LO (-0.25)
#define PURIF_C_HI 1.25
#define PURIF_TOL 1e-11
#define PURIF_STALL 8
#define PURIF_FLOOR 1e-8
__global__ void k_purif_finish(const double *__restrict__ part, int nblk, double *scal)
{
    if (threadIdx.x != 0) return;
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    if (scal[8] != 0.0) {
        scal[7] = nan;   // stopped: no update
        return;
    }
    double e = 0.0, t = 0.0, t2 = 0.0;
    for (int b = 0; b < nblk; b++) {
        e += part[3 * b];
        t += part[3 * b + 1];
        t2 += part[3 * b + 2];
    }
    const double c = t / t2;
    const bool ok = isfinite(c) && c >= PURIF_C_LO && c <= PURIF_C_HI;
    scal[6] = ok ? sqrt(e) : 0.0;
    scal[7] = ok ? c : nan;
    scal[9] += 1.0;
    if (ok) {
        if (scal[10] == 0.0 || scal[6] < 0.99 * scal[10]) {
            scal[10] = scal[6];
            scal[11] = 0.0;
        } else {
            scal[11] += 1.0;
        }
    }
    if (!ok || scal[6] < PURIF_TOL || (scal[10] < PURIF_FLOOR && scal[11] >= PURIF_STALL)) scal[8] = 1.0;
}

// steps between two host reads of the stop flag (FP64 phase)
#define PURIF_CHECK 4

// D update (pscf/purif.c:441-455)
__global__ void k_purif_update(double *__restrict__ D, const double *__restrict__ D2, const double *__restrict__ D3,
                               size_t nn, const double *scal)
{
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nn) return;
    const double c = scal[7];
    if (!isfinite(c)) return;
    if (c < 0.5) D[k] = ((1.0 - 2.0 * c) * D[k] + (1.0 + c) * D2[k] - D3[k]) / (1.0 - c);
    else D[k] = ((1.0 + c) * D2[k] - D3[k]) / c;
}

// D = (D + D^T) / 2 (the split-BF16 products are symmetric only to FP32
// rounding; the FP64 steps assume a symmetric D, as D D^T = D^2)
__global__ void k_symmetrize(double *__restrict__ D, int n)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= n || j <= i) return;
    const double v = 0.5 * (D[(size_t)i * n + j] + D[(size_t)j * n + i]);
    D[(size_t)i * n + j] = v;
    D[(size_t)j * n + i] = v;
}

// cur = W - W^T (F D S - (F D S)^T, pscf/purif.c:553-558)
__global__ void k_antisym(const double *__restrict__ W, double *__restrict__ cur, int n)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= n) return;
    cur[(size_t)i * n + j] = W[(size_t)i * n + j] - W[(size_t)j * n + i];
}

__global__ void k_diis_reset(DiisState *ds) { diis_reset(ds, threadIdx.x, blockDim.x); }

// slot of this iteration: the next free one, else the largest-error one
__global__ void k_diis_slot(DiisState *ds) { diis_slot(ds); }

// block partials of <e, e_k> for the stored vectors k < len, slot `cur`
// standing for e itself, which is stored into it on the way
__global__ void k_dots(const double *__restrict__ e, double *__restrict__ vecs, size_t nn, const DiisState *ds,
                       double *__restrict__ part)
{
    __shared__ double s[RED_THREADS];
    const int m = ds->len, cur = ds->cur;
    for (int k = 0; k < m; k++) {
        double *b = vecs + nn * k;
        double v = 0.0;
        for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += (size_t)gridDim.x * blockDim.x) {
            const double a = e[i];
            if (k == cur) {
                b[i] = a;
                v += a * a;
            } else {
                v += a * b[i];
            }
        }
        s[threadIdx.x] = v;
        __syncthreads();
        for (int st = RED_THREADS / 2; st > 0; st >>= 1) {
            if (threadIdx.x < st) s[threadIdx.x] += s[threadIdx.x + st];
            __syncthreads();
        }
        if (threadIdx.x == 0) part[blockIdx.x * PUR_MAX_DIIS + k] = s[0];
        __syncthreads();
    }
}

// New row and column of b from the block partials, then the largest-error
// slot and the coefficients (diis_coefficients).  One warp: lane i sums the
// partials of column i in block order.
__global__ void k_diis_solve(const double *__restrict__ part, DiisState *ds)
{
    __shared__ double dots[PUR_MAX_DIIS];
    const int lane = threadIdx.x;
    if (lane < ds->len) {
        double v = 0.0;
        for (int bk = 0; bk < RED_BLOCKS; bk++) v += part[bk * PUR_MAX_DIIS + lane];
        dots[lane] = v;
    }
    __syncwarp();
    diis_update_solve(ds, dots, lane);
}

// F = sum_i c_i F_i over the stored Fock matrices, slot `cur` standing for
// this iteration's X F X (Fx), which is stored into it on the way
__global__ void k_combine(double *__restrict__ F, double *__restrict__ Fvecs, const double *__restrict__ Fx, size_t nn,
                          const DiisState *ds)
{
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nn) return;
    const int m = ds->len, cur = ds->cur;
    const double fx = Fx[k];
    Fvecs[nn * cur + k] = fx;
    double v = 0.0;
    for (int i = 0; i < m; i++) v += ds->co[i] * (i == cur ? fx : Fvecs[nn * i + k]);
    F[k] = v;
}

extern "C" int gtf_purif_create(int nbf, int nocc, void *stream, gtf_purif_dev_t **out)
{
    *out = nullptr;
    if (nbf <= 0 || nocc < 0 || nocc > nbf) return GTF_ERR_INVALID;
    gtf_purif_dev *p = new gtf_purif_dev();
    memset(p, 0, sizeof(*p));
    p->n = nbf;
    p->nocc = nocc;
    p->st = (cudaStream_t)stream;
    if (!p->st) {
        CKP(cudaStreamCreateWithFlags(&p->st, cudaStreamNonBlocking));
        p->own_st = 1;
    }
    // device buffers from the stream-ordered pool on the object's stream,
    // pinned host scalars from the pinned pool (devmem.cu): creating and
    // destroying this object synchronizes nothing else
    const size_t nn = (size_t)nbf * nbf;
    double **bufs[] = {&p->S, &p->X, &p->D, &p->D2, &p->D3, &p->F, &p->W, &p->W2, &p->E};
    for (double **b : bufs) CKP(gtf_dmalloc((void **)b, sizeof(double) * nn, p->st));
    CKP(gtf_dmalloc((void **)&p->vecs, sizeof(double) * nn * PUR_MAX_DIIS, p->st));
    CKP(gtf_dmalloc((void **)&p->Fvecs, sizeof(double) * nn * PUR_MAX_DIIS, p->st));
    CKP(gtf_dmalloc((void **)&p->part, sizeof(double) * RED_BLOCKS * 16, p->st));
    CKP(gtf_dmalloc((void **)&p->scal, sizeof(double) * 16, p->st));
    p->h_scal = (double *)gtf_pinned_alloc(sizeof(double) * 16);
    if (!p->h_scal) return GTF_ERR_ALLOC;
    CKP(gtf_dmalloc((void **)&p->ds, sizeof(DiisState), p->st));
    CKP(cudaEventCreate(&p->e0));
    CKP(cudaEventCreate(&p->e1));
    k_diis_reset<<<1, 128, 0, p->st>>>(p->ds);
    CKP(cudaGetLastError());
    *out = p;
    return GTF_OK;
}

extern "C" int gtf_purif_set_mode(gtf_purif_dev_t *p, int mode)
{
    if (mode != 0 && mode != 1) return GTF_ERR_INVALID;
    if (mode == 1 && !p->bx) {
        const int r = gtf_bf16x3_create(p->n, p->st, &p->bx);
        if (r != GTF_OK) return r;
    }
    p->mode = mode;
    return GTF_OK;
}

extern "C" void gtf_purif_last_iters(gtf_purif_dev_t *p, int *bf16_iters, int *fp64_iters)
{
    if (bf16_iters) *bf16_iters = p->it_bf16;
    if (fp64_iters) *fp64_iters = p->it_fp64;
}

extern "C" void gtf_purif_destroy(gtf_purif_dev_t *p)
{
    if (!p) return;
    cudaStreamSynchronize(p->st);
    if (p->bx) gtf_bf16x3_destroy(p->bx);
    double *bufs[] = {p->S, p->X, p->D, p->D2, p->D3, p->F, p->W, p->W2, p->E, p->vecs, p->Fvecs, p->part, p->scal};
    for (double *b : bufs) gtf_dfree(b, p->st);
    gtf_dfree(p->ds, p->st);
    gtf_pinned_free(p->h_scal);
    if (p->e0) cudaEventDestroy(p->e0);
    if (p->e1) cudaEventDestroy(p->e1);
    if (p->own_st) cudaStreamDestroy(p->st);
    delete p;
}

// forget the DIIS history (a new SCF solve starts); stream-ordered
extern "C" void gtf_purif_reset(gtf_purif_dev_t *p)
{
    k_diis_reset<<<1, 128, 0, p->st>>>(p->ds);
    gtf_note_launches(1);
}

extern "C" int gtf_purif_set_sx(gtf_purif_dev_t *p, const double *S_host, const double *X_host)
{
    const size_t nn = (size_t)p->n * p->n;
    CKP(cudaMemcpyAsync(p->S, S_host, sizeof(double) * nn, cudaMemcpyHostToDevice, p->st));
    CKP(cudaMemcpyAsync(p->X, X_host, sizeof(double) * nn, cudaMemcpyHostToDevice, p->st));
    CKP(cudaStreamSynchronize(p->st));
    p->sx_set = 1;
    return GTF_OK;
}

extern "C" int gtf_purif_set_sx_dev(gtf_purif_dev_t *p, const double *S_dev, const double *X_dev)
{
    const size_t nn = (size_t)p->n * p->n;
    CKP(cudaMemcpyAsync(p->S, S_dev, sizeof(double) * nn, cudaMemcpyDeviceToDevice, p->st));
    CKP(cudaMemcpyAsync(p->X, X_dev, sizeof(double) * nn, cudaMemcpyDeviceToDevice, p->st));
    p->sx_set = 1;
    return GTF_OK;
}

extern "C" int gtf_purif_run_dev(gtf_purif_dev_t *p, const double *F_dev, double *D_dev, int *iters)
{
    BlasLease lease(p->st);
    if (!lease.h) return GTF_ERR_CUDA;
    p->blas = lease.h;
    const int n = p->n;
    const size_t nn = (size_t)n * n;
    const unsigned ge = (unsigned)((nn + 255) / 256);
    cudaStream_t st = p->st;
    CKP(cudaEventRecord(p->e0, st));
    k_gersh<<<RED_BLOCKS, RED_THREADS, 0, st>>>(F_dev, n, p->part);
    k_purif_init<<<1, 32, 0, st>>>(p->part, RED_BLOCKS, n, p->nocc, p->scal);
    k_purif_d0<<<ge, 256, 0, st>>>(F_dev, p->D, n, p->scal);
    CKP(cudaGetLastError());
    gtf_note_launches(3);
    int it;
    double err = 0.0;
    // split-BF16 phase: tensor-core products until the error stops falling
    // (their rounding sets a floor near 2^-16 relative), then FP64 steps
    p->it_bf16 = 0;
    if (p->mode == 1 && p->bx) {
        CKP(cudaMemsetAsync(p->scal + 8, 0, sizeof(double) * 4, st));
        double best = 1e300;
        int stall = 0;
        for (int k = 0; k < PUR_MAX_ITERS; k++) {
            if (gtf_bf16x3_abt(p->bx, p->D, p->D, p->D2, st)) return GTF_ERR_CUDA;
            if (gtf_bf16x3_abt(p->bx, p->D, p->D2, p->D3, st)) return GTF_ERR_CUDA;
            k_purif_stats<<<RED_BLOCKS, RED_THREADS, 0, st>>>(p->D, p->D2, p->D3, n, p->part);
            k_purif_finish<<<1, 32, 0, st>>>(p->part, RED_BLOCKS, p->scal);
            k_purif_update<<<ge, 256, 0, st>>>(p->D, p->D2, p->D3, nn, p->scal);
            k_symmetrize<<<dim3((n + 127) / 128, n), 128, 0, st>>>(p->D, n);
            CKP(cudaGetLastError());
            gtf_note_launches(4);
            CKP(cudaMemcpyAsync(p->h_scal + 6, p->scal + 6, sizeof(double) * 2, cudaMemcpyDeviceToHost, st));
            CKP(cudaStreamSynchronize(st));
            p->it_bf16++;
            const double e = p->h_scal[6];
            // hand over to FP64 once the error is small or stops falling
            // (BF16 rounding floor)
            if (!(e == e) || e < 1e-2) break;
            if (e < 0.99 * best) {
                best = e;
                stall = 0;
            } else if (++stall >= 3) {
                break;
            }
        }
    }
    // FP64 canonical steps (from the split-BF16 state in mode 1), PURIF_CHECK
    // launched per host read of the device-side stop flag
    CKP(cudaMemsetAsync(p->scal + 8, 0, sizeof(double) * 4, st));
    int steps = 0;
    bool stopped = false;
    for (it = 0; it < PUR_MAX_ITERS && !stopped;) {
        for (int k = 0; k < PURIF_CHECK && it < PUR_MAX_ITERS; k++, it++) {
            if (gemm_abt(p, p->D, p->D, p->D2)) return GTF_ERR_CUDA;
            if (gemm_ab(p, p->D, p->D2, p->D3)) return GTF_ERR_CUDA;
            k_purif_stats<<<RED_BLOCKS, RED_THREADS, 0, st>>>(p->D, p->D2, p->D3, n, p->part);
            k_purif_finish<<<1, 32, 0, st>>>(p->part, RED_BLOCKS, p->scal);
            k_purif_update<<<ge, 256, 0, st>>>(p->D, p->D2, p->D3, nn, p->scal);
            CKP(cudaGetLastError());
            gtf_note_launches(3);
        }
        CKP(cudaMemcpyAsync(p->h_scal + 6, p->scal + 6, sizeof(double) * 4, cudaMemcpyDeviceToHost, st));
        CKP(cudaStreamSynchronize(st));
        err = p->h_scal[6];
        steps = (int)p->h_scal[9];
        stopped = p->h_scal[8] != 0.0;
    }
    p->errnorm = err;
    // the counts of the reference's loop: steps run, and the index of the
    // step that met the tolerance
    p->it_fp64 = stopped ? steps : PUR_MAX_ITERS;
    it = (stopped ? steps - 1 : PUR_MAX_ITERS) + p->it_bf16;
    // D_AO = X D X (pscf/purif.c:469-476)
    if (gemm_abt(p, p->X, p->D, p->W)) return GTF_ERR_CUDA;
    if (gemm_abt(p, p->W, p->X, D_dev)) return GTF_ERR_CUDA;
    CKP(cudaEventRecord(p->e1, st));
    CKP(cudaEventSynchronize(p->e1));
    float ms = 0.0f;
    CKP(cudaEventElapsedTime(&ms, p->e0, p->e1));
    p->ms_total = ms;
    if (iters) *iters = (it < PUR_MAX_ITERS) ? it : PUR_MAX_ITERS;
    return GTF_OK;
}

extern "C" int gtf_purif_run(gtf_purif_dev_t *p, const double *F_host, double *D_host, int *iters)
{
    const size_t nn = (size_t)p->n * p->n;
    CKP(cudaMemcpyAsync(p->F, F_host, sizeof(double) * nn, cudaMemcpyHostToDevice, p->st));
    int r = gtf_purif_run_dev(p, p->F, p->D2, iters);
    if (r) return r;
    CKP(cudaMemcpyAsync(D_host, p->D2, sizeof(double) * nn, cudaMemcpyDeviceToHost, p->st));
    CKP(cudaStreamSynchronize(p->st));
    return GTF_OK;
}

// One DIIS step (pscf/purif.c:491-641) with its bookkeeping on the device:
// no host synchronisation.  iter <= 1: F = X F X only.
extern "C" int gtf_diis_step_dev(gtf_purif_dev_t *p, const double *D_dev, double *F_dev, int iter)
{
    BlasLease lease(p->st);
    if (!lease.h) return GTF_ERR_CUDA;
    p->blas = lease.h;
    const int n = p->n;
    const size_t nn = (size_t)n * n;
    cudaStream_t st = p->st;
    if (iter <= 1) {
        // F = X F X
        if (gemm_abt(p, p->X, F_dev, p->W)) return GTF_ERR_CUDA;
        if (gemm_abt(p, p->W, p->X, F_dev)) return GTF_ERR_CUDA;
        return GTF_OK;
    }
    k_diis_slot<<<1, 1, 0, st>>>(p->ds);
    // error vector e = X (F D S - S D F) X (pscf/purif.c:540-566)
    if (gemm_abt(p, F_dev, D_dev, p->W)) return GTF_ERR_CUDA;
    if (gemm_abt(p, p->W, p->S, p->W2)) return GTF_ERR_CUDA;
    dim3 g((n + 127) / 128, n);
    k_antisym<<<g, 128, 0, st>>>(p->W2, p->E, n);
    if (gemm_abt(p, p->X, p->E, p->W)) return GTF_ERR_CUDA;
    if (gemm_abt(p, p->W, p->X, p->E)) return GTF_ERR_CUDA;
    k_dots<<<RED_BLOCKS, RED_THREADS, 0, st>>>(p->E, p->vecs, nn, p->ds, p->part);
    k_diis_solve<<<1, 32, 0, st>>>(p->part, p->ds);
    // this iteration's X F X, then the extrapolation
    if (gemm_abt(p, p->X, F_dev, p->W)) return GTF_ERR_CUDA;
    if (gemm_abt(p, p->W, p->X, p->W2)) return GTF_ERR_CUDA;
    k_combine<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(F_dev, p->Fvecs, p->W2, nn, p->ds);
    CKP(cudaGetLastError());
    gtf_note_launches(5);
    return GTF_OK;
}

extern "C" int gtf_diis_step(gtf_purif_dev_t *p, const double *D_host, double *F_host, int iter)
{
    const size_t nn = (size_t)p->n * p->n;
    CKP(cudaMemcpyAsync(p->F, F_host, sizeof(double) * nn, cudaMemcpyHostToDevice, p->st));
    CKP(cudaMemcpyAsync(p->D3, D_host, sizeof(double) * nn, cudaMemcpyHostToDevice, p->st));
    int r = gtf_diis_step_dev(p, p->D3, p->F, iter);
    if (r) return r;
    CKP(cudaMemcpyAsync(F_host, p->F, sizeof(double) * nn, cudaMemcpyDeviceToHost, p->st));
    CKP(cudaStreamSynchronize(p->st));
    return GTF_OK;
}

extern "C" int gtf_purif_stats(gtf_purif_dev_t *p, double *ms_gemm, double *ms_total, double *errnorm,
                               double *idem_err, double *tr_err)
{
    if (ms_gemm) *ms_gemm = p->ms_gemm;
    if (ms_total) *ms_total = p->ms_total;
    if (errnorm) *errnorm = p->errnorm;
    if (idem_err) *idem_err = p->idem;
    if (tr_err) *tr_err = p->trerr;
    return GTF_OK;
}
