// batch_scf.cu -- many SCF jobs (molecules of different sizes) iterated in
// lock-step on one GPU.
//
// Every step runs one SCF iteration (pscf/scf.c:348-459) of every running
// job: one batched Fock build (one launch per class pair, precision part and
// slice for all jobs, gtf_fock_batch_compute), the energy of
// pscf/scf.c:80-102, DIIS (pscf/purif.c:491-641) and canonical purification
// (pscf/purif.c:257-488), each as a few launches that cover all jobs.  The
// dense products are batched tiled DGEMMs over per-job descriptors; the
// reductions (energy, DIIS dots, purification traces and norms) use one block
// per job in a fixed order, so a job's numbers do not depend on its
// neighbours.  The DIIS bookkeeping (bordered matrix, replacement of the
// vector with the largest error, the small solve) stays on the host as in the
// single-job path.
//
// Jobs may join (gtf_batch_add) and leave (gtf_batch_remove) between steps:
// the serving loop admits a request as soon as a slot and device memory are
// free, and its iterations then interleave with those of the jobs already
// running.
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <utility>
#include <vector>

#include "devmem.cuh"
#include "diis_dev.cuh"
#include "gtf_cuda.h"
#include "gtfock_b200.h"

extern "C" gtf_fock_dev_t *gtf_pfock_device(PFock_t pf);
extern "C" int gtf_initial_density(BasisSet_t basis, double *D, int n);
extern "C" void gtf_note_launches(int n);
extern "C" const char *gtf_last_error(void);

#define BJ_MAX_DIIS GTF_MAX_DIIS
#define BJ_THREADS 256
#define BJ_PUR_MAX 200
#define BJ_PUR_CHECK 8
#define BJ_EBLOCKS 64   // blocks per job of the energy reduction
// Jobs above BJ_BIG functions run DIIS and purification through the single-job
// path (cuBLAS DGEMM, multi-block reductions) on the batch's stream: their
// products are large enough to fill the GPU alone.
#define BJ_BIG 640

// ---------------------------------------------------------------------------
// device side
// ---------------------------------------------------------------------------
struct JobDev {
    double *D, *F;                 // engine density (AO, input of the Fock build) and Fock matrix
    // the Fock build's result: F itself, or for incremental builds the
    // engine's running sum, which the step must leave intact (F is then the
    // job's own copy that receives F + H and DIIS)
    const double *Fe;
    const double *H, *S, *X;
    double *P, *P2, *P3, *W, *W2;  // purification (orthogonal basis) and scratch
    double *vecs, *Fvecs;          // DIIS error vectors and Fock matrices
    DiisState *ds;                 // the job's DIIS bookkeeping (device)
    int n, nocc;
    int diis;                      // DIIS this iteration (else F = X F X only)
};

struct GemmDesc {
    const double *A, *B;
    double *C;
    int n;
    int job;                       // index into the active flags (-1: always)
};

// C = A B^T (TB) or C = A B, row-major n x n.  Block t of the launch is tile
// (ti, tj) of descriptor d, found in the exclusive tile prefix.  BM x BN
// output tiles, TM x TN per thread, KT-deep slabs of A and op(B) in
// shared memory (column-major in the slab so a thread's TM / TN values are
// contiguous 16-byte vectors), double-buffered: the next slab's global loads
// are in flight while the current one is multiplied.  Rows of the
// transposed slabs are padded by two doubles so the transposing stores of a
// warp spread over the banks.
template <bool TB, int BM, int BN, int TM, int TN, int KT>
__global__ void __launch_bounds__((BM / TM) * (BN / TN)) k_bgemm(const GemmDesc *__restrict__ ds,
                                                               const int *__restrict__ tile_prefix, int nd,
                                                               const int *__restrict__ active)
{
    constexpr int NT = (BM / TM) * (BN / TN);
    constexpr int NA = BM * KT / NT, NB = BN * KT / NT;   // slab elements per thread
    static_assert(BM * KT % NT == 0 && BN * KT % NT == 0 && TM % 2 == 0 && TN % 2 == 0, "tile shape");
    constexpr int PA = BM + 2, PB = TB ? BN + 2 : BN;
    __shared__ __align__(16) double As[2][KT][PA];
    __shared__ __align__(16) double Bs[2][KT][PB];
    const int t = blockIdx.x;
    int lo = 0, hi = nd;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (tile_prefix[mid] <= t) lo = mid;
        else hi = mid;
    }
    const GemmDesc g = ds[lo];
    if (g.job >= 0 && active && !active[g.job]) return;
    const int n = g.n;
    const int ntc = (n + BN - 1) / BN;
    const int local = t - tile_prefix[lo];
    const int r0 = (local / ntc) * BM, c0 = (local % ntc) * BN;
    const int tid = threadIdx.x;
    const int tx = tid % (BN / TN), ty = tid / (BN / TN);
    double ra[NA], rb[NB];
    // slab k0 -> registers (zero outside the matrix)
    auto load = [&](int k0) {
#pragma unroll
        for (int q = 0; q < NA; q++) {
            const int e = tid + q * NT, kk = e % KT, rr = e / KT;
            const int ar = r0 + rr, ak = k0 + kk;
            ra[q] = (ar < n && ak < n) ? __ldg(g.A + (size_t)ar * n + ak) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < NB; q++) {
            const int e = tid + q * NT;
            if (TB) {
                const int kk = e % KT, cc = e / KT, bc = c0 + cc, bk = k0 + kk;
                rb[q] = (bc < n && bk < n) ? __ldg(g.B + (size_t)bc * n + bk) : 0.0;
            } else {
                const int cc = e % BN, kk = e / BN, bc = c0 + cc, bk = k0 + kk;
                rb[q] = (bc < n && bk < n) ? __ldg(g.B + (size_t)bk * n + bc) : 0.0;
            }
        }
    };
    auto store = [&](int buf) {
#pragma unroll
        for (int q = 0; q < NA; q++) {
            const int e = tid + q * NT;
            As[buf][e % KT][e / KT] = ra[q];
        }
#pragma unroll
        for (int q = 0; q < NB; q++) {
            const int e = tid + q * NT;
            if (TB) Bs[buf][e % KT][e / KT] = rb[q];
            else Bs[buf][e / BN][e % BN] = rb[q];
        }
    };
    double acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; i++)
#pragma unroll
        for (int j = 0; j < TN; j++) acc[i][j] = 0.0;
    load(0);
    store(0);
    __syncthreads();
    int cur = 0;
    for (int k0 = 0; k0 < n; k0 += KT) {
        const bool more = k0 + KT < n;
        if (more) load(k0 + KT);
#pragma unroll
        for (int kk = 0; kk < KT; kk++) {
            double a[TM], b[TN];
#pragma unroll
            for (int i = 0; i < TM; i += 2) {
                const double2 v = *reinterpret_cast<const double2 *>(&As[cur][kk][ty * TM + i]);
                a[i] = v.x;
                a[i + 1] = v.y;
            }
#pragma unroll
            for (int j = 0; j < TN; j += 2) {
                const double2 v = *reinterpret_cast<const double2 *>(&Bs[cur][kk][tx * TN + j]);
                b[j] = v.x;
                b[j + 1] = v.y;
            }
#pragma unroll
            for (int i = 0; i < TM; i++)
#pragma unroll
                for (int j = 0; j < TN; j++) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        if (more) store(cur ^ 1);
        __syncthreads();
        cur ^= 1;
    }
#pragma unroll
    for (int i = 0; i < TM; i++) {
        const int r = r0 + ty * TM + i;
        if (r >= n) continue;
#pragma unroll
        for (int j = 0; j < TN; j++) {
            const int c = c0 + tx * TN + j;
            if (c < n) g.C[(size_t)r * n + c] = acc[i][j];
        }
    }
}

// Tile shapes the batched products can run with (the autotuner picks one per
// batch; 0 is the default).
struct BGemmShape {
    int bm, bn, tm, tn, kt;
};
static const BGemmShape BG_SHAPES[] = {{64, 64, 4, 4, 16}, {32, 32, 2, 2, 16}, {32, 64, 2, 4, 16},
                                       {128, 64, 8, 4, 8}};
#define BG_NSHAPES 4

template <bool TB>
static void launch_bgemm_shape(int shape, int ntiles, cudaStream_t st, const GemmDesc *gd, const int *tp, int m,
                               const int *active)
{
    switch (shape) {
        case 1: k_bgemm<TB, 32, 32, 2, 2, 16><<<ntiles, 256, 0, st>>>(gd, tp, m, active); break;
        case 2: k_bgemm<TB, 32, 64, 2, 4, 16><<<ntiles, 256, 0, st>>>(gd, tp, m, active); break;
        case 3: k_bgemm<TB, 128, 64, 8, 4, 8><<<ntiles, 256, 0, st>>>(gd, tp, m, active); break;
        default: k_bgemm<TB, 64, 64, 4, 4, 16><<<ntiles, 256, 0, st>>>(gd, tp, m, active); break;
    }
}

__device__ __forceinline__ double block_sum(double v, double *sh)
{
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int s = BJ_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

// job blockIdx.y: F += H and block partials of sum D (H + F) (pscf/scf.c:80-102);
// the host adds the BJ_EBLOCKS partials of a job in order
__global__ void __launch_bounds__(BJ_THREADS) k_j_energy(const JobDev *__restrict__ jobs, double *__restrict__ part)
{
    __shared__ double sh[BJ_THREADS];
    const JobDev j = jobs[blockIdx.y];
    const size_t nn = (size_t)j.n * j.n;
    double e = 0.0;
    for (size_t k = (size_t)blockIdx.x * BJ_THREADS + threadIdx.x; k < nn; k += (size_t)BJ_EBLOCKS * BJ_THREADS) {
        const double f = j.Fe[k] + j.H[k];
        j.F[k] = f;
        e += j.D[k] * (j.H[k] + f);
    }
    e = block_sum(e, sh);
    if (threadIdx.x == 0) part[blockIdx.y * BJ_EBLOCKS + blockIdx.x] = e;
}

__global__ void k_j_diis_reset(DiisState *ds) { diis_reset(ds, threadIdx.x, blockDim.x); }

// slot of this iteration's vectors, per DIIS job
__global__ void k_j_diis_slot(const JobDev *__restrict__ jobs, int m)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < m && jobs[q].diis) diis_slot(jobs[q].ds);
}

// P2 = W2 - W2^T, the commutator of the error vector (pscf/purif.c:553-558);
// P2 and P3 are free until the purification starts
__global__ void k_j_antisym(const JobDev *__restrict__ jobs)
{
    const JobDev j = jobs[blockIdx.y];
    if (!j.diis) return;
    const size_t nn = (size_t)j.n * j.n;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(k / j.n), c = (int)(k % j.n);
        j.P2[k] = j.W2[k] - j.W2[(size_t)c * j.n + r];
    }
}

// dots[job][i] = <e, vecs[i]>, i < len, with e = P2 the error vector in the
// orthogonal basis; slot cur stands for e, which is stored into it on the way
__global__ void __launch_bounds__(BJ_THREADS) k_j_dots(const JobDev *__restrict__ jobs, double *__restrict__ dots)
{
    __shared__ double sh[BJ_THREADS];
    const JobDev j = jobs[blockIdx.x];
    if (!j.diis) return;
    const size_t nn = (size_t)j.n * j.n;
    const double *a = j.P2;
    const int len = j.ds->len, cur = j.ds->cur;
    for (int i = 0; i < len; i++) {
        double *b = j.vecs + nn * i;
        double v = 0.0;
        if (i == cur) {
            for (size_t k = threadIdx.x; k < nn; k += BJ_THREADS) {
                const double x = a[k];
                b[k] = x;
                v += x * x;
            }
        } else {
            for (size_t k = threadIdx.x; k < nn; k += BJ_THREADS) v += a[k] * b[k];
        }
        v = block_sum(v, sh);
        if (threadIdx.x == 0) dots[blockIdx.x * BJ_MAX_DIIS + i] = v;
    }
}

// new row and column of the bordered matrix, then the coefficients: one warp per job
__global__ void k_j_diis_solve(const JobDev *__restrict__ jobs, const double *__restrict__ dots)
{
    const JobDev j = jobs[blockIdx.x];
    if (!j.diis) return;
    diis_update_solve(j.ds, dots + blockIdx.x * BJ_MAX_DIIS, threadIdx.x);
}

// F = sum_i c_i Fvecs_i, slot cur standing for this iteration's X F X (P3),
// which is stored into it on the way
__global__ void k_j_combine(const JobDev *__restrict__ jobs)
{
    const JobDev j = jobs[blockIdx.y];
    if (!j.diis) return;
    const size_t nn = (size_t)j.n * j.n;
    const int len = j.ds->len, cur = j.ds->cur;
    const double *c = j.ds->co;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += (size_t)gridDim.x * blockDim.x) {
        const double fx = j.P3[k];
        j.Fvecs[nn * cur + k] = fx;
        double v = 0.0;
        for (int i = 0; i < len; i++) v += c[i] * (i == cur ? fx : j.Fvecs[nn * i + k]);
        j.F[k] = v;
    }
}

// Gershgorin bounds and trace of F (orthogonal basis), initial P
// (pscf/purif.c:309-373); scal[job*8 + 0..1] hold the two coefficients
__global__ void __launch_bounds__(BJ_THREADS) k_j_pur_init(const JobDev *__restrict__ jobs, double *__restrict__ scal,
                                                          int *__restrict__ active)
{
    __shared__ double sh[BJ_THREADS];
    __shared__ double c01[2];
    const JobDev j = jobs[blockIdx.x];
    const int n = j.n;
    double lmin = DBL_MAX, lmax = -DBL_MAX, ltr = 0.0;
    for (int i = threadIdx.x; i < n; i += BJ_THREADS) {
        double off = 0.0, dg = 0.0;
        for (int r = 0; r < n; r++) {
            const double v = j.F[(size_t)r * n + i];
            off += fabs(v);
            if (r == i) dg = v;
        }
        off -= fabs(dg);
        lmin = fmin(lmin, dg - off);
        lmax = fmax(lmax, dg + off);
        ltr += dg;
    }
    // min / max / sum reductions in a fixed order
    sh[threadIdx.x] = lmin;
    __syncthreads();
    for (int s = BJ_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] = fmin(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    const double hmin = sh[0];
    __syncthreads();
    sh[threadIdx.x] = lmax;
    __syncthreads();
    for (int s = BJ_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    const double hmax = sh[0];
    __syncthreads();
    const double trF = block_sum(ltr, sh);
    if (threadIdx.x == 0) {
        const double mu_bar = trF / (double)n;
        const double lambda = fmin((double)j.nocc / (hmax - mu_bar), (double)(n - j.nocc) / (mu_bar - hmin));
        c01[0] = -lambda / n;
        c01[1] = lambda * mu_bar / (double)n + (double)j.nocc / n;
        scal[blockIdx.x * 8 + 0] = c01[0];
        scal[blockIdx.x * 8 + 1] = c01[1];
        scal[blockIdx.x * 8 + 3] = 0.0;   // best error so far (0: none yet)
        scal[blockIdx.x * 8 + 4] = 0.0;   // steps since it last fell by 1%
        active[blockIdx.x] = 1;
    }
    __syncthreads();
    const size_t nn = (size_t)n * n;
    for (size_t k = threadIdx.x; k < nn; k += BJ_THREADS) {
        double v = j.F[k] * c01[0];
        if (k / n == k % n) v += c01[1];
        j.P[k] = v;
    }
}

// ||P - P2||_F, c = tr(P2 - P3) / tr(P - P2), then the trace-conserving
// update (pscf/purif.c:394-455); a job stops once ||P - P2||_F < 1e-11, or
// once that error, already below 1e-8, has not fallen by 1% in 8 steps
// (rounding above the tolerance: the reference's loop would run to its cap
// without changing P), as the one-job path does.
// Block b serves job list[b] (the jobs still purifying).
__global__ void __launch_bounds__(BJ_THREADS) k_j_pur_step(const JobDev *__restrict__ jobs, const int *__restrict__ list,
                                                          double *__restrict__ scal, int *__restrict__ active,
                                                          int *__restrict__ iters)
{
    __shared__ double sh[BJ_THREADS];
    const int q = list[blockIdx.x];
    if (!active[q]) return;
    const JobDev j = jobs[q];
    const int n = j.n;
    const size_t nn = (size_t)n * n;
    double e = 0.0, t = 0.0, t2 = 0.0;
    for (size_t k = threadIdx.x; k < nn; k += BJ_THREADS) {
        const double d = j.P[k] - j.P2[k];
        e += d * d;
    }
    for (int i = threadIdx.x; i < n; i += BJ_THREADS) {
        const size_t k = (size_t)i * n + i;
        t += j.P2[k] - j.P3[k];
        t2 += j.P[k] - j.P2[k];
    }
    e = block_sum(e, sh);
    t = block_sum(t, sh);
    t2 = block_sum(t2, sh);
    const double c = t / t2;
    // 0/0 at an idempotent P, or c far outside [0, 1] (eigenvalues of P out
    // of [0, 1], the update diverging): stop and keep P, as the one-job path
    const bool ok = isfinite(c) && c >= -0.25 && c <= 1.25;
    const double err = ok ? sqrt(e) : 0.0;
    for (size_t k = threadIdx.x; k < nn && ok; k += BJ_THREADS) {
        if (c < 0.5) j.P[k] = ((1.0 - 2.0 * c) * j.P[k] + (1.0 + c) * j.P2[k] - j.P3[k]) / (1.0 - c);
        else j.P[k] = ((1.0 + c) * j.P2[k] - j.P3[k]) / c;
    }
    if (threadIdx.x == 0) {
        scal[q * 8 + 2] = err;
        iters[q] += 1;
        double &best = scal[q * 8 + 3], &stall = scal[q * 8 + 4];
        if (ok) {
            if (best == 0.0 || err < 0.99 * best) {
                best = err;
                stall = 0.0;
            } else {
                stall += 1.0;
            }
        }
        if (err < 1e-11 || (best < 1e-8 && stall >= 8.0)) active[q] = 0;
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct BJob {
    int used;
    int n, nocc, nbf_cart;
    double enuc;
    BasisSet_t basis;
    PFock_t pf;
    gtf_fock_dev_t *eng;
    gtf_purif_dev_t *pd;           // jobs above BJ_BIG functions: single-job DIIS / purification
    double *mem;
    double *fcopy;                 // incremental builds: the job's copy of F (see JobDev::Fe)
    int inc_since;                 // builds since the last full one (incremental builds)
    size_t bytes;
    JobDev dv;
    // SCF state
    int iter, max_iters, done, failed;
    double etol, e_prev;
    std::vector<double> energies;
    int pur_iters;
    long long pur_total;           // purification iterations over all steps
};

struct gtf_batch {
    int capacity;
    std::vector<BJob> jobs;
    cudaStream_t st;
    gtf_fock_batch_t *fb;
    std::vector<int> fb_members;   // slots in the current Fock batch
    int dirty;
    // the batched Fock build of the current membership, captured once as a
    // CUDA graph and replayed every step (null: launch directly)
    cudaGraphExec_t fock_exec;
    int fock_launches;
    int gshape;                    // tile shape of the batched products (BG_SHAPES)
    // device arrays (capacity-sized)
    JobDev *d_jobs;
    GemmDesc *d_gd;                // 10 call sets x capacity
    int *d_tp;                     // 10 call sets x (capacity + 1)
    double *d_energy, *d_dots, *d_scal;
    DiisState *d_diis;             // per slot: the job's DIIS bookkeeping
    int *d_active, *d_iters, *d_count, *d_list;
    // pinned mirrors
    JobDev *h_jobs;
    GemmDesc *h_gd;
    int *h_tp;
    double *h_energy;
    int *h_iters, *h_count, *h_act, *h_list;
    size_t dev_bytes_jobs;
    double ms_fock, ms_rest, ms_energy, ms_diis, ms_pur, pur_steps, nsteps;
    // incremental Fock builds for the jobs added while on (gtf_batch_set_incremental)
    int incr, incr_period;
    double incr_tau;
    std::vector<int> h_full;
    cudaEvent_t e0, e1, e2, e3, e4;
};

#define CKH(call)                                                                          \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            fprintf(stderr, "gtfock_b200 batch %s:%d %s\n", __FILE__, __LINE__, cudaGetErrorString(e_)); \
            return GTF_ERR_CUDA;                                                           \
        }                                                                                  \
    } while (0)

static const int NSETS = 10;

// device bytes of one job's batch buffers (beyond its Fock engine)
static size_t job_buffer_bytes(int n) { return sizeof(double) * (size_t)n * n * (5 + 2 * BJ_MAX_DIIS); }

extern "C" size_t gtf_batch_job_bytes(int nbf) { return job_buffer_bytes(nbf); }

// The job's buffers are on the batch's stream `st` (devmem.cu's pool); the
// caller has synchronized `st` or queued nothing on it that uses them.
static void job_free(BJob &j, cudaStream_t st)
{
    gtf_dfree(j.mem, st);
    gtf_dfree(j.fcopy, st);
    if (j.pd) gtf_purif_destroy(j.pd);
    if (j.pf) {
        PFock_destroyOvlMat(j.pf);
        PFock_destroyCoreHMat(j.pf);
        PFock_destroy(j.pf);
    }
    if (j.basis) CInt_destroyBasisSet(j.basis);
    j = BJob();
}

extern "C" void gtf_batch_destroy(gtf_batch_t *b)
{
    if (!b) return;
    cudaStreamSynchronize(b->st);
    if (b->fock_exec) cudaGraphExecDestroy(b->fock_exec);
    if (b->fb) gtf_fock_batch_destroy(b->fb);
    for (auto &j : b->jobs)
        if (j.used) job_free(j, b->st);
    void *dp[] = {b->d_jobs, b->d_gd, b->d_tp, b->d_energy, b->d_dots, b->d_diis, b->d_scal, b->d_active,
                  b->d_iters, b->d_count, b->d_list};
    for (void *p : dp)
        if (p) cudaFree(p);
    void *hp[] = {b->h_jobs, b->h_gd, b->h_tp, b->h_energy, b->h_iters, b->h_count, b->h_act, b->h_list};
    for (void *p : hp)
        if (p) cudaFreeHost(p);
    cudaEventDestroy(b->e0);
    cudaEventDestroy(b->e1);
    cudaEventDestroy(b->e2);
    cudaEventDestroy(b->e3);
    cudaEventDestroy(b->e4);
    cudaStreamDestroy(b->st);
    delete b;
}

extern "C" gtf_batch_t *gtf_batch_create(int capacity)
{
    if (capacity <= 0) return nullptr;
    gtf_batch *b = new gtf_batch();
    b->capacity = capacity;
    b->jobs.resize(capacity);
    b->fb = nullptr;
    b->dirty = 1;
    b->gshape = 0;
    b->ms_fock = b->ms_rest = b->ms_energy = b->ms_diis = b->ms_pur = b->pur_steps = b->nsteps = 0.0;
    bool ok = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && cudaEventCreate(&b->e0) == cudaSuccess && cudaEventCreate(&b->e1) == cudaSuccess &&
         cudaEventCreate(&b->e2) == cudaSuccess && cudaEventCreate(&b->e3) == cudaSuccess &&
         cudaEventCreate(&b->e4) == cudaSuccess;
    const size_t C = capacity;
    ok = ok && cudaMalloc(&b->d_jobs, sizeof(JobDev) * C) == cudaSuccess;
    ok = ok && cudaMalloc(&b->d_gd, sizeof(GemmDesc) * C * NSETS) == cudaSuccess;
    ok = ok && cudaMalloc(&b->d_tp, sizeof(int) * (C + 1) * NSETS) == cudaSuccess;
    ok = ok && cudaMalloc(&b->d_energy, sizeof(double) * C * BJ_EBLOCKS) == cudaSuccess;
    ok = ok && cudaMalloc(&b->d_dots, sizeof(double) * C * BJ_MAX_DIIS) == cudaSuccess;
    ok = ok && cudaMalloc(&b->d_diis, sizeof(DiisState) * C) == cudaSuccess;
    ok = ok && cudaMalloc(&b->d_scal, sizeof(double) * C * 8) == cudaSuccess;
    ok = ok && cudaMalloc(&b->d_active, sizeof(int) * C) == cudaSuccess;
    ok = ok && cudaMalloc(&b->d_iters, sizeof(int) * C) == cudaSuccess;
    ok = ok && cudaMalloc(&b->d_count, sizeof(int)) == cudaSuccess;
    ok = ok && cudaMalloc(&b->d_list, sizeof(int) * C) == cudaSuccess;
    ok = ok && cudaMallocHost(&b->h_act, sizeof(int) * C) == cudaSuccess;
    ok = ok && cudaMallocHost(&b->h_list, sizeof(int) * C) == cudaSuccess;
    ok = ok && cudaMallocHost(&b->h_jobs, sizeof(JobDev) * C) == cudaSuccess;
    ok = ok && cudaMallocHost(&b->h_gd, sizeof(GemmDesc) * C * NSETS) == cudaSuccess;
    ok = ok && cudaMallocHost(&b->h_tp, sizeof(int) * (C + 1) * NSETS) == cudaSuccess;
    ok = ok && cudaMallocHost(&b->h_energy, sizeof(double) * C * BJ_EBLOCKS) == cudaSuccess;
    ok = ok && cudaMallocHost(&b->h_iters, sizeof(int) * C) == cudaSuccess;
    ok = ok && cudaMallocHost(&b->h_count, sizeof(int)) == cudaSuccess;
    if (!ok) {
        fprintf(stderr, "gtfock_b200: batch allocation failed\n");
        gtf_batch_destroy(b);
        return nullptr;
    }
    return b;
}

// A job set up but not yet in a batch (gtf_batch_prepare / gtf_batch_attach).
struct gtf_batch_job {
    BJob j;
    int prec_mode;
};

// The part of a job's set-up that touches no batch: basis, engine (screening,
// pair data, task lists, precision, incremental builds), S, H_core and X, all
// on the engine's own stream, which is synchronized at the end.  Returns 0 or
// gtf_batch_add's error codes -3 .. -5.
static int job_prepare(BJob &j, const char *bsfile, const char *xyzfile, double tolscr, int prec_mode,
                       double fp32_cutoff, int incr, double incr_tau, int incr_period)
{
    j = BJob();
    if (CInt_createBasisSet(&j.basis) != CINT_STATUS_SUCCESS ||
        CInt_loadBasisSet(j.basis, (char *)bsfile, (char *)xyzfile) != CINT_STATUS_SUCCESS) {
        if (j.basis) CInt_destroyBasisSet(j.basis);
        j = BJob();
        return -3;
    }
    j.n = CInt_getNumFuncs(j.basis);
    j.nocc = CInt_getNumOccOrb(j.basis);
    j.enuc = CInt_getNucEnergy(j.basis);
    if (PFock_create(j.basis, 1, 1, 4, tolscr, 1, 1, &j.pf) != PFOCK_STATUS_SUCCESS) {
        j.pf = nullptr;
        job_free(j, nullptr);
        return -4;
    }
    j.used = 1;
    j.eng = gtf_pfock_device(j.pf);
    if ((prec_mode != 0 && gtf_pfock_set_precision(j.pf, prec_mode, fp32_cutoff) != PFOCK_STATUS_SUCCESS) ||
        PFock_createOvlMat(j.pf, j.basis) != PFOCK_STATUS_SUCCESS ||
        PFock_createCoreHMat(j.pf, j.basis) != PFOCK_STATUS_SUCCESS ||
        (incr && gtf_pfock_set_incremental(j.pf, 1, incr_tau, incr_period) != PFOCK_STATUS_SUCCESS) ||
        cudaStreamSynchronize((cudaStream_t)gtf_fock_stream(j.eng)) != cudaSuccess) {
        job_free(j, nullptr);
        return -5;
    }
    return 0;
}

// The job's batch buffers (on the batch's stream), its device descriptor and
// initial density, in `slot`; -6 / -7 on failure (the job is released).
static int job_attach(gtf_batch *b, int slot, BJob &&src, int prec_mode, int max_iters, double etol)
{
    BJob &j = b->jobs[slot];
    j = std::move(src);
    const size_t nn = (size_t)j.n * j.n;
    j.bytes = job_buffer_bytes(j.n);
    JobDev &d = j.dv;
    d.S = gtf_fock_onee_dev(j.eng, 0);
    d.X = gtf_fock_onee_dev(j.eng, 1);
    if (j.n > BJ_BIG) {
        // mixed precision: split-BF16 tensor-core purification products too
        if (gtf_purif_create(j.n, j.nocc, b->st, &j.pd) != GTF_OK ||
            gtf_purif_set_sx_dev(j.pd, d.S, d.X) != GTF_OK ||
            (prec_mode == 1 && gtf_purif_set_mode(j.pd, 1) != GTF_OK)) {
            j.pd = nullptr;
            job_free(j, b->st);
            return -6;
        }
    } else if (gtf_dmalloc((void **)&j.mem, j.bytes, b->st) != cudaSuccess) {
        j.mem = nullptr;
        job_free(j, b->st);
        return -6;
    }
    d.D = const_cast<double *>(gtf_fock_mat_dev(j.eng, 0, 0));
    d.F = const_cast<double *>(gtf_fock_mat_dev(j.eng, 1, 0));
    d.Fe = d.F;
    if (b->incr) {
        if (gtf_dmalloc((void **)&j.fcopy, sizeof(double) * nn, b->st) != cudaSuccess) {
            j.fcopy = nullptr;
            job_free(j, b->st);
            return -6;
        }
        j.bytes += sizeof(double) * nn;
        d.F = j.fcopy;
    }
    j.inc_since = 0;
    d.H = gtf_fock_onee_dev(j.eng, 2);
    if (j.mem) {
        d.P = j.mem;
        d.P2 = d.P + nn;
        d.P3 = d.P2 + nn;
        d.W = d.P3 + nn;
        d.W2 = d.W + nn;
        d.vecs = d.W2 + nn;
        d.Fvecs = d.vecs + nn * BJ_MAX_DIIS;
    }
    d.n = j.n;
    d.nocc = j.nocc;
    d.diis = 0;
    d.ds = b->d_diis + slot;
    k_j_diis_reset<<<1, 128, 0, b->st>>>(d.ds);
    // initial guess (pscf/scf.c:34-76) into the engine's density buffer; the
    // engine's set-up is complete (job_prepare), and the job's buffers on the
    // batch's stream are before the batch's launches use them; the other
    // lanes' work is not waited for
    std::vector<double> D0(nn);
    gtf_initial_density(j.basis, D0.data(), j.n);
    if (cudaMemcpyAsync(d.D, D0.data(), sizeof(double) * nn, cudaMemcpyHostToDevice, b->st) != cudaSuccess ||
        cudaStreamSynchronize(b->st) != cudaSuccess) {
        job_free(j, b->st);
        return -7;
    }
    j.iter = 0;
    j.max_iters = max_iters;
    j.etol = etol;
    j.e_prev = 0.0;
    j.done = 0;
    j.failed = 0;
    b->dirty = 1;
    return slot;
}

static int free_slot(const gtf_batch *b)
{
    for (int s = 0; s < b->capacity; s++)
        if (!b->jobs[s].used) return s;
    return -1;
}

// Set-up of one SCF job (pscf/scf.c:298-314, init_oedmat pscf/scf.c:131-185)
// in a free slot; returns the slot or a negative error.
extern "C" int gtf_batch_add(gtf_batch_t *b, const char *bsfile, const char *xyzfile, double tolscr, int prec_mode,
                             double fp32_cutoff, int max_iters, double etol)
{
    if (!b || !bsfile || !xyzfile || max_iters <= 0 || !(etol >= 0.0)) return -1;
    const int slot = free_slot(b);
    if (slot < 0) return -2;
    BJob j;
    const int r = job_prepare(j, bsfile, xyzfile, tolscr, prec_mode, fp32_cutoff, b->incr, b->incr_tau,
                              b->incr_period);
    if (r) return r;
    return job_attach(b, slot, std::move(j), prec_mode, max_iters, etol);
}

// gtf_batch_add in two parts, so that a server can set a job up while the
// batch it will join is stepping on another thread: gtf_batch_prepare touches
// no state of the batch but its (fixed) incremental setting; gtf_batch_attach
// takes a free slot and must not overlap a step of the batch.
extern "C" int gtf_batch_prepare(gtf_batch_t *b, const char *bsfile, const char *xyzfile, double tolscr,
                                 int prec_mode, double fp32_cutoff, gtf_batch_job_t **out)
{
    if (!out) return -1;
    *out = nullptr;
    if (!b || !bsfile || !xyzfile) return -1;
    gtf_batch_job *job = new gtf_batch_job();
    job->prec_mode = prec_mode;
    const int r = job_prepare(job->j, bsfile, xyzfile, tolscr, prec_mode, fp32_cutoff, b->incr, b->incr_tau,
                              b->incr_period);
    if (r) {
        delete job;
        return r;
    }
    *out = job;
    return 0;
}

extern "C" int gtf_batch_attach(gtf_batch_t *b, gtf_batch_job_t *job, int max_iters, double etol)
{
    if (!b || !job || max_iters <= 0 || !(etol >= 0.0)) {
        gtf_batch_job_free(job);
        return -1;
    }
    const int slot = free_slot(b);
    if (slot < 0) {
        gtf_batch_job_free(job);
        return -2;
    }
    const int r = job_attach(b, slot, std::move(job->j), job->prec_mode, max_iters, etol);
    delete job;
    return r;
}

extern "C" void gtf_batch_job_free(gtf_batch_job_t *job)
{
    if (!job) return;
    job_free(job->j, nullptr);
    delete job;
}

extern "C" int gtf_batch_remove(gtf_batch_t *b, int slot)
{
    if (!b || slot < 0 || slot >= b->capacity || !b->jobs[slot].used) return -1;
    cudaStreamSynchronize(b->st);
    job_free(b->jobs[slot], b->st);
    b->dirty = 1;
    return 0;
}

extern "C" int gtf_batch_result(gtf_batch_t *b, int slot, double *energies, int *niters, int *done)
{
    if (!b || slot < 0 || slot >= b->capacity || !b->jobs[slot].used) return -1;
    const BJob &j = b->jobs[slot];
    if (energies)
        for (size_t k = 0; k < j.energies.size(); k++) energies[k] = j.energies[k];
    if (niters) *niters = (int)j.energies.size();
    if (done) *done = j.done;
    return j.failed ? -2 : 0;
}

extern "C" int gtf_batch_density(gtf_batch_t *b, int slot, double *D)
{
    if (!b || slot < 0 || slot >= b->capacity || !b->jobs[slot].used || !D) return -1;
    CKH(cudaStreamSynchronize(b->st));
    const BJob &j = b->jobs[slot];
    CKH(cudaMemcpy(D, j.dv.D, sizeof(double) * j.n * j.n, cudaMemcpyDeviceToHost));
    return 0;
}

// one call set of batched GEMMs: descriptors of set `s` for `m` jobs
static int run_gemm(gtf_batch *b, int s, int m, bool tb, const int *active, int *launches)
{
    if (m == 0) return GTF_OK;
    const int ntiles = b->h_tp[s * (b->capacity + 1) + m];
    if (ntiles == 0) return GTF_OK;
    const GemmDesc *gd = b->d_gd + (size_t)s * b->capacity;
    const int *tp = b->d_tp + (size_t)s * (b->capacity + 1);
    if (tb) launch_bgemm_shape<true>(b->gshape, ntiles, b->st, gd, tp, m, active);
    else launch_bgemm_shape<false>(b->gshape, ntiles, b->st, gd, tp, m, active);
    CKH(cudaGetLastError());
    (*launches)++;
    return GTF_OK;
}

static void set_gemm(gtf_batch *b, int s, int k, const double *A, const double *B, double *C, int n, int job)
{
    GemmDesc &g = b->h_gd[(size_t)s * b->capacity + k];
    g.A = A;
    g.B = B;
    g.C = C;
    g.n = n;
    g.job = job;
    const BGemmShape &sh = BG_SHAPES[b->gshape];
    const int ntr = (n + sh.bm - 1) / sh.bm, ntc = (n + sh.bn - 1) / sh.bn;
    int *tp = b->h_tp + (size_t)s * (b->capacity + 1);
    if (k == 0) tp[0] = 0;
    tp[k + 1] = tp[k] + ntr * ntc;
}

// One SCF iteration of every running job.  Returns the number of jobs still
// running afterwards, or a negative error.
// sum of n^3 over the jobs whose dense products run batched (the size key of
// the tile-shape tuning)
static double batch_gemm_work(const gtf_batch *b, const std::vector<int> &run)
{
    double w = 0.0;
    for (int s : run)
        if (!b->jobs[s].pd) w += (double)b->jobs[s].n * b->jobs[s].n * b->jobs[s].n;
    return w;
}

// (Re)creates the batched Fock build for the jobs in `run`, picks the tile
// shape of the dense products from the tuning table, and captures the build
// as a CUDA graph for replay while the membership stays the same.
static int rebuild_fock_batch(gtf_batch *b, const std::vector<int> &run)
{
    if (b->fb) gtf_fock_batch_destroy(b->fb);
    b->fb = nullptr;
    std::vector<gtf_fock_dev_t *> eng;
    for (int s : run) eng.push_back(b->jobs[s].eng);
    if (gtf_fock_batch_create(eng.data(), (int)eng.size(), b->st, &b->fb) != GTF_OK) {
        fprintf(stderr, "gtfock_b200: batched Fock set-up failed: %s\n", gtf_last_error());
        return -2;
    }
    b->fb_members = run;
    b->dirty = 0;
    // capture the build (one launch per class pair, part and slice, plus
    // the transforms) for replay while the membership stays the same
    if (b->fock_exec) cudaGraphExecDestroy(b->fock_exec);
    b->fock_exec = nullptr;
    b->fock_launches = 0;
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        const int nl = gtf_fock_batch_compute(b->fb);
        const cudaError_t ce = cudaStreamEndCapture(b->st, &graph);
        if (nl >= 0 && ce == cudaSuccess && graph &&
            cudaGraphInstantiate(&b->fock_exec, graph, 0) == cudaSuccess) {
            b->fock_launches = nl;
            gtf_note_launches(-nl);   // counted when replayed, not when captured
        } else {
            b->fock_exec = nullptr;
        }
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
    }
    // tile shape of the dense products: tuned for this size, else the default
    b->gshape = 0;
    int shape = 0;
    if (gtf_tune_get(2, -1, -1, 0, batch_gemm_work(b, run), &shape, nullptr) && shape >= 0 && shape < BG_NSHAPES)
        b->gshape = shape;
    return 0;
}

extern "C" int gtf_batch_step(gtf_batch_t *b)
{
    if (!b) return -1;
    std::vector<int> run;
    for (int s = 0; s < b->capacity; s++)
        if (b->jobs[s].used && !b->jobs[s].done) run.push_back(s);
    if (run.empty()) return 0;
    int launches = 0;
    // ---- Fock build of every running job ----
    if (b->dirty || run != b->fb_members) {
        const int r = rebuild_fock_batch(b, run);
        if (r) return r;
    }
    if (b->incr) {
        // full or incremental build, per member, before the (captured) build reads the flags
        b->h_full.resize(run.size());
        for (size_t k = 0; k < run.size(); k++) {
            BJob &j = b->jobs[run[k]];
            const int full = (j.inc_since == 0 || j.inc_since >= b->incr_period) ? 1 : 0;
            b->h_full[k] = full;
            j.inc_since = full ? 1 : j.inc_since + 1;
        }
        if (gtf_fock_batch_set_full(b->fb, b->h_full.data()) != GTF_OK) {
            fprintf(stderr, "gtfock_b200: %s\n", gtf_last_error());
            return -3;
        }
    }
    CKH(cudaEventRecord(b->e0, b->st));
    if (b->fock_exec) {
        CKH(cudaGraphLaunch(b->fock_exec, b->st));
        gtf_note_launches(b->fock_launches);
    } else if (gtf_fock_batch_compute(b->fb) < 0) {
        fprintf(stderr, "gtfock_b200: batched Fock build failed: %s\n", gtf_last_error());
        return -3;
    }
    CKH(cudaEventRecord(b->e1, b->st));
    // ---- energies (pscf/scf.c:80-102, 339-375) ----
    const int M = (int)run.size();
    for (int k = 0; k < M; k++) {
        BJob &j = b->jobs[run[k]];
        j.dv.diis = 0;
        b->h_jobs[k] = j.dv;
    }
    CKH(cudaMemcpyAsync(b->d_jobs, b->h_jobs, sizeof(JobDev) * M, cudaMemcpyHostToDevice, b->st));
    k_j_energy<<<dim3(BJ_EBLOCKS, M), BJ_THREADS, 0, b->st>>>(b->d_jobs, b->d_energy);
    CKH(cudaGetLastError());
    launches++;
    CKH(cudaMemcpyAsync(b->h_energy, b->d_energy, sizeof(double) * M * BJ_EBLOCKS, cudaMemcpyDeviceToHost, b->st));
    CKH(cudaEventRecord(b->e3, b->st));
    CKH(cudaEventRecord(b->e4, b->st));
    CKH(cudaStreamSynchronize(b->st));
    // jobs that continue with DIIS + purification: batched (cont) or one by one (big)
    std::vector<int> cont, big;   // indices into run
    for (int k = 0; k < M; k++) {
        BJob &j = b->jobs[run[k]];
        double e = 0.0;
        for (int q = 0; q < BJ_EBLOCKS; q++) e += b->h_energy[k * BJ_EBLOCKS + q];
        j.energies.push_back(e + j.enuc);
        const int it = j.iter++;
        if ((it > 0 && fabs(e - j.e_prev) < j.etol) || j.iter >= j.max_iters) {
            j.done = 1;
            continue;
        }
        j.e_prev = e;
        if (j.pd) big.push_back(k);
        else cont.push_back(k);
    }
    const int C = (int)cont.size();
    if (C > 0) {
        // ---- DIIS (pscf/purif.c:491-641) ----
        // call sets: 0 W=F D^T, 1 W2=W S^T, 2 W=X cur^T, 3 cur=W X^T (DIIS jobs);
        //            4 W=X F^T, 5 target=W X^T (all); 6 P2=P P^T, 7 P3=P P2,
        //            8 W=X P^T, 9 D=W X^T (purification)
        int nd = 0;
        for (int q = 0; q < C; q++) {
            BJob &j = b->jobs[run[cont[q]]];
            JobDev &d = j.dv;
            const int it = j.iter - 1;   // this iteration's index
            // DIIS jobs: the error vector and X F X go through P2 and P3,
            // and the device bookkeeping stores them into the job's slot
            d.diis = it > 1;
            double *target = d.F;
            if (d.diis) {
                target = d.P3;
                set_gemm(b, 0, nd, d.F, d.D, d.W, j.n, -1);
                set_gemm(b, 1, nd, d.W, d.S, d.W2, j.n, -1);
                set_gemm(b, 2, nd, d.X, d.P2, d.W, j.n, -1);
                set_gemm(b, 3, nd, d.W, d.X, d.P2, j.n, -1);
                nd++;
            }
            set_gemm(b, 4, q, d.X, d.F, d.W, j.n, -1);
            set_gemm(b, 5, q, d.W, d.X, target, j.n, -1);
            set_gemm(b, 6, q, d.P, d.P, d.P2, j.n, q);
            set_gemm(b, 7, q, d.P, d.P2, d.P3, j.n, q);
            set_gemm(b, 8, q, d.X, d.P, d.W, j.n, -1);
            set_gemm(b, 9, q, d.W, d.X, d.D, j.n, -1);
            b->h_jobs[q] = d;
        }
        // DIIS-set descriptors come first in `cont` order; the slot, antisym,
        // dots, solve and combine kernels skip the jobs without DIIS
        const size_t C1 = b->capacity + 1;
        CKH(cudaMemcpyAsync(b->d_jobs, b->h_jobs, sizeof(JobDev) * C, cudaMemcpyHostToDevice, b->st));
        CKH(cudaMemcpyAsync(b->d_gd, b->h_gd, sizeof(GemmDesc) * b->capacity * NSETS, cudaMemcpyHostToDevice, b->st));
        CKH(cudaMemcpyAsync(b->d_tp, b->h_tp, sizeof(int) * C1 * NSETS, cudaMemcpyHostToDevice, b->st));
        int maxn = 0;
        for (int q = 0; q < C; q++) maxn = b->h_jobs[q].n > maxn ? b->h_jobs[q].n : maxn;
        const unsigned ge = (unsigned)(((size_t)maxn * maxn + 255) / 256 < 1024 ? ((size_t)maxn * maxn + 255) / 256 : 1024);
        if (nd > 0) {
            k_j_diis_slot<<<(C + 127) / 128, 128, 0, b->st>>>(b->d_jobs, C);
            CKH(cudaGetLastError());
            launches++;
            if (run_gemm(b, 0, nd, true, nullptr, &launches) || run_gemm(b, 1, nd, true, nullptr, &launches))
                return -4;
            k_j_antisym<<<dim3(ge, C), 256, 0, b->st>>>(b->d_jobs);
            CKH(cudaGetLastError());
            launches++;
            if (run_gemm(b, 2, nd, true, nullptr, &launches) || run_gemm(b, 3, nd, true, nullptr, &launches))
                return -4;
            k_j_dots<<<C, BJ_THREADS, 0, b->st>>>(b->d_jobs, b->d_dots);
            k_j_diis_solve<<<C, 32, 0, b->st>>>(b->d_jobs, b->d_dots);
            CKH(cudaGetLastError());
            launches += 2;
        }
        // F' = X F X^T (pscf/purif.c:620-636)
        if (run_gemm(b, 4, C, true, nullptr, &launches) || run_gemm(b, 5, C, true, nullptr, &launches)) return -4;
        if (nd > 0) {
            k_j_combine<<<dim3(ge, C), 256, 0, b->st>>>(b->d_jobs);
            CKH(cudaGetLastError());
            launches++;
        }
        // ---- canonical purification (pscf/purif.c:257-488) ----
        CKH(cudaEventRecord(b->e4, b->st));
        CKH(cudaMemsetAsync(b->d_iters, 0, sizeof(int) * C, b->st));
        k_j_pur_init<<<C, BJ_THREADS, 0, b->st>>>(b->d_jobs, b->d_scal, b->d_active);
        CKH(cudaGetLastError());
        launches++;
        // the launches cover the jobs still purifying: every BJ_PUR_CHECK steps
        // the active flags come back and the job list and the descriptors of
        // the two products are compacted to the jobs that remain
        int nact = C;
        for (int q = 0; q < C; q++) b->h_list[q] = q;
        CKH(cudaMemcpyAsync(b->d_list, b->h_list, sizeof(int) * C, cudaMemcpyHostToDevice, b->st));
        int step;
        for (step = 0; step < BJ_PUR_MAX; step++) {
            if (run_gemm(b, 6, nact, true, b->d_active, &launches) ||
                run_gemm(b, 7, nact, false, b->d_active, &launches))
                return -4;
            k_j_pur_step<<<nact, BJ_THREADS, 0, b->st>>>(b->d_jobs, b->d_list, b->d_scal, b->d_active, b->d_iters);
            CKH(cudaGetLastError());
            launches++;
            if ((step + 1) % BJ_PUR_CHECK == 0) {
                CKH(cudaMemcpyAsync(b->h_act, b->d_active, sizeof(int) * C, cudaMemcpyDeviceToHost, b->st));
                CKH(cudaStreamSynchronize(b->st));
                int m = 0;
                for (int q = 0; q < C; q++)
                    if (b->h_act[q]) {
                        const JobDev &d = b->h_jobs[q];
                        set_gemm(b, 6, m, d.P, d.P, d.P2, d.n, q);
                        set_gemm(b, 7, m, d.P, d.P2, d.P3, d.n, q);
                        b->h_list[m++] = q;
                    }
                if (m == 0) break;
                if (m < nact) {
                    nact = m;
                    const size_t C1 = b->capacity + 1;
                    CKH(cudaMemcpyAsync(b->d_gd + 6 * (size_t)b->capacity, b->h_gd + 6 * (size_t)b->capacity,
                                        sizeof(GemmDesc) * 2 * b->capacity, cudaMemcpyHostToDevice, b->st));
                    CKH(cudaMemcpyAsync(b->d_tp + 6 * C1, b->h_tp + 6 * C1, sizeof(int) * 2 * C1,
                                        cudaMemcpyHostToDevice, b->st));
                    CKH(cudaMemcpyAsync(b->d_list, b->h_list, sizeof(int) * nact, cudaMemcpyHostToDevice, b->st));
                }
            }
        }
        b->pur_steps += step + 1;
        // D_AO = X P X^T (pscf/purif.c:469-476), into the engine's density
        if (run_gemm(b, 8, C, true, nullptr, &launches) || run_gemm(b, 9, C, true, nullptr, &launches)) return -4;
        CKH(cudaMemcpyAsync(b->h_iters, b->d_iters, sizeof(int) * C, cudaMemcpyDeviceToHost, b->st));
    }
    // jobs above BJ_BIG functions: the single-job DIIS and purification
    for (int k : big) {
        BJob &j = b->jobs[run[k]];
        int it = 0;
        if (gtf_diis_step_dev(j.pd, j.dv.D, j.dv.F, j.iter - 1) != GTF_OK ||
            gtf_purif_run_dev(j.pd, j.dv.F, j.dv.D, &it) != GTF_OK) {
            j.failed = 1;
            j.done = 1;
        }
        j.pur_iters = it;
        j.pur_total += it;
    }
    CKH(cudaEventRecord(b->e2, b->st));
    CKH(cudaStreamSynchronize(b->st));
    for (int q = 0; q < C; q++) {
        BJob &j = b->jobs[run[cont[q]]];
        j.pur_iters = b->h_iters[q];
        j.pur_total += j.pur_iters;
    }
    float ms1 = 0.0f, ms2 = 0.0f, ms3 = 0.0f, ms4 = 0.0f;
    cudaEventElapsedTime(&ms1, b->e0, b->e1);
    cudaEventElapsedTime(&ms2, b->e1, b->e2);
    cudaEventElapsedTime(&ms3, b->e1, b->e3);
    cudaEventElapsedTime(&ms4, b->e4, b->e2);
    b->ms_fock += ms1;
    b->ms_rest += ms2;
    b->ms_energy += ms3;
    b->ms_pur += ms4;
    b->ms_diis += ms2 - ms3 - ms4;
    b->nsteps += 1;
    gtf_note_launches(launches);
    int left = 0;
    for (int s = 0; s < b->capacity; s++)
        if (b->jobs[s].used && !b->jobs[s].done) left++;
    return left;
}

// Tunes the batch for its current jobs: the launch shapes of the batched
// Fock build, then the tile shape of the dense products, timed on W = X X^T
// of every job whose products run batched (W is scratch between steps).  The
// next step re-captures the Fock graph with the tuned shapes.
extern "C" int gtf_batch_autotune(gtf_batch_t *b, int reps)
{
    if (!b) return GTF_ERR_INVALID;
    if (reps < 1) reps = 1;
    std::vector<int> run;
    for (int s = 0; s < b->capacity; s++)
        if (b->jobs[s].used && !b->jobs[s].done) run.push_back(s);
    if (run.empty()) return GTF_OK;
    if ((b->dirty || run != b->fb_members) && rebuild_fock_batch(b, run) != 0) return GTF_ERR_CUDA;
    const int rc = gtf_fock_batch_autotune(b->fb, reps);
    if (rc != GTF_OK) return rc;
    std::vector<int> small;
    for (int s : run)
        if (!b->jobs[s].pd) small.push_back(s);
    if (!small.empty()) {
        const int m = (int)small.size();
        const size_t C1 = b->capacity + 1;
        double best = -1.0;
        int bs = 0;
        for (int shape = 0; shape < BG_NSHAPES; shape++) {
            b->gshape = shape;
            for (int q = 0; q < m; q++) {
                const BJob &j = b->jobs[small[q]];
                set_gemm(b, 6, q, j.dv.X, j.dv.X, j.dv.W, j.n, -1);
            }
            CKH(cudaMemcpyAsync(b->d_gd + 6 * (size_t)b->capacity, b->h_gd + 6 * (size_t)b->capacity,
                                sizeof(GemmDesc) * m, cudaMemcpyHostToDevice, b->st));
            CKH(cudaMemcpyAsync(b->d_tp + 6 * C1, b->h_tp + 6 * C1, sizeof(int) * (m + 1), cudaMemcpyHostToDevice,
                                b->st));
            double tmin = 1e30;
            int launches = 0;
            for (int r = 0; r < reps + 1; r++) {   // the first run warms up
                CKH(cudaEventRecord(b->e0, b->st));
                if (run_gemm(b, 6, m, true, nullptr, &launches)) return GTF_ERR_CUDA;
                CKH(cudaEventRecord(b->e1, b->st));
                CKH(cudaEventSynchronize(b->e1));
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, b->e0, b->e1);
                if (r > 0 && ms < tmin) tmin = ms;
            }
            gtf_note_launches(launches);
            if (best < 0.0 || tmin < best) {
                best = tmin;
                bs = shape;
            }
        }
        gtf_tune_put(2, -1, -1, 0, batch_gemm_work(b, run), bs, 0, best);
        b->gshape = bs;
    }
    b->dirty = 1;
    return GTF_OK;
}

// Incremental Fock builds (gtf_pfock_set_incremental) for the jobs added from
// now on (on = 0: plain builds).  A batch must not mix the two: set it before
// the first job is added.
extern "C" int gtf_batch_set_incremental(gtf_batch_t *b, int on, double tau, int period)
{
    if (!b || (on && period < 1)) return -1;
    for (auto &j : b->jobs)
        if (j.used) return -2;
    b->incr = on ? 1 : 0;
    b->incr_tau = tau;
    b->incr_period = period;
    return 0;
}

extern "C" int gtf_batch_run(gtf_batch_t *b)
{
    int r;
    while ((r = gtf_batch_step(b)) > 0) {
    }
    return r;
}

extern "C" int gtf_batch_info(gtf_batch_t *b, int *nrunning, int *nused, double *ms_fock, double *ms_rest,
                              size_t *job_bytes)
{
    if (!b) return -1;
    int r = 0, u = 0;
    size_t by = 0;
    for (auto &j : b->jobs)
        if (j.used) {
            u++;
            if (!j.done) r++;
            by += j.bytes + gtf_fock_device_bytes(j.eng);
        }
    if (nrunning) *nrunning = r;
    if (nused) *nused = u;
    if (ms_fock) *ms_fock = b->ms_fock;
    if (ms_rest) *ms_rest = b->ms_rest;
    if (job_bytes) *job_bytes = by;
    return 0;
}

// per-job statistics: [0] basis functions, [1] SCF iterations run, [2]
// purification iterations of the last step, [3] over all steps; returns the
// count written (0 for an empty slot)
extern "C" int gtf_batch_job_stats(gtf_batch_t *b, int slot, double *out, int n)
{
    if (!b || !out || slot < 0 || slot >= b->capacity || !b->jobs[slot].used) return 0;
    const BJob &j = b->jobs[slot];
    const double v[4] = {(double)j.n, (double)j.iter, (double)j.pur_iters, (double)j.pur_total};
    const int m = n < 4 ? n : 4;
    for (int k = 0; k < m; k++) out[k] = v[k];
    return m;
}

// device bytes held by the job in `slot` (batch buffers and Fock engine); 0 if empty
extern "C" size_t gtf_batch_job_device_bytes(gtf_batch_t *b, int slot)
{
    if (!b || slot < 0 || slot >= b->capacity || !b->jobs[slot].used) return 0;
    const BJob &j = b->jobs[slot];
    return j.bytes + gtf_fock_device_bytes(j.eng);
}

// accumulated statistics: [0] ms of Fock builds, [1] energies, [2] DIIS,
// [3] purification (incl. jobs on the one-job path), [4] purification steps
// of the batched jobs, [5] batch steps; returns the number written
extern "C" int gtf_batch_stats(gtf_batch_t *b, double *out, int n)
{
    if (!b || !out) return -1;
    const double v[6] = {b->ms_fock, b->ms_energy, b->ms_diis, b->ms_pur, b->pur_steps, b->nsteps};
    const int m = n < 6 ? n : 6;
    for (int k = 0; k < m; k++) out[k] = v[k];
    return m;
}
