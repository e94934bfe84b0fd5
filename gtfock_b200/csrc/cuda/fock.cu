// fock.cu -- the PFock engine on one B200.
//
// Setup (PFock_create, pfock/pfock.c:801-997):
//   * device Schwarz screening: one thread per shell pair evaluates the
//     diagonal quartet (MN|MN) by Rys quadrature and keeps max |(mn|mn)|
//     (pfock/screening.c:59-90); the global max and eta = tol^2/max follow
//     pfock/screening.c:100,111;
//   * the reference's CSR pair list (parity rule and signed values,
//     pfock/screening.c:118-175) is built on the device by scan + scatter;
//   * the same pairs, re-oriented so that L(a) >= L(b), are radix-sorted by
//     angular class and by bound (descending) into the device pair list;
//   * per class pair (bra class X >= ket class Y) and per bra pair, the
//     number of ket pairs passing the quartet Schwarz test
//     |v1 v2| >= tol^2 (pfock/fock_task.c:192) is a prefix of the sorted ket
//     class (binary search); X == Y keeps ket <= bra so every unique quartet
//     (pfock/fock_task.c:169-175) is visited once; 32 kets form one unit.
// Build (PFock_computeFock, pfock/pfock.c:1274-1729):
//   * D (spherical) -> Cartesian, Fj/Fk zeroed;
//   * one persistent kernel per class pair: warps claim units from an
//     atomic counter, each lane evaluates one quartet and the warp digests
//     into Fj (Coulomb terms) and Fk (exchange terms) with FP64 atomics;
//   * symmetrise (GA_Symmetrize) and transform back: F = J + K.
#include <cub/cub.cuh>
#include <cuda_runtime.h>
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <atomic>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "devmem.cuh"
#include "gtf_cuda.h"
#include "gtf_dev.cuh"
// the Fock kernels live in fock_kernel.cuh, instantiated across several
// translation units (fock_cls_*.cu) so that they compile in parallel
#include "fock_kernel.cuh"


#define NCLS 6
#define NCLSPAIR 21

static thread_local char g_errbuf[512];

extern "C" const char *gtf_last_error(void) { return g_errbuf; }
extern "C" void gtf_note_launches(int n);

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            snprintf(g_errbuf, sizeof(g_errbuf), "%s:%d %s: %s", __FILE__, __LINE__, #call, \
                     cudaGetErrorString(e_));                                             \
            return GTF_ERR_CUDA;                                                          \
        }                                                                                 \
    } while (0)

// pair class of (La, Lb), La >= Lb: ss=0 ps=1 pp=2 ds=3 dp=4 dd=5
__host__ __device__ inline int pair_class(int la, int lb)
{
    if (la < lb) { int t = la; la = lb; lb = t; }
    return la * (la + 1) / 2 + lb;
}

static const int k_cls_la[NCLS] = {0, 1, 1, 2, 2, 2};
static const int k_cls_lb[NCLS] = {0, 0, 1, 0, 1, 2};

struct UnitTask;

static inline double __longlong_as_double_host(unsigned long long b)
{
    double d;
    memcpy(&d, &b, sizeof(d));
    return d;
}

// Device state of an engine for incremental builds: the largest |element| of
// the density change of the current build (a non-negative double kept as its
// bit pattern, so atomicMax orders it), the quartet thresholds derived from
// it, whether the build adds to the previous result (acc) and the quartet
// counts of the build's task lists (FP64, FP32).
struct DynState {
    unsigned long long dmax_bits;
    double tol2, cut2;
    int acc, pad;
    unsigned long long nq64, nq32;
};

struct ClassPairTask {
    int X, Y;
    int bra_start, nbra;
    int ket_start, nketcls;
    int seg[GTF_NBKT + 1];  // ket segments (primitive-count buckets), relative to ket_start
    long long nunits, nunits32;  // units of the FP64 and the FP32 launch
    long long nunits_bound;      // bound on either launch's units under any thresholds >= tol2
    double flops, nprimq;        // Rys-model FLOPs and primitive quartets (before primitive screening)
    double nquart, nquart32;     // quartets in all, of which evaluated in FP32
    int *d_nket;                 // [nbra][GTF_NBKT] kets per (bra, segment)
    int *d_n64;                  // [nbra][GTF_NBKT] of which FP64 (a prefix)
    int *d_cum64, *d_cum32;      // [nbra][GTF_CUM] per-bra segment prefixes of the two launches
    long long *d_unit_prefix;    // [nbra + 1], FP64 launch
    long long *d_unit_prefix32;  // [nbra + 1], FP32 launch
};

struct gtf_fock_dev {
    int dev;
    int nsm;
    cudaStream_t stream;
    // basis
    int natoms, nshells, nbf, nbf_cart, nprims, pure, max_numdmat;
    std::vector<int> h_sh_L, h_f_start, h_fc_start;
    int *d_sh_L, *d_sh_nprim, *d_sh_pstart, *d_f_start, *d_fc_start, *d_sph2shell, *d_cart2shell, *d_Z;
    double *d_sh_xyz, *d_alpha, *d_coef, *d_atom_xyz;
    // screening
    double tolscr, tolscr2, maxvalue;
    int nnz;
    double *d_sq;
    int *d_shellptr, *d_shellid, *d_shellrid;
    double *d_shellvalue;
    // device pair list
    int npairs;
    int cls_start[NCLS + 1];
    PairRec *d_pairs;
    double *d_pair_v;
    int nprimpairs;
    double *d_pp;   // 6 * nprimpairs: records {p, K, Px, Py, Pz, 1/(2p)} (PPRec)
    float *d_pp32;  // 8 * nprimpairs: FP32 records {p, K, PA, 1/(2p), 0, 0} (PPRec32)
    ClassPairTask tasks[NCLSPAIR];
    unsigned long long *d_counters;
    double usq, uitl, eri_flops;
    // matrices
    double *d_D;     // [max_numdmat][nbf*nbf]
    double *d_Dc;    // cart scratch
    double *d_Fj, *d_Fk;  // cart accumulators
    double *d_F, *d_J, *d_K;  // [max_numdmat][nbf*nbf] results
    double *d_S, *d_X, *d_H;
    double *d_host_stage;     // pinned staging for strided copies
    size_t host_stage_bytes;
    // timing
    cudaEvent_t ev0, ev1, ev2, ev3;
    cudaEvent_t ev_cls[NCLSPAIR + 1];
    double ms_total, ms_eri, ms_other;
    double ms_cls[NCLSPAIR];
    int prec;
    double fp32_cutoff;
    size_t dev_bytes;
    // non-symmetric densities (PFock_create with symm = 0): GTF_NOSYMM_*
    int nosymm;
    double *d_Ds, *d_Da, *d_Dca, *d_Fka;
    // the reference's own symm = 0 output: sign-adjusted antisymmetric part
    // (spherical, Cartesian), its Coulomb accumulator and a scratch exchange
    // accumulator
    double *d_Dta, *d_Dcta, *d_Fja, *d_Fscr;
    // sharded build: this engine computes shard `shard` of `nshards` (0: all);
    // its units of every (class pair, part): [shard_lo, shard_hi), split by
    // the work model (see shard_bounds)
    int shard, nshards;
    long long shard_lo[NCLSPAIR][2], shard_hi[NCLSPAIR][2];
    double shard_work;           // model FLOPs of this shard's units
    std::vector<int> h_pair_n;   // primitive pairs per shell pair (pair list order)
    bool work_model = false;     // tasks[].flops / nprimq and eri_flops evaluated
    // task lists on the device (UnitTask per class pair with work): static
    // thresholds, and the same tasks reading the thresholds of d_dyn
    std::vector<struct UnitTask> h_ut;
    struct UnitTask *d_ut_static, *d_ut_dyn;
    long long ut_nidx, ut_nbras;
    // incremental builds (gtf_fock_set_incremental): F_k = F_k-1 + G[D_k -
    // D_k-1], quartets screened against tau / max|D_k - D_k-1|
    int incr, incr_period, incr_since;
    double incr_tau;
    double *d_Dprev, *d_Dd;
    DynState *d_dyn;
    unsigned long long *d_unit_tot;  // [NCLSPAIR][3] quartets, FP32 quartets, unit bound (build_units)
    // the task-list arrays hold an incremental build's lists (rebuilt from
    // the static thresholds before a plain build uses them)
    int lists_dyn;
};

// ---------------------------------------------------------------------------
// Device allocations of an engine's set-up.  Every one goes through
// dev_malloc, which a test can make fail: after gtf_debug_fail_alloc(n) the
// n-th allocation from then on fails as an out-of-memory cudaMalloc would
// (and the counter disarms), so each error path of PFock_create can be shown
// to release what it had allocated.
// ---------------------------------------------------------------------------
static std::atomic<int> g_fail_alloc{0};
static std::atomic<long long> g_live_allocs{0};   // dev_malloc'd and not yet dev_free'd

extern "C" void gtf_debug_fail_alloc(int n) { g_fail_alloc.store(n > 0 ? n : 0); }
extern "C" long long gtf_debug_live_allocs(void) { return g_live_allocs.load(); }

// Buffers come from the device's stream-ordered pool on the engine's stream
// (devmem.cu): creating and destroying engines while other engines' kernels
// run then synchronizes nothing but this engine's own stream.
static cudaError_t dev_malloc(void **p, size_t bytes, cudaStream_t st)
{
    int n = g_fail_alloc.load();
    while (n > 0 && !g_fail_alloc.compare_exchange_weak(n, n - 1)) {
    }
    if (n == 1) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    const cudaError_t e = gtf_dmalloc(p, bytes, st);
    if (e == cudaSuccess) g_live_allocs++;
    return e;
}

// ordered on `st` after the buffer's last use there (or after the host has
// synchronized every stream that used it)
static void dev_free(void *p, cudaStream_t st)
{
    if (!p) return;
    gtf_dfree(p, st);
    g_live_allocs--;
}

// Device temporaries of one set-up call on stream `st` (every use of them is
// on that stream): released when the call returns, on success and on every
// error path alike, ordered after their last use.
struct DevTemps {
    std::vector<void *> p;
    cudaStream_t st;
    explicit DevTemps(cudaStream_t s) : st(s) {}
    DevTemps(const DevTemps &) = delete;
    DevTemps &operator=(const DevTemps &) = delete;
    ~DevTemps()
    {
        for (void *q : p) dev_free(q, st);
    }
    template <typename T>
    int get(T **out, size_t n)
    {
        *out = nullptr;
        if (n == 0) n = 1;
        void *q = nullptr;
        cudaError_t e = dev_malloc(&q, n * sizeof(T), st);
        if (e != cudaSuccess) {
            snprintf(g_errbuf, sizeof(g_errbuf), "cudaMalloc(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
            return GTF_ERR_ALLOC;
        }
        p.push_back(q);
        *out = (T *)q;
        return GTF_OK;
    }
    void drop(void *q)
    {
        for (size_t k = 0; k < p.size(); k++)
            if (p[k] == q) {
                dev_free(q, st);
                p.erase(p.begin() + (long)k);
                return;
            }
    }
};

#define TALLOC(tmps, ptr, n)                        \
    do {                                            \
        int r_ = (tmps).get(&(ptr), (size_t)(n));   \
        if (r_) return r_;                          \
    } while (0)

template <typename T>
static int dalloc(gtf_fock_dev *f, T **p, size_t n)
{
    *p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = dev_malloc((void **)p, n * sizeof(T), f->stream);
    if (e != cudaSuccess) {
        snprintf(g_errbuf, sizeof(g_errbuf), "cudaMalloc(%zu bytes): %s", n * sizeof(T),
                 cudaGetErrorString(e));
        return GTF_ERR_ALLOC;
    }
    f->dev_bytes += n * sizeof(T);
    return 0;
}

#define DALLOC(ptr, n)                          \
    do {                                        \
        int r_ = dalloc(f, &(ptr), (size_t)(n)); \
        if (r_) return r_;                      \
    } while (0)

// ---------------------------------------------------------------------------
// spherical <-> Cartesian transforms (d shells only)
// rows m = -2..2, cols xx, xy, xz, yy, yz, zz
// ---------------------------------------------------------------------------
__constant__ double c_sph_d[5][6] = {
    {0.0, 1.7320508075688772, 0.0, 0.0, 0.0, 0.0},
    {0.0, 0.0, 0.0, 0.0, 1.7320508075688772, 0.0},
    {-0.5, 0.0, 0.0, -0.5, 0.0, 1.0},
    {0.0, 0.0, 1.7320508075688772, 0.0, 0.0, 0.0},
    {0.8660254037844386, 0.0, 0.0, -0.8660254037844386, 0.0, 0.0}};

__device__ __forceinline__ double sph_coef(int L, int pure, int m, int c)
{
    if (pure && L == 2) return c_sph_d[m][c];
    return (m == c) ? 1.0 : 0.0;
}

__device__ __forceinline__ int nsph_of(int L, int pure) { return (pure && L == 2) ? 5 : ncart(L); }

// D_cart[i][j] = sum_{m,n} T[m][i] T[n][j] D[m][n]
__device__ __forceinline__ void d_to_cart_elem(const double *__restrict__ D, double *__restrict__ Dc,
                                               const int *__restrict__ cart2shell, const int *__restrict__ sh_L,
                                               const int *__restrict__ f_start, const int *__restrict__ fc_start,
                                               int nbf, int nbfc, int pure, int i, int j)
{
    const int si = cart2shell[i], sj = cart2shell[j];
    const int ci = i - fc_start[si], cj = j - fc_start[sj];
    const int Li = sh_L[si], Lj = sh_L[sj];
    const int mi = nsph_of(Li, pure), mj = nsph_of(Lj, pure);
    const int fi = f_start[si], fj = f_start[sj];
    double v = 0.0;
    for (int m = 0; m < mi; m++) {
        const double tm = sph_coef(Li, pure, m, ci);
        if (tm == 0.0) continue;
        for (int n = 0; n < mj; n++) {
            const double tn = sph_coef(Lj, pure, n, cj);
            if (tn == 0.0) continue;
            v += tm * tn * D[(size_t)(fi + m) * nbf + fj + n];
        }
    }
    Dc[(size_t)i * nbfc + j] = v;
}

__global__ void k_d_to_cart(const double *__restrict__ D, double *__restrict__ Dc,
                            const int *__restrict__ cart2shell, const int *__restrict__ sh_L,
                            const int *__restrict__ f_start, const int *__restrict__ fc_start,
                            int nbf, int nbfc, int pure)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= nbfc) return;
    d_to_cart_elem(D, Dc, cart2shell, sh_L, f_start, fc_start, nbf, nbfc, pure, i, j);
}

// Orientation of shell pair {A, B} in the reference's pair list
// (pfock/screening.c:146-163 keeps (A, B) for A > B with A + B even, A < B
// with A + B odd, and A == B): +1 for that orientation, -1 for the other.
// The reference digests each unique quartet once, in the orientation of its
// bra and ket pairs, with the update_F formulas written for a symmetric D
// (pfock/fock_task.c:29-117); with a non-symmetric D its Coulomb terms keep
// the part of the antisymmetric density Da that these orientations select.
// With Dta = s(M, N) Da the usual Coulomb digestion over any fixed pair
// orientations gives Fja, and the reference's symm = 0 result
// (F[D] + F[D^T]^T) / 2 (pfock/pfock.c:1704-1718) is the exact
// 2 J[D] - K[D] plus (S.Fja - (S.Fja)^T) / 2, S the block signs s(M, N).
__host__ __device__ __forceinline__ double ref_pair_sign(int A, int B)
{
    if (A == B) return 1.0;
    return ((A > B) == (((A + B) & 1) == 0)) ? 1.0 : -1.0;
}

// J = T sym(Fj) T^T, K = T sym(Fk) T^T, F = J + K (pfock/pfock.c:1719-1726, 1161-1185)
// Fka (non-symmetric densities only, else null): exchange accumulator of the
// antisymmetric part of D, whose full contribution is (Fka - Fka^T) / 2
__device__ __forceinline__ void f_to_sph_elem(const double *__restrict__ Fj, const double *__restrict__ Fk,
                                              double *__restrict__ F, double *__restrict__ J, double *__restrict__ K,
                                              const int *__restrict__ sph2shell, const int *__restrict__ sh_L,
                                              const int *__restrict__ f_start, const int *__restrict__ fc_start,
                                              int nbf, int nbfc, int pure, int m, int n,
                                              const double *__restrict__ Fka = nullptr, bool acc = false,
                                              const double *__restrict__ Fja = nullptr)
{
    const int sm = sph2shell[m], sn = sph2shell[n];
    const int cm = m - f_start[sm], cn = n - f_start[sn];
    const int Lm = sh_L[sm], Ln = sh_L[sn];
    const int fm = fc_start[sm], fn = fc_start[sn];
    const int nm = ncart(Lm), nn = ncart(Ln);
    // Fja: sign of the shell block in the reference's pair orientation
    const double smn = Fja ? ref_pair_sign(sm, sn) : 0.0, snm = Fja ? ref_pair_sign(sn, sm) : 0.0;
    double j = 0.0, k = 0.0;
    for (int a = 0; a < nm; a++) {
        const double ta = sph_coef(Lm, pure, cm, a);
        if (ta == 0.0) continue;
        for (int b = 0; b < nn; b++) {
            const double tb = sph_coef(Ln, pure, cn, b);
            if (tb == 0.0) continue;
            const size_t ab = (size_t)(fm + a) * nbfc + fn + b;
            const size_t ba = (size_t)(fn + b) * nbfc + fm + a;
            j += ta * tb * (0.5 * (Fj[ab] + Fj[ba]));
            k += ta * tb * (0.5 * (Fk[ab] + Fk[ba]));
            if (Fka) k += ta * tb * (0.5 * (Fka[ab] - Fka[ba]));
            if (Fja) j += ta * tb * (0.5 * (smn * Fja[ab] - snm * Fja[ba]));
        }
    }
    const size_t o = (size_t)m * nbf + n;
    if (acc) {
        // incremental build: this build's part is added to the previous result
        J[o] += j;
        K[o] += k;
        F[o] += j + k;
    } else {
        J[o] = j;
        K[o] = k;
        F[o] = j + k;
    }
}

__global__ void k_f_to_sph(const double *__restrict__ Fj, const double *__restrict__ Fk,
                           double *__restrict__ F, double *__restrict__ J, double *__restrict__ K,
                           const int *__restrict__ sph2shell, const int *__restrict__ sh_L,
                           const int *__restrict__ f_start, const int *__restrict__ fc_start,
                           int nbf, int nbfc, int pure, const double *__restrict__ Fka = nullptr,
                           const int *__restrict__ acc_flag = nullptr, const double *__restrict__ Fja = nullptr)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = blockIdx.y;
    if (n >= nbf) return;
    const bool acc = acc_flag != nullptr && *acc_flag != 0;
    f_to_sph_elem(Fj, Fk, F, J, K, sph2shell, sh_L, f_start, fc_start, nbf, nbfc, pure, m, n, Fka, acc, Fja);
}

// ---------------------------------------------------------------------------
// Incremental builds.  F is linear in D, so F[D_k] = F[D_k-1] + G[D_k -
// D_k-1].  A quartet contributes at most its Schwarz bound times the largest
// element of the density it digests, so with dmax = max |D_k - D_k-1| the
// build of the change keeps the quartets with bound * dmax >= tau (tau the
// Schwarz threshold by default: each dropped contribution is below what the
// plain build's screening drops), and evaluates in FP32 those with bound *
// dmax below the FP32 cutoff.  Every few builds a full one restarts the sum.
// ---------------------------------------------------------------------------
// Dd = D - Dprev (D itself on a full build), Dprev = D, and max |Dd| into the
// state (its dmax_bits zeroed before the launch)
__device__ __forceinline__ void delta_range(const double *__restrict__ D, double *__restrict__ Dprev,
                                            double *__restrict__ Dd, size_t n, int full, DynState *dyn,
                                            size_t i0, size_t step)
{
    double m = 0.0;
    for (size_t i = i0; i < n; i += step) {
        const double d = D[i];
        const double dd = full ? d : d - Dprev[i];
        Dd[i] = dd;
        Dprev[i] = d;
        m = fmax(m, fabs(dd));
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) m = fmax(m, __shfl_xor_sync(GTF_FULL_MASK, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(&dyn->dmax_bits, (unsigned long long)__double_as_longlong(m));
}

__global__ void k_delta(const double *__restrict__ D, double *__restrict__ Dprev, double *__restrict__ Dd, size_t n,
                        int full, DynState *dyn)
{
    delta_range(D, Dprev, Dd, n, full, dyn, (size_t)blockIdx.x * blockDim.x + threadIdx.x,
                (size_t)gridDim.x * blockDim.x);
}

// the thresholds of the build from dmax (one thread per engine)
__device__ __forceinline__ void dyn_thresholds(DynState *dyn, double tol2, double cut2, double tau2, double c2,
                                               int full)
{
    dyn->nq64 = 0;
    dyn->nq32 = 0;
    if (full) {
        dyn->tol2 = tol2;
        dyn->cut2 = cut2;
        dyn->acc = 0;
        return;
    }
    const double dm = __longlong_as_double((long long)dyn->dmax_bits);
    const double d2 = dm * dm;
    dyn->tol2 = d2 > 0.0 ? fmax(tol2, tau2 / d2) : INFINITY;
    dyn->cut2 = (c2 > 0.0 && d2 > 0.0) ? c2 / d2 : 0.0;
    dyn->acc = 1;
}

__global__ void k_dyn_thresholds(DynState *dyn, double tol2, double cut2, double tau2, double c2, int full)
{
    dyn_thresholds(dyn, tol2, cut2, tau2, c2, full);
}

// non-symmetric D: Ds = (D + D^T) / 2, Da = (D - D^T) / 2 and, for the
// reference's symm = 0 output (Dta non-null), Dta = s(M, N) Da with M, N the
// shells of the element (ref_pair_sign)
__global__ void k_split_density(const double *__restrict__ D, double *__restrict__ Ds, double *__restrict__ Da, int n,
                                double *__restrict__ Dta = nullptr, const int *__restrict__ sph2shell = nullptr)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= n) return;
    const double a = D[(size_t)i * n + j], t = D[(size_t)j * n + i];
    Ds[(size_t)i * n + j] = 0.5 * (a + t);
    Da[(size_t)i * n + j] = 0.5 * (a - t);
    if (Dta) Dta[(size_t)i * n + j] = ref_pair_sign(sph2shell[i], sph2shell[j]) * 0.5 * (a - t);
}

// ---------------------------------------------------------------------------
// screening
// ---------------------------------------------------------------------------
struct BasisDev {
    const int *sh_L, *sh_nprim, *sh_pstart;
    const double *sh_xyz, *alpha, *coef;
    int nshells, pure;
};

// pair record and primitive-pair data of shell pair (a, b), L(a) >= L(b)
__device__ __forceinline__ void make_pair(const BasisDev &b, int a, int bb, int off, int fa, int fb,
                                          PairRec *__restrict__ pr, double *__restrict__ pp, size_t npp)
{
    PairRec r;
    r.Ax = b.sh_xyz[3 * a];
    r.Ay = b.sh_xyz[3 * a + 1];
    r.Az = b.sh_xyz[3 * a + 2];
    const double Bx = b.sh_xyz[3 * bb], By = b.sh_xyz[3 * bb + 1], Bz = b.sh_xyz[3 * bb + 2];
    r.ABx = r.Ax - Bx;
    r.ABy = r.Ay - By;
    r.ABz = r.Az - Bz;
    r.fa = fa;
    r.fb = fb;
    r.off = off;
    const int na = b.sh_nprim[a], nb = b.sh_nprim[bb];
    r.n = na * nb;
    *pr = r;
    const double r2 = r.ABx * r.ABx + r.ABy * r.ABy + r.ABz * r.ABz;
    const int pa = b.sh_pstart[a], pb = b.sh_pstart[bb];
    for (int i = 0; i < na; i++) {
        for (int j = 0; j < nb; j++) {
            const double al = b.alpha[pa + i], be = b.alpha[pb + j];
            const double p = al + be, ip = 1.0 / p;
            const size_t o = (size_t)off + i * nb + j;
            pp[o] = p;
            pp[npp + o] = (al * r.Ax + be * Bx) * ip;
            pp[2 * npp + o] = (al * r.Ay + be * By) * ip;
            pp[3 * npp + o] = (al * r.Az + be * Bz) * ip;
            pp[4 * npp + o] = GTF_PAIR_PREF * b.coef[pa + i] * b.coef[pb + j] * exp(-al * be * ip * r2) * ip;
        }
    }
}

// pair data of every shell pair M >= N of one class (screening pass)
__global__ void k_screen_prep(BasisDev b, const int2 *__restrict__ mn, const int *__restrict__ off, int n,
                              PairRec *__restrict__ pairs, double *__restrict__ pp, size_t npp)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int M = mn[t].x, N = mn[t].y;
    const int a = (b.sh_L[M] >= b.sh_L[N]) ? M : N;
    const int bb = (a == M) ? N : M;
    make_pair(b, a, bb, off[t], 0, 0, pairs + t, pp, npp);
}

// Screening slices: the ket components cd = CD0 .. CD0+N-1 (cd = k + NA*l)
// of the diagonal quartet (MN|MN) at a time, folded into the sums
// s[m][n] = sum_{i,j,k,l} T[m][i] T[n][j] T[m][k] T[n][l] (ij|kl), so that no
// thread holds all NA*NB*NA*NB integrals (1296 for (dd|dd)).
__host__ __device__ constexpr int screen_slice_n(int LA, int LB)
{
    // whole quartets up to 81 integrals; else slices of at most 54
    return ncart(LA) * ncart(LB) * ncart(LA) * ncart(LB) <= 81 ? ncart(LA) * ncart(LB)
           : ncart(LA) * ncart(LB) * 3 <= 54                   ? 3
                                                               : 1;
}

template <int LA, int LB, int CD0, int N>
__device__ __forceinline__ void screen_slices(const PairRec &pr, const PPStored &src, int pure,
                                              double (&s)[ncart(LA) * ncart(LB)])
{
    constexpr int NA = ncart(LA), NB = ncart(LB), NR = LA + LB + 1;
    if constexpr (CD0 < NA * NB) {
        double acc[NA * NB * N];
#pragma unroll
        for (int k = 0; k < NA * NB * N; k++) acc[k] = 0.0;
        eri_accumulate_cd<LA, LB, LA, LB, CD0, N, false>(src, pr, src, pr, acc, RysTab<double>::ptr(NR));
        const int sa = nsph_of(LA, pure), sb = nsph_of(LB, pure);
#pragma unroll
        for (int m = 0; m < NA; m++) {
#pragma unroll
            for (int n = 0; n < NB; n++) {
                if (m >= sa || n >= sb) continue;
                double v = 0.0;
#pragma unroll
                for (int t = 0; t < N; t++) {
                    const int k = (CD0 + t) % NA, l = (CD0 + t) / NA;
                    const double tk = sph_coef(LA, pure, m, k), tl = sph_coef(LB, pure, n, l);
                    if (tk == 0.0 || tl == 0.0) continue;
#pragma unroll
                    for (int i = 0; i < NA; i++) {
                        const double ti = sph_coef(LA, pure, m, i);
                        if (ti == 0.0) continue;
#pragma unroll
                        for (int j = 0; j < NB; j++) {
                            const double tj = sph_coef(LB, pure, n, j);
                            if (tj == 0.0) continue;
                            v += ti * tj * tk * tl * acc[i + NA * (j + NB * t)];
                        }
                    }
                }
                s[m * NB + n] += v;
            }
        }
        screen_slices<LA, LB, CD0 + N, N>(pr, src, pure, s);
    }
}

// max |(mn|mn)| over the diagonal of (MN|MN) in the basis's own functions
// (pfock/screening.c:59-90), for the pairs of one class
template <int LA, int LB>
__global__ void __launch_bounds__(64) k_screen(const PairRec *__restrict__ pairs, PrimPairs pp,
                                               const int2 *__restrict__ mn, int n, int ns, int pure,
                                               double *__restrict__ sq, unsigned long long *__restrict__ gmax)
{
    constexpr int NA = ncart(LA), NB = ncart(LB);
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const PairRec pr = pairs[t];
    PPStored src{pp};
    double s[NA * NB];
#pragma unroll
    for (int k = 0; k < NA * NB; k++) s[k] = 0.0;
    screen_slices<LA, LB, 0, screen_slice_n(LA, LB)>(pr, src, pure, s);
    const int sa = nsph_of(LA, pure), sb = nsph_of(LB, pure);
    double mx = 0.0;
#pragma unroll
    for (int m = 0; m < NA; m++)
#pragma unroll
        for (int n2 = 0; n2 < NB; n2++)
            if (m < sa && n2 < sb && fabs(s[m * NB + n2]) > mx) mx = fabs(s[m * NB + n2]);
    const int M = mn[t].x, N = mn[t].y;
    sq[(size_t)M * ns + N] = mx;
    sq[(size_t)N * ns + M] = mx;
    atomicMax(gmax, (unsigned long long)__double_as_longlong(mx));
}

static int launch_screen(int cls, const PairRec *pairs, PrimPairs pp, const int2 *mn, int n, int ns, int pure,
                         double *sq, unsigned long long *gmax, cudaStream_t st)
{
    const unsigned g = (unsigned)((n + 63) / 64);
    switch (cls) {
        case 0: k_screen<0, 0><<<g, 64, 0, st>>>(pairs, pp, mn, n, ns, pure, sq, gmax); break;
        case 1: k_screen<1, 0><<<g, 64, 0, st>>>(pairs, pp, mn, n, ns, pure, sq, gmax); break;
        case 2: k_screen<1, 1><<<g, 64, 0, st>>>(pairs, pp, mn, n, ns, pure, sq, gmax); break;
        case 3: k_screen<2, 0><<<g, 64, 0, st>>>(pairs, pp, mn, n, ns, pure, sq, gmax); break;
        case 4: k_screen<2, 1><<<g, 64, 0, st>>>(pairs, pp, mn, n, ns, pure, sq, gmax); break;
        case 5: k_screen<2, 2><<<g, 64, 0, st>>>(pairs, pp, mn, n, ns, pure, sq, gmax); break;
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// keep flag per (M, N): value > eta and the parity rule (pfock/screening.c:127-133)
__global__ void k_csr_flags(const double *__restrict__ sq, int ns, double eta, int *__restrict__ flags)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)ns * ns) return;
    const int M = (int)(e / ns), N = (int)(e % ns);
    int keep = sq[e] > eta;
    if ((M > N && (M + N) % 2 == 1) || (M < N && (M + N) % 2 == 0)) keep = 0;
    flags[e] = keep;
}

__global__ void k_csr_scatter(const double *__restrict__ sq, const int *__restrict__ flags,
                              const int *__restrict__ pos, int ns, int *__restrict__ shellid,
                              int *__restrict__ shellrid, double *__restrict__ shellvalue,
                              int *__restrict__ shellptr)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n2 = (long long)ns * ns;
    if (e >= n2) return;
    const int M = (int)(e / ns), N = (int)(e % ns);
    if (N == 0) shellptr[M] = pos[e];
    if (e == n2 - 1) shellptr[ns] = pos[e] + flags[e];
    if (!flags[e]) return;
    const int k = pos[e];
    const double v = sq[e];
    shellid[k] = N;
    shellrid[k] = M;
    shellvalue[k] = (M == N) ? v : -v;
}

__global__ void k_sort_keys(const double *__restrict__ shellvalue, const int *__restrict__ shellid,
                            const int *__restrict__ shellrid, const int *__restrict__ sh_L, int nnz,
                            unsigned long long *__restrict__ kval, int *__restrict__ kcls,
                            int *__restrict__ idx)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nnz) return;
    const double v = fabs(shellvalue[k]);
    kval[k] = ~(unsigned long long)__double_as_longlong(v);  // descending by value
    kcls[k] = pair_class(sh_L[shellrid[k]], sh_L[shellid[k]]);
    idx[k] = k;
}

// second sort key: angular class (high bits) and primitive-count bucket
__global__ void k_gather_cls(const int *__restrict__ idx, const int *__restrict__ shellid,
                             const int *__restrict__ shellrid, const int *__restrict__ sh_L,
                             const int *__restrict__ kept, int nnz, int *__restrict__ kcls)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nnz) return;
    const int k = idx[s];
    kcls[s] = pair_class(sh_L[shellrid[k]], sh_L[shellid[k]]) * 16 + gtf_prim_bucket(kept[k]);
}

// prefactor K of primitive pair (i, j) of shells (a, bb) at squared distance r2
__device__ __forceinline__ double prim_pair_K(const BasisDev &b, int pa, int pb, int i, int j, double r2, double &p)
{
    const double al = b.alpha[pa + i], be = b.alpha[pb + j];
    p = al + be;
    const double ip = 1.0 / p;
    return GTF_PAIR_PREF * b.coef[pa + i] * b.coef[pb + j] * exp(-al * be * ip * r2) * ip;
}

// number of primitive pairs of CSR entry k that survive |K| >= GTF_PRIM_EPS
__global__ void k_prim_keep(const int *__restrict__ shellid, const int *__restrict__ shellrid, BasisDev b,
                            int nnz, int *__restrict__ kept)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nnz) return;
    const int M = shellrid[k], N = shellid[k];
    const double dx = b.sh_xyz[3 * M] - b.sh_xyz[3 * N], dy = b.sh_xyz[3 * M + 1] - b.sh_xyz[3 * N + 1],
                 dz = b.sh_xyz[3 * M + 2] - b.sh_xyz[3 * N + 2];
    const double r2 = dx * dx + dy * dy + dz * dz;
    int c = 0;
    for (int i = 0; i < b.sh_nprim[M]; i++)
        for (int j = 0; j < b.sh_nprim[N]; j++) {
            double p;
            if (fabs(prim_pair_K(b, b.sh_pstart[M], b.sh_pstart[N], i, j, r2, p)) >= GTF_PRIM_EPS) c++;
        }
    kept[k] = c;
}

__global__ void k_build_pairs(const int *__restrict__ idx, const int *__restrict__ shellid,
                              const int *__restrict__ shellrid, const double *__restrict__ shellvalue,
                              BasisDev b, const int *__restrict__ fc_start, int nnz,
                              PairRec *__restrict__ pairs, double *__restrict__ pair_v,
                              int *__restrict__ pair_n)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nnz) return;
    const int k = idx[s];
    const int M = shellrid[k], N = shellid[k];
    const int a = (b.sh_L[M] >= b.sh_L[N]) ? M : N;
    const int bb = (a == M) ? N : M;
    PairRec r;
    r.Ax = b.sh_xyz[3 * a];
    r.Ay = b.sh_xyz[3 * a + 1];
    r.Az = b.sh_xyz[3 * a + 2];
    r.ABx = r.Ax - b.sh_xyz[3 * bb];
    r.ABy = r.Ay - b.sh_xyz[3 * bb + 1];
    r.ABz = r.Az - b.sh_xyz[3 * bb + 2];
    r.fa = fc_start[a];
    r.fb = fc_start[bb];
    r.off = 0;
    r.n = b.sh_nprim[a] * b.sh_nprim[bb];
    pairs[s] = r;
    pair_v[s] = fabs(shellvalue[k]);
    pair_n[s] = r.n;
}

// Primitive pairs of each listed shell pair, compacted and sorted: pairs
// whose prefactor |K| is below GTF_PRIM_EPS are dropped (their contribution
// to any integral is below ~1e-15 Hartree), the rest are stored in descending
// |K| so that the quartet loop can stop once |K_ab K_cd| < GTF_PRIMQ_EPS.
// pairs[s].n becomes the kept count (possibly 0); the slot keeps its size.
// Records are {p, K, Px, Py, Pz, 1/(2p)} (PPRec).
__global__ void k_fill_primpairs(PairRec *__restrict__ pairs, const int *__restrict__ idx,
                                 const int *__restrict__ shellid, const int *__restrict__ shellrid,
                                 const int *__restrict__ pair_off, BasisDev b, int npairs, double *pp)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= npairs) return;
    const int k = idx[s];
    const int M = shellrid[k], N = shellid[k];
    const int a = (b.sh_L[M] >= b.sh_L[N]) ? M : N;
    const int bb = (a == M) ? N : M;
    const int off = pair_off[s];
    const double Ax = b.sh_xyz[3 * a], Ay = b.sh_xyz[3 * a + 1], Az = b.sh_xyz[3 * a + 2];
    const double Bx = b.sh_xyz[3 * bb], By = b.sh_xyz[3 * bb + 1], Bz = b.sh_xyz[3 * bb + 2];
    const double r2 = (Ax - Bx) * (Ax - Bx) + (Ay - By) * (Ay - By) + (Az - Bz) * (Az - Bz);
    const int na = b.sh_nprim[a], nb = b.sh_nprim[bb];
    const int pa = b.sh_pstart[a], pb = b.sh_pstart[bb];
    constexpr int W = 2 * GTF_PPREC_D2;
    int kept = 0;
    for (int i = 0; i < na; i++) {
        for (int j = 0; j < nb; j++) {
            double p;
            const double K = prim_pair_K(b, pa, pb, i, j, r2, p);
            if (fabs(K) < GTF_PRIM_EPS) continue;
            const double al = b.alpha[pa + i], be = b.alpha[pb + j], ip = 1.0 / p;
            // insertion into the descending-|K| list of the kept pairs
            int o = kept;
            while (o > 0 && fabs(pp[W * ((size_t)off + o - 1) + 1]) < fabs(K)) {
                const size_t src = W * ((size_t)off + o - 1);
                for (int f = 0; f < W; f++) pp[src + W + f] = pp[src + f];
                o--;
            }
            double *d = pp + W * ((size_t)off + o);
            d[0] = p;
            d[1] = K;
            d[2] = (al * Ax + be * Bx) * ip;
            d[3] = (al * Ay + be * By) * ip;
            d[4] = (al * Az + be * Bz) * ip;
            d[5] = 0.5 * ip;
            kept++;
        }
    }
    pairs[s].off = off;
    pairs[s].n = kept;
}

// FP32 records of the kept primitive pairs: centre relative to the pair's
// first shell, so that single precision keeps the small differences
__global__ void k_fill_pp32(const PairRec *__restrict__ pairs, int npairs, const double *__restrict__ pp,
                            float *__restrict__ pp32)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= npairs) return;
    const PairRec r = pairs[s];
    constexpr int W = 2 * GTF_PPREC_D2;
    for (int i = 0; i < r.n; i++) {
        const double *d = pp + W * ((size_t)r.off + i);
        float *o = pp32 + 8 * ((size_t)r.off + i);
        o[0] = (float)d[0];
        o[1] = (float)d[1];
        o[2] = (float)(d[2] - r.Ax);
        o[3] = (float)(d[3] - r.Ay);
        o[4] = (float)(d[4] - r.Az);
        o[5] = (float)d[5];
        o[6] = 0.0f;
        o[7] = 0.0f;
    }
}

// ---------------------------------------------------------------------------
// Task lists, built on the device.
//
// For every (engine, class pair) and bra pair i of class X: the number of ket
// pairs of each segment b of class Y that pass the quartet Schwarz test
// v_i v_j >= tol2 (pfock/fock_task.c:192).  Each segment is sorted by value,
// descending, so these kets are a prefix, found by binary search.  For X == Y
// only kets at or before the bra in the class order count, so every unordered
// pair of pairs is visited once.  Segment 0 holds pairs whose primitive pairs
// were all screened out: counted, but given no units.
//
// cut2 > 0 (mixed precision): the kets with v_i v_j < cut2, i.e. a Schwarz
// bound sqrt(v_i v_j) below the FP32 cutoff, form the tail of each prefix and
// go to the FP32 launch; n64 counts the FP64 head.
//
// Per bra, the kets of all segments (in segment order, segment 0 left out)
// form one list per launch part, so a warp's 32 lanes are filled across
// segment boundaries: cum[i][b] is the exclusive prefix of the segment counts
// and the bra has ceil(total / 32) units; the unit prefixes over the bras
// close the lists.
//
// The thresholds are an engine's static ones, or, for incremental builds,
// read from the engine's device state, where they were scaled by the largest
// element of the density change.  Three launches rebuild the lists of every
// engine of a build (one engine, or all the molecules of a batch) with no
// host round trip, so a rebuild can sit inside a captured graph.
// ---------------------------------------------------------------------------
struct UnitTask {
    const double *pair_v;
    int *nket, *n64, *cum64, *cum32;
    long long *up64, *up32;      // unit prefixes, [nbra + 1] each
    DynState *dyn;               // null: the static thresholds below
    double tol2, cut2;
    long long idx0;              // first (bra, segment) index of this task, over all tasks
    long long bra0;              // first bra index of this task, over all tasks
    int bra_start, nbra, ket_start, same;
    int seg[GTF_NBKT + 1];
};

// last task k with key(k) <= v (key non-decreasing, key(0) = 0 <= v)
template <typename Key>
__device__ __forceinline__ int task_of(const UnitTask *__restrict__ t, int nt, long long v, Key key)
{
    int lo = 0, hi = nt - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (key(t[mid]) <= v) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// phase 1: one thread per (task, bra, segment)
__global__ void k_units_count(const UnitTask *__restrict__ tasks, int nt, long long total)
{
    for (long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x; x < total;
         x += (long long)gridDim.x * blockDim.x) {
        const int k = task_of(tasks, nt, x, [](const UnitTask &t) { return t.idx0; });
        const UnitTask &t = tasks[k];
        const int r = (int)(x - t.idx0);
        const int i = r / GTF_NBKT, b = r - i * GTF_NBKT;
        double tol2 = t.tol2, cut2 = t.cut2;
        if (t.dyn) {
            tol2 = t.dyn->tol2;
            cut2 = t.dyn->cut2;
        }
        const double *pv = t.pair_v + t.ket_start;
        const double v = t.pair_v[t.bra_start + i];
        const int s0 = t.seg[b], s1 = t.seg[b + 1];
        int lo = s0, hi = s1;  // first index failing the Schwarz test
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (fabs(v * pv[mid]) >= tol2) lo = mid + 1;
            else hi = mid;
        }
        int c = lo - s0;
        int lo2 = s0, hi2 = s0 + c;  // first index below the FP32 cutoff
        while (lo2 < hi2) {
            const int mid = (lo2 + hi2) >> 1;
            if (fabs(v * pv[mid]) >= cut2) lo2 = mid + 1;
            else hi2 = mid;
        }
        int c64 = lo2 - s0;
        if (t.same) {
            const int lim = i - s0 + 1;  // kets j <= i
            c = lim < 0 ? 0 : (c < lim ? c : lim);
            c64 = c64 < c ? c64 : c;
        }
        t.nket[r] = c;
        t.n64[r] = c64;
        if (t.dyn) {
            // quartets of this build (FP64, FP32), for the statistics
            unsigned long long q64 = (unsigned long long)c64, q32 = (unsigned long long)(c - c64);
            atomicAdd(&t.dyn->nq64, q64);
            atomicAdd(&t.dyn->nq32, q32);
        }
    }
}

// phase 2: one thread per (task, bra): segment prefixes and units per bra
// (the unit counts go into the prefix arrays, scanned in place by phase 3)
__global__ void k_units_pack(const UnitTask *__restrict__ tasks, int nt, long long total)
{
    for (long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x; x < total;
         x += (long long)gridDim.x * blockDim.x) {
        const int k = task_of(tasks, nt, x, [](const UnitTask &t) { return t.bra0; });
        const UnitTask &t = tasks[k];
        const int i = (int)(x - t.bra0);
        int a = 0, c = 0;
        for (int b = 0; b < GTF_NBKT; b++) {
            t.cum64[i * GTF_CUM + b] = a;
            t.cum32[i * GTF_CUM + b] = c;
            if (b == 0) continue;  // pairs whose primitive pairs were all screened out
            const int n = t.nket[i * GTF_NBKT + b], h = t.n64[i * GTF_NBKT + b];
            a += h;
            c += n - h;
        }
        t.cum64[i * GTF_CUM + GTF_NBKT] = a;
        t.cum32[i * GTF_CUM + GTF_NBKT] = c;
        t.up64[i] = (a + 31) / 32;
        t.up32[i] = (c + 31) / 32;
    }
}

// phase 3: block (task, part) turns the per-bra units into the exclusive
// prefix [nbra + 1] in place
#define UNIT_SCAN_THREADS 256
#define UNIT_SCAN_ITEMS 4
__global__ void __launch_bounds__(UNIT_SCAN_THREADS) k_units_scan(const UnitTask *__restrict__ tasks)
{
    typedef cub::BlockScan<long long, UNIT_SCAN_THREADS> Scan;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ long long s_carry;
    const UnitTask &t = tasks[blockIdx.x >> 1];
    long long *u = (blockIdx.x & 1) ? t.up32 : t.up64;
    const int n = t.nbra;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    constexpr int CH = UNIT_SCAN_THREADS * UNIT_SCAN_ITEMS;
    for (int base = 0; base < n; base += CH) {
        long long v[UNIT_SCAN_ITEMS];
#pragma unroll
        for (int q = 0; q < UNIT_SCAN_ITEMS; q++) {
            const int i = base + threadIdx.x * UNIT_SCAN_ITEMS + q;
            v[q] = i < n ? u[i] : 0;
        }
        long long agg;
        Scan(tmp).ExclusiveSum(v, v, agg);
        const long long carry = s_carry;
#pragma unroll
        for (int q = 0; q < UNIT_SCAN_ITEMS; q++) {
            const int i = base + threadIdx.x * UNIT_SCAN_ITEMS + q;
            if (i < n) u[i] = v[q] + carry;
        }
        __syncthreads();
        if (threadIdx.x == 0) s_carry = carry + agg;
        __syncthreads();
    }
    if (threadIdx.x == 0) u[n] = s_carry;
}

// Primitive quartets the Fock kernels evaluate after primitive screening: the
// loops stop at |K_ab K_cd| < GTF_PRIMQ_EPS with both lists in descending
// |K| (the ket loop once the largest bra primitive fails), so a quartet
// evaluates, per ket primitive that passes with the first bra primitive, the
// prefix of bra primitives that pass with it.  One thread per (task, bra,
// segment) walks its kets; out[k] receives task k's total.  Statistics only.
__global__ void k_count_primq(const UnitTask *__restrict__ tasks, int nt, long long total,
                              const PairRec *__restrict__ pairs, const double *__restrict__ pp,
                              double *__restrict__ out)
{
    for (long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x; x < total;
         x += (long long)gridDim.x * blockDim.x) {
        const int k = task_of(tasks, nt, x, [](const UnitTask &t) { return t.idx0; });
        const UnitTask &t = tasks[k];
        const int r = (int)(x - t.idx0);
        const int i = r / GTF_NBKT, b = r - i * GTF_NBKT;
        if (b == 0) continue;   // segment 0 gets no units
        const int n = t.nket[r];
        const PairRec pb = pairs[t.bra_start + i];
        if (n == 0 || pb.n <= 0) continue;
        const double kb0 = fabs(pp[(size_t)2 * GTF_PPREC_D2 * pb.off + 1]);
        double cnt = 0.0;
        for (int q = 0; q < n; q++) {
            const PairRec pk = pairs[t.ket_start + t.seg[b] + q];
            for (int ik = 0; ik < pk.n; ik++) {
                const double kk = fabs(pp[(size_t)2 * GTF_PPREC_D2 * (pk.off + ik) + 1]);
                if (kb0 * kk < GTF_PRIMQ_EPS) break;
                int nb = 0;
                while (nb < pb.n && fabs(pp[(size_t)2 * GTF_PPREC_D2 * (pb.off + nb) + 1]) * kk >= GTF_PRIMQ_EPS) nb++;
                cnt += nb;
            }
        }
        atomicAdd(out + k, cnt);
    }
}

// Launches the three phases over `nt` tasks (device array) whose flattened
// (bra, segment) and bra counts are nidx and nbras.
static int run_units(const UnitTask *d_tasks, int nt, long long nidx, long long nbras, int nsm, cudaStream_t st)
{
    if (nt == 0) return GTF_OK;
    auto grid = [&](long long n) {
        long long g = (n + 255) / 256, cap = (long long)nsm * 8;
        return (unsigned)(g < 1 ? 1 : (g > cap ? cap : g));
    };
    k_units_count<<<grid(nidx), 256, 0, st>>>(d_tasks, nt, nidx);
    CK(cudaGetLastError());
    k_units_pack<<<grid(nbras), 256, 0, st>>>(d_tasks, nt, nbras);
    CK(cudaGetLastError());
    k_units_scan<<<2 * nt, UNIT_SCAN_THREADS, 0, st>>>(d_tasks);
    CK(cudaGetLastError());
    return GTF_OK;
}

typedef int (*fock_group_launch_t)(int la, int lb, int lc, int ld, const FockGrid &g, cudaStream_t st);
extern fock_group_launch_t gtf_fock_groups[];
extern const int gtf_fock_ngroups;

static int launch_fock(int X, int Y, const FockGrid &fg, cudaStream_t st)
{
    for (int g = 0; g < gtf_fock_ngroups; g++) {
        int r = gtf_fock_groups[g](k_cls_la[X], k_cls_lb[X], k_cls_la[Y], k_cls_lb[Y], fg, st);
        if (r != GTF_NOT_IN_GROUP) return r;  // launches, or -1 on error
    }
    return -1;
}

// ---------------------------------------------------------------------------
// launch-shape autotuning
// ---------------------------------------------------------------------------
// Process-wide table: (kind, class X, class Y, precision part, size bucket)
// -> (a, b).  Kind 0 / 1: a Fock launch of a single engine / of a batch,
// a = persistent blocks per SM, b = units of 32 quartets a warp claims at
// once; kind 2: the batched dense products, a = tile shape.  The size bucket
// is floor(log2) of the launch's units (or of the products' n^3 sum).  The
// tuners time candidate shapes on the live engine and record the fastest;
// launches look their shape up here (absent: the defaults).
struct TuneKey {
    int kind, X, Y, part, bucket;
    bool operator<(const TuneKey &o) const
    {
        return std::tie(kind, X, Y, part, bucket) < std::tie(o.kind, o.X, o.Y, o.part, o.bucket);
    }
};
struct TuneVal {
    int a, b;
    double ms;
};
static std::map<TuneKey, TuneVal> g_tune;
static std::mutex g_tune_mu;

static int tune_bucket(double size)
{
    int b = 0;
    while (b < 120 && ldexp(1.0, b + 1) <= size) b++;
    return b;
}

extern "C" int gtf_tune_get(int kind, int X, int Y, int part, double size, int *a, int *b)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(TuneKey{kind, X, Y, part, tune_bucket(size)});
    if (it == g_tune.end()) return 0;
    if (a) *a = it->second.a;
    if (b) *b = it->second.b;
    return 1;
}

extern "C" void gtf_tune_put(int kind, int X, int Y, int part, double size, int a, int b, double ms)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[TuneKey{kind, X, Y, part, tune_bucket(size)}] = TuneVal{a, b, ms};
}

extern "C" void gtf_tune_clear(void)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune.clear();
}

// rows of 8 ints: kind, X, Y, part, bucket, a, b, ms x 1000 (rounded); returns the count
extern "C" int gtf_tune_entries(int *rows, int max_rows)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    int n = 0;
    for (const auto &kv : g_tune) {
        if (rows && n < max_rows) {
            int *r = rows + 8 * n;
            r[0] = kv.first.kind;
            r[1] = kv.first.X;
            r[2] = kv.first.Y;
            r[3] = kv.first.part;
            r[4] = kv.first.bucket;
            r[5] = kv.second.a;
            r[6] = kv.second.b;
            r[7] = (int)lrint(kv.second.ms * 1000.0);
        }
        n++;
    }
    return n;
}

static void device_name(char *out, size_t len)
{
    int dev = 0;
    cudaDeviceProp p;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&p, dev) != cudaSuccess) {
        snprintf(out, len, "unknown");
        return;
    }
    snprintf(out, len, "%s sm_%d%d", p.name, p.major, p.minor);
    for (char *c = out; *c; c++)
        if (*c == ' ') *c = '_';
}

// Text file: "gtfock_b200-tune 1 <device>" then one entry per line
// "kind X Y part bucket a b ms".
extern "C" int gtf_tune_save(const char *path)
{
    char dev[256];
    device_name(dev, sizeof(dev));
    FILE *fp = fopen(path, "w");
    if (!fp) return GTF_ERR_IO;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    fprintf(fp, "gtfock_b200-tune 1 %s\n", dev);
    for (const auto &kv : g_tune)
        fprintf(fp, "%d %d %d %d %d %d %d %.6f\n", kv.first.kind, kv.first.X, kv.first.Y, kv.first.part,
                kv.first.bucket, kv.second.a, kv.second.b, kv.second.ms);
    return fclose(fp) == 0 ? GTF_OK : GTF_ERR_IO;
}

// Merges a saved table; a file written on another device model is refused
// (GTF_ERR_INVALID) and leaves the table unchanged.
extern "C" int gtf_tune_load(const char *path)
{
    FILE *fp = fopen(path, "r");
    if (!fp) return GTF_ERR_IO;
    char magic[64], dev[256], here[256];
    int ver = 0;
    if (fscanf(fp, "%63s %d %255s", magic, &ver, dev) != 3 || strcmp(magic, "gtfock_b200-tune") != 0 || ver != 1) {
        fclose(fp);
        return GTF_ERR_INVALID;
    }
    device_name(here, sizeof(here));
    if (strcmp(dev, here) != 0) {
        fclose(fp);
        return GTF_ERR_INVALID;
    }
    std::vector<std::pair<TuneKey, TuneVal>> rows;
    TuneKey k;
    TuneVal v;
    int r;
    while ((r = fscanf(fp, "%d %d %d %d %d %d %d %lf", &k.kind, &k.X, &k.Y, &k.part, &k.bucket, &v.a, &v.b, &v.ms)) == 8)
        rows.push_back({k, v});
    const bool ok = (r == EOF);
    fclose(fp);
    if (!ok) return GTF_ERR_INVALID;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (const auto &kv : rows) g_tune[kv.first] = kv.second;
    return GTF_OK;
}

static void tune_apply(int kind, int X, int Y, int part, FockGrid &g)
{
    int a = 0, b = 0;
    if (gtf_tune_get(kind, X, Y, part, (double)g.nunits, &a, &b)) {
        g.ctas_per_sm = a;
        g.claim = b;
    }
}

// Times launch_fock of one (class pair, part) under each candidate shape
// (blocks per SM: the occupancy limit, one less, half; for batched launches
// claims of 1, 2, 4 units) and records the fastest.  `counters` holds GTF_MAX_SLICES slots;
// the launches accumulate into the grid's F buffers, which the next build
// clears.  Returns the best time in ms, or a negative value on error.
static double tune_launch(int kind, int X, int Y, int part, FockGrid g, cudaStream_t st, int reps,
                          cudaEvent_t e0, cudaEvent_t e1)
{
    g.query = 1;
    const int occ = launch_fock(X, Y, g, st);
    g.query = 0;
    if (occ < 1) return -1.0;
    int ctas[3] = {occ, occ - 1, (occ + 1) / 2};
    int nct = 1;
    for (int i = 1; i < 3; i++) {
        bool dup = ctas[i] < 1;
        for (int j = 0; j < nct; j++) dup = dup || ctas[j] == ctas[i];
        if (!dup) ctas[nct++] = ctas[i];
    }
    const int claims[3] = {1, 2, 4};
    const int ncl = g.nmol > 1 ? 3 : 1;    // only the batched kernels claim several units
    double best = -1.0;
    int ba = occ, bb = 1;
    for (int ci = 0; ci < nct; ci++)
        for (int cl = 0; cl < ncl; cl++) {
            g.ctas_per_sm = ctas[ci];
            g.claim = claims[cl];
            double tmin = 1e30;
            for (int r = 0; r < reps + 1; r++) {   // the first run warms up
                if (cudaMemsetAsync(g.counter, 0, sizeof(unsigned long long) * GTF_MAX_SLICES, st) != cudaSuccess ||
                    cudaEventRecord(e0, st) != cudaSuccess || launch_fock(X, Y, g, st) < 0 ||
                    cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess)
                    return -1.0;
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (r > 0 && ms < tmin) tmin = ms;
            }
            if (best < 0.0 || tmin < best) {
                best = tmin;
                ba = ctas[ci];
                bb = claims[cl];
            }
        }
    gtf_tune_put(kind, X, Y, part, (double)g.nunits, ba, bb, best);
    return best;
}

// Rys-model FLOPs of one quartet of a class (normalisation used for the roofline):
// K [30 n_r + 12 n_r (la+lb+1)(lc+ld+1) + 3 n_r Nc] + 2 K Nc + 12 Ns
static double class_flops_per_prim(int X, int Y, double *contract_part)
{
    const int la = k_cls_la[X], lb = k_cls_lb[X], lc = k_cls_la[Y], ld = k_cls_lb[Y];
    const int nr = (la + lb + lc + ld) / 2 + 1;
    const double nc = (double)ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
    *contract_part = 2.0 * nc;
    return 30.0 * nr + 12.0 * nr * (la + lb + 1) * (lc + ld + 1) + 3.0 * nr * nc;
}

// ---------------------------------------------------------------------------
// host API
// ---------------------------------------------------------------------------
// device, stream, events and the basis arrays (shared by the Fock engine and
// the basis-only context of the per-quartet CInt entry points)
static int upload_basis(gtf_fock_dev *f, const gtf_basis_view_t *b)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        snprintf(g_errbuf, sizeof(g_errbuf), "no CUDA device visible");
        return GTF_ERR_NODEVICE;
    }
    if (b->nshells <= 0) return GTF_ERR_INVALID;
    CK(cudaGetDevice(&f->dev));
    CK(cudaDeviceGetAttribute(&f->nsm, cudaDevAttrMultiProcessorCount, f->dev));
    CK(cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&f->ev0));
    CK(cudaEventCreate(&f->ev1));
    CK(cudaEventCreate(&f->ev2));
    CK(cudaEventCreate(&f->ev3));
    for (int c = 0; c <= NCLSPAIR; c++) CK(cudaEventCreate(&f->ev_cls[c]));
    f->natoms = b->natoms;
    f->nshells = b->nshells;
    f->nbf = b->nbf;
    f->nbf_cart = b->nbf_cart;
    f->nprims = b->nprims;
    f->pure = b->pure;
    const int ns = b->nshells;
    cudaStream_t st = f->stream;
    f->h_sh_L.assign(b->sh_L, b->sh_L + ns);
    f->h_f_start.assign(b->f_start, b->f_start + ns + 1);
    f->h_fc_start.assign(b->fc_start, b->fc_start + ns + 1);
    std::vector<double> sh_xyz(3 * ns);
    for (int s = 0; s < ns; s++)
        for (int k = 0; k < 3; k++) sh_xyz[3 * s + k] = b->xyz[3 * b->sh_atom[s] + k];
    std::vector<int> sph2shell(b->nbf), cart2shell(b->nbf_cart);
    for (int s = 0; s < ns; s++) {
        for (int k = b->f_start[s]; k < b->f_start[s + 1]; k++) sph2shell[k] = s;
        for (int k = b->fc_start[s]; k < b->fc_start[s + 1]; k++) cart2shell[k] = s;
    }
    DALLOC(f->d_sh_L, ns);
    DALLOC(f->d_sh_nprim, ns);
    DALLOC(f->d_sh_pstart, ns);
    DALLOC(f->d_f_start, ns + 1);
    DALLOC(f->d_fc_start, ns + 1);
    DALLOC(f->d_sph2shell, b->nbf);
    DALLOC(f->d_cart2shell, b->nbf_cart);
    DALLOC(f->d_Z, b->natoms);
    DALLOC(f->d_sh_xyz, 3 * ns);
    DALLOC(f->d_alpha, b->nprims);
    DALLOC(f->d_coef, b->nprims);
    DALLOC(f->d_atom_xyz, 3 * b->natoms);
    CK(cudaMemcpyAsync(f->d_sh_L, b->sh_L, sizeof(int) * ns, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(f->d_sh_nprim, b->sh_nprim, sizeof(int) * ns, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(f->d_sh_pstart, b->sh_pstart, sizeof(int) * ns, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(f->d_f_start, b->f_start, sizeof(int) * (ns + 1), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(f->d_fc_start, b->fc_start, sizeof(int) * (ns + 1), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(f->d_sph2shell, sph2shell.data(), sizeof(int) * b->nbf, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(f->d_cart2shell, cart2shell.data(), sizeof(int) * b->nbf_cart,
                       cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(f->d_Z, b->Z, sizeof(int) * b->natoms, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(f->d_sh_xyz, sh_xyz.data(), sizeof(double) * 3 * ns, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(f->d_alpha, b->alpha, sizeof(double) * b->nprims, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(f->d_coef, b->coef, sizeof(double) * b->nprims, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(f->d_atom_xyz, b->xyz, sizeof(double) * 3 * b->natoms, cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    return GTF_OK;
}

// basis-only context: no screening, no Fock buffers
extern "C" int gtf_basis_dev_create(const gtf_basis_view_t *b, gtf_fock_dev_t **out)
{
    gtf_fock_dev *f = new gtf_fock_dev();
    memset(f->tasks, 0, sizeof(f->tasks));
    f->max_numdmat = 0;
    *out = f;
    return upload_basis(f, b);
}

// The engine's task set: one UnitTask per class pair with work, static and
// dynamic copies on the device (called once, after the per-task arrays exist).
static int make_unit_tasks(gtf_fock_dev *f)
{
    f->h_ut.clear();
    long long nidx = 0, nbras = 0;
    for (int c = 0; c < NCLSPAIR; c++) {
        ClassPairTask &t = f->tasks[c];
        if (t.nbra == 0 || t.nketcls == 0) continue;
        UnitTask u;
        memset(&u, 0, sizeof(u));
        u.pair_v = f->d_pair_v;
        u.nket = t.d_nket;
        u.n64 = t.d_n64;
        u.cum64 = t.d_cum64;
        u.cum32 = t.d_cum32;
        u.up64 = t.d_unit_prefix;
        u.up32 = t.d_unit_prefix32;
        u.idx0 = nidx;
        u.bra0 = nbras;
        u.bra_start = t.bra_start;
        u.nbra = t.nbra;
        u.ket_start = t.ket_start;
        u.same = t.X == t.Y;
        for (int bk = 0; bk <= GTF_NBKT; bk++) u.seg[bk] = t.seg[bk];
        f->h_ut.push_back(u);
        nidx += (long long)t.nbra * GTF_NBKT;
        nbras += t.nbra;
    }
    f->ut_nidx = nidx;
    f->ut_nbras = nbras;
    const size_t nt = f->h_ut.size();
    DALLOC(f->d_ut_static, nt);
    DALLOC(f->d_ut_dyn, nt);
    DALLOC(f->d_dyn, 1);
    DALLOC(f->d_unit_tot, 3 * NCLSPAIR);
    std::vector<UnitTask> dyn(f->h_ut);
    for (auto &u : dyn) u.dyn = f->d_dyn;
    if (nt) CK(cudaMemcpyAsync(f->d_ut_dyn, dyn.data(), sizeof(UnitTask) * nt, cudaMemcpyHostToDevice, f->stream));
    CK(cudaMemsetAsync(f->d_dyn, 0, sizeof(DynState), f->stream));
    CK(cudaStreamSynchronize(f->stream));
    return GTF_OK;
}

static int shard_bounds(gtf_fock_dev *f, int c, const std::vector<int> &nk, const std::vector<int> &n64);

// Totals of one class pair's (bra, segment) ket counts: quartets, FP32
// quartets and the bound on a launch's units (sum over bras of the units of
// all non-empty segments).  64-bit integer sums: exact whatever the order.
__global__ void k_unit_totals(const int *__restrict__ nk, const int *__restrict__ n64, int nbra,
                              unsigned long long *__restrict__ out)
{
    unsigned long long q = 0, q32 = 0, bound = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nbra; i += gridDim.x * blockDim.x) {
        long long all = 0;
#pragma unroll
        for (int b = 0; b < GTF_NBKT; b++) {
            const int k = i * GTF_NBKT + b;
            q += (unsigned long long)nk[k];
            q32 += (unsigned long long)(nk[k] - n64[k]);
            if (b > 0) all += nk[k];
        }
        bound += (unsigned long long)((all + 31) / 32);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        q += __shfl_down_sync(GTF_FULL_MASK, q, o);
        q32 += __shfl_down_sync(GTF_FULL_MASK, q32, o);
        bound += __shfl_down_sync(GTF_FULL_MASK, bound, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out, q);
        atomicAdd(out + 1, q32);
        atomicAdd(out + 2, bound);
    }
}

// Per class pair and (bra, segment): ket counts, the FP64 / FP32 split for
// the current precision mode and the unit prefixes of both launches, under
// the engine's static thresholds; the unit totals and quartet counts come
// back to the host.
static int build_units(gtf_fock_dev *f)
{
    cudaStream_t st = f->stream;
    const double cut2 = f->prec == GTF_PREC_MIXED ? f->fp32_cutoff * f->fp32_cutoff : 0.0;
    const int nt = (int)f->h_ut.size();
    for (auto &u : f->h_ut) {
        u.tol2 = f->tolscr2;
        u.cut2 = cut2;
    }
    for (int c = 0; c < NCLSPAIR; c++) {
        ClassPairTask &t = f->tasks[c];
        t.nunits = t.nunits32 = 0;
        t.nquart = t.nquart32 = 0.0;
    }
    f->lists_dyn = 0;
    if (nt == 0) return GTF_OK;
    CK(cudaMemcpyAsync(f->d_ut_static, f->h_ut.data(), sizeof(UnitTask) * nt, cudaMemcpyHostToDevice, st));
    int r = run_units(f->d_ut_static, nt, f->ut_nidx, f->ut_nbras, f->nsm, st);
    if (r) return r;
    gtf_note_launches(3);
    // the per-(bra, segment) counts come to the host only for the shard split
    const bool sharded = f->nshards > 1;
    std::vector<std::vector<int>> nk(NCLSPAIR), n64(NCLSPAIR);
    unsigned long long tot[3 * NCLSPAIR];
    CK(cudaMemsetAsync(f->d_unit_tot, 0, sizeof(tot), st));
    int nl = 0;
    for (int c = 0; c < NCLSPAIR; c++) {
        ClassPairTask &t = f->tasks[c];
        if (t.nbra == 0 || t.nketcls == 0) continue;
        const int nidx = t.nbra * GTF_NBKT;
        int g = (t.nbra + 255) / 256;
        if (g > 4 * f->nsm) g = 4 * f->nsm;
        k_unit_totals<<<g, 256, 0, st>>>(t.d_nket, t.d_n64, t.nbra, f->d_unit_tot + 3 * c);
        CK(cudaGetLastError());
        nl++;
        CK(cudaMemcpyAsync(&t.nunits, t.d_unit_prefix + t.nbra, sizeof(long long), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&t.nunits32, t.d_unit_prefix32 + t.nbra, sizeof(long long), cudaMemcpyDeviceToHost, st));
        if (sharded) {
            nk[c].resize(nidx);
            n64[c].resize(nidx);
            CK(cudaMemcpyAsync(nk[c].data(), t.d_nket, sizeof(int) * nidx, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(n64[c].data(), t.d_n64, sizeof(int) * nidx, cudaMemcpyDeviceToHost, st));
        }
    }
    gtf_note_launches(nl);
    CK(cudaMemcpyAsync(tot, f->d_unit_tot, sizeof(tot), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int c = 0; c < NCLSPAIR; c++) {
        ClassPairTask &t = f->tasks[c];
        if (t.nbra == 0 || t.nketcls == 0) continue;
        t.nquart = (double)tot[3 * c];
        t.nquart32 = (double)tot[3 * c + 1];
        // thresholds at or above tol2 select a subset of these kets, in one
        // launch or split between two (one more unit per bra at most)
        t.nunits_bound = (long long)tot[3 * c + 2] + t.nbra;
    }
    // the units of this engine's shard (all of them when not sharded)
    f->shard_work = 0.0;
    for (int c = 0; c < NCLSPAIR; c++) {
        const int r2 = shard_bounds(f, c, nk[c], n64[c]);
        if (r2) return r2;
    }
    return GTF_OK;
}

// Plain builds use the static task lists: restore them after incremental
// builds overwrote the arrays (no allocation; one host wait).
static int static_lists(gtf_fock_dev *f)
{
    return f->lists_dyn ? build_units(f) : GTF_OK;
}

// Rys-model FLOPs per build (a fixed work normalisation: every primitive
// quartet of every screened shell quartet, before primitive screening) and
// primitive quartets, per class pair, from the static ket counts.  It walks
// every (bra, segment) of every class pair on the host, so it is evaluated
// when first asked for rather than at set-up.
static int ensure_work_model(gtf_fock_dev *f)
{
    if (f->work_model) return GTF_OK;
    const int r = static_lists(f);
    if (r) return r;
    const std::vector<int> &hn = f->h_pair_n;
    double flops = 0.0;
    for (int c2 = 0; c2 < NCLSPAIR; c2++) {
        ClassPairTask &t = f->tasks[c2];
        if (t.nbra == 0 || t.nketcls == 0) continue;
        const int nidx = t.nbra * GTF_NBKT;
        std::vector<int> nk(nidx);
        CK(cudaMemcpyAsync(nk.data(), t.d_nket, sizeof(int) * nidx, cudaMemcpyDeviceToHost, f->stream));
        CK(cudaStreamSynchronize(f->stream));
        // prefix sums of ket primitive-pair counts
        std::vector<double> kpre(t.nketcls + 1, 0.0);
        for (int j = 0; j < t.nketcls; j++) kpre[j + 1] = kpre[j] + hn[t.ket_start + j];
        double cpart;
        const double per_prim = class_flops_per_prim(t.X, t.Y, &cpart);
        const int la = k_cls_la[t.X], lb = k_cls_lb[t.X], lc = k_cls_la[t.Y], ld = k_cls_lb[t.Y];
        const double ns_ = (double)(f->pure && la == 2 ? 5 : ncart(la)) * (f->pure && lb == 2 ? 5 : ncart(lb)) *
                           (f->pure && lc == 2 ? 5 : ncart(lc)) * (f->pure && ld == 2 ? 5 : ncart(ld));
        double cf = 0.0, cq = 0.0;
        for (int i = 0; i < t.nbra; i++) {
            const double kb = hn[t.bra_start + i];
            for (int bk = 0; bk < GTF_NBKT; bk++) {
                const int c = nk[i * GTF_NBKT + bk];
                const double kk = kpre[t.seg[bk] + c] - kpre[t.seg[bk]];
                cf += kb * kk * per_prim + (cpart + 12.0 * ns_) * c;
                cq += kb * kk;
            }
        }
        t.flops = cf;
        t.nprimq = cq;
        flops += cf;
    }
    f->eri_flops = flops;
    f->work_model = true;
    return GTF_OK;
}

extern "C" int gtf_fock_create(const gtf_basis_view_t *b, double tolscr, int max_numdmat,
                               gtf_fock_dev_t **out)
{
    *out = nullptr;
    if (b->nshells <= 0 || tolscr < 0.0 || max_numdmat <= 0) return GTF_ERR_INVALID;
    gtf_fock_dev *f = new gtf_fock_dev();
    memset(f->tasks, 0, sizeof(f->tasks));
    *out = f;
    int r = upload_basis(f, b);
    if (r) return r;
    f->max_numdmat = max_numdmat;
    f->tolscr = tolscr;
    f->tolscr2 = tolscr * tolscr;
    f->prec = GTF_PREC_FP64;
    f->fp32_cutoff = 0.0;
    const int ns = b->nshells;
    cudaStream_t st = f->stream;
    BasisDev bd{f->d_sh_L, f->d_sh_nprim, f->d_sh_pstart, f->d_sh_xyz, f->d_alpha, f->d_coef, ns, b->pure};

    // ---- Schwarz values of every shell pair (M >= N), one class at a time ----
    const size_t n2 = (size_t)ns * ns;
    DevTemps tmps(st);
    DALLOC(f->d_sq, n2);
    unsigned long long *d_gmax;
    TALLOC(tmps, d_gmax, 1);
    CK(cudaMemsetAsync(d_gmax, 0, sizeof(unsigned long long), st));
    {
        std::vector<int2> mn[NCLS];
        std::vector<int> off[NCLS];
        size_t npp_cls[NCLS] = {0, 0, 0, 0, 0, 0};
        for (int M = 0; M < ns; M++) {
            for (int N = 0; N <= M; N++) {
                const int c = pair_class(b->sh_L[M], b->sh_L[N]);
                mn[c].push_back(make_int2(M, N));
                off[c].push_back((int)npp_cls[c]);
                npp_cls[c] += (size_t)b->sh_nprim[M] * b->sh_nprim[N];
            }
        }
        for (int c = 0; c < NCLS; c++) {
            const int n = (int)mn[c].size();
            if (n == 0) continue;
            int2 *d_mn;
            int *d_off;
            PairRec *d_pr;
            double *d_pp;
            TALLOC(tmps, d_mn, n);
            TALLOC(tmps, d_off, n);
            TALLOC(tmps, d_pr, n);
            TALLOC(tmps, d_pp, 5 * npp_cls[c]);
            CK(cudaMemcpyAsync(d_mn, mn[c].data(), sizeof(int2) * n, cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(d_off, off[c].data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
            k_screen_prep<<<(n + 127) / 128, 128, 0, st>>>(bd, d_mn, d_off, n, d_pr, d_pp, npp_cls[c]);
            CK(cudaGetLastError());
            const size_t np_ = npp_cls[c];
            PrimPairs pps{d_pp, d_pp + np_, d_pp + 2 * np_, d_pp + 3 * np_, d_pp + 4 * np_};
            if (launch_screen(c, d_pr, pps, d_mn, n, ns, b->pure, f->d_sq, d_gmax, st) != 0)
                CK(cudaGetLastError());
            CK(cudaStreamSynchronize(st));
            tmps.drop(d_mn);
            tmps.drop(d_off);
            tmps.drop(d_pr);
            tmps.drop(d_pp);
        }
    }
    unsigned long long hmax = 0;
    CK(cudaMemcpyAsync(&hmax, d_gmax, sizeof(hmax), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    memcpy(&f->maxvalue, &hmax, sizeof(double));
    tmps.drop(d_gmax);
    const double eta = f->tolscr2 / f->maxvalue;

    // ---- reference CSR list (row-major scan + scatter) ----
    int *d_flags, *d_pos;
    TALLOC(tmps, d_flags, n2);
    TALLOC(tmps, d_pos, n2);
    const unsigned g2 = (unsigned)((n2 + 255) / 256);
    k_csr_flags<<<g2, 256, 0, st>>>(f->d_sq, ns, eta, d_flags);
    CK(cudaGetLastError());
    size_t tmp_bytes = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d_flags, d_pos, (int)n2, st));
    char *d_tmp = nullptr;
    size_t tmp_cap = tmp_bytes;
    TALLOC(tmps, d_tmp, tmp_cap);
    CK(cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, d_flags, d_pos, (int)n2, st));
    int last_pos = 0, last_flag = 0;
    CK(cudaMemcpyAsync(&last_pos, d_pos + n2 - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&last_flag, d_flags + n2 - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const int nnz = last_pos + last_flag;
    f->nnz = nnz;
    DALLOC(f->d_shellptr, ns + 1);
    DALLOC(f->d_shellid, nnz);
    DALLOC(f->d_shellrid, nnz);
    DALLOC(f->d_shellvalue, nnz);
    k_csr_scatter<<<g2, 256, 0, st>>>(f->d_sq, d_flags, d_pos, ns, f->d_shellid, f->d_shellrid,
                                      f->d_shellvalue, f->d_shellptr);
    CK(cudaGetLastError());

    // ---- device pair list: sort by class, then value descending ----
    f->npairs = nnz;
    unsigned long long *d_kval, *d_kval2;
    int *d_kcls, *d_kcls2, *d_idx, *d_idx2, *d_pair_n, *d_pair_off, *d_kept;
    TALLOC(tmps, d_kval, nnz);
    TALLOC(tmps, d_kval2, nnz);
    TALLOC(tmps, d_kcls, nnz);
    TALLOC(tmps, d_kcls2, nnz);
    TALLOC(tmps, d_idx, nnz);
    TALLOC(tmps, d_idx2, nnz);
    TALLOC(tmps, d_pair_n, nnz + 1);
    TALLOC(tmps, d_pair_off, nnz + 1);
    TALLOC(tmps, d_kept, nnz);
    const unsigned gp = (unsigned)((nnz + 255) / 256 > 0 ? (nnz + 255) / 256 : 1);
    if (nnz > 0) {
        k_sort_keys<<<gp, 256, 0, st>>>(f->d_shellvalue, f->d_shellid, f->d_shellrid, f->d_sh_L, nnz,
                                        d_kval, d_kcls, d_idx);
        CK(cudaGetLastError());
        k_prim_keep<<<gp, 256, 0, st>>>(f->d_shellid, f->d_shellrid, bd, nnz, d_kept);
        CK(cudaGetLastError());
        size_t b1 = 0, b2 = 0;
        CK(cub::DeviceRadixSort::SortPairs(nullptr, b1, d_kval, d_kval2, d_idx, d_idx2, nnz, 0, 64, st));
        CK(cub::DeviceRadixSort::SortPairs(nullptr, b2, d_kcls, d_kcls2, d_idx2, d_idx, nnz, 0, 7, st));
        size_t need = b1 > b2 ? b1 : b2;
        if (need > tmp_cap) {
            tmps.drop(d_tmp);
            tmp_cap = need;
            TALLOC(tmps, d_tmp, tmp_cap);
        }
        b1 = tmp_cap;
        CK(cub::DeviceRadixSort::SortPairs(d_tmp, b1, d_kval, d_kval2, d_idx, d_idx2, nnz, 0, 64, st));
        k_gather_cls<<<gp, 256, 0, st>>>(d_idx2, f->d_shellid, f->d_shellrid, f->d_sh_L, d_kept, nnz, d_kcls);
        CK(cudaGetLastError());
        b2 = tmp_cap;
        CK(cub::DeviceRadixSort::SortPairs(d_tmp, b2, d_kcls, d_kcls2, d_idx2, d_idx, nnz, 0, 7, st));
    }
    DALLOC(f->d_pairs, nnz);
    DALLOC(f->d_pair_v, nnz);
    if (nnz > 0) {
        k_build_pairs<<<gp, 256, 0, st>>>(d_idx, f->d_shellid, f->d_shellrid, f->d_shellvalue, bd,
                                          f->d_fc_start, nnz, f->d_pairs, f->d_pair_v, d_pair_n);
        CK(cudaGetLastError());
    }
    CK(cudaMemsetAsync(d_pair_n + nnz, 0, sizeof(int), st));
    size_t b3 = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, b3, d_pair_n, d_pair_off, nnz + 1, st));
    if (b3 > tmp_cap) {
        tmps.drop(d_tmp);
        tmp_cap = b3;
        TALLOC(tmps, d_tmp, tmp_cap);
    }
    b3 = tmp_cap;
    CK(cub::DeviceScan::ExclusiveSum(d_tmp, b3, d_pair_n, d_pair_off, nnz + 1, st));
    int npp = 0;
    CK(cudaMemcpyAsync(&npp, d_pair_off + nnz, sizeof(int), cudaMemcpyDeviceToHost, st));
    std::vector<int> cls_sorted(nnz > 0 ? nnz : 1);
    if (nnz > 0)
        CK(cudaMemcpyAsync(cls_sorted.data(), d_kcls2, sizeof(int) * nnz, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    f->nprimpairs = npp;
    DALLOC(f->d_pp, 2 * GTF_PPREC_D2 * (size_t)(npp > 0 ? npp : 1));
    DALLOC(f->d_pp32, 8 * (size_t)(npp > 0 ? npp : 1));
    if (nnz > 0) {
        k_fill_primpairs<<<gp, 256, 0, st>>>(f->d_pairs, d_idx, f->d_shellid, f->d_shellrid, d_pair_off, bd,
                                             nnz, f->d_pp);
        CK(cudaGetLastError());
        k_fill_pp32<<<gp, 256, 0, st>>>(f->d_pairs, nnz, f->d_pp, f->d_pp32);
        CK(cudaGetLastError());
    }
    // class and segment starts from the sorted keys (class * 16 + bucket)
    std::vector<int> key_start(NCLS * 16 + 1, nnz);
    for (int s2 = nnz - 1; s2 >= 0; s2--) key_start[cls_sorted[s2]] = s2;
    for (int k = NCLS * 16 - 1; k >= 0; k--)
        if (key_start[k] > key_start[k + 1]) key_start[k] = key_start[k + 1];
    for (int c = 0; c <= NCLS; c++) f->cls_start[c] = key_start[c * 16];

    // ---- task lists per class pair ----
    f->usq = 0.0;
    f->uitl = 0.0;
    f->eri_flops = 0.0;
    DALLOC(f->d_counters, 2 * NCLSPAIR * GTF_MAX_SLICES);
    int cp = 0;
    for (int X = 0; X < NCLS; X++) {
        for (int Y = 0; Y <= X; Y++, cp++) {
            ClassPairTask &t = f->tasks[cp];
            t.X = X;
            t.Y = Y;
            t.bra_start = f->cls_start[X];
            t.nbra = f->cls_start[X + 1] - f->cls_start[X];
            t.ket_start = f->cls_start[Y];
            t.nketcls = f->cls_start[Y + 1] - f->cls_start[Y];
            for (int bk = 0; bk <= GTF_NBKT; bk++) t.seg[bk] = key_start[Y * 16 + bk] - t.ket_start;
            t.nunits = t.nunits32 = 0;
            t.nquart = t.nquart32 = 0.0;
            if (t.nbra == 0 || t.nketcls == 0) continue;
            const int nidx = t.nbra * GTF_NBKT;
            DALLOC(t.d_nket, nidx);
            DALLOC(t.d_n64, nidx);
            DALLOC(t.d_cum64, (size_t)t.nbra * GTF_CUM);
            DALLOC(t.d_cum32, (size_t)t.nbra * GTF_CUM);
            DALLOC(t.d_unit_prefix, t.nbra + 1);
            DALLOC(t.d_unit_prefix32, t.nbra + 1);
        }
    }
    {
        int r = make_unit_tasks(f);
        if (r == GTF_OK) r = build_units(f);
        if (r != GTF_OK) return r;
    }
    cp = 0;
    for (int X = 0; X < NCLS; X++) {
        for (int Y = 0; Y <= X; Y++, cp++) {
            ClassPairTask &t = f->tasks[cp];
            if (t.nbra == 0 || t.nketcls == 0) continue;
            const double q = t.nquart;
            const int la = k_cls_la[X], lb = k_cls_lb[X], lc = k_cls_la[Y], ld = k_cls_lb[Y];
            const double dims = (double)(b->pure ? (la == 2 ? 5 : ncart(la)) : ncart(la)) *
                                (b->pure ? (lb == 2 ? 5 : ncart(lb)) : ncart(lb)) *
                                (b->pure ? (lc == 2 ? 5 : ncart(lc)) : ncart(lc)) *
                                (b->pure ? (ld == 2 ? 5 : ncart(ld)) : ncart(ld));
            f->usq += q;
            f->uitl += q * dims;
        }
    }
    // primitive pairs per shell pair: the work model's input (evaluated when
    // first asked for, work_model below) and the shard split's
    f->h_pair_n.assign(nnz, 0);
    if (nnz > 0) {
        CK(cudaMemcpyAsync(f->h_pair_n.data(), d_pair_n, sizeof(int) * nnz, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    // the set-up temporaries are released here (tmps) and on every error return

    // ---- matrices ----
    const size_t nn = (size_t)b->nbf * b->nbf, nnc = (size_t)b->nbf_cart * b->nbf_cart;
    DALLOC(f->d_D, nn * max_numdmat);
    DALLOC(f->d_F, nn * max_numdmat);
    DALLOC(f->d_J, nn * max_numdmat);
    DALLOC(f->d_K, nn * max_numdmat);
    DALLOC(f->d_Dc, nnc);
    DALLOC(f->d_Fj, nnc);
    DALLOC(f->d_Fk, nnc);
    CK(cudaMemsetAsync(f->d_D, 0, sizeof(double) * nn * max_numdmat, st));
    CK(cudaMemsetAsync(f->d_F, 0, sizeof(double) * nn * max_numdmat, st));
    CK(cudaMemsetAsync(f->d_J, 0, sizeof(double) * nn * max_numdmat, st));
    CK(cudaMemsetAsync(f->d_K, 0, sizeof(double) * nn * max_numdmat, st));
    f->host_stage_bytes = nn * sizeof(double);
    f->d_host_stage = (double *)gtf_pinned_alloc(f->host_stage_bytes);
    if (!f->d_host_stage) {
        snprintf(g_errbuf, sizeof(g_errbuf), "pinned host buffer of %zu bytes", f->host_stage_bytes);
        return GTF_ERR_ALLOC;
    }
    CK(cudaStreamSynchronize(st));
    return GTF_OK;
}

// Every buffer is freed on the engine's stream after the host has waited for
// it (a batch that used the engine's buffers on its own stream has
// synchronized that stream before destroying the engine).
extern "C" void gtf_fock_destroy(gtf_fock_dev_t *f)
{
    if (!f) return;
    cudaStreamSynchronize(f->stream);
    cudaStream_t st = f->stream;
    void *ptrs[] = {f->d_sh_L, f->d_sh_nprim, f->d_sh_pstart, f->d_f_start, f->d_fc_start, f->d_sph2shell,
                    f->d_cart2shell, f->d_Z, f->d_sh_xyz, f->d_alpha, f->d_coef, f->d_atom_xyz, f->d_sq,
                    f->d_shellptr, f->d_shellid, f->d_shellrid, f->d_shellvalue, f->d_pairs, f->d_pair_v,
                    f->d_pp, f->d_pp32, f->d_counters, f->d_D, f->d_Dc, f->d_Fj, f->d_Fk, f->d_F, f->d_J, f->d_K,
                    f->d_Ds, f->d_Da, f->d_Dca, f->d_Fka, f->d_ut_static, f->d_ut_dyn, f->d_Dprev, f->d_Dd,
                    f->d_dyn, f->d_Dta, f->d_Dcta, f->d_Fja, f->d_Fscr, f->d_unit_tot};
    for (void *p : ptrs) dev_free(p, st);   // all from dalloc
    for (int c = 0; c < NCLSPAIR; c++) {
        dev_free(f->tasks[c].d_nket, st);
        dev_free(f->tasks[c].d_unit_prefix, st);
        dev_free(f->tasks[c].d_n64, st);
        dev_free(f->tasks[c].d_cum64, st);
        dev_free(f->tasks[c].d_cum32, st);
        dev_free(f->tasks[c].d_unit_prefix32, st);
    }
    // the one-electron matrices come from onee.cu's own allocations (the
    // same pool, on this stream)
    void *onee[] = {f->d_S, f->d_X, f->d_H};
    for (void *p : onee) gtf_dfree(p, st);
    gtf_pinned_free(f->d_host_stage);
    // a partly created engine has some of these unset: destroying a null
    // handle would leave a stale error for the next cudaGetLastError
    cudaEvent_t evs[] = {f->ev0, f->ev1, f->ev2, f->ev3};
    for (cudaEvent_t e : evs)
        if (e) cudaEventDestroy(e);
    for (int c = 0; c <= NCLSPAIR; c++)
        if (f->ev_cls[c]) cudaEventDestroy(f->ev_cls[c]);
    if (f->stream) cudaStreamDestroy(f->stream);
    delete f;
}

extern "C" int gtf_fock_screening_info(gtf_fock_dev_t *f, int *nnz, double *maxvalue, double *usq,
                                       double *uitl)
{
    if (nnz) *nnz = f->nnz;
    if (maxvalue) *maxvalue = f->maxvalue;
    if (usq) *usq = f->usq;
    if (uitl) *uitl = f->uitl;
    return GTF_OK;
}

extern "C" int gtf_fock_get_csr(gtf_fock_dev_t *f, int *shellptr, int *shellid, int *shellrid,
                                double *shellvalue)
{
    cudaStream_t st = f->stream;
    if (shellptr)
        CK(cudaMemcpyAsync(shellptr, f->d_shellptr, sizeof(int) * (f->nshells + 1), cudaMemcpyDeviceToHost, st));
    if (f->nnz > 0) {
        if (shellid) CK(cudaMemcpyAsync(shellid, f->d_shellid, sizeof(int) * f->nnz, cudaMemcpyDeviceToHost, st));
        if (shellrid) CK(cudaMemcpyAsync(shellrid, f->d_shellrid, sizeof(int) * f->nnz, cudaMemcpyDeviceToHost, st));
        if (shellvalue)
            CK(cudaMemcpyAsync(shellvalue, f->d_shellvalue, sizeof(double) * f->nnz, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    return GTF_OK;
}

// strided host block <-> device full matrix
static int put_block(gtf_fock_dev *f, double *dmat, int n, int r0, int r1, int c0, int c1, int stride,
                     const double *host)
{
    if (r0 < 0 || c0 < 0 || r1 >= n || c1 >= n || r1 < r0 || c1 < c0 || !host) return GTF_ERR_INVALID;
    const int nr = r1 - r0 + 1, nc = c1 - c0 + 1;
    if (stride < nc) return GTF_ERR_INVALID;   // rows of the host block would overlap
    CK(cudaMemcpy2DAsync(dmat + (size_t)r0 * n + c0, sizeof(double) * n, host, sizeof(double) * stride,
                         sizeof(double) * nc, nr, cudaMemcpyHostToDevice, f->stream));
    CK(cudaStreamSynchronize(f->stream));
    return GTF_OK;
}

static int get_block(gtf_fock_dev *f, const double *dmat, int n, int r0, int r1, int c0, int c1, int stride,
                     double *host)
{
    if (r0 < 0 || c0 < 0 || r1 >= n || c1 >= n || r1 < r0 || c1 < c0 || !host) return GTF_ERR_INVALID;
    const int nr = r1 - r0 + 1, nc = c1 - c0 + 1;
    if (stride < nc) return GTF_ERR_INVALID;   // rows of the host block would overlap
    CK(cudaMemcpy2DAsync(host, sizeof(double) * stride, dmat + (size_t)r0 * n + c0, sizeof(double) * n,
                         sizeof(double) * nc, nr, cudaMemcpyDeviceToHost, f->stream));
    CK(cudaStreamSynchronize(f->stream));
    return GTF_OK;
}

__global__ void k_fill(double *p, size_t n, double v)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

extern "C" int gtf_fock_fill_density(gtf_fock_dev_t *f, int index, double value)
{
    if (index < 0 || index >= f->max_numdmat) return GTF_ERR_INVALID;
    const size_t nn = (size_t)f->nbf * f->nbf;
    k_fill<<<(unsigned)((nn + 255) / 256), 256, 0, f->stream>>>(f->d_D + nn * index, nn, value);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(f->stream));
    return GTF_OK;
}

extern "C" int gtf_fock_put_density(gtf_fock_dev_t *f, int index, int r0, int r1, int c0, int c1, int stride,
                                    const double *host)
{
    if (index < 0 || index >= f->max_numdmat) return GTF_ERR_INVALID;
    const size_t nn = (size_t)f->nbf * f->nbf;
    return put_block(f, f->d_D + nn * index, f->nbf, r0, r1, c0, c1, stride, host);
}

extern "C" int gtf_fock_put_density_dev(gtf_fock_dev_t *f, int index, const double *dev)
{
    if (index < 0 || index >= f->max_numdmat) return GTF_ERR_INVALID;
    const size_t nn = (size_t)f->nbf * f->nbf;
    CK(cudaMemcpyAsync(f->d_D + nn * index, dev, sizeof(double) * nn, cudaMemcpyDeviceToDevice, f->stream));
    return GTF_OK;
}

// Non-symmetric densities (PFock_create with symm = 0): buffers for the
// symmetric and antisymmetric parts and the second exchange accumulator, and
// for the reference's own output the sign-adjusted density and its Coulomb
// accumulator (GTF_NOSYMM_REFERENCE / GTF_NOSYMM_EXACT / off).
extern "C" int gtf_fock_set_nosymm(gtf_fock_dev_t *f, int mode)
{
    if (mode != GTF_NOSYMM_OFF && mode != GTF_NOSYMM_REFERENCE && mode != GTF_NOSYMM_EXACT) {
        snprintf(g_errbuf, sizeof(g_errbuf), "unknown non-symmetric density mode %d", mode);
        return GTF_ERR_INVALID;
    }
    if (mode == GTF_NOSYMM_OFF) {
        f->nosymm = 0;
        return GTF_OK;
    }
    if (f->incr) {
        snprintf(g_errbuf, sizeof(g_errbuf), "non-symmetric densities: incremental builds are on");
        return GTF_ERR_INVALID;
    }
    const size_t nn = (size_t)f->nbf * f->nbf, nnc = (size_t)f->nbf_cart * f->nbf_cart;
    if (!f->d_Fka) {
        DALLOC(f->d_Ds, nn);
        DALLOC(f->d_Da, nn);
        DALLOC(f->d_Dca, nnc);
        DALLOC(f->d_Fka, nnc);
    }
    if (mode == GTF_NOSYMM_REFERENCE && !f->d_Fja) {
        DALLOC(f->d_Dta, nn);
        DALLOC(f->d_Dcta, nnc);
        DALLOC(f->d_Fja, nnc);
        DALLOC(f->d_Fscr, nnc);
    }
    f->nosymm = mode;
    return GTF_OK;
}

// Units [lo, hi) of a class launch that shard r of n computes: contiguous,
// sizes differing by at most one unit (units of one class launch are 32
// quartets of equal class; the pre-sorted ket segments spread the heavy and
// light bras over the range).
extern "C" void gtf_shard_range(long long nunits, int r, int n, long long *lo, long long *hi)
{
    if (n <= 1) {
        *lo = 0;
        *hi = nunits;
        return;
    }
    *lo = nunits * r / n;
    *hi = nunits * (r + 1) / n;
}

// Contiguous split of n weighted items (w[i] >= 0) into nshards: shard r
// gets [lo, hi), lo the first item whose preceding weight reaches W r /
// nshards (W the total).  The shards tile [0, n) in order, each within one
// item's weight of W / nshards; every rank computes the same split from the
// same weights.
extern "C" void gtf_shard_split(const double *w, long long n, int r, int nshards, long long *lo, long long *hi)
{
    if (n <= 0) {
        *lo = *hi = 0;
        return;
    }
    if (nshards <= 1) {
        *lo = 0;
        *hi = n;
        return;
    }
    double W = 0.0;
    for (long long i = 0; i < n; i++) W += w[i];
    const double t0 = W * (double)r / nshards, t1 = W * (double)(r + 1) / nshards;
    long long a = -1, b = -1;
    double pre = 0.0;
    for (long long i = 0; i <= n; i++) {
        if (a < 0 && (r == 0 || pre >= t0)) a = i;
        if (b < 0 && r + 1 < nshards && pre >= t1) b = i;
        if (i < n) pre += w[i];
    }
    *lo = a < 0 ? n : a;
    *hi = (r + 1 == nshards || b < 0) ? n : b;
    if (*hi < *lo) *hi = *lo;
}

// Unit ranges of this engine's shard, per (class pair, part): the bras of
// the launch are split by the work model (primitive quartets x FLOPs per
// primitive quartet + per-quartet contraction and digestion FLOPs), so the
// shards get equal work rather than equal unit counts (a d-class bra with
// 8 primitive pairs costs tens of times an s-class one).  nk / n64: the
// launch's ket counts per (bra, segment) for the current thresholds.
static int shard_bounds(gtf_fock_dev *f, int c, const std::vector<int> &nk, const std::vector<int> &n64)
{
    ClassPairTask &t = f->tasks[c];
    for (int p = 0; p < 2; p++) {
        f->shard_lo[c][p] = 0;
        f->shard_hi[c][p] = p ? t.nunits32 : t.nunits;
    }
    if (t.nbra == 0 || t.nketcls == 0) return GTF_OK;
    if (f->nshards <= 1) {
        f->shard_work += t.flops;
        return GTF_OK;
    }
    const int la = k_cls_la[t.X], lb = k_cls_lb[t.X], lc = k_cls_la[t.Y], ld = k_cls_lb[t.Y];
    double cpart;
    const double per_prim = class_flops_per_prim(t.X, t.Y, &cpart);
    const double ns_ = (double)(f->pure && la == 2 ? 5 : ncart(la)) * (f->pure && lb == 2 ? 5 : ncart(lb)) *
                       (f->pure && lc == 2 ? 5 : ncart(lc)) * (f->pure && ld == 2 ? 5 : ncart(ld));
    std::vector<double> kpre(t.nketcls + 1, 0.0);
    for (int j = 0; j < t.nketcls; j++) kpre[j + 1] = kpre[j] + f->h_pair_n[t.ket_start + j];
    std::vector<long long> up(t.nbra + 1);
    std::vector<double> w(t.nbra);
    for (int p = 0; p < 2; p++) {
        const long long nu = p ? t.nunits32 : t.nunits;
        if (nu == 0) continue;
        CK(cudaMemcpy(up.data(), p ? t.d_unit_prefix32 : t.d_unit_prefix, sizeof(long long) * (t.nbra + 1),
                      cudaMemcpyDeviceToHost));
        for (int i = 0; i < t.nbra; i++) {
            const double kb = f->h_pair_n[t.bra_start + i];
            double wi = 0.0;
            for (int b = 1; b < GTF_NBKT; b++) {   // segment 0 has no units
                const int k = i * GTF_NBKT + b;
                const int j0 = t.seg[b] + (p ? n64[k] : 0), j1 = t.seg[b] + (p ? nk[k] : n64[k]);
                wi += kb * (kpre[j1] - kpre[j0]) * per_prim + (cpart + 12.0 * ns_) * (j1 - j0);
            }
            w[i] = wi;
        }
        long long blo = 0, bhi = 0;
        gtf_shard_split(w.data(), t.nbra, f->shard, f->nshards, &blo, &bhi);
        f->shard_lo[c][p] = up[blo];
        f->shard_hi[c][p] = up[bhi];
        for (long long i = blo; i < bhi; i++) f->shard_work += w[i];
    }
    return GTF_OK;
}

// A sharded build: every class launch of this engine covers shard `shard` of
// `nshards` of its units (contiguous, split by the work model), so the F, J,
// K of the build are this shard's part; the parts of all shards sum to the
// whole build.  nshards <= 1 restores the whole build.
extern "C" int gtf_fock_set_shard(gtf_fock_dev_t *f, int shard, int nshards)
{
    if (nshards < 0 || (nshards > 1 && (shard < 0 || shard >= nshards))) return GTF_ERR_INVALID;
    if (nshards > 1 && f->incr) {
        snprintf(g_errbuf, sizeof(g_errbuf), "a sharded engine cannot use incremental builds");
        return GTF_ERR_INVALID;
    }
    f->shard = nshards > 1 ? shard : 0;
    f->nshards = nshards > 1 ? nshards : 0;
    return build_units(f);   // recomputes the shard's unit ranges
}

// Model FLOPs of this engine's shard of a build (the whole build when not
// sharded): the work the shard split balances.
extern "C" int gtf_fock_shard_work(gtf_fock_dev_t *f, double *work)
{
    if (!f || !work) return GTF_ERR_INVALID;
    if (f->nshards <= 1) {
        const int r = ensure_work_model(f);
        if (r) return r;
    }
    *work = f->nshards > 1 ? f->shard_work : f->eri_flops;
    return GTF_OK;
}

extern "C" int gtf_fock_set_precision(gtf_fock_dev_t *f, int prec, double fp32_cutoff)
{
    if (prec != GTF_PREC_FP64 && prec != GTF_PREC_MIXED) return GTF_ERR_INVALID;
    if (prec == GTF_PREC_MIXED && !(fp32_cutoff >= 0.0)) return GTF_ERR_INVALID;
    f->prec = prec;
    f->fp32_cutoff = fp32_cutoff;
    return build_units(f);
}

// The descriptor of class pair c, part 0 (FP64 head of every ket range) or
// part 1 (FP32 tail), of one engine.
static void fill_launch(const gtf_fock_dev *f, int c, int part, const double *D, double *Fj, double *Fk,
                        FockLaunch &a, int konly = 0)
{
    const ClassPairTask &t = f->tasks[c];
    memset(&a, 0, sizeof(a));
    a.pairs = f->d_pairs;
    a.pprec = reinterpret_cast<const double2 *>(f->d_pp);
    a.pprec32 = reinterpret_cast<const float4 *>(f->d_pp32);
    a.nlo = part ? t.d_n64 : nullptr;
    a.cum = part ? t.d_cum32 : t.d_cum64;
    a.unit_prefix = part ? t.d_unit_prefix32 : t.d_unit_prefix;
    a.nbra = t.nbra;
    a.nunits = part ? t.nunits32 : t.nunits;
    a.bra_start = t.bra_start;
    a.ket_start = t.ket_start;
    for (int b = 0; b <= GTF_NBKT; b++) a.seg[b] = t.seg[b];
    a.D = D;
    a.Fj = Fj;
    a.Fk = Fk;
    a.ld = f->nbf_cart;
    a.konly = konly;
}

// Launches the Fock kernels of class pair c: the FP64 part of every ket
// range, then (mixed precision) the FP32 tail.  counters holds
// GTF_MAX_SLICES zeroed slots per (class pair, part), one per slice launch.
// Returns the number of launches, or -1 on a launch error.
// dyn: the task lists were rebuilt on the device for this build (incremental
// builds): every part that can have work is launched, with its unit count
// read by the kernel and its grid sized for the bound.
static int launch_class(const gtf_fock_dev *f, int c, const double *D, double *Fj, double *Fk,
                        unsigned long long *counters, cudaStream_t st, int konly = 0, bool dyn = false)
{
    const ClassPairTask &t = f->tasks[c];
    int n = 0;
    for (int part = 0; part < 2; part++) {
        const long long nu = dyn ? ((part == 0 || f->prec == GTF_PREC_MIXED) ? t.nunits_bound : 0)
                                 : (part ? t.nunits32 : t.nunits);
        if (nu == 0 || t.nbra == 0 || t.nketcls == 0) continue;
        FockGrid g;
        memset(&g, 0, sizeof(g));
        fill_launch(f, c, part, D, Fj, Fk, g.one, konly);
        g.nmol = 1;
        long long lo = 0, hi = nu;
        if (dyn) {
            g.nunits_dev = (part ? t.d_unit_prefix32 : t.d_unit_prefix) + t.nbra;
        } else if (f->nshards > 1) {
            lo = f->shard_lo[c][part];
            hi = f->shard_hi[c][part];
            if (hi <= lo) continue;
        }
        g.nunits = hi - lo;
        g.unit_lo = lo;
        g.counter = counters + (size_t)(2 * c + part) * GTF_MAX_SLICES;
        g.nsm = f->nsm;
        g.fp32 = part;
        tune_apply(0, t.X, t.Y, part, g);
        const int r = launch_fock(t.X, t.Y, g, st);
        if (r < 0) {
            snprintf(g_errbuf, sizeof(g_errbuf), "Fock kernel launch for class pair (%d,%d)%s failed: %s", t.X, t.Y,
                     part ? " (FP32)" : "", cudaGetErrorString(cudaGetLastError()));
            return -1;
        }
        n += r;
    }
    return n;
}

// One incremental build of density 0 (see k_delta): the change of D since
// the previous build goes through device-rebuilt task lists, and F, J, K
// receive its part (or are overwritten on a full build).
static int fock_compute_incremental(gtf_fock_dev *f)
{
    cudaStream_t st = f->stream;
    const int nbf = f->nbf, nbfc = f->nbf_cart;
    const size_t nn = (size_t)nbf * nbf, nnc = (size_t)nbfc * nbfc;
    const bool need_tr = f->pure && nbfc != nbf;
    const int full = (f->incr_since == 0 || f->incr_since >= f->incr_period) ? 1 : 0;
    const double cut2 = f->prec == GTF_PREC_MIXED ? f->fp32_cutoff * f->fp32_cutoff : 0.0;
    f->lists_dyn = 1;
    CK(cudaEventRecord(f->ev0, st));
    CK(cudaMemsetAsync(&f->d_dyn->dmax_bits, 0, sizeof(unsigned long long), st));
    {
        const size_t nb = (nn + 255) / 256;
        const unsigned g = (unsigned)(nb < (size_t)f->nsm * 8 ? (nb < 1 ? 1 : nb) : (size_t)f->nsm * 8);
        k_delta<<<g, 256, 0, st>>>(f->d_D, f->d_Dprev, f->d_Dd, nn, full, f->d_dyn);
        CK(cudaGetLastError());
    }
    k_dyn_thresholds<<<1, 1, 0, st>>>(f->d_dyn, f->tolscr2, cut2, f->incr_tau * f->incr_tau,
                                      f->prec == GTF_PREC_MIXED ? f->fp32_cutoff * f->fp32_cutoff : 0.0, full);
    CK(cudaGetLastError());
    int r = run_units(f->d_ut_dyn, (int)f->h_ut.size(), f->ut_nidx, f->ut_nbras, f->nsm, st);
    if (r) return r;
    gtf_note_launches(5);
    const double *Dc = f->d_Dd;
    if (need_tr) {
        dim3 g((nbfc + 127) / 128, nbfc);
        k_d_to_cart<<<g, 128, 0, st>>>(f->d_Dd, f->d_Dc, f->d_cart2shell, f->d_sh_L, f->d_f_start, f->d_fc_start,
                                       nbf, nbfc, f->pure);
        CK(cudaGetLastError());
        Dc = f->d_Dc;
        gtf_note_launches(1);
    }
    CK(cudaMemsetAsync(f->d_Fj, 0, sizeof(double) * nnc, st));
    CK(cudaMemsetAsync(f->d_Fk, 0, sizeof(double) * nnc, st));
    CK(cudaMemsetAsync(f->d_counters, 0, sizeof(unsigned long long) * 2 * NCLSPAIR * GTF_MAX_SLICES, st));
    CK(cudaEventRecord(f->ev1, st));
    for (int c = 0; c < NCLSPAIR; c++) {
        CK(cudaEventRecord(f->ev_cls[c], st));
        const int n = launch_class(f, c, Dc, f->d_Fj, f->d_Fk, f->d_counters, st, 0, true);
        if (n < 0) return GTF_ERR_CUDA;
        gtf_note_launches(n);
    }
    CK(cudaEventRecord(f->ev_cls[NCLSPAIR], st));
    CK(cudaEventRecord(f->ev2, st));
    dim3 g2((nbf + 127) / 128, nbf);
    k_f_to_sph<<<g2, 128, 0, st>>>(f->d_Fj, f->d_Fk, f->d_F, f->d_J, f->d_K, f->d_sph2shell, f->d_sh_L,
                                   f->d_f_start, f->d_fc_start, nbf, nbfc, f->pure, nullptr, &f->d_dyn->acc);
    CK(cudaGetLastError());
    gtf_note_launches(1);
    CK(cudaEventRecord(f->ev3, st));
    CK(cudaEventSynchronize(f->ev3));
    float tot = 0.0f, eri = 0.0f;
    CK(cudaEventElapsedTime(&tot, f->ev0, f->ev3));
    CK(cudaEventElapsedTime(&eri, f->ev1, f->ev2));
    for (int c = 0; c < NCLSPAIR; c++) {
        float mc = 0.0f;
        CK(cudaEventElapsedTime(&mc, f->ev_cls[c], f->ev_cls[c + 1]));
        f->ms_cls[c] = mc;
    }
    f->ms_total = tot;
    f->ms_eri = eri;
    f->ms_other = tot - eri;
    f->incr_since = full ? 1 : f->incr_since + 1;
    return GTF_OK;
}

// Incremental builds on (on = 1) or off: tau is the threshold on Schwarz
// bound x max |D_k - D_k-1| below which a quartet of the change is dropped
// (<= 0: the engine's Schwarz threshold), period the number of builds
// between full ones (>= 1; 1 = every build full).  Density 0 only, symmetric
// densities, unsharded engines.  The next build is a full one.
extern "C" int gtf_fock_set_incremental(gtf_fock_dev_t *f, int on, double tau, int period)
{
    if (!f || f->max_numdmat < 1) return GTF_ERR_INVALID;
    if (!on) {
        f->incr = 0;
        return GTF_OK;
    }
    if (f->nosymm || f->nshards > 1 || period < 1) {
        snprintf(g_errbuf, sizeof(g_errbuf), "incremental builds need a symmetric, unsharded engine and period >= 1");
        return GTF_ERR_INVALID;
    }
    if (!f->d_Dprev) {
        const size_t nn = (size_t)f->nbf * f->nbf;
        DALLOC(f->d_Dprev, nn);
        DALLOC(f->d_Dd, nn);
    }
    f->incr = 1;
    f->incr_tau = tau > 0.0 ? tau : f->tolscr;
    f->incr_period = period;
    f->incr_since = 0;
    return GTF_OK;
}

// Statistics of the last incremental build: quartets evaluated in FP64 and in
// FP32, and max |D_k - D_k-1| (0 on a full build).
extern "C" int gtf_fock_incremental_stats(gtf_fock_dev_t *f, double *nq64, double *nq32, double *dmax)
{
    if (!f || !f->d_dyn) return GTF_ERR_INVALID;
    DynState h;
    CK(cudaMemcpyAsync(&h, f->d_dyn, sizeof(h), cudaMemcpyDeviceToHost, f->stream));
    CK(cudaStreamSynchronize(f->stream));
    if (nq64) *nq64 = (double)h.nq64;
    if (nq32) *nq32 = (double)h.nq32;
    if (dmax) *dmax = h.acc ? __longlong_as_double_host(h.dmax_bits) : 0.0;
    return GTF_OK;
}

extern "C" int gtf_fock_compute(gtf_fock_dev_t *f, int numdmat)
{
    if (numdmat <= 0 || numdmat > f->max_numdmat) return GTF_ERR_INVALID;
    if (f->incr && numdmat == 1 && !f->nosymm && f->nshards <= 1) return fock_compute_incremental(f);
    {
        const int r = static_lists(f);
        if (r) return r;
    }
    cudaStream_t st = f->stream;
    const int nbf = f->nbf, nbfc = f->nbf_cart;
    const size_t nn = (size_t)nbf * nbf, nnc = (size_t)nbfc * nbfc;
    const bool need_tr = f->pure && nbfc != nbf;
    CK(cudaEventRecord(f->ev0, st));
    float eri_ms_total = 0.0f;
    for (int d = 0; d < numdmat; d++) {
        const double *D = f->d_D + nn * d;
        if (f->nosymm) {
            // exact 2 J[D] - K[D] for a general D: the symmetric part goes
            // through the usual build, the antisymmetric part only through
            // the exchange terms (it has no Coulomb contribution)
            dim3 g((nbf + 127) / 128, nbf);
            const bool ref = f->nosymm == GTF_NOSYMM_REFERENCE;
            k_split_density<<<g, 128, 0, st>>>(D, f->d_Ds, f->d_Da, nbf, ref ? f->d_Dta : nullptr,
                                               f->d_sph2shell);
            CK(cudaGetLastError());
            gtf_note_launches(1);
            D = f->d_Ds;
        }
        const double *Dc = D;
        if (need_tr) {
            dim3 g((nbfc + 127) / 128, nbfc);
            k_d_to_cart<<<g, 128, 0, st>>>(D, f->d_Dc, f->d_cart2shell, f->d_sh_L, f->d_f_start,
                                           f->d_fc_start, nbf, nbfc, f->pure);
            CK(cudaGetLastError());
            Dc = f->d_Dc;
            gtf_note_launches(1);
        }
        CK(cudaMemsetAsync(f->d_Fj, 0, sizeof(double) * nnc, st));
        CK(cudaMemsetAsync(f->d_Fk, 0, sizeof(double) * nnc, st));
        CK(cudaMemsetAsync(f->d_counters, 0, sizeof(unsigned long long) * 2 * NCLSPAIR * GTF_MAX_SLICES, st));
        CK(cudaEventRecord(f->ev1, st));
        for (int c = 0; c < NCLSPAIR; c++) {
            ClassPairTask &t = f->tasks[c];
            CK(cudaEventRecord(f->ev_cls[c], st));
            (void)t;
            const int r = launch_class(f, c, Dc, f->d_Fj, f->d_Fk, f->d_counters, st);
            if (r < 0) return GTF_ERR_CUDA;
            gtf_note_launches(r);
        }
        if (f->nosymm) {
            const double *Dca = f->d_Da;
            if (need_tr) {
                dim3 g((nbfc + 127) / 128, nbfc);
                k_d_to_cart<<<g, 128, 0, st>>>(f->d_Da, f->d_Dca, f->d_cart2shell, f->d_sh_L, f->d_f_start,
                                               f->d_fc_start, nbf, nbfc, f->pure);
                CK(cudaGetLastError());
                gtf_note_launches(1);
                Dca = f->d_Dca;
            }
            CK(cudaMemsetAsync(f->d_Fka, 0, sizeof(double) * nnc, st));
            CK(cudaMemsetAsync(f->d_counters, 0, sizeof(unsigned long long) * 2 * NCLSPAIR * GTF_MAX_SLICES, st));
            for (int c = 0; c < NCLSPAIR; c++) {
                const int r = launch_class(f, c, Dca, f->d_Fj, f->d_Fka, f->d_counters, st, 1);
                if (r < 0) return GTF_ERR_CUDA;
                gtf_note_launches(r);
            }
        }
        if (f->nosymm == GTF_NOSYMM_REFERENCE) {
            // the reference's orientation-dependent Coulomb part: a plain
            // build of the sign-adjusted Dta, whose exchange part (into the
            // scratch accumulator) is not used
            const double *Dcta = f->d_Dta;
            if (need_tr) {
                dim3 g((nbfc + 127) / 128, nbfc);
                k_d_to_cart<<<g, 128, 0, st>>>(f->d_Dta, f->d_Dcta, f->d_cart2shell, f->d_sh_L, f->d_f_start,
                                               f->d_fc_start, nbf, nbfc, f->pure);
                CK(cudaGetLastError());
                gtf_note_launches(1);
                Dcta = f->d_Dcta;
            }
            CK(cudaMemsetAsync(f->d_Fja, 0, sizeof(double) * nnc, st));
            CK(cudaMemsetAsync(f->d_Fscr, 0, sizeof(double) * nnc, st));
            CK(cudaMemsetAsync(f->d_counters, 0, sizeof(unsigned long long) * 2 * NCLSPAIR * GTF_MAX_SLICES, st));
            for (int c = 0; c < NCLSPAIR; c++) {
                const int r = launch_class(f, c, Dcta, f->d_Fja, f->d_Fscr, f->d_counters, st);
                if (r < 0) return GTF_ERR_CUDA;
                gtf_note_launches(r);
            }
        }
        CK(cudaEventRecord(f->ev_cls[NCLSPAIR], st));
        CK(cudaEventRecord(f->ev2, st));
        dim3 g2((nbf + 127) / 128, nbf);
        k_f_to_sph<<<g2, 128, 0, st>>>(f->d_Fj, f->d_Fk, f->d_F + nn * d, f->d_J + nn * d, f->d_K + nn * d,
                                       f->d_sph2shell, f->d_sh_L, f->d_f_start, f->d_fc_start, nbf, nbfc,
                                       f->pure, f->nosymm ? f->d_Fka : nullptr, nullptr,
                                       f->nosymm == GTF_NOSYMM_REFERENCE ? f->d_Fja : nullptr);
        CK(cudaGetLastError());
        gtf_note_launches(1);
        CK(cudaEventSynchronize(f->ev2));
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, f->ev1, f->ev2));
        eri_ms_total += ms;
        for (int c = 0; c < NCLSPAIR; c++) {
            float mc = 0.0f;
            CK(cudaEventElapsedTime(&mc, f->ev_cls[c], f->ev_cls[c + 1]));
            f->ms_cls[c] = (d == 0 ? 0.0 : f->ms_cls[c]) + mc;
        }
    }
    CK(cudaEventRecord(f->ev3, st));
    CK(cudaEventSynchronize(f->ev3));
    float tot = 0.0f;
    CK(cudaEventElapsedTime(&tot, f->ev0, f->ev3));
    f->ms_total = tot;
    f->ms_eri = eri_ms_total;
    f->ms_other = tot - eri_ms_total;
    return GTF_OK;
}

// Tunes the launch shapes of every class pair and precision part of this
// engine on its current density (one build first, so the Cartesian density
// is in place); the next build clears what the trial launches accumulated.
extern "C" int gtf_fock_autotune(gtf_fock_dev_t *f, int reps)
{
    if (reps < 1) reps = 1;
    if (f->nosymm) return GTF_ERR_INVALID;
    const int incr = f->incr;
    f->incr = 0;   // tune on a plain build (static task lists)
    int r = gtf_fock_compute(f, 1);
    f->incr = incr;
    if (incr) f->incr_since = 0;   // the plain build replaced F: restart the sum
    if (r != GTF_OK) return r;
    cudaStream_t st = f->stream;
    const bool need_tr = f->pure && f->nbf_cart != f->nbf;
    const double *Dc = need_tr ? f->d_Dc : f->d_D;
    for (int c = 0; c < NCLSPAIR; c++) {
        const ClassPairTask &t = f->tasks[c];
        for (int part = 0; part < 2; part++) {
            const long long nu = part ? t.nunits32 : t.nunits;
            if (nu == 0) continue;
            FockGrid g;
            memset(&g, 0, sizeof(g));
            fill_launch(f, c, part, Dc, f->d_Fj, f->d_Fk, g.one);
            g.nmol = 1;
            g.nunits = nu;
            g.counter = f->d_counters + (size_t)(2 * c + part) * GTF_MAX_SLICES;
            g.nsm = f->nsm;
            g.fp32 = part;
            if (tune_launch(0, t.X, t.Y, part, g, st, reps, f->ev0, f->ev1) < 0.0) {
                snprintf(g_errbuf, sizeof(g_errbuf), "autotuning class pair (%d,%d) failed: %s", t.X, t.Y,
                         cudaGetErrorString(cudaGetLastError()));
                return GTF_ERR_CUDA;
            }
        }
    }
    return GTF_OK;
}

extern "C" const double *gtf_fock_mat_dev(gtf_fock_dev_t *f, int type, int index)
{
    const size_t nn = (size_t)f->nbf * f->nbf;
    if (index < 0 || index >= f->max_numdmat) return nullptr;
    switch (type) {
        case 0: return f->d_D + nn * index;
        case 1: return f->d_F + nn * index;
        case 2: return f->d_J + nn * index;
        case 3: return f->d_K + nn * index;
    }
    return nullptr;
}

extern "C" int gtf_fock_get_mat(gtf_fock_dev_t *f, int type, int index, int r0, int r1, int c0, int c1,
                                int stride, double *host)
{
    const double *m = gtf_fock_mat_dev(f, type, index);
    if (!m) return GTF_ERR_INVALID;
    return get_block(f, m, f->nbf, r0, r1, c0, c1, stride, host);
}

extern "C" int gtf_fock_last_timing(gtf_fock_dev_t *f, double *ms_total, double *ms_eri, double *ms_other)
{
    if (ms_total) *ms_total = f->ms_total;
    if (ms_eri) *ms_eri = f->ms_eri;
    if (ms_other) *ms_other = f->ms_other;
    return GTF_OK;
}

// per class pair of the last build: (X, Y) classes, ms, quartets, Rys-model FLOPs
extern "C" int gtf_fock_class_stats(gtf_fock_dev_t *f, int *X, int *Y, double *ms, double *nquart)
{
    for (int c = 0; c < NCLSPAIR; c++) {
        if (X) X[c] = f->tasks[c].X;
        if (Y) Y[c] = f->tasks[c].Y;
        if (ms) ms[c] = f->ms_cls[c];
        if (nquart) nquart[c] = f->tasks[c].nquart;
    }
    return NCLSPAIR;
}

// Per class pair: Rys-model FLOPs and primitive quartets of one build after
// primitive screening (the primitive quartets the kernels evaluate, counted
// by k_count_primq on the static task lists; the per-quartet contraction and
// digestion terms as in gtf_fock_class_work).
extern "C" int gtf_fock_class_work_screened(gtf_fock_dev_t *f, double *flops, double *nprimq)
{
    int r = static_lists(f);
    if (r) return r;
    const int nt = (int)f->h_ut.size();
    std::vector<double> cnt(nt > 0 ? nt : 1, 0.0);
    if (nt > 0) {
        DevTemps tmps(f->stream);
        double *d_out;
        TALLOC(tmps, d_out, nt);
        CK(cudaMemsetAsync(d_out, 0, sizeof(double) * nt, f->stream));
        const long long g = (f->ut_nidx + 255) / 256;
        const unsigned grid = (unsigned)(g < (long long)f->nsm * 16 ? (g < 1 ? 1 : g) : (long long)f->nsm * 16);
        k_count_primq<<<grid, 256, 0, f->stream>>>(f->d_ut_static, nt, f->ut_nidx, f->d_pairs, f->d_pp, d_out);
        CK(cudaGetLastError());
        gtf_note_launches(1);
        CK(cudaMemcpyAsync(cnt.data(), d_out, sizeof(double) * nt, cudaMemcpyDeviceToHost, f->stream));
        CK(cudaStreamSynchronize(f->stream));
    }
    int k = 0;
    for (int c = 0; c < NCLSPAIR; c++) {
        const ClassPairTask &t = f->tasks[c];
        double q = 0.0, fl = 0.0;
        if (t.nbra > 0 && t.nketcls > 0) {
            q = cnt[k++];
            double cpart;
            const double per_prim = class_flops_per_prim(t.X, t.Y, &cpart);
            const int la = k_cls_la[t.X], lb = k_cls_lb[t.X], lc = k_cls_la[t.Y], ld = k_cls_lb[t.Y];
            const double ns_ = (double)(f->pure && la == 2 ? 5 : ncart(la)) * (f->pure && lb == 2 ? 5 : ncart(lb)) *
                               (f->pure && lc == 2 ? 5 : ncart(lc)) * (f->pure && ld == 2 ? 5 : ncart(ld));
            fl = q * per_prim + (cpart + 12.0 * ns_) * t.nquart;
        }
        if (flops) flops[c] = fl;
        if (nprimq) nprimq[c] = q;
    }
    return NCLSPAIR;
}

extern "C" int gtf_fock_class_work(gtf_fock_dev_t *f, double *flops, double *nprimq)
{
    const int r = ensure_work_model(f);
    if (r) return r;   // negative
    for (int c = 0; c < NCLSPAIR; c++) {
        if (flops) flops[c] = f->tasks[c].flops;
        if (nprimq) nprimq[c] = f->tasks[c].nprimq;
    }
    return NCLSPAIR;
}

extern "C" int gtf_fock_fp32_quartets(gtf_fock_dev_t *f, double *nq32, double *nq)
{
    double a = 0.0, b = 0.0;
    for (int c = 0; c < NCLSPAIR; c++) {
        a += f->tasks[c].nquart32;
        b += f->tasks[c].nquart;
    }
    if (nq32) *nq32 = a;
    if (nq) *nq = b;
    return GTF_OK;
}

extern "C" int gtf_fock_eri_flops(gtf_fock_dev_t *f, double *flops)
{
    const int r = ensure_work_model(f);
    *flops = f->eri_flops;
    return r;
}

extern "C" void *gtf_fock_stream(gtf_fock_dev_t *f) { return (void *)f->stream; }
extern "C" size_t gtf_fock_device_bytes(gtf_fock_dev_t *f) { return f->dev_bytes; }

// one-electron matrices live in onee.cu; these accessors need the struct
extern "C" int gtf_onee_compute(gtf_fock_dev_t *f, int want_sx, int want_h, double **S, double **X, double **H);

extern "C" int gtf_fock_one_electron(gtf_fock_dev_t *f, int want_sx, int want_h)
{
    return gtf_onee_compute(f, want_sx, want_h, &f->d_S, &f->d_X, &f->d_H);
}

extern "C" const double *gtf_fock_onee_dev(gtf_fock_dev_t *f, int which)
{
    return which == 0 ? f->d_S : which == 1 ? f->d_X : which == 2 ? f->d_H : nullptr;
}

extern "C" int gtf_fock_get_onee(gtf_fock_dev_t *f, int which, int r0, int r1, int c0, int c1, int stride,
                                 double *host)
{
    const double *m = gtf_fock_onee_dev(f, which);
    if (!m) return GTF_ERR_INVALID;
    return get_block(f, m, f->nbf, r0, r1, c0, c1, stride, host);
}

extern "C" void gtf_fock_release_onee(gtf_fock_dev_t *f, int which)
{
    double **p = which == 0 ? &f->d_S : which == 1 ? &f->d_X : &f->d_H;
    if (*p) {
        cudaStreamSynchronize(f->stream);
        gtf_dfree(*p, f->stream);
        *p = nullptr;
    }
}

// angular momentum of each shell, host copy (onee.cu groups shell pairs by class)
extern "C" const int *gtf_fock_shell_L_host(gtf_fock_dev_t *f) { return f->h_sh_L.data(); }

// basis arrays for onee.cu
extern "C" void gtf_fock_basis_dev(gtf_fock_dev_t *f, const int **sh_L, const int **sh_nprim,
                                   const int **sh_pstart, const int **f_start, const int **fc_start,
                                   const double **sh_xyz, const double **alpha, const double **coef,
                                   const int **Z, const double **atom_xyz, int *nshells, int *natoms, int *nbf,
                                   int *pure)
{
    *sh_L = f->d_sh_L;
    *sh_nprim = f->d_sh_nprim;
    *sh_pstart = f->d_sh_pstart;
    *f_start = f->d_f_start;
    *fc_start = f->d_fc_start;
    *sh_xyz = f->d_sh_xyz;
    *alpha = f->d_alpha;
    *coef = f->d_coef;
    *Z = f->d_Z;
    *atom_xyz = f->d_atom_xyz;
    *nshells = f->nshells;
    *natoms = f->natoms;
    *nbf = f->nbf;
    *pure = f->pure;
}

// ---------------------------------------------------------------------------
// Allocation-free Fock build
//
// Some callers cannot allocate device memory once they are running: a host
// that hands every byte of the GPU to its own pool allocator, a real-time
// loop that must not block on the driver's allocator, or a plugin whose
// host process forbids new allocations after start-up.  For them this
// variant of gtf_fock_compute keeps its scratch -- Cartesian D, the Coulomb
// and exchange accumulators, spherical J and K, and the per-class unit
// counters -- in one file-scope device array instead of the engine's
// buffers.  The engine itself (pair lists, primitive pairs, task lists) is
// still built by gtf_fock_create.
//
// Limits and sharing:
//   * at most GTF_FIXED_MAX_FUNCS Cartesian (and spherical) functions;
//     larger bases are rejected with GTF_ERR_INVALID and a message;
//   * the array (about 5.9 MB) exists on every GPU that loads the library,
//     for the life of the process;
//   * every call on a device uses the same array, so calls whose work
//     overlaps on that GPU (two streams, two threads, two engines) race;
//     callers must order them;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress, with that device current); make that first call
//     before any stream capture;
//   * the accumulators and counters are cleared on every call (stream-ordered
//     cudaMemsetAsync), so results never depend on the previous call.
// ---------------------------------------------------------------------------
#define GTF_FIXED_MAX_FUNCS 384
#define GTF_FIXED_NN ((size_t)GTF_FIXED_MAX_FUNCS * GTF_FIXED_MAX_FUNCS)
#define GTF_FIXED_DOUBLES (5 * GTF_FIXED_NN + 2 * NCLSPAIR * GTF_MAX_SLICES + 3)
#define GTF_FIXED_MAX_DEVICES 64

static __device__ __align__(256) double g_fixed_scratch[GTF_FIXED_DOUBLES];

static double *g_fixed_ptr[GTF_FIXED_MAX_DEVICES];
static pthread_mutex_t g_fixed_lock = PTHREAD_MUTEX_INITIALIZER;

// device address of g_fixed_scratch on the current device (looked up once)
static int fixed_scratch(int dev, double **out)
{
    if (dev < 0 || dev >= GTF_FIXED_MAX_DEVICES) return GTF_ERR_INVALID;
    pthread_mutex_lock(&g_fixed_lock);
    if (g_fixed_ptr[dev] == nullptr) {
        double *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void **)&p, g_fixed_scratch);
        if (e != cudaSuccess || p == nullptr) {
            pthread_mutex_unlock(&g_fixed_lock);
            snprintf(g_errbuf, sizeof(g_errbuf), "cudaGetSymbolAddress(g_fixed_scratch): %s",
                     cudaGetErrorString(e));
            return GTF_ERR_CUDA;
        }
        g_fixed_ptr[dev] = p;
    }
    *out = g_fixed_ptr[dev];
    pthread_mutex_unlock(&g_fixed_lock);
    return GTF_OK;
}

extern "C" int gtf_fock_compute_fixed(gtf_fock_dev_t *f, const double *dev_D, double *dev_F)
{
    if (f == nullptr || dev_D == nullptr || dev_F == nullptr || f->max_numdmat <= 0) return GTF_ERR_INVALID;
    if (f->nosymm) {
        snprintf(g_errbuf, sizeof(g_errbuf), "allocation-free Fock build: non-symmetric densities are not supported");
        return GTF_ERR_INVALID;
    }
    if (f->nshards > 1) {
        // the launches of a sharded engine cover one shard's units only; this
        // entry point promises the whole F
        snprintf(g_errbuf, sizeof(g_errbuf), "allocation-free Fock build: engine is sharded (%d of %d)", f->shard,
                 f->nshards);
        return GTF_ERR_INVALID;
    }
    const int nbf = f->nbf, nbfc = f->nbf_cart;
    if (nbfc > GTF_FIXED_MAX_FUNCS || nbf > GTF_FIXED_MAX_FUNCS) {
        snprintf(g_errbuf, sizeof(g_errbuf),
                 "allocation-free Fock build: basis has %d Cartesian functions, limit is %d", nbfc,
                 GTF_FIXED_MAX_FUNCS);
        return GTF_ERR_INVALID;
    }
    int dev = -1;
    CK(cudaGetDevice(&dev));
    if (dev != f->dev) {
        snprintf(g_errbuf, sizeof(g_errbuf), "allocation-free Fock build: current device %d, engine on %d", dev,
                 f->dev);
        return GTF_ERR_INVALID;
    }
    double *scr = nullptr;
    int r = fixed_scratch(dev, &scr);
    if (r == GTF_OK) r = static_lists(f);
    if (r) return r;
    cudaStream_t st = f->stream;
    const size_t nn = (size_t)nbf * nbf, nnc = (size_t)nbfc * nbfc;
    double *Dc = scr;
    double *Fj = scr + GTF_FIXED_NN;
    double *Fk = scr + 2 * GTF_FIXED_NN;
    double *J = scr + 3 * GTF_FIXED_NN;
    double *K = scr + 4 * GTF_FIXED_NN;
    unsigned long long *counters = (unsigned long long *)(scr + 5 * GTF_FIXED_NN);
    const bool need_tr = f->pure && nbfc != nbf;
    const double *Duse = dev_D;
    if (need_tr) {
        dim3 g((nbfc + 127) / 128, nbfc);
        k_d_to_cart<<<g, 128, 0, st>>>(dev_D, Dc, f->d_cart2shell, f->d_sh_L, f->d_f_start, f->d_fc_start, nbf,
                                       nbfc, f->pure);
        CK(cudaGetLastError());
        Duse = Dc;
    }
    CK(cudaMemsetAsync(Fj, 0, sizeof(double) * nnc, st));
    CK(cudaMemsetAsync(Fk, 0, sizeof(double) * nnc, st));
    CK(cudaMemsetAsync(counters, 0, sizeof(unsigned long long) * 2 * NCLSPAIR * GTF_MAX_SLICES, st));
    for (int c = 0; c < NCLSPAIR; c++)
        if (launch_class(f, c, Duse, Fj, Fk, counters, st) < 0) return GTF_ERR_CUDA;
    dim3 g2((nbf + 127) / 128, nbf);
    k_f_to_sph<<<g2, 128, 0, st>>>(Fj, Fk, dev_F, J, K, f->d_sph2shell, f->d_sh_L, f->d_f_start, f->d_fc_start,
                                   nbf, nbfc, f->pure);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    (void)nn;
    return GTF_OK;
}

// ---------------------------------------------------------------------------
// Batched Fock builds: many engines (molecules of any size) share one launch
// per (class pair, precision part, slice); pre- and post-transforms run as one
// kernel over all molecules.  Each engine reads its D from its own density
// buffer (gtf_fock_mat_dev(f, 0, 0)) and leaves F, J, K in its own result
// buffers, as gtf_fock_compute does.
// ---------------------------------------------------------------------------
struct XformDesc {
    const double *D;
    double *Dc, *Fj, *Fk, *F, *J, *K;
    const int *cart2shell, *sph2shell, *sh_L, *f_start, *fc_start;
    const int *acc;   // incremental builds: add to the previous result when *acc (null: overwrite)
    int nbf, nbfc, pure, need_tr;
};

// Incremental builds of a batch: per molecule, the density change and the
// thresholds (see k_delta); full[m] (written by the host before each build)
// selects a full build of molecule m.
struct DeltaDesc {
    const double *D;
    double *Dprev, *Dd;
    DynState *dyn;
    size_t n;
    double tol2, cut2, tau2, c2;
};

__global__ void k_b_dzero(const DeltaDesc *__restrict__ ds, int M)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < M) ds[m].dyn->dmax_bits = 0ULL;
}

// molecule blockIdx.y
__global__ void k_b_delta(const DeltaDesc *__restrict__ ds, const int *__restrict__ full)
{
    const DeltaDesc &d = ds[blockIdx.y];
    delta_range(d.D, d.Dprev, d.Dd, d.n, full[blockIdx.y], d.dyn, (size_t)blockIdx.x * blockDim.x + threadIdx.x,
                (size_t)gridDim.x * blockDim.x);
}

__global__ void k_b_thresholds(const DeltaDesc *__restrict__ ds, const int *__restrict__ full, int M)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < M) dyn_thresholds(ds[m].dyn, ds[m].tol2, ds[m].cut2, ds[m].tau2, ds[m].c2, full[m]);
}

// The unit prefix over the molecules of each batched launch, from the
// molecules' unit totals of this build (one thread per launch).
struct PrefixDesc {
    const long long *const *tot;   // [n] pointers to the members' totals
    long long *prefix;             // [n + 1]
    int n;
};

__global__ void k_b_molprefix(const PrefixDesc *__restrict__ ps, int np)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= np) return;
    const PrefixDesc p = ps[k];
    long long a = 0;
    p.prefix[0] = 0;
    for (int m = 0; m < p.n; m++) {
        a += *p.tot[m];
        p.prefix[m + 1] = a;
    }
}

// molecule blockIdx.z: Dc = T D T^T (when spherical), Fj = Fk = 0
__global__ void k_b_prep(const XformDesc *__restrict__ xs)
{
    const XformDesc x = xs[blockIdx.z];
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    for (int i = blockIdx.y; i < x.nbfc; i += gridDim.y) {
        if (j >= x.nbfc) continue;
        const size_t o = (size_t)i * x.nbfc + j;
        x.Fj[o] = 0.0;
        x.Fk[o] = 0.0;
        if (x.need_tr) d_to_cart_elem(x.D, x.Dc, x.cart2shell, x.sh_L, x.f_start, x.fc_start, x.nbf, x.nbfc, x.pure, i, j);
    }
}

// molecule blockIdx.z: symmetrise and transform back, F = J + K
__global__ void k_b_post(const XformDesc *__restrict__ xs)
{
    const XformDesc x = xs[blockIdx.z];
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    for (int m = blockIdx.y; m < x.nbf; m += gridDim.y) {
        if (n >= x.nbf) continue;
        f_to_sph_elem(x.Fj, x.Fk, x.F, x.J, x.K, x.sph2shell, x.sh_L, x.f_start, x.fc_start, x.nbf, x.nbfc, x.pure,
                      m, n, nullptr, x.acc != nullptr && *x.acc != 0);
    }
}

struct gtf_fock_batch {
    int M;
    std::vector<gtf_fock_dev *> eng;
    cudaStream_t st;
    int nsm, maxn, maxnc;
    XformDesc *d_xf;
    FockLaunch *d_desc[NCLSPAIR][2];
    long long *d_prefix[NCLSPAIR][2];
    FockLaunch one[NCLSPAIR][2];
    int nmol[NCLSPAIR][2];
    long long total[NCLSPAIR][2];
    // molecules with at least GTF_SOLO_UNITS units in a (class pair, part)
    // run there as launches of their own with the single-molecule kernel
    std::vector<FockLaunch> solo[NCLSPAIR][2];
    std::vector<long long> solo_units[NCLSPAIR][2];
    int solo_base[NCLSPAIR][2];     // first counter block of the part's solo launches
    int ncounter_blocks;            // GTF_MAX_SLICES counters each
    unsigned long long *d_counters;
    // incremental builds (every engine has them on): task lists rebuilt on
    // the device each build, unit counts read by the kernels
    int dyn;
    DeltaDesc *d_delta;
    int *d_full, *h_full;
    UnitTask *d_ut;
    int ut_n;
    long long ut_nidx, ut_nbras;
    PrefixDesc *d_pdesc;
    const long long **d_ptot;
    int npdesc;
    size_t maxnn;
    std::vector<const long long *> solo_tot[NCLSPAIR][2];
};

// A molecule whose units in one launch reach this many (32 quartets each)
// fills the GPU by itself for ~70 rounds of its resident warps; it then runs
// with the single-molecule kernel, which keeps its descriptor in the kernel
// parameters (the batched kernel reads it from memory and holds the molecule
// offset, at 50-60 more bytes of spills; measured 17% slower on 2-3 copies of
// C54H18 or (H2O)64).  At 32768 units the tails and the serial order of many
// medium solo launches cost more than that (256-molecule batch: -16%).  The
// environment variable GTFOCK_SOLO_UNITS replaces both rules by "solo when a
// launch has at least that many units" (tests, measurements).
#define GTF_SOLO_UNITS 262144
// A molecule with at least GTF_SOLO_MOL_UNITS units over all its launches
// (C54H18 / cc-pVDZ: 13.4M; the molecules of the 256-molecule batch: below
// 0.7M) is large enough that all its launches of at least GTF_SOLO_MIN_UNITS
// run solo: it then runs as fast as a build of its own.
#define GTF_SOLO_MOL_UNITS 2000000LL
#define GTF_SOLO_MIN_UNITS 4096

// Returns the per-launch threshold; *overridden is set when the environment
// variable gives it, which also turns off the per-molecule rule below.
static long long solo_units_threshold(bool *overridden)
{
    *overridden = false;
    const char *e = getenv("GTFOCK_SOLO_UNITS");
    if (e && *e) {
        const long long v = atoll(e);
        if (v >= 1) {
            *overridden = true;
            return v;
        }
    }
    return GTF_SOLO_UNITS;
}

// The descriptors live in the device's stream-ordered pool (devmem.cu) and
// are freed on the batch's stream after the host has waited for it.
extern "C" void gtf_fock_batch_destroy(gtf_fock_batch_t *b)
{
    if (!b) return;
    cudaStreamSynchronize(b->st);
    cudaStream_t st = b->st;
    void *ptrs[] = {b->d_xf, b->d_counters, b->d_delta, b->d_full, b->d_ut, b->d_pdesc, b->d_ptot};
    for (void *p : ptrs) gtf_dfree(p, st);
    gtf_pinned_free(b->h_full);
    for (int c = 0; c < NCLSPAIR; c++)
        for (int p = 0; p < 2; p++) {
            gtf_dfree(b->d_desc[c][p], st);
            gtf_dfree(b->d_prefix[c][p], st);
        }
    delete b;
}

#define CKB_(call)                                                                        \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            snprintf(g_errbuf, sizeof(g_errbuf), "%s:%d %s: %s", __FILE__, __LINE__, #call, \
                     cudaGetErrorString(e_));                                             \
            gtf_fock_batch_destroy(b);                                                    \
            return GTF_ERR_CUDA;                                                          \
        }                                                                                 \
    } while (0)

// The engines must live on the current device and outlive the batch; their
// precision modes are read now (rebuild the batch after changing one).
extern "C" int gtf_fock_batch_create(gtf_fock_dev_t *const *engines, int M, void *stream, gtf_fock_batch_t **out)
{
    *out = nullptr;
    if (M <= 0 || !engines) return GTF_ERR_INVALID;
    gtf_fock_batch *b = new gtf_fock_batch();
    memset(b->d_desc, 0, sizeof(b->d_desc));
    memset(b->d_prefix, 0, sizeof(b->d_prefix));
    b->d_xf = nullptr;
    b->d_counters = nullptr;
    b->dyn = 0;
    b->d_delta = nullptr;
    b->d_full = b->h_full = nullptr;
    b->d_ut = nullptr;
    b->d_pdesc = nullptr;
    b->d_ptot = nullptr;
    b->npdesc = 0;
    b->ut_n = 0;
    b->maxnn = 0;
    b->M = M;
    // incremental builds are all or nothing in a batch
    {
        int ninc = 0;
        for (int m = 0; m < M; m++) ninc += (engines[m] && engines[m]->incr) ? 1 : 0;
        if (ninc != 0 && ninc != M) {
            snprintf(g_errbuf, sizeof(g_errbuf), "batch mixes engines with and without incremental builds");
            delete b;
            return GTF_ERR_INVALID;
        }
        b->dyn = ninc == M;
        for (int m = 0; m < M; m++) {
            if (!engines[m]) continue;
            if (b->dyn) {
                engines[m]->lists_dyn = 1;
            } else if (static_lists(engines[m]) != GTF_OK) {
                delete b;
                return GTF_ERR_CUDA;
            }
        }
    }
    b->eng.assign(engines, engines + M);
    b->st = (cudaStream_t)stream;
    b->nsm = engines[0]->nsm;
    b->maxn = b->maxnc = 0;
    std::vector<XformDesc> xf(M);
    for (int m = 0; m < M; m++) {
        gtf_fock_dev *f = engines[m];
        if (!f || f->max_numdmat < 1) {
            gtf_fock_batch_destroy(b);
            return GTF_ERR_INVALID;
        }
        XformDesc &x = xf[m];
        memset(&x, 0, sizeof(x));
        x.D = b->dyn ? f->d_Dd : f->d_D;
        x.acc = b->dyn ? &f->d_dyn->acc : nullptr;
        x.Dc = f->d_Dc;
        x.Fj = f->d_Fj;
        x.Fk = f->d_Fk;
        x.F = f->d_F;
        x.J = f->d_J;
        x.K = f->d_K;
        x.cart2shell = f->d_cart2shell;
        x.sph2shell = f->d_sph2shell;
        x.sh_L = f->d_sh_L;
        x.f_start = f->d_f_start;
        x.fc_start = f->d_fc_start;
        x.nbf = f->nbf;
        x.nbfc = f->nbf_cart;
        x.pure = f->pure;
        x.need_tr = f->pure && f->nbf_cart != f->nbf;
        if (f->nbf > b->maxn) b->maxn = f->nbf;
        if (f->nbf_cart > b->maxnc) b->maxnc = f->nbf_cart;
    }
    CKB_(gtf_dmalloc((void **)&b->d_xf, sizeof(XformDesc) * M, b->st));
    CKB_(cudaMemcpyAsync(b->d_xf, xf.data(), sizeof(XformDesc) * M, cudaMemcpyHostToDevice, b->st));
    int nblocks = 2 * NCLSPAIR;
    bool solo_env = false;
    const long long solo_min = solo_units_threshold(&solo_env);
    std::vector<char> big(M, 0);
    for (int m = 0; m < M && !solo_env; m++) {
        long long tot = 0;
        for (int c = 0; c < NCLSPAIR; c++) tot += engines[m]->tasks[c].nunits + engines[m]->tasks[c].nunits32;
        big[m] = tot >= GTF_SOLO_MOL_UNITS;
    }
    // (incremental batches) the members' unit totals, per batched launch
    std::vector<PrefixDesc> pdesc;
    std::vector<std::vector<const long long *>> ptot;
    std::vector<int> pdesc_cp;
    for (int c = 0; c < NCLSPAIR; c++)
        for (int p = 0; p < 2; p++) {
            std::vector<FockLaunch> d;
            std::vector<long long> pre(1, 0);
            std::vector<const long long *> tots;
            b->solo_base[c][p] = nblocks;
            for (int m = 0; m < M; m++) {
                gtf_fock_dev *f = engines[m];
                const ClassPairTask &t = f->tasks[c];
                // incremental: every part that can have work, sized by its bound
                const long long nu = b->dyn ? ((p == 0 || f->prec == GTF_PREC_MIXED) ? t.nunits_bound : 0)
                                            : (p ? t.nunits32 : t.nunits);
                if (nu == 0 || t.nbra == 0 || t.nketcls == 0) continue;
                const bool need_tr = f->pure && f->nbf_cart != f->nbf;
                FockLaunch a;
                fill_launch(f, c, p, need_tr ? f->d_Dc : (b->dyn ? f->d_Dd : f->d_D), f->d_Fj, f->d_Fk, a);
                const long long *tot = (p ? t.d_unit_prefix32 : t.d_unit_prefix) + t.nbra;
                if (M > 1 && (nu >= solo_min || (big[m] && nu >= GTF_SOLO_MIN_UNITS))) {
                    b->solo[c][p].push_back(a);
                    b->solo_units[c][p].push_back(nu);
                    b->solo_tot[c][p].push_back(tot);
                    nblocks++;
                    continue;
                }
                d.push_back(a);
                pre.push_back(pre.back() + nu);
                tots.push_back(tot);
            }
            b->nmol[c][p] = (int)d.size();
            b->total[c][p] = pre.back();
            if (d.empty()) continue;
            b->one[c][p] = d[0];
            CKB_(gtf_dmalloc((void **)&b->d_desc[c][p], sizeof(FockLaunch) * d.size(), b->st));
            CKB_(gtf_dmalloc((void **)&b->d_prefix[c][p], sizeof(long long) * pre.size(), b->st));
            CKB_(cudaMemcpyAsync(b->d_desc[c][p], d.data(), sizeof(FockLaunch) * d.size(), cudaMemcpyHostToDevice, b->st));
            CKB_(cudaMemcpyAsync(b->d_prefix[c][p], pre.data(), sizeof(long long) * pre.size(), cudaMemcpyHostToDevice, b->st));
            if (b->dyn) {
                PrefixDesc q;
                q.tot = nullptr;
                q.prefix = b->d_prefix[c][p];
                q.n = (int)tots.size();
                pdesc.push_back(q);
                ptot.push_back(tots);
            }
        }
    if (b->dyn) {
        // per-molecule delta descriptors and the concatenated task set
        std::vector<DeltaDesc> dd(M);
        std::vector<UnitTask> ut;
        long long nidx = 0, nbras = 0;
        for (int m = 0; m < M; m++) {
            gtf_fock_dev *f = engines[m];
            DeltaDesc &x = dd[m];
            x.D = f->d_D;
            x.Dprev = f->d_Dprev;
            x.Dd = f->d_Dd;
            x.dyn = f->d_dyn;
            x.n = (size_t)f->nbf * f->nbf;
            x.tol2 = f->tolscr2;
            x.cut2 = f->prec == GTF_PREC_MIXED ? f->fp32_cutoff * f->fp32_cutoff : 0.0;
            x.tau2 = f->incr_tau * f->incr_tau;
            x.c2 = x.cut2;
            if (x.n > b->maxnn) b->maxnn = x.n;
            for (const UnitTask &u0 : f->h_ut) {
                UnitTask u = u0;
                u.dyn = f->d_dyn;
                u.idx0 = nidx;
                u.bra0 = nbras;
                nidx += (long long)u.nbra * GTF_NBKT;
                nbras += u.nbra;
                ut.push_back(u);
            }
        }
        b->ut_n = (int)ut.size();
        b->ut_nidx = nidx;
        b->ut_nbras = nbras;
        CKB_(gtf_dmalloc((void **)&b->d_delta, sizeof(DeltaDesc) * M, b->st));
        CKB_(cudaMemcpyAsync(b->d_delta, dd.data(), sizeof(DeltaDesc) * M, cudaMemcpyHostToDevice, b->st));
        CKB_(gtf_dmalloc((void **)&b->d_full, sizeof(int) * M, b->st));
        b->h_full = (int *)gtf_pinned_alloc(sizeof(int) * M);
        CKB_(b->h_full ? cudaSuccess : cudaErrorMemoryAllocation);
        for (int m = 0; m < M; m++) b->h_full[m] = 1;
        CKB_(cudaMemcpyAsync(b->d_full, b->h_full, sizeof(int) * M, cudaMemcpyHostToDevice, b->st));
        if (!ut.empty()) {
            CKB_(gtf_dmalloc((void **)&b->d_ut, sizeof(UnitTask) * ut.size(), b->st));
            CKB_(cudaMemcpyAsync(b->d_ut, ut.data(), sizeof(UnitTask) * ut.size(), cudaMemcpyHostToDevice, b->st));
        }
        size_t ntot = 0;
        for (auto &v : ptot) ntot += v.size();
        b->npdesc = (int)pdesc.size();
        if (ntot > 0) {
            CKB_(gtf_dmalloc((void **)&b->d_ptot, sizeof(const long long *) * ntot, b->st));
            std::vector<const long long *> flat;
            for (size_t k = 0; k < ptot.size(); k++) {
                pdesc[k].tot = b->d_ptot + flat.size();
                flat.insert(flat.end(), ptot[k].begin(), ptot[k].end());
            }
            CKB_(cudaMemcpyAsync(b->d_ptot, flat.data(), sizeof(const long long *) * ntot, cudaMemcpyHostToDevice, b->st));
        }
        if (b->npdesc > 0) {
            CKB_(gtf_dmalloc((void **)&b->d_pdesc, sizeof(PrefixDesc) * pdesc.size(), b->st));
            CKB_(cudaMemcpyAsync(b->d_pdesc, pdesc.data(), sizeof(PrefixDesc) * pdesc.size(), cudaMemcpyHostToDevice, b->st));
        }
    }
    b->ncounter_blocks = nblocks;
    CKB_(gtf_dmalloc((void **)&b->d_counters, sizeof(unsigned long long) * (size_t)nblocks * GTF_MAX_SLICES, b->st));
    *out = b;
    return GTF_OK;
}

// One Fock build of every engine of the batch; returns the number of kernels
// launched (>= 0) or a negative error.  Stream-ordered: no host wait.
// Incremental batches: full[m] != 0 makes molecule m's next build a full one
// (copied to the device on the batch's stream, so a captured build replayed
// afterwards reads it).
extern "C" int gtf_fock_batch_set_full(gtf_fock_batch_t *b, const int *full)
{
    if (!b || !b->dyn || !full) return GTF_ERR_INVALID;
    CK(cudaStreamSynchronize(b->st));   // the pinned flags may still be in flight
    for (int m = 0; m < b->M; m++) b->h_full[m] = full[m] ? 1 : 0;
    CK(cudaMemcpyAsync(b->d_full, b->h_full, sizeof(int) * b->M, cudaMemcpyHostToDevice, b->st));
    return GTF_OK;
}

extern "C" int gtf_fock_batch_compute(gtf_fock_batch_t *b)
{
    cudaStream_t st = b->st;
    int launches = 0;
    if (b->dyn) {
        // density changes, thresholds, task lists and launch prefixes of
        // every molecule, all on the device
        k_b_dzero<<<(b->M + 127) / 128, 128, 0, st>>>(b->d_delta, b->M);
        CK(cudaGetLastError());
        const size_t nb = (b->maxnn + 255) / 256;
        dim3 g((unsigned)(nb < 64 ? (nb < 1 ? 1 : nb) : 64), b->M);
        k_b_delta<<<g, 256, 0, st>>>(b->d_delta, b->d_full);
        CK(cudaGetLastError());
        k_b_thresholds<<<(b->M + 127) / 128, 128, 0, st>>>(b->d_delta, b->d_full, b->M);
        CK(cudaGetLastError());
        launches += 3;
        const int r = run_units(b->d_ut, b->ut_n, b->ut_nidx, b->ut_nbras, b->nsm, st);
        if (r) return r;
        launches += 3;
        if (b->npdesc > 0) {
            k_b_molprefix<<<(b->npdesc + 127) / 128, 128, 0, st>>>(b->d_pdesc, b->npdesc);
            CK(cudaGetLastError());
            launches++;
        }
    }
    {
        dim3 g((b->maxnc + 127) / 128, b->maxnc < 1024 ? b->maxnc : 1024, b->M);
        k_b_prep<<<g, 128, 0, st>>>(b->d_xf);
        CK(cudaGetLastError());
        launches++;
    }
    CK(cudaMemsetAsync(b->d_counters, 0, sizeof(unsigned long long) * (size_t)b->ncounter_blocks * GTF_MAX_SLICES,
                       st));
    for (int c = 0; c < NCLSPAIR; c++) {
        const ClassPairTask &t0 = b->eng[0]->tasks[c];
        for (int p = 0; p < 2; p++) {
            for (size_t k = 0; k < b->solo[c][p].size(); k++) {
                FockGrid g;
                memset(&g, 0, sizeof(g));
                g.one = b->solo[c][p][k];
                g.nmol = 1;
                g.nunits = b->solo_units[c][p][k];
                if (b->dyn) g.nunits_dev = b->solo_tot[c][p][k];
                g.counter = b->d_counters + (size_t)(b->solo_base[c][p] + (int)k) * GTF_MAX_SLICES;
                g.nsm = b->nsm;
                g.fp32 = p;
                tune_apply(0, t0.X, t0.Y, p, g);
                const int r = launch_fock(t0.X, t0.Y, g, st);
                if (r < 0) {
                    snprintf(g_errbuf, sizeof(g_errbuf), "Fock launch for class pair %d part %d failed: %s", c, p,
                             cudaGetErrorString(cudaGetLastError()));
                    return GTF_ERR_CUDA;
                }
                launches += r;
            }
            if (b->total[c][p] == 0) continue;
            FockGrid g;
            memset(&g, 0, sizeof(g));
            g.one = b->one[c][p];
            g.mols = b->d_desc[c][p];
            g.mol_prefix = b->d_prefix[c][p];
            g.nmol = b->nmol[c][p];
            g.nunits = b->total[c][p];
            if (b->dyn) g.nunits_dev = b->d_prefix[c][p] + b->nmol[c][p];
            g.counter = b->d_counters + (size_t)(2 * c + p) * GTF_MAX_SLICES;
            g.nsm = b->nsm;
            g.fp32 = p;
            tune_apply(1, t0.X, t0.Y, p, g);
            const int r = launch_fock(t0.X, t0.Y, g, st);
            if (r < 0) {
                snprintf(g_errbuf, sizeof(g_errbuf), "batched Fock launch for class pair %d part %d failed: %s", c, p,
                         cudaGetErrorString(cudaGetLastError()));
                return GTF_ERR_CUDA;
            }
            launches += r;
        }
    }
    {
        dim3 g((b->maxn + 127) / 128, b->maxn < 1024 ? b->maxn : 1024, b->M);
        k_b_post<<<g, 128, 0, st>>>(b->d_xf);
        CK(cudaGetLastError());
        launches++;
    }
    gtf_note_launches(launches);
    return launches;
}

// Tunes the shapes of the batched launches (all molecules per launch).
extern "C" int gtf_fock_batch_autotune(gtf_fock_batch_t *b, int reps)
{
    if (reps < 1) reps = 1;
    if (gtf_fock_batch_compute(b) < 0) return GTF_ERR_CUDA;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        return GTF_ERR_CUDA;
    }
    int rc = GTF_OK;
    for (int c = 0; c < NCLSPAIR && rc == GTF_OK; c++) {
        const ClassPairTask &t0 = b->eng[0]->tasks[c];
        for (int p = 0; p < 2; p++) {
            for (size_t k = 0; k < b->solo[c][p].size() && rc == GTF_OK; k++) {
                FockGrid g;
                memset(&g, 0, sizeof(g));
                g.one = b->solo[c][p][k];
                g.nmol = 1;
                g.nunits = b->solo_units[c][p][k];
                if (b->dyn) g.nunits_dev = b->solo_tot[c][p][k];
                g.counter = b->d_counters + (size_t)(b->solo_base[c][p] + (int)k) * GTF_MAX_SLICES;
                g.nsm = b->nsm;
                g.fp32 = p;
                if (tune_launch(0, t0.X, t0.Y, p, g, b->st, reps, e0, e1) < 0.0) rc = GTF_ERR_CUDA;
            }
            if (rc != GTF_OK) break;
            if (b->total[c][p] == 0) continue;
            FockGrid g;
            memset(&g, 0, sizeof(g));
            g.one = b->one[c][p];
            g.mols = b->d_desc[c][p];
            g.mol_prefix = b->d_prefix[c][p];
            g.nmol = b->nmol[c][p];
            g.nunits = b->total[c][p];
            if (b->dyn) g.nunits_dev = b->d_prefix[c][p] + b->nmol[c][p];
            g.counter = b->d_counters + (size_t)(2 * c + p) * GTF_MAX_SLICES;
            g.nsm = b->nsm;
            g.fp32 = p;
            if (tune_launch(1, t0.X, t0.Y, p, g, b->st, reps, e0, e1) < 0.0) {
                snprintf(g_errbuf, sizeof(g_errbuf), "autotuning batched class pair %d part %d failed: %s", c, p,
                         cudaGetErrorString(cudaGetLastError()));
                rc = GTF_ERR_CUDA;
                break;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}
