// fock_kernel.cuh -- the persistent Fock kernel (one instantiation per
// angular class pair) and its launcher; included by fock.cu and by the
// fock_cls_*.cu translation units that instantiate it.
#pragma once

#include <cuda_runtime.h>

#include "gtf_cuda.h"
#include "gtf_dev.cuh"

#define FOCK_THREADS 128

// Ket pairs of one angular class are stored in segments of similar
// primitive-pair count (gtf_prim_bucket), each sorted by Schwarz bound, so the
// 32 lanes of a warp loop over about the same number of primitive quartets.
#define GTF_NBKT 15
__host__ __device__ inline int gtf_prim_bucket(int n)
{
    if (n <= 2) return n < 0 ? 0 : n;
    if (n <= 4) return 3;
    if (n <= 6) return 4;
    if (n <= 9) return 5;
    if (n <= 12) return 6;
    if (n <= 16) return 7;
    if (n <= 20) return 8;
    if (n <= 25) return 9;
    if (n <= 32) return 10;
    if (n <= 40) return 11;
    if (n <= 48) return 12;
    if (n <= 64) return 13;
    return 14;
}

struct FockLaunch {
    const PairRec *pairs;
    const double2 *pprec;          // primitive-pair records (PPRec)
    const int *nlo;                // [nbra][GTF_NBKT] first ket of this launch in the segment prefix (null: 0)
    const int *nket;               // [nbra][GTF_NBKT] end of this launch's kets in the segment prefix
    const long long *unit_prefix;  // exclusive prefix of units over (bra, segment)
    int nbra;
    long long nunits;
    int bra_start, ket_start;
    int seg[GTF_NBKT + 1];         // segment starts, relative to ket_start
    unsigned long long *counter;
    const double *D;
    double *Fj, *Fk;
    int ld;
    int nsm;
    int fp32;                      // evaluate the integrals in FP32 (digestion stays FP64)
};

// ---------------------------------------------------------------------------
// the Fock kernel: persistent warps claim units of 32 quartets
// ---------------------------------------------------------------------------
// Ket components per slice: quartets with up to 64 Cartesian integrals are
// done in one pass; larger ones are split so that a slice keeps at most
// ~54 accumulators in registers (the Rys roots and 2-D tables are
// recomputed per slice, which costs less than spilling the accumulators).
// FP32 values take one register each, so the FP32 kernels keep quartets of
// up to 81 integrals in one pass; larger FP32 slices spill like the FP64 ones
// (the FP32 2-D tables and roots are live at the same time).
__host__ __device__ constexpr int fock_slice(int LA, int LB, int LC, int LD, int fp32)
{
    const int nab = ncart(LA) * ncart(LB), ncd = ncart(LC) * ncart(LD);
    if (nab * ncd <= (fp32 ? 81 : 64)) return ncd;
    const int s = 54 / nab;
    return s < 1 ? 1 : (s > ncd ? ncd : s);
}

template <int LA, int LB, int LC, int LD, typename R, int CD0>
__device__ __forceinline__ void fock_slices(const PPRec &src, const PairRec &pb, const PairRec &pk, bool active,
                                            bool same, const double *__restrict__ D, double *__restrict__ Fj,
                                            double *__restrict__ Fk, int ld, int lane)
{
    constexpr int NCD = ncart(LC) * ncart(LD);
    constexpr int S = fock_slice(LA, LB, LC, LD, sizeof(R) == 4 ? 1 : 0);
    if constexpr (CD0 < NCD) {
        constexpr int N = (NCD - CD0 < S) ? NCD - CD0 : S;
        R acc[ncart(LA) * ncart(LB) * N];
#pragma unroll
        for (int k = 0; k < ncart(LA) * ncart(LB) * N; k++) acc[k] = (R)0;
        if (active) eri_accumulate_cd<LA, LB, LC, LD, CD0, N, true>(src, pb, src, pk, acc);
        digest_cd<LA, LB, LC, LD, CD0, N>(acc, active, pb, pk, same, D, Fj, Fk, ld, lane);
        fock_slices<LA, LB, LC, LD, R, CD0 + N>(src, pb, pk, active, same, D, Fj, Fk, ld, lane);
    }
}

// unit u -> (bra i, segment b, chunk of 32 kets): binary search of the
// exclusive unit prefix over the flattened (bra, segment) index
template <int LA, int LB, int LC, int LD, typename R>
__global__ void __launch_bounds__(FOCK_THREADS) k_fock(const FockLaunch a)
{
    const int lane = threadIdx.x & 31;
    const PPRec src{a.pprec};
    const int nidx = a.nbra * GTF_NBKT;
    for (;;) {
        unsigned long long u = 0;
        if (lane == 0) u = atomicAdd(a.counter, 1ULL);
        u = __shfl_sync(GTF_FULL_MASK, u, 0);
        if (u >= (unsigned long long)a.nunits) break;
        int lo = 0, hi = nidx;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (__ldg(a.unit_prefix + mid) <= (long long)u) lo = mid;
            else hi = mid;
        }
        const int i = lo / GTF_NBKT, b = lo - i * GTF_NBKT;
        const long long chunk = (long long)u - __ldg(a.unit_prefix + lo);
        const int jj = (int)(chunk * 32) + lane;
        const int k0 = a.nlo ? __ldg(a.nlo + lo) : 0;
        const bool active = jj < __ldg(a.nket + lo) - k0;
        const int j = a.seg[b] + k0 + jj;
        const PairRec pb = a.pairs[a.bra_start + i];
        const PairRec pk = active ? a.pairs[a.ket_start + j] : pb;
        const bool same = (a.bra_start + i) == (a.ket_start + j);
        fock_slices<LA, LB, LC, LD, R, 0>(src, pb, pk, active, same, a.D, a.Fj, a.Fk, a.ld, lane);
    }
}

template <int LA, int LB, int LC, int LD, typename R>
int launch_fock_t(const FockLaunch &a, cudaStream_t st)
{
    auto k = k_fock<LA, LB, LC, LD, R>;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)k, FOCK_THREADS, 0);
    if (per_sm < 1) per_sm = 1;
    long long want = (a.nunits + (FOCK_THREADS / 32) - 1) / (FOCK_THREADS / 32);
    long long grid = (long long)a.nsm * per_sm;
    if (want < grid) grid = want;
    if (grid < 1) grid = 1;
    k<<<(unsigned)grid, FOCK_THREADS, 0, st>>>(a);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// returns 0 when launched, -1 on a launch error, 1 when the class pair is not in this group
#define FOCK_GROUP_CASE(A, B, C, D) \
    if (la == A && lb == B && lc == C && ld == D)                                                       \
        return a.fp32 ? launch_fock_t<A, B, C, D, float>(a, st) : launch_fock_t<A, B, C, D, double>(a, st);
