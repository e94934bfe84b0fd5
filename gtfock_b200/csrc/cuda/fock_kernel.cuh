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
#define GTF_CUM 16   // per-bra segment prefix: GTF_NBKT + 1 entries
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

// One molecule's part of a class-pair launch (its task lists, pair data, D
// and accumulators).
struct FockLaunch {
    const PairRec *pairs;
    const double2 *pprec;          // primitive-pair records (PPRec)
    const float4 *pprec32;         // FP32 primitive-pair records (PPRec32)
    const int *nlo;                // [nbra][GTF_NBKT] first ket of this launch in each segment prefix (null: 0)
    const int *cum;                // [nbra][GTF_CUM] exclusive prefix over segments of this launch's kets
    const long long *unit_prefix;  // [nbra + 1] exclusive prefix of units (32 kets) over bras
    int nbra;
    long long nunits;
    int bra_start, ket_start;
    int seg[GTF_NBKT + 1];         // segment starts, relative to ket_start
    const double *D;
    double *Fj, *Fk;
    int ld;
    int konly;                     // exchange terms only (antisymmetric part of a non-symmetric D)
};

// A launch over one molecule (nmol == 1: `one`) or a batch of molecules
// (mols[0..nmol), units concatenated in mol_prefix order): the persistent
// warps of one kernel serve every molecule of the batch.
struct FockGrid {
    FockLaunch one;
    const FockLaunch *mols;         // device array, nmol > 1
    const long long *mol_prefix;    // device, [nmol + 1] exclusive prefix of units
    int nmol;
    long long nunits;               // all units of the launch (with nunits_dev: an upper bound)
    // task lists rebuilt on the device (incremental builds): the launch's
    // unit count is read here when the kernel starts; null: nunits
    const long long *nunits_dev;
    unsigned long long *counter;    // GTF_MAX_SLICES zeroed counters, one per slice launch
    int nsm;
    int fp32;                       // evaluate the integrals in FP32 (digestion stays FP64)
    // launch shape (autotuned; 0 = default): persistent blocks per SM (capped
    // by the occupancy limit) and, in batched launches, units of 32 quartets
    // a warp claims at once
    int ctas_per_sm;
    int claim;
    int query;                      // launch nothing: return the first slice's occupancy limit
    // single-molecule launches of a sharded build: this launch covers units
    // [unit_lo, unit_lo + nunits) of the class's unit range
    long long unit_lo;
};

// ---------------------------------------------------------------------------
// the Fock kernel: persistent warps claim units of 32 quartets
// ---------------------------------------------------------------------------
// Ket components per slice: quartets with up to 64 Cartesian integrals are
// done in one pass; larger ones are split so that a slice keeps at most
// ~54 accumulators in registers (the Rys roots and 2-D tables are
// recomputed per slice, which costs less than spilling the accumulators).
// FP32 values take one register each, so the FP32 kernels keep quartets of
// up to 81 integrals in one pass and slices of up to ~72 accumulators.  FP64
// (dd| classes also take 72 (2 ket components): their spills cost less than
// recomputing the roots and 2-D tables for twice as many slices, which is not
// so for the (dp| classes (measured on C54H18).
__host__ __device__ constexpr int fock_slice(int LA, int LB, int LC, int LD, int fp32)
{
    const int nab = ncart(LA) * ncart(LB), ncd = ncart(LC) * ncart(LD);
    if (nab * ncd <= (fp32 ? 81 : 64)) return ncd;
    const int s = (fp32 || nab >= 36 ? 72 : 54) / nab;
    return s < 1 ? 1 : (s > ncd ? ncd : s);
}

// One launch per slice (CD0 = first ket component of the slice): each
// kernel holds the code of a single slice, which keeps the instruction
// footprint of the d-class kernels small.  The Rys table block of this class
// (NR roots, precision R) is staged in shared memory by every block.
// Blocks per SM the register allocation must allow: small quartets run
// latency-bound dependency chains (Rys polynomial, recurrences), so more
// resident warps pay off more than the registers they give up.
__host__ __device__ constexpr int fock_min_blocks(int LA, int LB, int LC, int LD, int slice)
{
    const int nq = ncart(LA) * ncart(LB) * slice;
    return nq <= 3 ? 6 : nq <= 9 ? 4 : nq <= 27 ? 3 : 2;
}

template <int LA, int LB, int LC, int LD, typename R, int CD0, bool BATCH>
__global__ void __launch_bounds__(FOCK_THREADS,
                                  fock_min_blocks(LA, LB, LC, LD,
                                                  fock_slice(LA, LB, LC, LD, sizeof(R) == 4 ? 1 : 0)))
    k_fock(const FockGrid g, unsigned long long *counter)
{
    constexpr int NR = (LA + LB + LC + LD) / 2 + 1;
    constexpr int NCD = ncart(LC) * ncart(LD);
    constexpr int S = fock_slice(LA, LB, LC, LD, sizeof(R) == 4 ? 1 : 0);
    constexpr int N = (NCD - CD0 < S) ? NCD - CD0 : S;
    __shared__ __align__(16) R tab[RysTab<R>::slen(NR)];
    // the launch's unit count, kept in shared memory rather than a register
    // across the integral loops (visible after the staging's barrier)
    __shared__ unsigned long long s_nunits;
    if (threadIdx.x == 0) s_nunits = (unsigned long long)(g.nunits_dev ? *g.nunits_dev : g.nunits);
    rys_stage<R, NR>(tab);
    const int lane = threadIdx.x & 31;
    // batched launches: per-warp slots for the claimed range of units and the
    // molecule of the current unit, so that neither holds registers across
    // the integral loops
    constexpr int NW = FOCK_THREADS / 32;
    __shared__ unsigned long long s_claim[BATCH ? 2 * NW : 1];
    __shared__ int s_mol[BATCH ? NW : 1];
    const int wib = threadIdx.x >> 5;
    if constexpr (BATCH) {
        if (lane == 0) {
            s_claim[2 * wib] = 0;
            s_claim[2 * wib + 1] = 0;
        }
        __syncwarp();
    }
    for (;;) {
        unsigned long long uu;
        if constexpr (BATCH) {
            // a warp claims g.claim units at once (fewer atomics on the
            // counter when the molecules' units are small)
            volatile unsigned long long *sc = s_claim + 2 * wib;
            unsigned long long u = sc[0], uend = sc[1];
            if (u >= uend) {
                const unsigned claim = g.claim > 1 ? (unsigned)g.claim : 1u;
                unsigned long long c0 = 0;
                if (lane == 0) c0 = atomicAdd(counter, (unsigned long long)claim);
                u = __shfl_sync(GTF_FULL_MASK, c0, 0);
                uend = u + claim;
            }
            if (u >= *(volatile unsigned long long *)&s_nunits) break;
            uu = u;
            __syncwarp();
            if (lane == 0) {
                sc[0] = u + 1;
                sc[1] = uend;
            }
            __syncwarp();
        } else {
            unsigned long long c0 = 0;
            if (lane == 0) c0 = atomicAdd(counter, 1ULL);
            uu = __shfl_sync(GTF_FULL_MASK, c0, 0);
            if (uu >= *(volatile unsigned long long *)&s_nunits) break;
            uu += (unsigned long long)g.unit_lo;
        }
        // molecule of the unit (batched launches); the fields are read from
        // the kernel parameter (one molecule, no registers held for them) or
        // from the descriptor array
        constexpr bool bt = BATCH;
        const FockLaunch *mp = g.mols;   // reassigned after the integral loops (batched)
        if constexpr (BATCH) {
            const int m = warp_find_le(g.mol_prefix, g.nmol, (long long)uu, lane);
            mp += m;
            uu -= (unsigned long long)__ldg(g.mol_prefix + m);
            __syncwarp();
            if (lane == 0) s_mol[wib] = m;
            __syncwarp();
        }
#define GTF_FLD(x) (bt ? mp->x : g.one.x)
        const long long *unit_prefix = GTF_FLD(unit_prefix);
        // unit u -> (bra i, chunk of 32 kets) by a warp search of the unit
        // prefix over bras; lane v of the chunk -> segment b and position in
        // it from the bra's segment prefix (the kets of consecutive segments
        // share a warp)
        const int nbra = GTF_FLD(nbra);
        const int i = warp_find_le(unit_prefix, nbra, (long long)uu, lane);
        const int v = (int)((long long)uu - __ldg(unit_prefix + i)) * 32 + lane;
        const int4 *cq = reinterpret_cast<const int4 *>(GTF_FLD(cum) + (size_t)i * GTF_CUM);
        const int4 c0 = __ldg(cq), c1 = __ldg(cq + 1), c2 = __ldg(cq + 2), c3 = __ldg(cq + 3);
        const int cum[GTF_CUM] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w,
                                  c2.x, c2.y, c2.z, c2.w, c3.x, c3.y, c3.z, c3.w};
        const bool active = v < cum[GTF_NBKT];
        int b = 0, cb = 0;
#pragma unroll
        for (int k = 1; k < GTF_NBKT; k++)
            if (cum[k] <= v) {
                b = k;
                cb = cum[k];
            }
        const int *nlo = GTF_FLD(nlo);
        const int k0 = nlo ? __ldg(nlo + (size_t)i * GTF_NBKT + b) : 0;
        const int j = GTF_FLD(seg[b]) + k0 + (v - cb);
        const PairRec *pairs = GTF_FLD(pairs);
        const int bra_start = GTF_FLD(bra_start), ket_start = GTF_FLD(ket_start);
        const PairRec pb = pairs[bra_start + i];
        const PairRec pk = active ? pairs[ket_start + j] : pb;
        const bool same = (bra_start + i) == (ket_start + j);
        R acc[ncart(LA) * ncart(LB) * N];
#pragma unroll
        for (int k = 0; k < ncart(LA) * ncart(LB) * N; k++) acc[k] = (R)0;
        if constexpr (sizeof(R) == 4) {
            const PPRec32 src{GTF_FLD(pprec32)};
            if (active) eri_accumulate_cd32<LA, LB, LC, LD, CD0, N, true, true>(src, pb, pk, acc, tab);
        } else {
            const PPRec src{GTF_FLD(pprec)};
            if (active) eri_accumulate_cd<LA, LB, LC, LD, CD0, N, true, true>(src, pb, src, pk, acc, tab);
        }
        if constexpr (BATCH) mp = g.mols + ((volatile int *)s_mol)[wib];   // reloaded after the loops
        digest_cd<LA, LB, LC, LD, CD0, N>(acc, active, pb, pk, same, GTF_FLD(D), GTF_FLD(Fj), GTF_FLD(Fk),
                                          GTF_FLD(ld), lane, GTF_FLD(konly) != 0);
#undef GTF_FLD
    }
}

// Number of slice launches of a class pair; g.counter points at that many
// zeroed counters.
__host__ __device__ constexpr int fock_nslices(int LA, int LB, int LC, int LD, int fp32)
{
    const int ncd = ncart(LC) * ncart(LD), s = fock_slice(LA, LB, LC, LD, fp32);
    return (ncd + s - 1) / s;
}
#define GTF_MAX_SLICES 64

template <int LA, int LB, int LC, int LD, typename R, int CD0>
int launch_fock_slices(const FockGrid &g, cudaStream_t st, int slice)
{
    constexpr int NCD = ncart(LC) * ncart(LD);
    if constexpr (CD0 < NCD) {
        constexpr int S = fock_slice(LA, LB, LC, LD, sizeof(R) == 4 ? 1 : 0);
        auto k = g.nmol > 1 ? k_fock<LA, LB, LC, LD, R, CD0, true> : k_fock<LA, LB, LC, LD, R, CD0, false>;
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)k, FOCK_THREADS, 0);
        if (per_sm < 1) per_sm = 1;
        if (g.query) return per_sm;
        if (g.ctas_per_sm > 0 && g.ctas_per_sm < per_sm) per_sm = g.ctas_per_sm;
        long long want = (g.nunits + (FOCK_THREADS / 32) - 1) / (FOCK_THREADS / 32);
        long long grid = (long long)g.nsm * per_sm;
        if (want < grid) grid = want;
        if (grid < 1) grid = 1;
        k<<<(unsigned)grid, FOCK_THREADS, 0, st>>>(g, g.counter + slice);
        if (cudaGetLastError() != cudaSuccess) return -1;
        const int r = launch_fock_slices<LA, LB, LC, LD, R, CD0 + S>(g, st, slice + 1);
        return r < 0 ? r : r + 1;
    } else {
        return 0;
    }
}

// returns the number of kernels launched, or -1 on a launch error
template <int LA, int LB, int LC, int LD, typename R>
int launch_fock_t(const FockGrid &g, cudaStream_t st)
{
    static_assert(fock_nslices(LA, LB, LC, LD, sizeof(R) == 4 ? 1 : 0) <= GTF_MAX_SLICES, "slice counters");
    return launch_fock_slices<LA, LB, LC, LD, R, 0>(g, st, 0);
}

// returns the number of launches, -1 on a launch error, GTF_NOT_IN_GROUP when the
// class pair is not in this group
#define GTF_NOT_IN_GROUP (-2)
#define FOCK_GROUP_CASE(A, B, C, D) \
    if (la == A && lb == B && lc == C && ld == D)                                                       \
        return g.fp32 ? launch_fock_t<A, B, C, D, float>(g, st) : launch_fock_t<A, B, C, D, double>(g, st);
