// gtf_dev.cuh -- device building blocks of the Fock build (sm_100a).
//
// Replaces the integral engine behind CInt_computeShellQuartet
// (libcint/include/CInt.h:159-167, called at pfock/fock_task.c:197-198) and
// the J/K digestion update_F (pfock/fock_task.c:29-117):
//   * rys_roots<N>: N-point Rys quadrature for the Boys weight from the
//     generated Chebyshev-fitted table (rys_table.h), large-T Hermite form;
//   * eri_accumulate<LA,LB,LC,LD>: contracted Cartesian (ab|cd) by Rys
//     quadrature -- per primitive quartet and root the 2-D integrals
//     G(i,k) by the Rys recurrences (C00, C00', B10, B01, B00), horizontal
//     transfer to (a b | c d) per Cartesian direction, and the product
//     Ix*Iy*Iz accumulated in registers; integrals never leave the thread;
//   * digest_cd<...>: the six J/K updates of one unique quartet into F with
//     the reference's degeneracy factors; the bra block (uniform across a
//     warp) is warp-reduced before its atomics.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define RYS_QUAL __device__ __align__(16)
#define RYS_QUAL_SMALL __constant__
#include "rys_table.h"

#define GTF_FULL_MASK 0xffffffffu
#define GTF_MAXL 2

// sqrt(2) * pi^(5/4): the per-pair share of 2 pi^(5/2) / (p q sqrt(p+q))
#define GTF_PAIR_PREF 5.9149671727956130

// primitive screening in the Fock build: a primitive pair is dropped when its
// prefactor K is below GTF_PRIM_EPS; a primitive quartet is skipped when
// |K_ab K_cd| is below GTF_PRIMQ_EPS (pairs are stored in descending |K|, so
// the loops stop there).  A primitive integral is at most |K_ab K_cd| /
// sqrt(p+q) times angular factors of order 10 for s-d shells, so a skipped one
// is below ~1e-14 Ha.  Against the reference-pinned Fock matrices of C54H18 /
// cc-pVDZ, (H2O)64 / 6-31G and C96H24 / cc-pVDZ the largest element error is
// 1.8e-12, 4.1e-13 and 2.0e-12 Ha (1.1e-12, 4.2e-13, 1.4e-12 at 1e-17, where
// the atomics' rounding dominates), and the builds are 6% faster than at 1e-17.
#define GTF_PRIM_EPS 1e-15
#define GTF_PRIMQ_EPS 1e-15

// ---------------------------------------------------------------------------
// Cartesian component tables (lexicographic: xx, xy, xz, yy, yz, zz)
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int ncart(int L) { return (L + 1) * (L + 2) / 2; }

__host__ __device__ constexpr int cart_x(int L, int c)
{
    int x = L;
    int first = 0;  // index of the first component with this x
    while (x >= 0) {
        int cnt = L - x + 1;
        if (c < first + cnt) return x;
        first += cnt;
        x--;
    }
    return 0;
}

__host__ __device__ constexpr int cart_y(int L, int c)
{
    int x = L;
    int first = 0;
    while (x >= 0) {
        int cnt = L - x + 1;
        if (c < first + cnt) return (L - x) - (c - first);
        first += cnt;
        x--;
    }
    return 0;
}

__host__ __device__ constexpr int cart_z(int L, int c) { return L - cart_x(L, c) - cart_y(L, c); }

// ---------------------------------------------------------------------------
// Shell-pair record (64 bytes, coalesced by lane)
// ---------------------------------------------------------------------------
struct __align__(16) PairRec {
    double Ax, Ay, Az;     // centre of shell a
    double ABx, ABy, ABz;  // A - B
    int fa, fb;            // first Cartesian function of a and b
    int off, n;            // primitive-pair offset and count
};

// primitive-pair data, structure of arrays
struct PrimPairs {
    const double *p;   // a + b
    const double *Px, *Py, *Pz;
    const double *K;   // GTF_PAIR_PREF * ca * cb * exp(-ab/p |AB|^2) / p
};

// one primitive pair: exponent sum p, centre P, prefactor K, h = 1/(2p)
struct PrimVals {
    double p, Px, Py, Pz, K, h;
};

// FP32 form of a primitive pair, centre relative to the pair's first shell:
// {p, K, PAx, PAy}, {PAz, 1/(2p), 0, 0} (32 bytes, two 16-byte loads)
struct PrimVals32 {
    float p, K, PAx, PAy, PAz, h;
};
struct PPRec32 {
    const float4 *r;
    __device__ __forceinline__ PrimVals32 get(const PairRec &pr, int i) const
    {
        const float4 *q = r + 2 * (size_t)(pr.off + i);
        const float4 a = __ldg(q), b = __ldg(q + 1);
        PrimVals32 v;
        v.p = a.x;
        v.K = a.y;
        v.PAx = a.z;
        v.PAy = a.w;
        v.PAz = b.x;
        v.h = b.y;
        return v;
    }
};


__device__ __forceinline__ double gfma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float gfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double grsqrt(double x) { return rsqrt(x); }
__device__ __forceinline__ float grsqrt(float x) { return rsqrtf(x); }

// ---------------------------------------------------------------------------
// Rys roots and weights
// ---------------------------------------------------------------------------
// interval width and polynomial degree of the N-root FP64 table
__host__ __device__ constexpr double rys_h(int n)
{
    constexpr double h[] = {RYS_H_LIST};
    return h[n];
}
__host__ __device__ constexpr int rys_deg(int n)
{
    constexpr int d[] = {RYS_DEG_LIST};
    return d[n];
}

// The N-root block of each table is [off(N), off(N+1)); its extent is known
// at compile time so kernels can stage it in shared memory.  rows(N) values
// per interval; a lane reads one interval's row as 2-value vectors (16 bytes
// FP64, 8 bytes FP32).  The lanes of a warp read different intervals, so the
// shared-memory copy pads each interval to srows(N), an odd number of vectors:
// consecutive intervals then start in different banks (unpadded, the FP64
// 4-root rows are 48 vectors long and every interval starts in the same bank).
template <typename R>
struct RysTab;
template <>
struct RysTab<double> {
    static __host__ __device__ constexpr int off(int n)
    {
        constexpr int o[] = {RYS_OFF_LIST, RYS_TABLE_LEN};
        return o[n];
    }
    static __host__ __device__ constexpr int len(int n) { return off(n + 1) - off(n); }
    static __host__ __device__ constexpr int rows(int n) { return (rys_deg(n) + 1) * 2 * n; }
    static __host__ __device__ constexpr int srows(int n) { return (rows(n) / 2) % 2 == 0 ? rows(n) + 2 : rows(n); }
    static __host__ __device__ constexpr int slen(int n) { return len(n) / rows(n) * srows(n); }
    static __device__ __forceinline__ const double *ptr(int n) { return RYS_TABLE + off(n); }
};
template <>
struct RysTab<float> {
    static __host__ __device__ constexpr int off(int n)
    {
        constexpr int o[] = {RYS32_OFF_LIST, RYS32_TABLE_LEN};
        return o[n];
    }
    static __host__ __device__ constexpr int len(int n) { return off(n + 1) - off(n); }
    static __host__ __device__ constexpr int rows(int n) { return (RYS32_DEG + 1) * 2 * n; }
    static __host__ __device__ constexpr int srows(int n) { return (rows(n) / 2) % 2 == 0 ? rows(n) + 2 : rows(n); }
    static __host__ __device__ constexpr int slen(int n) { return len(n) / rows(n) * srows(n); }
    static __device__ __forceinline__ const float *ptr(int n) { return RYS32_TABLE + off(n); }
};

// Stages the N-root block into shared memory with the padded row stride.
template <typename R, int N>
__device__ __forceinline__ void rys_stage(R *stab)
{
    constexpr int RW = RysTab<R>::rows(N), SR = RysTab<R>::srows(N), TL = RysTab<R>::len(N);
    static_assert(TL % RW == 0, "whole intervals");
    const R *gt = RysTab<R>::ptr(N);
    for (int k = threadIdx.x; k < TL; k += blockDim.x) stab[(k / RW) * SR + k % RW] = __ldg(gt + k);
    __syncthreads();
}

// tab: the N-root block of RYS_TABLE (global, STRIDE = rows) or its padded
// shared-memory copy (STRIDE = srows)
template <int N, int STRIDE = RysTab<double>::rows(N)>
__device__ __forceinline__ void rys_roots(double T, double (&u)[N], double (&w)[N], const double *tab)
{
    constexpr double H = rys_h(N), INV_H = 1.0 / rys_h(N);
    constexpr int DEG = rys_deg(N);
    if (T >= RYS_TMAX[N]) {
        const double it = 1.0 / T;
        const double rs = rsqrt(T);
#pragma unroll
        for (int i = 0; i < N; i++) {
            u[i] = RYS_LARGE_X2[N][i] * it;
            w[i] = RYS_LARGE_W[N][i] * rs;
        }
        return;
    }
    const int k = (int)(T * INV_H);
    const double s = T - ((double)k * H + 0.5 * H);
    static_assert(STRIDE % 2 == 0 && STRIDE >= (DEG + 1) * 2 * N, "interval stride");
    const double *c = tab + k * STRIDE;
    // rows of 2N coefficients start on 16-byte boundaries (even offsets)
    const double2 *c2 = reinterpret_cast<const double2 *>(c);
    double a[2 * N];
#pragma unroll
    for (int f = 0; f < N; f++) {
        const double2 t = c2[DEG * N + f];
        a[2 * f] = t.x;
        a[2 * f + 1] = t.y;
    }
#pragma unroll
    for (int j = DEG - 1; j >= 0; j--) {
#pragma unroll
        for (int f = 0; f < N; f++) {
            const double2 t = c2[j * N + f];
            a[2 * f] = fma(a[2 * f], s, t.x);
            a[2 * f + 1] = fma(a[2 * f + 1], s, t.y);
        }
    }
#pragma unroll
    for (int i = 0; i < N; i++) {
        u[i] = a[i];
        w[i] = a[N + i];
    }
}

// FP32 form for quartets evaluated in single precision: degree-7 fit of the
// same functions on the same intervals (RYS32_TABLE), same large-T form
template <int N, int STRIDE = RysTab<float>::rows(N)>
__device__ __forceinline__ void rys_roots(float T, float (&u)[N], float (&w)[N], const float *tab)
{
    if (T >= (float)RYS_TMAX[N]) {
        const float it = 1.0f / T;
        const float rs = rsqrtf(T);
#pragma unroll
        for (int i = 0; i < N; i++) {
            u[i] = (float)RYS_LARGE_X2[N][i] * it;
            w[i] = (float)RYS_LARGE_W[N][i] * rs;
        }
        return;
    }
    const int k = (int)(T * RYS32_INV_H);
    const float s = T - ((float)k * (float)RYS32_H + 0.5f * (float)RYS32_H);
    static_assert(STRIDE % 2 == 0 && STRIDE >= (RYS32_DEG + 1) * 2 * N, "interval stride");
    const float2 *c2 = reinterpret_cast<const float2 *>(tab + k * STRIDE);
    float a[2 * N];
#pragma unroll
    for (int f = 0; f < N; f++) {
        const float2 t = c2[RYS32_DEG * N + f];
        a[2 * f] = t.x;
        a[2 * f + 1] = t.y;
    }
#pragma unroll
    for (int j = RYS32_DEG - 1; j >= 0; j--) {
#pragma unroll
        for (int f = 0; f < N; f++) {
            const float2 t = c2[j * N + f];
            a[2 * f] = fmaf(a[2 * f], s, t.x);
            a[2 * f + 1] = fmaf(a[2 * f + 1], s, t.y);
        }
    }
#pragma unroll
    for (int i = 0; i < N; i++) {
        u[i] = a[i];
        w[i] = a[N + i];
    }
}

// ---------------------------------------------------------------------------
// one-dimensional horizontal transfer:
// t(a, b+1) = t(a+1, b) + dist * t(a, b); input v[0..L1+L2], output o[a][b]
// ---------------------------------------------------------------------------
template <int L1, int L2, typename R>
__device__ __forceinline__ void hrr1d(const R (&v)[L1 + L2 + 1], R (&o)[L1 + 1][L2 + 1], R dist)
{
    R t[L1 + L2 + 1][L2 + 1];
#pragma unroll
    for (int a = 0; a <= L1 + L2; a++) t[a][0] = v[a];
#pragma unroll
    for (int b = 0; b < L2; b++) {
#pragma unroll
        for (int a = 0; a <= L1 + L2 - b - 1; a++) t[a][b + 1] = gfma(dist, t[a][b], t[a + 1][b]);
    }
#pragma unroll
    for (int a = 0; a <= L1; a++) {
#pragma unroll
        for (int b = 0; b <= L2; b++) o[a][b] = t[a][b];
    }
}

// 2-D Rys integrals G[i][k] (i on centre A, k on centre C) for one direction
template <int NI, int NK, typename R>
__device__ __forceinline__ void rys_2d(R (&G)[NI][NK], R g00, R C00, R C0p, R B10, R B01, R B00)
{
    G[0][0] = g00;
    if (NI > 1) G[1][0] = C00 * g00;
#pragma unroll
    for (int i = 1; i < NI - 1; i++) G[i + 1][0] = gfma(C00, G[i][0], (R)i * B10 * G[i - 1][0]);
    if (NK > 1) G[0][1] = C0p * g00;
#pragma unroll
    for (int k = 1; k < NK - 1; k++) G[0][k + 1] = gfma(C0p, G[0][k], (R)k * B01 * G[0][k - 1]);
#pragma unroll
    for (int k = 1; k < NK; k++) {
#pragma unroll
        for (int i = 0; i < NI - 1; i++) {
            R v = gfma(C00, G[i][k], (R)k * B00 * G[i][k - 1]);
            if (i > 0) v = gfma((R)i * B10, G[i - 1][k], v);
            G[i + 1][k] = v;
        }
    }
}

// full 1-D transfer: G[i][k] -> I[a][b][c][d]
template <int LA, int LB, int LC, int LD, typename R>
__device__ __forceinline__ void hrr_abcd(const R (&G)[LA + LB + 1][LC + LD + 1],
                                         R (&I)[LA + 1][LB + 1][LC + 1][LD + 1], R ab, R cd)
{
    constexpr int NI = LA + LB + 1;
    R K[NI][LC + 1][LD + 1];
#pragma unroll
    for (int i = 0; i < NI; i++) {
        R v[LC + LD + 1];
#pragma unroll
        for (int k = 0; k <= LC + LD; k++) v[k] = G[i][k];
        R o[LC + 1][LD + 1];
        hrr1d<LC, LD>(v, o, cd);
#pragma unroll
        for (int c = 0; c <= LC; c++)
#pragma unroll
            for (int d = 0; d <= LD; d++) K[i][c][d] = o[c][d];
    }
#pragma unroll
    for (int c = 0; c <= LC; c++) {
#pragma unroll
        for (int d = 0; d <= LD; d++) {
            R v[NI];
#pragma unroll
            for (int i = 0; i < NI; i++) v[i] = K[i][c][d];
            R o[LA + 1][LB + 1];
            hrr1d<LA, LB>(v, o, ab);
#pragma unroll
            for (int a = 0; a <= LA; a++)
#pragma unroll
                for (int b = 0; b <= LB; b++) I[a][b][c][d] = o[a][b];
        }
    }
}

// ---------------------------------------------------------------------------
// contracted Cartesian (ab|cd), accumulated into acc[ia + NA*(ib + NB*(ic + NC*id))]
// ---------------------------------------------------------------------------
// SKIP: primitive pairs are sorted by descending |K| (Fock-build pair list),
// so the primitive-quartet cutoff may end the ket loop early
// Restricted to the ket components cd = CD0 .. CD0+N-1 (cd = ic + NC*id):
// acc[ia + NA*(ib + NB*t)] with t = cd - CD0.  The output-split Fock kernels
// call it once per slice so that a slice's accumulators fit in registers.
// R = double, or float for quartets evaluated in single precision (the
// differences of centres are formed in double first, then rounded).
// rtab: the NR-root block of the Rys table of precision R.
// Loop order: ket primitive pairs outside (one per lane), bra primitive pairs
// inside -- the bra is shared by the warp, so its records are warp-uniform
// loads that stay in L1, and each lane reads its ket's records once.
template <int LA, int LB, int LC, int LD, int CD0, int N, bool SKIP, bool SPAD = false, class PPB, class PPK,
          typename R>
__device__ __forceinline__ void eri_accumulate_cd(const PPB &bra, const PairRec &pb, const PPK &ket,
                                                  const PairRec &pk, R (&acc)[ncart(LA) * ncart(LB) * N],
                                                  const R *rtab)
{
    constexpr int NR = (LA + LB + LC + LD) / 2 + 1;
    constexpr int NI = LA + LB + 1, NK = LC + LD + 1;
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    if (pb.n <= 0) return;
    const R ABx = (R)pb.ABx, ABy = (R)pb.ABy, ABz = (R)pb.ABz;
    const R CDx = (R)pk.ABx, CDy = (R)pk.ABy, CDz = (R)pk.ABz;
    const PrimVals b0 = bra.get(pb, 0);
    PrimVals nk;
    if (pk.n > 0) nk = ket.get(pk, 0);
    for (int ik = 0; ik < pk.n; ik++) {
        const PrimVals kq = nk;
        if (ik + 1 < pk.n) nk = ket.get(pk, ik + 1);
        if (SKIP && fabs(b0.K * kq.K) < GTF_PRIMQ_EPS) break;  // both lists are in descending |K|
        const R q_ = (R)kq.p, h2q = (R)kq.h;
        const R QCx = (R)(kq.Px - pk.Ax), QCy = (R)(kq.Py - pk.Ay), QCz = (R)(kq.Pz - pk.Az);
        // the next bra primitive pair is loaded while the current one is used
        PrimVals nb = b0;
        for (int ib = 0; ib < pb.n; ib++) {
            const PrimVals bq = nb;
            if (ib + 1 < pb.n) nb = bra.get(pb, ib + 1);
            if (SKIP && fabs(bq.K * kq.K) < GTF_PRIMQ_EPS) break;
            const R p_ = (R)bq.p, h2p = (R)bq.h;
            const R PAx = (R)(bq.Px - pb.Ax), PAy = (R)(bq.Py - pb.Ay), PAz = (R)(bq.Pz - pb.Az);
            const R rpq = grsqrt((R)(bq.p + kq.p));
            const R ipq = rpq * rpq;
            const R PQx = (R)(bq.Px - kq.Px), PQy = (R)(bq.Py - kq.Py), PQz = (R)(bq.Pz - kq.Pz);
            const R rho = p_ * q_ * ipq;
            const R T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
            const R pref = (R)(bq.K * kq.K) * rpq;
            R u[NR], w[NR];
            rys_roots<NR, SPAD ? RysTab<R>::srows(NR) : RysTab<R>::rows(NR)>(T, u, w, rtab);
            const R qf = q_ * ipq, pf = p_ * ipq;
#pragma unroll
            for (int r = 0; r < NR; r++) {
                const R ur = u[r];
                const R B00 = (R)0.5 * ur * ipq;
                const R B10 = h2p * ((R)1 - qf * ur);
                const R B01 = h2q * ((R)1 - pf * ur);
                const R cq = qf * ur, cp = pf * ur;
                R Gx[NI][NK], Gy[NI][NK], Gz[NI][NK];
                rys_2d<NI, NK>(Gx, (R)1, PAx - cq * PQx, QCx + cp * PQx, B10, B01, B00);
                rys_2d<NI, NK>(Gy, (R)1, PAy - cq * PQy, QCy + cp * PQy, B10, B01, B00);
                rys_2d<NI, NK>(Gz, w[r] * pref, PAz - cq * PQz, QCz + cp * PQz, B10, B01, B00);
                R Ix[LA + 1][LB + 1][LC + 1][LD + 1];
                R Iy[LA + 1][LB + 1][LC + 1][LD + 1];
                R Iz[LA + 1][LB + 1][LC + 1][LD + 1];
                hrr_abcd<LA, LB, LC, LD>(Gx, Ix, ABx, CDx);
                hrr_abcd<LA, LB, LC, LD>(Gy, Iy, ABy, CDy);
                hrr_abcd<LA, LB, LC, LD>(Gz, Iz, ABz, CDz);
#pragma unroll
                for (int t = 0; t < N; t++) {
                    const int ic = (CD0 + t) % NC, id = (CD0 + t) / NC;
#pragma unroll
                    for (int ibb = 0; ibb < NB; ibb++)
#pragma unroll
                        for (int ia = 0; ia < NA; ia++) {
                            const R xy = Ix[cart_x(LA, ia)][cart_x(LB, ibb)][cart_x(LC, ic)][cart_x(LD, id)] *
                                         Iy[cart_y(LA, ia)][cart_y(LB, ibb)][cart_y(LC, ic)][cart_y(LD, id)];
                            R &dst = acc[ia + NA * (ibb + NB * t)];
                            dst = gfma(xy, Iz[cart_z(LA, ia)][cart_z(LB, ibb)][cart_z(LC, ic)][cart_z(LD, id)],
                                       dst);
                        }
                }
            }
        }
    }
    (void)ND;
}

// FP32 quartets: everything in single precision, from the FP32 records (centres
// relative to each pair's first shell; P - Q = PA - QC + (A - C) with A - C
// formed in double once per quartet).  Same structure as eri_accumulate_cd.
template <int LA, int LB, int LC, int LD, int CD0, int N, bool SKIP, bool SPAD = false>
__device__ __forceinline__ void eri_accumulate_cd32(const PPRec32 &src, const PairRec &pb, const PairRec &pk,
                                                    float (&acc)[ncart(LA) * ncart(LB) * N], const float *rtab)
{
    constexpr int NR = (LA + LB + LC + LD) / 2 + 1;
    constexpr int NI = LA + LB + 1, NK = LC + LD + 1;
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC);
    if (pb.n <= 0) return;
    const float ABx = (float)pb.ABx, ABy = (float)pb.ABy, ABz = (float)pb.ABz;
    const float CDx = (float)pk.ABx, CDy = (float)pk.ABy, CDz = (float)pk.ABz;
    const float ACx = (float)(pb.Ax - pk.Ax), ACy = (float)(pb.Ay - pk.Ay), ACz = (float)(pb.Az - pk.Az);
    const PrimVals32 b0 = src.get(pb, 0);
    PrimVals32 nk;
    if (pk.n > 0) nk = src.get(pk, 0);
    for (int ik = 0; ik < pk.n; ik++) {
        const PrimVals32 kq = nk;
        if (ik + 1 < pk.n) nk = src.get(pk, ik + 1);
        if (SKIP && fabsf(b0.K * kq.K) < (float)GTF_PRIMQ_EPS) break;
        const float q = kq.p, h2q = kq.h;
        const float QCx = kq.PAx, QCy = kq.PAy, QCz = kq.PAz;
        const float dx = ACx - QCx, dy = ACy - QCy, dz = ACz - QCz;
        PrimVals32 nb = b0;
        for (int ib = 0; ib < pb.n; ib++) {
            const PrimVals32 bq = nb;
            if (ib + 1 < pb.n) nb = src.get(pb, ib + 1);
            if (SKIP && fabsf(bq.K * kq.K) < (float)GTF_PRIMQ_EPS) break;
            const float p = bq.p, h2p = bq.h;
            const float PAx = bq.PAx, PAy = bq.PAy, PAz = bq.PAz;
            const float rpq = rsqrtf(p + q);
            const float ipq = rpq * rpq;
            const float PQx = PAx + dx, PQy = PAy + dy, PQz = PAz + dz;
            const float rho = p * q * ipq;
            const float T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
            const float pref = bq.K * kq.K * rpq;
            float u[NR], w[NR];
            rys_roots<NR, SPAD ? RysTab<float>::srows(NR) : RysTab<float>::rows(NR)>(T, u, w, rtab);
            const float qf = q * ipq, pf = p * ipq;
#pragma unroll
            for (int r = 0; r < NR; r++) {
                const float ur = u[r];
                const float B00 = 0.5f * ur * ipq;
                const float B10 = h2p * (1.0f - qf * ur);
                const float B01 = h2q * (1.0f - pf * ur);
                const float cq = qf * ur, cp = pf * ur;
                float Gx[NI][NK], Gy[NI][NK], Gz[NI][NK];
                rys_2d<NI, NK>(Gx, 1.0f, PAx - cq * PQx, QCx + cp * PQx, B10, B01, B00);
                rys_2d<NI, NK>(Gy, 1.0f, PAy - cq * PQy, QCy + cp * PQy, B10, B01, B00);
                rys_2d<NI, NK>(Gz, w[r] * pref, PAz - cq * PQz, QCz + cp * PQz, B10, B01, B00);
                float Ix[LA + 1][LB + 1][LC + 1][LD + 1];
                float Iy[LA + 1][LB + 1][LC + 1][LD + 1];
                float Iz[LA + 1][LB + 1][LC + 1][LD + 1];
                hrr_abcd<LA, LB, LC, LD>(Gx, Ix, ABx, CDx);
                hrr_abcd<LA, LB, LC, LD>(Gy, Iy, ABy, CDy);
                hrr_abcd<LA, LB, LC, LD>(Gz, Iz, ABz, CDz);
#pragma unroll
                for (int t = 0; t < N; t++) {
                    const int ic = (CD0 + t) % NC, id = (CD0 + t) / NC;
#pragma unroll
                    for (int ibb = 0; ibb < NB; ibb++)
#pragma unroll
                        for (int ia = 0; ia < NA; ia++) {
                            const float xy = Ix[cart_x(LA, ia)][cart_x(LB, ibb)][cart_x(LC, ic)][cart_x(LD, id)] *
                                             Iy[cart_y(LA, ia)][cart_y(LB, ibb)][cart_y(LC, ic)][cart_y(LD, id)];
                            float &dst = acc[ia + NA * (ibb + NB * t)];
                            dst = fmaf(xy, Iz[cart_z(LA, ia)][cart_z(LB, ibb)][cart_z(LC, ic)][cart_z(LD, id)], dst);
                        }
                }
            }
        }
    }
}

// the whole quartet: acc[ia + NA*(ib + NB*(ic + NC*id))]
template <int LA, int LB, int LC, int LD, bool SKIP = false, class PPB, class PPK>
__device__ __forceinline__ void eri_accumulate(const PPB &bra, const PairRec &pb, const PPK &ket,
                                               const PairRec &pk,
                                               double (&acc)[ncart(LA) * ncart(LB) * ncart(LC) * ncart(LD)])
{
    constexpr int NR = (LA + LB + LC + LD) / 2 + 1;
    eri_accumulate_cd<LA, LB, LC, LD, 0, ncart(LC) * ncart(LD), SKIP>(bra, pb, ket, pk, acc,
                                                                      RysTab<double>::ptr(NR));
}

// primitive pairs read from the precomputed pair arrays (SoA)
struct PPStored {
    PrimPairs pp;
    __device__ __forceinline__ PrimVals get(const PairRec &pr, int i) const
    {
        const int k = pr.off + i;
        PrimVals v;
        v.p = __ldg(pp.p + k);
        v.Px = __ldg(pp.Px + k);
        v.Py = __ldg(pp.Py + k);
        v.Pz = __ldg(pp.Pz + k);
        v.K = __ldg(pp.K + k);
        v.h = 0.5 / v.p;
        return v;
    }
};

// primitive pairs of the Fock build: one 48-byte record per pair,
// {p, K}, {Px, Py}, {Pz, 1/(2p)}, read with three 16-byte loads
#define GTF_PPREC_D2 3
struct PPRec {
    const double2 *r;
    __device__ __forceinline__ PrimVals get(const PairRec &pr, int i) const
    {
        const double2 *q = r + (size_t)GTF_PPREC_D2 * (pr.off + i);
        const double2 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
        PrimVals v;
        v.p = a.x;
        v.K = a.y;
        v.Px = b.x;
        v.Py = b.y;
        v.Pz = c.x;
        v.h = c.y;
        return v;
    }
};

// ---------------------------------------------------------------------------
// Warp sum of M values per lane (M <= 32) by recursive halving: at each of
// the first log2(MP) butterfly steps a lane keeps half of its values and
// sends the other half to its partner, so the whole reduction costs MP-1
// shuffles (MP = M rounded up to a power of two) instead of 5 M.  Afterwards
// lane l holds the total of value index m = l >> (5 - log2 MP); the lanes
// with (l & (32/MP - 1)) == 0 and m < M each own one distinct total.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int pow2_ceil(int m) { return m <= 1 ? 1 : 2 * pow2_ceil((m + 1) / 2); }
__host__ __device__ constexpr int ilog2c(int m) { return m <= 1 ? 0 : 1 + ilog2c(m / 2); }

// Last i in [0, n) with prefix[i] <= u, for a non-decreasing prefix with
// prefix[0] = 0 <= u, searched by the whole warp (u and n warp-uniform, all
// lanes active): each step probes 32 positions and keeps the sub-range after
// the last probe that is <= u, so the search takes ceil(log32 n) dependent
// loads instead of log2 n.
__device__ __forceinline__ int warp_find_le(const long long *__restrict__ prefix, int n, long long u, int lane)
{
    int lo = 0, hi = n;
    while (hi - lo > 32) {
        const long long span = hi - lo;
        const int p = lo + (int)(span * lane / 32);
        const unsigned m = __ballot_sync(GTF_FULL_MASK, __ldg(prefix + p) <= u);
        const int j = 31 - __clz(m);
        const int nlo = lo + (int)(span * j / 32);
        hi = (j == 31) ? hi : lo + (int)(span * (j + 1) / 32);
        lo = nlo;
    }
    const bool le = (lane < hi - lo) && __ldg(prefix + lo + lane) <= u;
    const unsigned m = __ballot_sync(GTF_FULL_MASK, le);
    return lo + 31 - __clz(m);
}

template <int M, class Sink>
__device__ __forceinline__ void warp_sum_values(const double *v, int lane, Sink &&sink)
{
    static_assert(M >= 1 && M <= 32, "at most 32 values per call");
    constexpr int MP = pow2_ceil(M), LG = ilog2c(MP);
    double w[MP];
#pragma unroll
    for (int k = 0; k < MP; k++) w[k] = k < M ? v[k] : 0.0;
    int m = 0;
#pragma unroll
    for (int st = 0; st < LG; st++) {
        const int h = MP >> (st + 1), o = 16 >> st;
        const bool up = (lane & o) != 0;
#pragma unroll
        for (int k = 0; k < h; k++) {
            const double send = up ? w[k] : w[k + h];
            const double keep = up ? w[k + h] : w[k];
            w[k] = keep + __shfl_xor_sync(GTF_FULL_MASK, send, o);
        }
        if (up) m += h;
    }
#pragma unroll
    for (int o = 16 >> LG; o >= 1; o >>= 1) w[0] += __shfl_xor_sync(GTF_FULL_MASK, w[0], o);
    if ((lane & ((32 >> LG) - 1)) == 0 && m < M) sink(m, w[0]);
}

// any M: chunks of 32 values
template <int M, int C0 = 0, class Sink>
__device__ __forceinline__ void warp_sum_many(const double (&v)[M], int lane, Sink &&sink)
{
    if constexpr (C0 < M) {
        constexpr int n = (M - C0 < 32) ? M - C0 : 32;
        warp_sum_values<n>(v + C0, lane, [&](int m, double t) { sink(C0 + m, t); });
        warp_sum_many<M, C0 + 32>(v, lane, sink);
    }
}

// ---------------------------------------------------------------------------
// J/K digestion of one unique quartet (pfock/fock_task.c:29-117 semantics):
//   Fj[a][b] += 2(1+f1)(1+f2)         sum_cd D[c][d] I
//   Fj[c][d] += 2 f3 (1+f1)(1+f2)     sum_ab D[a][b] I
//   Fk[a][c] -= (1+f3)                sum_bd D[b][d] I
//   Fk[b][c] -= f1 (1+f3)             sum_ad D[a][d] I
//   Fk[a][d] -= f2 (1+f3)             sum_bc D[b][c] I
//   Fk[b][d] -= f1 f2 (1+f3)          sum_ac D[a][c] I
// f1 = a!=b, f2 = c!=d, f3 = bra pair != ket pair.  The caller symmetrises
// Fj and Fk afterwards (GA_Symmetrize, pfock/pfock.c:1719-1726).
// The bra pair is shared by the 32 lanes of the warp; `active` lanes carry a
// quartet, inactive lanes contribute zeros to the warp reductions.
// digest_cd<..., CD0, N> digests the slice of ket components
// cd = CD0 .. CD0+N-1 (cd = ic + NC*id) of the quartet; terms whose
// destination sums over the sliced index (Fj[a][b], Fk[a][c], Fk[b][c])
// receive a partial sum per slice.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr bool slice_has_c(int CD0, int N, int NC, int ic)
{
    for (int t = 0; t < N; t++)
        if ((CD0 + t) % NC == ic) return true;
    return false;
}

__host__ __device__ constexpr bool slice_has_d(int CD0, int N, int NC, int id)
{
    for (int t = 0; t < N; t++)
        if ((CD0 + t) / NC == id) return true;
    return false;
}

template <int LA, int LB, int LC, int LD, int CD0, int N, typename R>
__device__ __forceinline__ void digest_cd(const R (&I)[ncart(LA) * ncart(LB) * N], bool active,
                                          const PairRec &pb, const PairRec &pk, bool same_pair,
                                          const double *__restrict__ D, double *__restrict__ Fj,
                                          double *__restrict__ Fk, int ld, int lane, bool konly = false)
{
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    const int fa = pb.fa, fb = pb.fb, fc = pk.fa, fd = pk.fb;
    const double f1 = (fa != fb) ? 1.0 : 0.0;
    const double f2 = (fc != fd) ? 1.0 : 0.0;
    const double f3 = same_pair ? 0.0 : 1.0;
    const double sJab = 2.0 * (1.0 + f1) * (1.0 + f2);
    const double sJcd = f3 * sJab;
    const double sKac = -(1.0 + f3);
    const double sKbc = f1 * sKac, sKad = f2 * sKac, sKbd = f1 * f2 * sKac;
    // bra block J (warp-uniform destination), partial over the slice; konly
    // (warp-uniform) skips both Coulomb terms
    if (!konly) {
        double dcd[N];
#pragma unroll
        for (int t = 0; t < N; t++) {
            const int ic = (CD0 + t) % NC, id = (CD0 + t) / NC;
            dcd[t] = active ? __ldg(D + (size_t)(fc + ic) * ld + fd + id) : 0.0;
        }
        double vab[NA * NB];
#pragma unroll
        for (int k = 0; k < NA * NB; k++) {
            double v = 0.0;
#pragma unroll
            for (int t = 0; t < N; t++) v = fma((double)I[k + NA * NB * t], dcd[t], v);
            vab[k] = v * sJab;  // the factor depends on the lane's ket
        }
        warp_sum_many<NA * NB>(vab, lane, [&](int k, double t) {
            atomicAdd(Fj + (size_t)(fa + k % NA) * ld + fb + k / NA, t);
        });
    }
    if (!active) return;
    // ket block J: complete per (c, d)
    if (f3 != 0.0 && !konly) {
        double dab[NA * NB];
#pragma unroll
        for (int ia = 0; ia < NA; ia++)
#pragma unroll
            for (int ibb = 0; ibb < NB; ibb++) dab[ia + NA * ibb] = __ldg(D + (size_t)(fa + ia) * ld + fb + ibb);
#pragma unroll
        for (int t = 0; t < N; t++) {
            const int ic = (CD0 + t) % NC, id = (CD0 + t) / NC;
            double v = 0.0;
#pragma unroll
            for (int ibb = 0; ibb < NB; ibb++)
#pragma unroll
                for (int ia = 0; ia < NA; ia++) v = fma((double)I[ia + NA * (ibb + NB * t)], dab[ia + NA * ibb], v);
            atomicAdd(Fj + (size_t)(fc + ic) * ld + fd + id, sJcd * v);
        }
    }
    // K[a][c] -= (1+f3) sum_bd D[b][d] I   and   K[b][c] -= f1 (1+f3) sum_ad D[a][d] I
#pragma unroll
    for (int ic = 0; ic < NC; ic++) {
        if (!slice_has_c(CD0, N, NC, ic)) continue;
#pragma unroll
        for (int ia = 0; ia < NA; ia++) {
            double v = 0.0;
#pragma unroll
            for (int t = 0; t < N; t++) {
                if ((CD0 + t) % NC != ic) continue;
                const int id = (CD0 + t) / NC;
#pragma unroll
                for (int ibb = 0; ibb < NB; ibb++)
                    v = fma((double)I[ia + NA * (ibb + NB * t)], __ldg(D + (size_t)(fb + ibb) * ld + fd + id), v);
            }
            atomicAdd(Fk + (size_t)(fa + ia) * ld + fc + ic, sKac * v);
        }
        if (f1 != 0.0) {
#pragma unroll
            for (int ibb = 0; ibb < NB; ibb++) {
                double v = 0.0;
#pragma unroll
                for (int t = 0; t < N; t++) {
                    if ((CD0 + t) % NC != ic) continue;
                    const int id = (CD0 + t) / NC;
#pragma unroll
                    for (int ia = 0; ia < NA; ia++)
                        v = fma((double)I[ia + NA * (ibb + NB * t)], __ldg(D + (size_t)(fa + ia) * ld + fd + id), v);
                }
                atomicAdd(Fk + (size_t)(fb + ibb) * ld + fc + ic, sKbc * v);
            }
        }
    }
    // K[a][d] -= f2 (1+f3) sum_bc D[b][c] I   and   K[b][d] -= f1 f2 (1+f3) sum_ac D[a][c] I
    if (f2 != 0.0) {
#pragma unroll
        for (int id = 0; id < ND; id++) {
            if (!slice_has_d(CD0, N, NC, id)) continue;
#pragma unroll
            for (int ia = 0; ia < NA; ia++) {
                double v = 0.0;
#pragma unroll
                for (int t = 0; t < N; t++) {
                    if ((CD0 + t) / NC != id) continue;
                    const int ic = (CD0 + t) % NC;
#pragma unroll
                    for (int ibb = 0; ibb < NB; ibb++)
                        v = fma((double)I[ia + NA * (ibb + NB * t)], __ldg(D + (size_t)(fb + ibb) * ld + fc + ic), v);
                }
                atomicAdd(Fk + (size_t)(fa + ia) * ld + fd + id, sKad * v);
            }
            if (f1 != 0.0) {
#pragma unroll
                for (int ibb = 0; ibb < NB; ibb++) {
                    double v = 0.0;
#pragma unroll
                    for (int t = 0; t < N; t++) {
                        if ((CD0 + t) / NC != id) continue;
                        const int ic = (CD0 + t) % NC;
#pragma unroll
                        for (int ia = 0; ia < NA; ia++)
                            v = fma((double)I[ia + NA * (ibb + NB * t)], __ldg(D + (size_t)(fa + ia) * ld + fc + ic), v);
                    }
                    atomicAdd(Fk + (size_t)(fb + ibb) * ld + fd + id, sKbd * v);
                }
            }
        }
    }
}
