// onee.cu -- one-electron matrices on the device (pfock/one_electron.c:28-119,
// pfock/pfock.c:1732-1867): overlap S, core Hamiltonian H = T + V and
// X = U diag(lambda^-1/2) U^T from the eigen-decomposition of S.
//
//   * S and T: each 1-D factor is an exact 4-point Gauss-Hermite quadrature
//     of the product Gaussian (polynomial degree <= 6 for L <= 2);
//   * V: Rys quadrature of 1/|r - C| with the same root table as the ERIs;
//   * eigenvectors of S: cuSOLVER dsyevd (setup only), X by one DGEMM.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>
#include <stdio.h>

#include <vector>

#include "devmem.cuh"
#include "gtf_cuda.h"
#include "gtf_dev.cuh"

extern "C" void gtf_fock_basis_dev(gtf_fock_dev_t *f, const int **sh_L, const int **sh_nprim,
                                   const int **sh_pstart, const int **f_start, const int **fc_start,
                                   const double **sh_xyz, const double **alpha, const double **coef,
                                   const int **Z, const double **atom_xyz, int *nshells, int *natoms, int *nbf,
                                   int *pure);
extern "C" void *gtf_fock_stream(gtf_fock_dev_t *f);
extern "C" const int *gtf_fock_shell_L_host(gtf_fock_dev_t *f);

__constant__ double c_gh_x[4] = {-1.6506801238857845559, -0.52464762327529031788, 0.52464762327529031788,
                                 1.6506801238857845559};
__constant__ double c_gh_w[4] = {0.081312835447245177143, 0.80491409000551283651, 0.80491409000551283651,
                                 0.081312835447245177143};
__constant__ double c_sph_d1[5][6] = {
    {0.0, 1.7320508075688772, 0.0, 0.0, 0.0, 0.0},
    {0.0, 0.0, 0.0, 0.0, 1.7320508075688772, 0.0},
    {-0.5, 0.0, 0.0, -0.5, 0.0, 1.0},
    {0.0, 0.0, 1.7320508075688772, 0.0, 0.0, 0.0},
    {0.8660254037844386, 0.0, 0.0, -0.8660254037844386, 0.0, 0.0}};

// One warp per unordered shell pair {A, B}, oriented so that L(A) >= L(B).
// The lanes share out the pair's primitive pairs for S and T, and its
// (primitive pair, nucleus) terms for V; the warp sums are taken by shuffles
// in a fixed order, so the matrices are the same from run to run.  The block
// of (A, B) is written together with its transpose, so S and H come out
// exactly symmetric.  One launch per angular class pair keeps every
// per-pair array in registers.
struct OneePair {
    int a, b;
};

template <int N>
__device__ __forceinline__ void warp_sum(double (&v)[N])
{
#pragma unroll
    for (int k = 0; k < N; k++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
}

// spherical (pure d) or Cartesian block of c1 (+ c2 when given) at rows
// fa.., columns fb.., and at the mirrored place.  A diagonal block (fa == fb)
// is evaluated on and above its diagonal and mirrored, since the two
// triangles of c1 agree only to rounding (contracted multiply-adds).
template <int LA, int LB>
__device__ __forceinline__ void onee_put(const double (&c1)[ncart(LA) * ncart(LB)], const double *c2, int pure,
                                         int fa, int fb, int nbf, double *__restrict__ M)
{
    constexpr int NA = ncart(LA), NB = ncart(LB);
    const int sa = (pure && LA == 2) ? 5 : NA, sb = (pure && LB == 2) ? 5 : NB;
    const bool diag = fa == fb;
    for (int m = 0; m < sa; m++) {
        for (int n = diag ? m : 0; n < sb; n++) {
            double v1 = 0.0, v2 = 0.0;
#pragma unroll
            for (int ia = 0; ia < NA; ia++) {
                const double tm = (pure && LA == 2) ? c_sph_d1[m][ia] : (m == ia ? 1.0 : 0.0);
#pragma unroll
                for (int ib = 0; ib < NB; ib++) {
                    const double tn = (pure && LB == 2) ? c_sph_d1[n][ib] : (n == ib ? 1.0 : 0.0);
                    v1 += tm * tn * c1[ia + NA * ib];
                    if (c2) v2 += tm * tn * c2[ia + NA * ib];
                }
            }
            const double v = c2 ? v1 + v2 : v1;
            M[(size_t)(fa + m) * nbf + fb + n] = v;
            M[(size_t)(fb + n) * nbf + fa + m] = v;
        }
    }
}

template <int LA, int LB, bool WANT_V>
__global__ void __launch_bounds__(128)
    k_onee(const OneePair *__restrict__ pairs, int npairs, const int *__restrict__ sh_nprim,
           const int *__restrict__ sh_pstart, const int *__restrict__ f_start, const double *__restrict__ sh_xyz,
           const double *__restrict__ alpha, const double *__restrict__ coef, const int *__restrict__ Z,
           const double *__restrict__ atom_xyz, int natoms, int nbf, int pure, double *__restrict__ S,
           double *__restrict__ H, double *__restrict__ Tout, double *__restrict__ Vout)
{
    constexpr int NA = ncart(LA), NB = ncart(LB), NR = (LA + LB) / 2 + 1;
    __shared__ double s_t[4][NA * NB];  // the warp's T block, kept across the V loop
    const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    if (w >= npairs) return;  // the same for every lane of the warp
    const int A = pairs[w].a, B = pairs[w].b;
    const double Ac[3] = {sh_xyz[3 * A], sh_xyz[3 * A + 1], sh_xyz[3 * A + 2]};
    const double Bc[3] = {sh_xyz[3 * B], sh_xyz[3 * B + 1], sh_xyz[3 * B + 2]};
    const double AB[3] = {Ac[0] - Bc[0], Ac[1] - Bc[1], Ac[2] - Bc[2]};
    const double R2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
    const int npa = sh_nprim[A], npb = sh_nprim[B], pa0 = sh_pstart[A], pb0 = sh_pstart[B];
    const int npp = npa * npb;
    const int fa = f_start[A], fb = f_start[B];

    // S and T: lanes over primitive pairs
    double Sc[NA * NB], Tc[NA * NB];
#pragma unroll
    for (int k = 0; k < NA * NB; k++) {
        Sc[k] = 0.0;
        Tc[k] = 0.0;
    }
    for (int q = lane; q < npp; q += 32) {
        const int i = q / npb, j = q - i * npb;
        const double a = alpha[pa0 + i], b = alpha[pb0 + j];
        const double p = a + b, ip = 1.0 / p;
        const double K = coef[pa0 + i] * coef[pb0 + j] * exp(-a * b * ip * R2);
        // 1-D overlap factors s[d][ia][jb] (4-point Gauss-Hermite, exact to degree 7)
        double s[3][LA + 1][LB + 3];
        const double rsp = rsqrt(p);
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const double P = (a * Ac[d] + b * Bc[d]) * ip;
            const double PA = P - Ac[d], PB = P - Bc[d];
#pragma unroll
            for (int ia = 0; ia <= LA; ia++)
#pragma unroll
                for (int jb = 0; jb <= LB + 2; jb++) s[d][ia][jb] = 0.0;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const double x = c_gh_x[k] * rsp;
                const double xa = x + PA, xb = x + PB;
                double pa = 1.0;
#pragma unroll
                for (int ia = 0; ia <= LA; ia++) {
                    double pb = 1.0;
#pragma unroll
                    for (int jb = 0; jb <= LB + 2; jb++) {
                        s[d][ia][jb] += c_gh_w[k] * pa * pb;
                        pb *= xb;
                    }
                    pa *= xa;
                }
            }
#pragma unroll
            for (int ia = 0; ia <= LA; ia++)
#pragma unroll
                for (int jb = 0; jb <= LB + 2; jb++) s[d][ia][jb] *= rsp;
        }
#pragma unroll
        for (int ib = 0; ib < NB; ib++) {
#pragma unroll
            for (int ia = 0; ia < NA; ia++) {
                const int ex[3] = {cart_x(LA, ia), cart_y(LA, ia), cart_z(LA, ia)};
                const int eb[3] = {cart_x(LB, ib), cart_y(LB, ib), cart_z(LB, ib)};
                const double sv = s[0][ex[0]][eb[0]] * s[1][ex[1]][eb[1]] * s[2][ex[2]][eb[2]];
                double tv = 0.0;
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    const int ii = ex[d], jj = eb[d];
                    double v = -2.0 * b * (2 * jj + 1) * s[d][ii][jj] + 4.0 * b * b * s[d][ii][jj + 2];
                    if (jj >= 2) v += jj * (jj - 1) * s[d][ii][jj >= 2 ? jj - 2 : 0];
                    double o = 1.0;
#pragma unroll
                    for (int e = 0; e < 3; e++)
                        if (e != d) o *= s[e][ex[e]][eb[e]];
                    tv += -0.5 * v * o;
                }
                Sc[ia + NA * ib] += K * sv;
                Tc[ia + NA * ib] += K * tv;
            }
        }
    }
    warp_sum(Sc);
    warp_sum(Tc);
    if (lane == 0) {
        if (S) onee_put<LA, LB>(Sc, nullptr, pure, fa, fb, nbf, S);
        if (Tout) onee_put<LA, LB>(Tc, nullptr, pure, fa, fb, nbf, Tout);
#pragma unroll
        for (int k = 0; k < NA * NB; k++) s_t[wib][k] = Tc[k];
    }
    if constexpr (WANT_V) {
        // V: lanes over (primitive pair, nucleus), Rys quadrature of 1/|r - C|
        double Vc[NA * NB];
#pragma unroll
        for (int k = 0; k < NA * NB; k++) Vc[k] = 0.0;
        const int nq = npp * natoms;
        for (int q = lane; q < nq; q += 32) {
            const int pp = q / natoms, c = q - pp * natoms;
            const int i = pp / npb, j = pp - i * npb;
            const double a = alpha[pa0 + i], b = alpha[pb0 + j];
            const double p = a + b, ip = 1.0 / p;
            const double K = coef[pa0 + i] * coef[pb0 + j] * exp(-a * b * ip * R2);
            double PA[3], PC[3];
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const double P = (a * Ac[d] + b * Bc[d]) * ip;
                PA[d] = P - Ac[d];
                PC[d] = P - atom_xyz[3 * c + d];
            }
            const double T = p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
            double u[NR], wt[NR];
            rys_roots<NR>(T, u, wt, RysTab<double>::ptr(NR));
            const double pref = -(double)Z[c] * 2.0 * M_PI * ip * K;
#pragma unroll
            for (int r = 0; r < NR; r++) {
                const double Bv = (1.0 - u[r]) * 0.5 * ip;
                double I1[3][LA + 1][LB + 1];  // [dim][ia][jb]
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    const double C = PA[d] - u[r] * PC[d];
                    double g[LA + LB + 1];
                    g[0] = 1.0;
                    if (LA + LB >= 1) g[LA + LB >= 1 ? 1 : 0] = C;
#pragma unroll
                    for (int e = 1; e < LA + LB; e++) g[e + 1] = C * g[e] + e * Bv * g[e - 1];
                    // transfer to (ia, jb): t(a, b+1) = t(a+1, b) + AB t(a, b)
                    double tt[LA + LB + 1][LB + 1];
#pragma unroll
                    for (int e = 0; e <= LA + LB; e++) tt[e][0] = g[e];
#pragma unroll
                    for (int jb = 0; jb < LB; jb++)
#pragma unroll
                        for (int e = 0; e <= LA + LB - jb - 1; e++) tt[e][jb + 1] = tt[e + 1][jb] + AB[d] * tt[e][jb];
#pragma unroll
                    for (int ia = 0; ia <= LA; ia++)
#pragma unroll
                        for (int jb = 0; jb <= LB; jb++) I1[d][ia][jb] = tt[ia][jb];
                }
                const double wr = wt[r] * pref;
#pragma unroll
                for (int ib = 0; ib < NB; ib++)
#pragma unroll
                    for (int ia = 0; ia < NA; ia++)
                        Vc[ia + NA * ib] += wr * I1[0][cart_x(LA, ia)][cart_x(LB, ib)] *
                                            I1[1][cart_y(LA, ia)][cart_y(LB, ib)] *
                                            I1[2][cart_z(LA, ia)][cart_z(LB, ib)];
            }
        }
        warp_sum(Vc);
        if (lane == 0) {
            if (Vout) onee_put<LA, LB>(Vc, nullptr, pure, fa, fb, nbf, Vout);
            if (H) {
                double Tk[NA * NB];
#pragma unroll
                for (int k = 0; k < NA * NB; k++) Tk[k] = s_t[wib][k];
                onee_put<LA, LB>(Tk, Vc, pure, fa, fb, nbf, H);
            }
        }
    }
}

__global__ void k_scale_cols(double *Y, const double *V, const double *w, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;  // row
    const int k = blockIdx.y;                             // eigenvector (column-major column)
    if (i >= n) return;
    Y[(size_t)k * n + i] = V[(size_t)k * n + i] * rsqrt(w[k]);
}

#define CKC(call)                                                                       \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            fprintf(stderr, "gtfock_b200 %s:%d %s\n", __FILE__, __LINE__, cudaGetErrorString(e_)); \
            return GTF_ERR_CUDA;                                                        \
        }                                                                               \
    } while (0)

// class index of an oriented pair L(A) >= L(B): ss, ps, pp, ds, dp, dd
static int onee_class(int la, int lb) { return la * (la + 1) / 2 + lb; }

template <bool WANT_V>
static void onee_launch_class(int cls, unsigned grid, cudaStream_t st, const OneePair *pairs, int n,
                              const int *sh_nprim, const int *sh_pstart, const int *f_start,
                              const double *sh_xyz, const double *alpha, const double *coef, const int *Z,
                              const double *atom_xyz, int natoms, int nbf, int pure, double *S, double *H,
                              double *T, double *V)
{
#define GTF_ONEE(LA, LB)                                                                                  \
    k_onee<LA, LB, WANT_V><<<grid, 128, 0, st>>>(pairs, n, sh_nprim, sh_pstart, f_start, sh_xyz, alpha, \
                                                 coef, Z, atom_xyz, natoms, nbf, pure, S, H, T, V)
    switch (cls) {
    case 0: GTF_ONEE(0, 0); break;
    case 1: GTF_ONEE(1, 0); break;
    case 2: GTF_ONEE(1, 1); break;
    case 3: GTF_ONEE(2, 0); break;
    case 4: GTF_ONEE(2, 1); break;
    default: GTF_ONEE(2, 2); break;
    }
#undef GTF_ONEE
}

// S, H = T + V, T and V of the whole basis into the given device arrays (any
// may be null; V is evaluated only when H or V is asked for).  One warp per
// unordered shell pair, one launch per angular class pair, ordered on st.
static int onee_matrices(gtf_fock_dev_t *f, cudaStream_t st, double *S, double *H, double *T, double *V)
{
    const int *sh_L, *sh_nprim, *sh_pstart, *f_start, *fc_start, *Z;
    const double *sh_xyz, *alpha, *coef, *atom_xyz;
    int ns, natoms, nbf, pure;
    gtf_fock_basis_dev(f, &sh_L, &sh_nprim, &sh_pstart, &f_start, &fc_start, &sh_xyz, &alpha, &coef, &Z, &atom_xyz,
                       &ns, &natoms, &nbf, &pure);
    const int *hL = gtf_fock_shell_L_host(f);
    // the unordered pairs grouped by class, each oriented L(a) >= L(b)
    int count[6] = {0, 0, 0, 0, 0, 0};
    for (int A = 0; A < ns; A++) {
        if (hL[A] < 0 || hL[A] > 2) return GTF_ERR_INVALID;
        for (int B = 0; B <= A; B++) count[onee_class(hL[A] > hL[B] ? hL[A] : hL[B], hL[A] > hL[B] ? hL[B] : hL[A])]++;
    }
    int start[7] = {0};
    for (int c = 0; c < 6; c++) start[c + 1] = start[c] + count[c];
    std::vector<OneePair> h(start[6]);
    int fill[6];
    for (int c = 0; c < 6; c++) fill[c] = start[c];
    for (int A = 0; A < ns; A++)
        for (int B = 0; B <= A; B++) {
            const bool swap = hL[B] > hL[A];
            const OneePair pr = swap ? OneePair{B, A} : OneePair{A, B};
            h[fill[onee_class(hL[pr.a], hL[pr.b])]++] = pr;
        }
    OneePair *d = nullptr;
    CKC(gtf_dmalloc((void **)&d, sizeof(OneePair) * h.size(), st));
    CKC(cudaMemcpyAsync(d, h.data(), sizeof(OneePair) * h.size(), cudaMemcpyHostToDevice, st));
    const bool want_v = H || V;
    for (int c = 0; c < 6; c++) {
        if (!count[c]) continue;
        const unsigned grid = (unsigned)((count[c] + 3) / 4);  // 4 warps per block
        if (want_v)
            onee_launch_class<true>(c, grid, st, d + start[c], count[c], sh_nprim, sh_pstart, f_start, sh_xyz,
                                    alpha, coef, Z, atom_xyz, natoms, nbf, pure, S, H, T, V);
        else
            onee_launch_class<false>(c, grid, st, d + start[c], count[c], sh_nprim, sh_pstart, f_start, sh_xyz,
                                     alpha, coef, Z, atom_xyz, natoms, nbf, pure, S, H, T, V);
    }
    const cudaError_t e = cudaGetLastError();
    gtf_dfree(d, st);
    // h is read by the copy above: keep it until the stream has passed it
    const cudaError_t e2 = cudaStreamSynchronize(st);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        fprintf(stderr, "gtfock_b200 one-electron kernels: %s\n",
                cudaGetErrorString(e != cudaSuccess ? e : e2));
        return GTF_ERR_CUDA;
    }
    return GTF_OK;
}

extern "C" int gtf_onee_compute(gtf_fock_dev_t *f, int want_sx, int want_h, double **S, double **X, double **H)
{
    const int *sh_L, *sh_nprim, *sh_pstart, *f_start, *fc_start, *Z;
    const double *sh_xyz, *alpha, *coef, *atom_xyz;
    int ns, natoms, nbf, pure;
    gtf_fock_basis_dev(f, &sh_L, &sh_nprim, &sh_pstart, &f_start, &fc_start, &sh_xyz, &alpha, &coef, &Z, &atom_xyz,
                       &ns, &natoms, &nbf, &pure);
    cudaStream_t st = (cudaStream_t)gtf_fock_stream(f);
    const size_t nn = (size_t)nbf * nbf;
    double *dS = nullptr, *dH = nullptr;
    // S, H and X live in the device's stream-ordered pool on the engine's
    // stream, which frees them (devmem.cu); so do the eigensolver's buffers
    if (want_sx) {
        if (!*S) CKC(gtf_dmalloc((void **)S, sizeof(double) * nn, st));
        dS = *S;
    }
    if (want_h) {
        if (!*H) CKC(gtf_dmalloc((void **)H, sizeof(double) * nn, st));
        dH = *H;
    }
    {
        const int e = onee_matrices(f, st, dS, dH, nullptr, nullptr);
        if (e != GTF_OK) return e;
    }
    if (want_sx) {
        if (!*X) CKC(gtf_dmalloc((void **)X, sizeof(double) * nn, st));
        SolverLease sl(st);
        BlasLease bl(st);
        if (!sl.h || !bl.h) return GTF_ERR_CUDA;
        cusolverDnHandle_t sh = sl.h;
        cublasHandle_t bh = bl.h;
        double *V, *w, *Y, *work;
        int *info, lwork = 0;
        CKC(gtf_dmalloc((void **)&V, sizeof(double) * nn, st));
        CKC(gtf_dmalloc((void **)&Y, sizeof(double) * nn, st));
        CKC(gtf_dmalloc((void **)&w, sizeof(double) * nbf, st));
        CKC(gtf_dmalloc((void **)&info, sizeof(int), st));
        CKC(cudaMemcpyAsync(V, dS, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st));
        cusolverDnDsyevd_bufferSize(sh, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, nbf, V, nbf, w, &lwork);
        CKC(gtf_dmalloc((void **)&work, sizeof(double) * (lwork > 0 ? lwork : 1), st));
        cusolverStatus_t ss =
            cusolverDnDsyevd(sh, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, nbf, V, nbf, w, work, lwork, info);
        int hinfo = 0;
        CKC(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, st));
        CKC(cudaStreamSynchronize(st));
        int ret = GTF_OK;
        if (ss != CUSOLVER_STATUS_SUCCESS || hinfo != 0) {
            fprintf(stderr, "gtfock_b200: dsyevd of S failed (status %d, info %d)\n", (int)ss, hinfo);
            ret = GTF_ERR_CUDA;
        } else {
            dim3 g((nbf + 127) / 128, nbf);
            k_scale_cols<<<g, 128, 0, st>>>(Y, V, w, nbf);
            // column-major: X = Y V^T (symmetric, so the row-major copy is the same)
            const double one = 1.0, zero = 0.0;
            cublasDgemm(bh, CUBLAS_OP_N, CUBLAS_OP_T, nbf, nbf, nbf, &one, Y, nbf, V, nbf, &zero, *X, nbf);
            CKC(cudaStreamSynchronize(st));
        }
        gtf_dfree(V, st);
        gtf_dfree(Y, st);
        gtf_dfree(w, st);
        gtf_dfree(info, st);
        gtf_dfree(work, st);
        if (ret) return ret;
    }
    CKC(cudaStreamSynchronize(st));
    return GTF_OK;
}

// S, T and V of the whole basis into host arrays (any may be NULL); used by
// the per-pair CInt one-electron entry points
extern "C" int gtf_onee_full(gtf_fock_dev_t *f, double *S_host, double *T_host, double *V_host)
{
    const int *sh_L, *sh_nprim, *sh_pstart, *f_start, *fc_start, *Z;
    const double *sh_xyz, *alpha, *coef, *atom_xyz;
    int ns, natoms, nbf, pure;
    gtf_fock_basis_dev(f, &sh_L, &sh_nprim, &sh_pstart, &f_start, &fc_start, &sh_xyz, &alpha, &coef, &Z, &atom_xyz,
                       &ns, &natoms, &nbf, &pure);
    cudaStream_t st = (cudaStream_t)gtf_fock_stream(f);
    const size_t nn = (size_t)nbf * nbf;
    double *buf;
    CKC(gtf_dmalloc((void **)&buf, sizeof(double) * nn * 3, st));
    {
        const int e = onee_matrices(f, st, buf, nullptr, buf + nn, buf + 2 * nn);
        if (e != GTF_OK) {
            gtf_dfree(buf, st);
            return e;
        }
    }
    if (S_host) CKC(cudaMemcpyAsync(S_host, buf, sizeof(double) * nn, cudaMemcpyDeviceToHost, st));
    if (T_host) CKC(cudaMemcpyAsync(T_host, buf + nn, sizeof(double) * nn, cudaMemcpyDeviceToHost, st));
    if (V_host) CKC(cudaMemcpyAsync(V_host, buf + 2 * nn, sizeof(double) * nn, cudaMemcpyDeviceToHost, st));
    CKC(cudaStreamSynchronize(st));
    gtf_dfree(buf, st);
    return GTF_OK;
}
