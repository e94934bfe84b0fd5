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

#include "devmem.cuh"
#include "gtf_cuda.h"
#include "gtf_dev.cuh"

extern "C" void gtf_fock_basis_dev(gtf_fock_dev_t *f, const int **sh_L, const int **sh_nprim,
                                   const int **sh_pstart, const int **f_start, const int **fc_start,
                                   const double **sh_xyz, const double **alpha, const double **coef,
                                   const int **Z, const double **atom_xyz, int *nshells, int *natoms, int *nbf,
                                   int *pure);
extern "C" void *gtf_fock_stream(gtf_fock_dev_t *f);

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

__device__ __forceinline__ int cx_of(int L, int c) { return cart_x(L, c); }
__device__ __forceinline__ int cy_of(int L, int c) { return cart_y(L, c); }
__device__ __forceinline__ int cz_of(int L, int c) { return cart_z(L, c); }

template <int N>
__device__ void nuclear_rys(double T, double (&u)[3], double (&w)[3])
{
    double uu[N], ww[N];
    rys_roots<N>(T, uu, ww, RysTab<double>::ptr(N));
#pragma unroll
    for (int i = 0; i < N; i++) {
        u[i] = uu[i];
        w[i] = ww[i];
    }
}

__global__ void __launch_bounds__(128) k_onee(const int *__restrict__ sh_L, const int *__restrict__ sh_nprim,
                                              const int *__restrict__ sh_pstart, const int *__restrict__ f_start,
                                              const double *__restrict__ sh_xyz, const double *__restrict__ alpha,
                                              const double *__restrict__ coef, const int *__restrict__ Z,
                                              const double *__restrict__ atom_xyz, int ns, int natoms, int nbf,
                                              int pure, double *__restrict__ S, double *__restrict__ H,
                                              double *__restrict__ Tout, double *__restrict__ Vout)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)ns * ns) return;
    const int A = (int)(t / ns), B = (int)(t % ns);
    const int LA = sh_L[A], LB = sh_L[B];
    const int na = ncart(LA), nb = ncart(LB);
    const double Ax = sh_xyz[3 * A], Ay = sh_xyz[3 * A + 1], Az = sh_xyz[3 * A + 2];
    const double Bx = sh_xyz[3 * B], By = sh_xyz[3 * B + 1], Bz = sh_xyz[3 * B + 2];
    const double R2 = (Ax - Bx) * (Ax - Bx) + (Ay - By) * (Ay - By) + (Az - Bz) * (Az - Bz);
    double Sc[36], Tc[36], Vc[36];
    for (int k = 0; k < 36; k++) {
        Sc[k] = 0.0;
        Tc[k] = 0.0;
        Vc[k] = 0.0;
    }
    const int nroot = (LA + LB) / 2 + 1;
    for (int i = 0; i < sh_nprim[A]; i++) {
        for (int j = 0; j < sh_nprim[B]; j++) {
            const double a = alpha[sh_pstart[A] + i], b = alpha[sh_pstart[B] + j];
            const double p = a + b, ip = 1.0 / p;
            const double K = coef[sh_pstart[A] + i] * coef[sh_pstart[B] + j] * exp(-a * b * ip * R2);
            const double P[3] = {(a * Ax + b * Bx) * ip, (a * Ay + b * By) * ip, (a * Az + b * Bz) * ip};
            const double PA[3] = {P[0] - Ax, P[1] - Ay, P[2] - Az};
            const double PB[3] = {P[0] - Bx, P[1] - By, P[2] - Bz};
            // 1-D overlap factors s[d][ia][jb], ia <= 2, jb <= 4 (Gauss-Hermite, exact)
            double s[3][3][5];
            const double rsp = rsqrt(p);
            for (int d = 0; d < 3; d++) {
                for (int ia = 0; ia <= LA; ia++)
                    for (int jb = 0; jb <= LB + 2; jb++) s[d][ia][jb] = 0.0;
                for (int k = 0; k < 4; k++) {
                    const double x = c_gh_x[k] * rsp;
                    const double xa = x + PA[d], xb = x + PB[d];
                    double pa = 1.0;
                    for (int ia = 0; ia <= LA; ia++) {
                        double pb = 1.0;
                        for (int jb = 0; jb <= LB + 2; jb++) {
                            s[d][ia][jb] += c_gh_w[k] * pa * pb;
                            pb *= xb;
                        }
                        pa *= xa;
                    }
                }
                for (int ia = 0; ia <= LA; ia++)
                    for (int jb = 0; jb <= LB + 2; jb++) s[d][ia][jb] *= rsp;
            }
            // nuclear attraction: Rys quadrature per nucleus
            double V[36];
            for (int k = 0; k < na * nb; k++) V[k] = 0.0;
            for (int c = 0; c < natoms; c++) {
                const double PC[3] = {P[0] - atom_xyz[3 * c], P[1] - atom_xyz[3 * c + 1], P[2] - atom_xyz[3 * c + 2]};
                const double T = p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
                double u[3], w[3];
                if (nroot == 1) nuclear_rys<1>(T, u, w);
                else if (nroot == 2) nuclear_rys<2>(T, u, w);
                else nuclear_rys<3>(T, u, w);
                const double pref = -(double)Z[c] * 2.0 * M_PI * ip * K;
                for (int r = 0; r < nroot; r++) {
                    const double Bv = (1.0 - u[r]) * 0.5 * ip;
                    double I1[3][3][3];  // [dim][ia][jb]
                    for (int d = 0; d < 3; d++) {
                        const double C = PA[d] - u[r] * PC[d];
                        const double AB = (d == 0 ? Ax - Bx : d == 1 ? Ay - By : Az - Bz);
                        double g[5];
                        g[0] = 1.0;
                        if (LA + LB >= 1) g[1] = C;
                        for (int e = 1; e < LA + LB; e++) g[e + 1] = C * g[e] + e * Bv * g[e - 1];
                        // transfer to (ia, jb): t(a, b+1) = t(a+1, b) + AB t(a, b)
                        double tt[5][3];
                        for (int e = 0; e <= LA + LB; e++) tt[e][0] = g[e];
                        for (int jb = 0; jb < LB; jb++)
                            for (int e = 0; e <= LA + LB - jb - 1; e++) tt[e][jb + 1] = tt[e + 1][jb] + AB * tt[e][jb];
                        for (int ia = 0; ia <= LA; ia++)
                            for (int jb = 0; jb <= LB; jb++) I1[d][ia][jb] = tt[ia][jb];
                    }
                    const double wr = w[r] * pref;
                    for (int ib = 0; ib < nb; ib++)
                        for (int ia = 0; ia < na; ia++)
                            V[ia + na * ib] += wr * I1[0][cx_of(LA, ia)][cx_of(LB, ib)] *
                                               I1[1][cy_of(LA, ia)][cy_of(LB, ib)] *
                                               I1[2][cz_of(LA, ia)][cz_of(LB, ib)];
                }
            }
            for (int ib = 0; ib < nb; ib++) {
                const int bx = cx_of(LB, ib), by = cy_of(LB, ib), bz = cz_of(LB, ib);
                for (int ia = 0; ia < na; ia++) {
                    const int ax = cx_of(LA, ia), ay = cy_of(LA, ia), az = cz_of(LA, ia);
                    const int ex[3] = {ax, ay, az}, eb[3] = {bx, by, bz};
                    const double sv = s[0][ax][bx] * s[1][ay][by] * s[2][az][bz];
                    double tv = 0.0;
                    for (int d = 0; d < 3; d++) {
                        const int ii = ex[d], jj = eb[d];
                        double v = -2.0 * b * (2 * jj + 1) * s[d][ii][jj] + 4.0 * b * b * s[d][ii][jj + 2];
                        if (jj >= 2) v += jj * (jj - 1) * s[d][ii][jj - 2];
                        double o = 1.0;
                        for (int e = 0; e < 3; e++)
                            if (e != d) o *= s[e][ex[e]][eb[e]];
                        tv += -0.5 * v * o;
                    }
                    Sc[ia + na * ib] += K * sv;
                    Tc[ia + na * ib] += K * tv;
                    Vc[ia + na * ib] += V[ia + na * ib];
                }
            }
        }
    }
    const int sa = (pure && LA == 2) ? 5 : na, sb = (pure && LB == 2) ? 5 : nb;
    const int fa = f_start[A], fb = f_start[B];
    for (int m = 0; m < sa; m++) {
        for (int n = 0; n < sb; n++) {
            double vs = 0.0, vt = 0.0, vv = 0.0;
            for (int ia = 0; ia < na; ia++) {
                const double tm = (pure && LA == 2) ? c_sph_d1[m][ia] : (m == ia ? 1.0 : 0.0);
                if (tm == 0.0) continue;
                for (int ib = 0; ib < nb; ib++) {
                    const double tn = (pure && LB == 2) ? c_sph_d1[n][ib] : (n == ib ? 1.0 : 0.0);
                    if (tn == 0.0) continue;
                    vs += tm * tn * Sc[ia + na * ib];
                    vt += tm * tn * Tc[ia + na * ib];
                    vv += tm * tn * Vc[ia + na * ib];
                }
            }
            const size_t o = (size_t)(fa + m) * nbf + fb + n;
            if (S) S[o] = vs;
            if (H) H[o] = vt + vv;
            if (Tout) Tout[o] = vt;
            if (Vout) Vout[o] = vv;
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
    const long long npair = (long long)ns * ns;
    k_onee<<<(unsigned)((npair + 127) / 128), 128, 0, st>>>(sh_L, sh_nprim, sh_pstart, f_start, sh_xyz, alpha,
                                                            coef, Z, atom_xyz, ns, natoms, nbf, pure, dS, dH,
                                                            nullptr, nullptr);
    CKC(cudaGetLastError());
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
    const long long npair = (long long)ns * ns;
    k_onee<<<(unsigned)((npair + 127) / 128), 128, 0, st>>>(sh_L, sh_nprim, sh_pstart, f_start, sh_xyz, alpha,
                                                            coef, Z, atom_xyz, ns, natoms, nbf, pure, buf, nullptr,
                                                            buf + nn, buf + 2 * nn);
    CKC(cudaGetLastError());
    if (S_host) CKC(cudaMemcpyAsync(S_host, buf, sizeof(double) * nn, cudaMemcpyDeviceToHost, st));
    if (T_host) CKC(cudaMemcpyAsync(T_host, buf + nn, sizeof(double) * nn, cudaMemcpyDeviceToHost, st));
    if (V_host) CKC(cudaMemcpyAsync(V_host, buf + 2 * nn, sizeof(double) * nn, cudaMemcpyDeviceToHost, st));
    CKC(cudaStreamSynchronize(st));
    gtf_dfree(buf, st);
    return GTF_OK;
}
