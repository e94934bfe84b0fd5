/*
 * cint_oracle.c -- CPU FP64 integral engine of the oracle (test
 * infrastructure only: linked by tests/, the bench's CPU-baseline leg and the
 * reference-source build under oracle/ref/; never by the product library).
 *
 * Implements the integral half of GTFock's CInt interface
 * (libcint/include/CInt.h:90-181) whose reference implementation (OptErd via
 * libcint) ships only as a binary:
 *   - ERIs by Obara-Saika vertical recursion to [e0|f0] over primitives,
 *     contraction, then Head-Gordon-Pople horizontal recursion
 *     (Obara & Saika, J. Chem. Phys. 84, 3963 (1986); Head-Gordon & Pople,
 *     J. Chem. Phys. 89, 5777 (1988));
 *   - Boys function by its power series with downward recursion for T < 40
 *     and by the erf closed form with upward recursion above;
 *   - overlap / kinetic / nuclear attraction by the Obara-Saika recursions.
 * This is deliberately a different formulation from the GPU kernels (Rys
 * quadrature with fitted roots), so that agreement between the two checks both.
 *
 * Layout conventions follow include/CInt.h (first shell index fastest;
 * Cartesian order xx,xy,xz,yy,yz,zz; spherical d order m=-2..2).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "gtf_basis.h"

#define OR_MAXL 2
#define OR_MAXLT (4 * OR_MAXL)        /* max total L of a quartet */
#define OR_NT(L) (((L) + 1) * ((L) + 2) * ((L) + 3) / 6)
#define OR_NTRIP OR_NT(OR_MAXLT)      /* 165 triples with sum <= 8 */
#define OR_NT2 OR_NT(2 * OR_MAXL)     /* 35 triples with sum <= 4 */
#define OR_MAXCART 6
#define OR_MAXQ (OR_MAXCART * OR_MAXCART * OR_MAXCART * OR_MAXCART)

/* ---- Cartesian triple tables ---- */
static int g_tri_init = 0;
static int g_tri_idx[OR_MAXLT + 1][OR_MAXLT + 1][OR_MAXLT + 1];
static int g_tri[OR_NTRIP][3];

static void tri_init(void)
{
    if (g_tri_init) return;
    int n = 0;
    for (int L = 0; L <= OR_MAXLT; L++) {
        for (int x = L; x >= 0; x--) {
            for (int y = L - x; y >= 0; y--) {
                int z = L - x - y;
                g_tri_idx[x][y][z] = n;
                g_tri[n][0] = x;
                g_tri[n][1] = y;
                g_tri[n][2] = z;
                n++;
            }
        }
    }
    g_tri_init = 1;
}

/* index of the first triple of total L, and count of triples of total L */
static inline int tri_first(int L) { return L * (L + 1) * (L + 2) / 6; }
static inline int tri_count(int L) { return (L + 1) * (L + 2) / 2; }

/* ---- Boys function ---- */
static void boys(int mmax, double T, double *F)
{
    if (T < 40.0) {
        double et = exp(-T);
        double twoT = 2.0 * T;
        double term = 1.0 / (2 * mmax + 1);
        double sum = term;
        for (int k = 1; k < 400; k++) {
            term *= twoT / (2 * mmax + 2 * k + 1);
            sum += term;
            if (term < 1e-18 * sum) break;
        }
        F[mmax] = et * sum;
        for (int m = mmax; m > 0; m--) F[m - 1] = (twoT * F[m] + et) / (2 * m - 1);
    } else {
        double et = exp(-T);
        F[0] = 0.5 * sqrt(M_PI / T) * erf(sqrt(T));
        for (int m = 0; m < mmax; m++) F[m + 1] = ((2 * m + 1) * F[m] - et) / (2.0 * T);
    }
}

/* ---- spherical d transform (rows m=-2..2, cols xx,xy,xz,yy,yz,zz) ---- */
static const double k_s3 = 1.7320508075688772935;
static void sph_d_matrix(double c[5][6])
{
    memset(c, 0, sizeof(double) * 30);
    c[0][1] = k_s3;
    c[1][4] = k_s3;
    c[2][0] = -0.5;
    c[2][3] = -0.5;
    c[2][5] = 1.0;
    c[3][2] = k_s3;
    c[4][0] = 0.5 * k_s3;
    c[4][3] = -0.5 * k_s3;
}

/* Transform index `pos` (0..3) of a 4-index array with dims n[4] (first index
 * fastest) from 6 Cartesian d components to 5 spherical ones. */
static void sph_transform_index(double *in, double *out, int n[], int nidx, int pos)
{
    double c[5][6];
    sph_d_matrix(c);
    int stride = 1;
    for (int k = 0; k < pos; k++) stride *= n[k];
    int outer = 1;
    for (int k = pos + 1; k < nidx; k++) outer *= n[k];
    int nout = 5;
    for (int o = 0; o < outer; o++) {
        for (int s = 0; s < stride; s++) {
            for (int m = 0; m < nout; m++) {
                double v = 0.0;
                for (int k = 0; k < 6; k++) {
                    if (c[m][k] != 0.0) v += c[m][k] * in[s + stride * (k + 6 * o)];
                }
                out[s + stride * (m + nout * o)] = v;
            }
        }
    }
    n[pos] = nout;
}

/* ------------------------------------------------------------------------ */
/* ERI                                                                       */
/* ------------------------------------------------------------------------ */

typedef struct {
    double vrr[(OR_MAXLT + 1) * OR_NT2 * OR_NT2];
    double con[OR_NT2 * OR_NT2];
    double hb[OR_NT2 * 10 * OR_NT2];   /* bra HRR, [a][b][f] */
    double hb2[OR_NT2 * 10 * OR_NT2];
    double cart[OR_MAXQ];
    double tmp[OR_MAXQ];
    double out[OR_MAXQ];
} eri_ws_t;

struct ERD {
    int nthreads;
    eri_ws_t *ws;
};

/* Contracted Cartesian ERI block (ab|cd) for shells A,B,C,D; result in
 * w->cart with first index fastest. */
static void eri_cart(BasisSet_t bs, eri_ws_t *w, int A, int B, int C, int D)
{
    tri_init();
    const int la = bs->sh_L[A], lb = bs->sh_L[B], lc = bs->sh_L[C], ld = bs->sh_L[D];
    const int LB = la + lb, LK = lc + ld, L = LB + LK;
    const double *Ac = &bs->xyz[3 * bs->sh_atom[A]];
    const double *Bc = &bs->xyz[3 * bs->sh_atom[B]];
    const double *Cc = &bs->xyz[3 * bs->sh_atom[C]];
    const double *Dc = &bs->xyz[3 * bs->sh_atom[D]];
    double AB[3], CD[3];
    double rab2 = 0.0, rcd2 = 0.0;
    for (int i = 0; i < 3; i++) {
        AB[i] = Ac[i] - Bc[i];
        CD[i] = Cc[i] - Dc[i];
        rab2 += AB[i] * AB[i];
        rcd2 += CD[i] * CD[i];
    }
    const int ne = OR_NT(LB);      /* e triples with |e| <= LB */
    const int nf = OR_NT(LK);
    const int e0 = tri_first(la);  /* first needed e */
    const int f0 = tri_first(lc);
    memset(w->con, 0, sizeof(double) * ne * nf);
#define VRR(m, e, f) w->vrr[((m) * ne + (e)) * nf + (f)]
    const double *al = bs->alpha, *co = bs->coef;
    const int pa = bs->sh_pstart[A], pb = bs->sh_pstart[B];
    const int pc = bs->sh_pstart[C], pd = bs->sh_pstart[D];
    double Fm[OR_MAXLT + 1];
    for (int i = 0; i < bs->sh_nprim[A]; i++) {
        for (int j = 0; j < bs->sh_nprim[B]; j++) {
            const double a = al[pa + i], b = al[pb + j];
            const double p = a + b;
            const double Kab = exp(-a * b / p * rab2) * co[pa + i] * co[pb + j];
            double P[3];
            for (int x = 0; x < 3; x++) P[x] = (a * Ac[x] + b * Bc[x]) / p;
            for (int k = 0; k < bs->sh_nprim[C]; k++) {
                for (int l = 0; l < bs->sh_nprim[D]; l++) {
                    const double c = al[pc + k], d = al[pd + l];
                    const double q = c + d;
                    const double Kcd = exp(-c * d / q * rcd2) * co[pc + k] * co[pd + l];
                    double Q[3], W[3], PA[3], WP[3], QC[3], WQ[3];
                    double rpq2 = 0.0;
                    for (int x = 0; x < 3; x++) {
                        Q[x] = (c * Cc[x] + d * Dc[x]) / q;
                        W[x] = (p * P[x] + q * Q[x]) / (p + q);
                        PA[x] = P[x] - Ac[x];
                        WP[x] = W[x] - P[x];
                        QC[x] = Q[x] - Cc[x];
                        WQ[x] = W[x] - Q[x];
                        rpq2 += (P[x] - Q[x]) * (P[x] - Q[x]);
                    }
                    const double rho = p * q / (p + q);
                    const double T = rho * rpq2;
                    const double pref = 2.0 * pow(M_PI, 2.5) / (p * q * sqrt(p + q)) * Kab * Kcd;
                    boys(L, T, Fm);
                    for (int m = 0; m <= L; m++) VRR(m, 0, 0) = pref * Fm[m];
                    const double o2p = 0.5 / p, o2q = 0.5 / q, o2pq = 0.5 / (p + q);
                    const double rp = rho / p, rq = rho / q;
                    /* bra build-up: [e0|00]^(m) */
                    for (int le = 1; le <= LB; le++) {
                        for (int t = tri_first(le); t < tri_first(le) + tri_count(le); t++) {
                            const int *e = g_tri[t];
                            int i_ = (e[0] > 0) ? 0 : (e[1] > 0 ? 1 : 2);
                            int em[3] = {e[0], e[1], e[2]};
                            em[i_]--;
                            const int t1 = g_tri_idx[em[0]][em[1]][em[2]];
                            const int n1 = em[i_];
                            int t2 = -1;
                            if (n1 > 0) {
                                em[i_]--;
                                t2 = g_tri_idx[em[0]][em[1]][em[2]];
                            }
                            for (int m = 0; m <= L - le; m++) {
                                double v = PA[i_] * VRR(m, t1, 0) + WP[i_] * VRR(m + 1, t1, 0);
                                if (t2 >= 0) v += n1 * o2p * (VRR(m, t2, 0) - rp * VRR(m + 1, t2, 0));
                                VRR(m, t, 0) = v;
                            }
                        }
                    }
                    /* ket build-up: [e0|f0]^(m) */
                    for (int lf = 1; lf <= LK; lf++) {
                        for (int u = tri_first(lf); u < tri_first(lf) + tri_count(lf); u++) {
                            const int *f = g_tri[u];
                            int j_ = (f[0] > 0) ? 0 : (f[1] > 0 ? 1 : 2);
                            int fm[3] = {f[0], f[1], f[2]};
                            fm[j_]--;
                            const int u1 = g_tri_idx[fm[0]][fm[1]][fm[2]];
                            const int n1 = fm[j_];
                            int u2 = -1;
                            if (n1 > 0) {
                                fm[j_]--;
                                u2 = g_tri_idx[fm[0]][fm[1]][fm[2]];
                            }
                            for (int t = 0; t < ne; t++) {
                                const int *e = g_tri[t];
                                const int le = e[0] + e[1] + e[2];
                                int t3 = -1;
                                if (e[j_] > 0) {
                                    int ee[3] = {e[0], e[1], e[2]};
                                    ee[j_]--;
                                    t3 = g_tri_idx[ee[0]][ee[1]][ee[2]];
                                }
                                int mtop = LK - lf;
                                if (mtop > L - le - lf) mtop = L - le - lf;
                                for (int m = 0; m <= mtop; m++) {
                                    double v = QC[j_] * VRR(m, t, u1) + WQ[j_] * VRR(m + 1, t, u1);
                                    if (u2 >= 0) v += n1 * o2q * (VRR(m, t, u2) - rq * VRR(m + 1, t, u2));
                                    if (t3 >= 0) v += e[j_] * o2pq * VRR(m + 1, t3, u1);
                                    VRR(m, t, u) = v;
                                }
                            }
                        }
                    }
                    for (int t = e0; t < ne; t++) {
                        for (int u = f0; u < nf; u++) w->con[t * nf + u] += VRR(0, t, u);
                    }
                }
            }
        }
    }
#undef VRR
    /* bra HRR: (a b|f) from (e 0|f), |a| = la, |b| = lb */
    const int nbt = OR_NT(lb);
#define HB(buf, a, b, f) (buf)[((a) * nbt + (b)) * nf + (f)]
    double *cur = w->hb, *nxt = w->hb2;
    for (int t = e0; t < ne; t++)
        for (int u = f0; u < nf; u++) HB(cur, t, 0, u) = w->con[t * nf + u];
    for (int kb = 1; kb <= lb; kb++) {
        for (int t = tri_first(la); t < OR_NT(LB - kb); t++) {
            for (int s = tri_first(kb); s < tri_first(kb) + tri_count(kb); s++) {
                const int *bb = g_tri[s];
                int i_ = (bb[0] > 0) ? 0 : (bb[1] > 0 ? 1 : 2);
                int bm[3] = {bb[0], bb[1], bb[2]};
                bm[i_]--;
                const int s1 = g_tri_idx[bm[0]][bm[1]][bm[2]];
                const int *aa = g_tri[t];
                int ap[3] = {aa[0], aa[1], aa[2]};
                ap[i_]++;
                const int t1 = g_tri_idx[ap[0]][ap[1]][ap[2]];
                for (int u = f0; u < nf; u++)
                    HB(cur, t, s, u) = HB(cur, t1, s1, u) + AB[i_] * HB(cur, t, s1, u);
            }
        }
    }
    (void)nxt;
    /* ket HRR and final write: (ab|cd) */
    const int na = tri_count(la), nb = tri_count(lb), nc = tri_count(lc), nd = tri_count(ld);
    const int ndt = OR_NT(ld);
    double kt[OR_NT2 * 10];
#define KT(c, d) kt[(c) * ndt + (d)]
    for (int ia = 0; ia < na; ia++) {
        for (int ib = 0; ib < nb; ib++) {
            const int t = tri_first(la) + ia, s = tri_first(lb) + ib;
            for (int u = f0; u < nf; u++) KT(u, 0) = HB(cur, t, s, u);
            for (int kd = 1; kd <= ld; kd++) {
                for (int u = tri_first(lc); u < OR_NT(LK - kd); u++) {
                    for (int v = tri_first(kd); v < tri_first(kd) + tri_count(kd); v++) {
                        const int *dd = g_tri[v];
                        int j_ = (dd[0] > 0) ? 0 : (dd[1] > 0 ? 1 : 2);
                        int dm[3] = {dd[0], dd[1], dd[2]};
                        dm[j_]--;
                        const int v1 = g_tri_idx[dm[0]][dm[1]][dm[2]];
                        const int *cc = g_tri[u];
                        int cp[3] = {cc[0], cc[1], cc[2]};
                        cp[j_]++;
                        const int u1 = g_tri_idx[cp[0]][cp[1]][cp[2]];
                        KT(u, v) = KT(u1, v1) + CD[j_] * KT(u, v1);
                    }
                }
            }
            for (int ic = 0; ic < nc; ic++) {
                for (int id = 0; id < nd; id++) {
                    w->cart[ia + na * (ib + nb * (ic + nc * id))] =
                        KT(tri_first(lc) + ic, tri_first(ld) + id);
                }
            }
        }
    }
#undef KT
#undef HB
}

CIntStatus_t CInt_createERD(BasisSet_t basis, ERD_t *erd, int nthreads)
{
    (void)basis;
    if (erd == NULL || nthreads <= 0) return CINT_STATUS_INVALID_VALUE;
    ERD_t e = (ERD_t)calloc(1, sizeof(struct ERD));
    if (e == NULL) return CINT_STATUS_ALLOC_FAILED;
    e->nthreads = nthreads;
    e->ws = (eri_ws_t *)calloc((size_t)nthreads, sizeof(eri_ws_t));
    if (e->ws == NULL) { free(e); return CINT_STATUS_ALLOC_FAILED; }
    tri_init();
    *erd = e;
    return CINT_STATUS_SUCCESS;
}

CIntStatus_t CInt_destroyERD(ERD_t erd)
{
    if (erd == NULL) return CINT_STATUS_INVALID_VALUE;
    free(erd->ws);
    free(erd);
    return CINT_STATUS_SUCCESS;
}

void CInt_getMaxMemory(ERD_t erd, double *memsize)
{
    *memsize = erd ? (double)erd->nthreads * sizeof(eri_ws_t) : 0.0;
}

/* Contracted ERI block in the basis's own functions (spherical d when the
 * basis is pure), first index fastest. */
CIntStatus_t CInt_computeShellQuartet(BasisSet_t basis, ERD_t erd, int tid,
                                      int A, int B, int C, int D,
                                      double **integrals, int *nints)
{
    if (erd == NULL || tid < 0 || tid >= erd->nthreads) return CINT_STATUS_INVALID_VALUE;
    eri_ws_t *w = &erd->ws[tid];
    eri_cart(basis, w, A, B, C, D);
    int sh[4] = {A, B, C, D};
    int n[4];
    for (int k = 0; k < 4; k++) n[k] = tri_count(basis->sh_L[sh[k]]);
    double *src = w->cart, *dst = w->tmp;
    if (basis->pure) {
        for (int k = 0; k < 4; k++) {
            if (basis->sh_L[sh[k]] == 2) {
                sph_transform_index(src, dst, n, 4, k);
                double *t = src; src = dst; dst = t;
            }
        }
    }
    int total = n[0] * n[1] * n[2] * n[3];
    if (src != w->out) memcpy(w->out, src, sizeof(double) * total);
    *integrals = w->out;
    *nints = total;
    return CINT_STATUS_SUCCESS;
}

CIntStatus_t CInt_computeShellQuartets(BasisSet_t basis, ERD_t erd, uint32_t threadId,
                                       uint32_t shellIndixA, const uint32_t *shellIndicesB,
                                       uint32_t shellIndixC, const uint32_t *shellIndicesD,
                                       uint32_t shellIndicesCount,
                                       double **integrals, int *integralsCount)
{
    /* batched variant: concatenates the blocks of (A B_i | C D_i) into a
     * per-thread buffer owned by the ERD object */
    static __thread double *buf = NULL;
    static __thread size_t cap = 0;
    size_t need = (size_t)shellIndicesCount * OR_MAXQ;
    if (need > cap) {
        free(buf);
        buf = (double *)malloc(sizeof(double) * need);
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

/* ------------------------------------------------------------------------ */
/* one-electron integrals                                                    */
/* ------------------------------------------------------------------------ */

struct OED {
    double buf[OR_MAXCART * OR_MAXCART];
    double tmp[OR_MAXCART * OR_MAXCART];
    double out[OR_MAXCART * OR_MAXCART];
};

CIntStatus_t CInt_createOED(BasisSet_t basis, OED_t *oed)
{
    (void)basis;
    if (oed == NULL) return CINT_STATUS_INVALID_VALUE;
    *oed = (OED_t)calloc(1, sizeof(struct OED));
    tri_init();
    return *oed ? CINT_STATUS_SUCCESS : CINT_STATUS_ALLOC_FAILED;
}

CIntStatus_t CInt_destroyOED(OED_t oed)
{
    free(oed);
    return CINT_STATUS_SUCCESS;
}

/* 1-D overlap table S[i][j], i <= imax, j <= jmax, for one dimension */
static void ovl1d(double PA, double PB, double p, double s00, int imax, int jmax, double S[7][7])
{
    const double o2p = 0.5 / p;
    S[0][0] = s00;
    for (int i = 0; i <= imax; i++) {
        for (int j = 0; j <= jmax; j++) {
            if (i == 0 && j == 0) continue;
            double v;
            if (i > 0) {
                v = PA * S[i - 1][j];
                if (i > 1) v += (i - 1) * o2p * S[i - 2][j];
                if (j > 0) v += j * o2p * S[i - 1][j - 1];
            } else {
                v = PB * S[i][j - 1];
                if (j > 1) v += (j - 1) * o2p * S[i][j - 2];
            }
            S[i][j] = v;
        }
    }
}

enum { OED_OVL = 0, OED_KIN = 1, OED_POT = 2 };

/* contracted Cartesian one-electron block, first index fastest */
static void oed_cart(BasisSet_t bs, int A, int B, int kind, double *out)
{
    const int la = bs->sh_L[A], lb = bs->sh_L[B];
    const int na = tri_count(la), nb = tri_count(lb);
    const double *Ac = &bs->xyz[3 * bs->sh_atom[A]];
    const double *Bc = &bs->xyz[3 * bs->sh_atom[B]];
    double AB[3], rab2 = 0.0;
    for (int x = 0; x < 3; x++) {
        AB[x] = Ac[x] - Bc[x];
        rab2 += AB[x] * AB[x];
    }
    memset(out, 0, sizeof(double) * na * nb);
    const int pa = bs->sh_pstart[A], pb = bs->sh_pstart[B];
    for (int i = 0; i < bs->sh_nprim[A]; i++) {
        for (int j = 0; j < bs->sh_nprim[B]; j++) {
            const double a = bs->alpha[pa + i], b = bs->alpha[pb + j];
            const double p = a + b, mu = a * b / p;
            const double cab = bs->coef[pa + i] * bs->coef[pb + j];
            double P[3], PA[3], PB[3];
            for (int x = 0; x < 3; x++) {
                P[x] = (a * Ac[x] + b * Bc[x]) / p;
                PA[x] = P[x] - Ac[x];
                PB[x] = P[x] - Bc[x];
            }
            if (kind == OED_OVL || kind == OED_KIN) {
                double S[3][7][7];
                for (int x = 0; x < 3; x++) {
                    double s00 = sqrt(M_PI / p) * exp(-mu * AB[x] * AB[x]);
                    ovl1d(PA[x], PB[x], p, s00, la, lb + 2, S[x]);
                }
                for (int ib = 0; ib < nb; ib++) {
                    const int *bj = g_tri[tri_first(lb) + ib];
                    for (int ia = 0; ia < na; ia++) {
                        const int *ai = g_tri[tri_first(la) + ia];
                        double v;
                        if (kind == OED_OVL) {
                            v = S[0][ai[0]][bj[0]] * S[1][ai[1]][bj[1]] * S[2][ai[2]][bj[2]];
                        } else {
                            v = 0.0;
                            for (int x = 0; x < 3; x++) {
                                const int ii = ai[x], jj = bj[x];
                                double t = -2.0 * b * (2 * jj + 1) * S[x][ii][jj] +
                                           4.0 * b * b * S[x][ii][jj + 2];
                                if (jj >= 2) t += jj * (jj - 1) * S[x][ii][jj - 2];
                                double o = 1.0;
                                for (int y = 0; y < 3; y++)
                                    if (y != x) o *= S[y][ai[y]][bj[y]];
                                v += -0.5 * t * o;
                            }
                        }
                        out[ia + na * ib] += cab * v;
                    }
                }
            } else {
                /* nuclear attraction: VRR on e = a+b then HRR */
                const int LT = la + lb;
                const int ne = OR_NT(LT);
                double th[OR_NT2][2 * OR_MAXL + 1];
                double acc[OR_NT2];
                memset(acc, 0, sizeof(acc));
                for (int cnuc = 0; cnuc < bs->natoms; cnuc++) {
                    const double *Cn = &bs->xyz[3 * cnuc];
                    double PC[3], rpc2 = 0.0;
                    for (int x = 0; x < 3; x++) {
                        PC[x] = P[x] - Cn[x];
                        rpc2 += PC[x] * PC[x];
                    }
                    double Fm[2 * OR_MAXL + 1];
                    boys(LT, p * rpc2, Fm);
                    const double pref = 2.0 * M_PI / p * exp(-mu * rab2);
                    for (int m = 0; m <= LT; m++) th[0][m] = pref * Fm[m];
                    for (int le = 1; le <= LT; le++) {
                        for (int t = tri_first(le); t < tri_first(le) + tri_count(le); t++) {
                            const int *e = g_tri[t];
                            int i_ = (e[0] > 0) ? 0 : (e[1] > 0 ? 1 : 2);
                            int em[3] = {e[0], e[1], e[2]};
                            em[i_]--;
                            const int t1 = g_tri_idx[em[0]][em[1]][em[2]];
                            const int n1 = em[i_];
                            int t2 = -1;
                            if (n1 > 0) {
                                em[i_]--;
                                t2 = g_tri_idx[em[0]][em[1]][em[2]];
                            }
                            for (int m = 0; m <= LT - le; m++) {
                                double v = PA[i_] * th[t1][m] - PC[i_] * th[t1][m + 1];
                                if (t2 >= 0) v += n1 * 0.5 / p * (th[t2][m] - th[t2][m + 1]);
                                th[t][m] = v;
                            }
                        }
                    }
                    for (int t = 0; t < ne; t++) acc[t] += -bs->Z[cnuc] * th[t][0];
                }
                /* HRR (a, b+1_i) = (a+1_i, b) + AB_i (a, b) */
                double hr[OR_NT2][10];
                for (int t = 0; t < ne; t++) hr[t][0] = acc[t];
                for (int kb = 1; kb <= lb; kb++) {
                    for (int t = tri_first(la); t < OR_NT(LT - kb); t++) {
                        for (int s = tri_first(kb); s < tri_first(kb) + tri_count(kb); s++) {
                            const int *bb = g_tri[s];
                            int i_ = (bb[0] > 0) ? 0 : (bb[1] > 0 ? 1 : 2);
                            int bm[3] = {bb[0], bb[1], bb[2]};
                            bm[i_]--;
                            const int s1 = g_tri_idx[bm[0]][bm[1]][bm[2]];
                            const int *aa = g_tri[t];
                            int ap[3] = {aa[0], aa[1], aa[2]};
                            ap[i_]++;
                            const int t1 = g_tri_idx[ap[0]][ap[1]][ap[2]];
                            hr[t][s] = hr[t1][s1] + AB[i_] * hr[t][s1];
                        }
                    }
                }
                for (int ib = 0; ib < nb; ib++)
                    for (int ia = 0; ia < na; ia++)
                        out[ia + na * ib] += cab * hr[tri_first(la) + ia][tri_first(lb) + ib];
            }
        }
    }
}

static CIntStatus_t oed_pair(BasisSet_t bs, OED_t oed, int A, int B, int kind,
                             double **integrals, int *nints)
{
    tri_init();
    int n[2] = {tri_count(bs->sh_L[A]), tri_count(bs->sh_L[B])};
    if (kind == -1) {
        double tmpk[OR_MAXCART * OR_MAXCART];
        oed_cart(bs, A, B, OED_KIN, oed->buf);
        oed_cart(bs, A, B, OED_POT, tmpk);
        for (int k = 0; k < n[0] * n[1]; k++) oed->buf[k] += tmpk[k];
    } else {
        oed_cart(bs, A, B, kind, oed->buf);
    }
    double *src = oed->buf, *dst = oed->tmp;
    int sh[2] = {A, B};
    if (bs->pure) {
        for (int k = 0; k < 2; k++) {
            if (bs->sh_L[sh[k]] == 2) {
                sph_transform_index(src, dst, n, 2, k);
                double *t = src; src = dst; dst = t;
            }
        }
    }
    memcpy(oed->out, src, sizeof(double) * n[0] * n[1]);
    *integrals = oed->out;
    *nints = n[0] * n[1];
    return CINT_STATUS_SUCCESS;
}

CIntStatus_t CInt_computePairOvl(BasisSet_t b, OED_t o, int A, int B, double **I, int *n)
{
    return oed_pair(b, o, A, B, OED_OVL, I, n);
}

CIntStatus_t CInt_computePairKin(BasisSet_t b, OED_t o, int A, int B, double **I, int *n)
{
    return oed_pair(b, o, A, B, OED_KIN, I, n);
}

CIntStatus_t CInt_computePairPot(BasisSet_t b, OED_t o, int A, int B, double **I, int *n)
{
    return oed_pair(b, o, A, B, OED_POT, I, n);
}

CIntStatus_t CInt_computePairCoreH(BasisSet_t b, OED_t o, int A, int B, double **I, int *n)
{
    return oed_pair(b, o, A, B, -1, I, n);
}
