"""Generate gtfock_b200/csrc/cuda/rys_table.h: Rys quadrature roots and weights.

The electron-repulsion kernels evaluate (ab|cd) by Rys quadrature: with
u = t^2, the Boys weight dmu(u) = u^(-1/2) exp(-T u) / 2 on [0, 1] has moments
F_k(T) (the Boys function), and an n-point Gauss rule {u_i, w_i} for it makes
the 2-D integral products exact for total angular momentum L <= 2n - 1.

Method (published, restated here):
  * moments F_k(T) = 1F1(k+1/2; k+3/2; -T) / (2k+1), evaluated with mpmath at
    60 significant digits;
  * Jacobi matrix from the moments by Gautschi's Chebyshev algorithm
    (W. Gautschi, "Orthogonal Polynomials: Computation and Approximation",
    Oxford 2004, sec. 2.1.7), nodes and weights by Golub-Welsch;
  * on each interval [T0, T0 + H_n) every u_i(T) and w_i(T) is interpolated at
    DEG_n+1 Chebyshev points and stored as a monomial series in
    s = T - (T0+H_n/2); the interval and degree depend on the root count n
    (narrower intervals and lower degrees for the few-root tables, which the
    light shell classes evaluate most often);
  * for T >= TMAX[n] the large-T form is exact to double precision:
    u_i = x_i^2 / T, w_i = W_i / sqrt(T) with x_i > 0 the roots of the Hermite
    polynomial H_2n and W_i their Gauss-Hermite weights.
Accuracy of the double table against the 60-digit values: <= 1e-15 relative
(checked by tests/test_oracle.py against values recomputed here).

Run:  python -m gtfock_b200.gen_rys_table   (about a minute on 8 cores)
"""
import multiprocessing as mproc
import os
import sys

import mpmath as mp

NMAX = 5            # roots needed for (dd|dd): L = 8 -> n = 5
# interval width in T and polynomial degree per root count n (FP64 table):
# each choice fits u_i and w_i to <= 6e-16 relative (measured at 9 points per
# interval on sample intervals); the N-root block must fit in 48 KB of
# shared memory, which keeps n = 5 on the wider intervals
H64 = {1: 0.5, 2: 0.5, 3: 2.0, 4: 1.0, 5: 2.0}
DEG64 = {1: 9, 2: 9, 3: 13, 4: 11, 5: 13}
TMAX = {1: 40.0, 2: 48.0, 3: 56.0, 4: 62.0, 5: 70.0}
# single-precision table for the mixed-precision kernels
H32 = 2.0
DEG32 = 7
DPS = 60


def boys_moments(T, n):
    T = mp.mpf(T)
    return [mp.hyp1f1(k + mp.mpf(1) / 2, k + mp.mpf(3) / 2, -T) / (2 * k + 1)
            for k in range(2 * n)]


def gauss_rule(T, n):
    """n-point Gauss rule (nodes u ascending, weights) for the Boys weight at T."""
    with mp.workdps(DPS):
        mu = boys_moments(T, n)
        sig_prev = [mp.mpf(0)] * (2 * n)
        sig = list(mu)
        alpha = [mu[1] / mu[0]]
        beta = [mu[0]]
        for k in range(1, n):
            new = [mp.mpf(0)] * (2 * n)
            for l in range(k, 2 * n - k):
                new[l] = sig[l + 1] - alpha[k - 1] * sig[l] - beta[k - 1] * sig_prev[l]
            alpha.append(new[k + 1] / new[k] - sig[k] / sig[k - 1])
            beta.append(new[k] / sig[k - 1])
            sig_prev, sig = sig, new
        J = mp.matrix(n, n)
        for i in range(n):
            J[i, i] = alpha[i]
            if i + 1 < n:
                J[i, i + 1] = J[i + 1, i] = mp.sqrt(beta[i + 1])
        E, Q = mp.eigsy(J)
        order = sorted(range(n), key=lambda i: E[i])
        return [E[i] for i in order], [mu[0] * Q[0, i] ** 2 for i in order]


def hermite_large_t(n):
    """(x_i^2, W_i) for the positive roots of H_2n, ascending."""
    with mp.workdps(DPS):
        m = 2 * n
        out = []
        # initial guesses from the asymptotic root spacing refined by findroot
        import numpy as np
        xs, _ = np.polynomial.hermite.hermgauss(m)
        for x0 in xs:
            if x0 <= 0:
                continue
            r = mp.findroot(lambda t: mp.hermite(m, t), mp.mpf(x0))
            wt = 2 ** (m - 1) * mp.factorial(m) * mp.sqrt(mp.pi) / (m ** 2 * mp.hermite(m - 1, r) ** 2)
            out.append((r * r, wt))
        out.sort()
        return out


def fit_interval(args):
    n, T0, h, deg = args
    with mp.workdps(DPS):
        xs = [mp.cos(mp.pi * (2 * k + 1) / (2 * (deg + 1))) for k in range(deg + 1)]
        vals = []
        for x in xs:
            u, w = gauss_rule(T0 + h * (x + 1) / 2, n)
            vals.append(u + w)
        V = mp.matrix([[(h * x / 2) ** j for j in range(deg + 1)] for x in xs])
        coefs = []
        for f in range(2 * n):
            c = mp.lu_solve(V, mp.matrix([v[f] for v in vals]))
            coefs.append([c[j] for j in range(deg + 1)])
        return coefs   # [func][coef]


def build_table(h, deg, pool):
    """h, deg: per root count (dict) or one value for all"""
    tables = {}
    for n in range(1, NMAX + 1):
        hn = h[n] if isinstance(h, dict) else h
        dn = deg[n] if isinstance(deg, dict) else deg
        nint = int(round(TMAX[n] / hn))
        res = pool.map(fit_interval, [(n, k * hn, hn, dn) for k in range(nint)])
        tables[n] = res
    return tables


def fmt(x, single=False):
    if single:
        return "%.9ef" % float(x)
    return "%.17e" % float(x)


def main(out_path=None):
    if out_path is None:
        out_path = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                "csrc", "cuda", "rys_table.h")
    with mproc.get_context("spawn").Pool(os.cpu_count()) as pool:
        t64 = build_table(H64, DEG64, pool)
        t32 = build_table(H32, DEG32, pool)
    lines = []
    w = lines.append
    w("/* rys_table.h -- generated by gtfock_b200/gen_rys_table.py; do not edit.")
    w(" * Rys quadrature for the Boys weight: per root count n, per interval of")
    w(" * width H_n in T (RYS_H_LIST), DEG_n+1 monomial coefficients (RYS_DEG_LIST)")
    w(" * in s = T - (T0 + H_n/2) for u_1..u_n then w_1..w_n, stored")
    w(" * [interval][coef][func]; above RYS_TMAX[n] the Hermite large-T form")
    w(" * u = x^2/T, w = W/sqrt(T) applies.  The FP32 table uses RYS32_H and")
    w(" * RYS32_DEG for every n. */")
    w("#pragma once")
    w("#ifndef RYS_QUAL")
    w("#define RYS_QUAL static")
    w("#endif")
    w("#ifndef RYS_QUAL_SMALL")
    w("#define RYS_QUAL_SMALL static")
    w("#endif")
    w("#define RYS_NMAX %d" % NMAX)
    w("#define RYS_H_LIST 0.0, %s" % ", ".join("%.2f" % H64[n] for n in range(1, NMAX + 1)))
    w("#define RYS_DEG_LIST 0, %s" % ", ".join("%d" % DEG64[n] for n in range(1, NMAX + 1)))
    w("#define RYS32_H %.1f" % H32)
    w("#define RYS32_INV_H %.9ef" % (1.0 / H32))
    w("#define RYS32_DEG %d" % DEG32)
    off = 0
    offs = {}
    flat = []
    for n in range(1, NMAX + 1):
        offs[n] = off
        for iv in t64[n]:
            for j in range(DEG64[n] + 1):
                for f in range(2 * n):
                    flat.append(iv[f][j])
        off = len(flat)
    w("RYS_QUAL_SMALL const double RYS_TMAX[RYS_NMAX + 1] = {0.0, %s};" %
      ", ".join("%.1f" % TMAX[n] for n in range(1, NMAX + 1)))
    w("RYS_QUAL_SMALL const int RYS_OFF[RYS_NMAX + 1] = {0, %s};" %
      ", ".join(str(offs[n]) for n in range(1, NMAX + 1)))
    w("#define RYS_OFF_LIST 0, %s" % ", ".join(str(offs[n]) for n in range(1, NMAX + 1)))
    w("#define RYS_TABLE_LEN %d" % len(flat))
    w("RYS_QUAL const double RYS_TABLE[RYS_TABLE_LEN] = {")
    for i in range(0, len(flat), 4):
        w("  " + ", ".join(fmt(x) for x in flat[i:i + 4]) + ",")
    w("};")
    off = 0
    offs32 = {}
    flat32 = []
    for n in range(1, NMAX + 1):
        offs32[n] = off
        for iv in t32[n]:
            for j in range(DEG32 + 1):
                for f in range(2 * n):
                    flat32.append(iv[f][j])
        off = len(flat32)
    w("RYS_QUAL_SMALL const int RYS32_OFF[RYS_NMAX + 1] = {0, %s};" %
      ", ".join(str(offs32[n]) for n in range(1, NMAX + 1)))
    w("#define RYS32_OFF_LIST 0, %s" % ", ".join(str(offs32[n]) for n in range(1, NMAX + 1)))
    w("#define RYS32_TABLE_LEN %d" % len(flat32))
    w("RYS_QUAL const float RYS32_TABLE[RYS32_TABLE_LEN] = {")
    for i in range(0, len(flat32), 6):
        w("  " + ", ".join(fmt(x, True) for x in flat32[i:i + 6]) + ",")
    w("};")
    # large-T constants
    w("RYS_QUAL_SMALL const double RYS_LARGE_X2[RYS_NMAX + 1][RYS_NMAX] = {")
    w("  {0.0},")
    hl = {n: hermite_large_t(n) for n in range(1, NMAX + 1)}
    for n in range(1, NMAX + 1):
        w("  {" + ", ".join(fmt(x2) for x2, _ in hl[n]) + "},")
    w("};")
    w("RYS_QUAL_SMALL const double RYS_LARGE_W[RYS_NMAX + 1][RYS_NMAX] = {")
    w("  {0.0},")
    for n in range(1, NMAX + 1):
        w("  {" + ", ".join(fmt(wt) for _, wt in hl[n]) + "},")
    w("};")
    with open(out_path, "w") as f:
        f.write("\n".join(lines) + "\n")
    print("wrote", out_path, len(flat), "doubles,", len(flat32), "floats")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else None)
