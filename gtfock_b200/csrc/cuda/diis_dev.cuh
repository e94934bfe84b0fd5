// diis_dev.cuh -- DIIS bookkeeping on the device (pscf/purif.c:491-641),
// shared by the single-job path (purif.cu) and the batched engine
// (batch_scf.cu).  Nothing of it returns to the host: the slot of each
// iteration, the bordered matrix and the extrapolation coefficients stay in
// device memory and are read by the launches that follow on the same stream.
#pragma once

#include <float.h>

#define GTF_MAX_DIIS 10
#define GTF_DIIS_LDB (GTF_MAX_DIIS + 1)

// The bordered matrix b (order len + 1, leading dimension GTF_DIIS_LDB):
// entries (i, j), i, j < len, are the dot products <e_i, e_j> of the stored
// error vectors, the rest -1 off the diagonal and 0 on it, so that row and
// column len form the border of the system of order len + 1.  `cur` is the
// slot of this iteration's vectors: the next free one, else the one with the
// largest <e_i, e_i> (bmax_id, pscf/purif.c:575-600).
struct DiisState {
    int len, cur, bmax_id, pad;
    double bmax;
    double b[GTF_DIIS_LDB * GTF_DIIS_LDB];
    double co[GTF_MAX_DIIS];
};

// thread t of nt
__device__ __forceinline__ void diis_reset(DiisState *ds, int t, int nt)
{
    if (t == 0) {
        ds->len = 0;
        ds->cur = -1;
        ds->bmax_id = -1;
        ds->bmax = DBL_MIN;
    }
    for (int k = t; k < GTF_DIIS_LDB * GTF_DIIS_LDB; k += nt)
        ds->b[k] = (k / GTF_DIIS_LDB != k % GTF_DIIS_LDB) ? -1.0 : 0.0;
    for (int k = t; k < GTF_MAX_DIIS; k += nt) ds->co[k] = 0.0;
}

// one thread
__device__ __forceinline__ void diis_slot(DiisState *ds)
{
    if (ds->len < GTF_MAX_DIIS) {
        ds->cur = ds->len;
        ds->len++;
    } else {
        ds->cur = ds->bmax_id;
    }
}

// One thread, after row and column `cur` of b hold this iteration's dot
// products: the largest-error slot and the coefficients c_i = -inv[i][len]
// of the bordered system, inverted by Gauss-Jordan elimination with partial
// pivoting (pscf/purif.c:603-623).  A singular system (two identical error
// vectors) gives non-finite coefficients: this iteration's F is then kept
// unextrapolated (c = e_cur).
__device__ __forceinline__ void diis_coefficients(DiisState *ds)
{
    const int m = ds->len, cur = ds->cur;
    double bmax = -DBL_MAX;
    int bmax_id = ds->bmax_id;
    for (int i = 0; i < m; i++) {
        const double v = ds->b[i * GTF_DIIS_LDB + i];
        if (bmax < v) {
            bmax = v;
            bmax_id = i;
        }
    }
    ds->bmax = bmax;
    ds->bmax_id = bmax_id;
    const int sz = m + 1;
    double a[GTF_DIIS_LDB][2 * GTF_DIIS_LDB];
    for (int i = 0; i < sz; i++)
        for (int j = 0; j < sz; j++) {
            a[i][j] = ds->b[i * GTF_DIIS_LDB + j];
            a[i][sz + j] = (i == j) ? 1.0 : 0.0;
        }
    for (int c = 0; c < sz; c++) {
        int piv = c;
        for (int r = c + 1; r < sz; r++)
            if (fabs(a[r][c]) > fabs(a[piv][c])) piv = r;
        if (piv != c)
            for (int j = 0; j < 2 * sz; j++) {
                const double t = a[c][j];
                a[c][j] = a[piv][j];
                a[piv][j] = t;
            }
        const double d = a[c][c];
        for (int j = 0; j < 2 * sz; j++) a[c][j] /= d;
        for (int r = 0; r < sz; r++) {
            if (r == c) continue;
            const double f = a[r][c];
            if (f == 0.0) continue;
            for (int j = 0; j < 2 * sz; j++) a[r][j] -= f * a[c][j];
        }
    }
    bool finite = true;
    for (int i = 0; i < m; i++) finite = finite && isfinite(a[i][2 * sz - 1]);
    for (int i = 0; i < GTF_MAX_DIIS; i++)
        ds->co[i] = (i >= m) ? 0.0 : finite ? -a[i][2 * sz - 1] : (i == cur ? 1.0 : 0.0);
}

// lane i < len of one warp stores dot product dots[i] = <e, e_i> into row
// and column `cur`; then lane 0 forms the coefficients
__device__ __forceinline__ void diis_update_solve(DiisState *ds, const double *dots, int lane)
{
    const int m = ds->len, cur = ds->cur;
    if (lane < m) {
        ds->b[cur * GTF_DIIS_LDB + lane] = dots[lane];
        ds->b[lane * GTF_DIIS_LDB + cur] = dots[lane];
    }
    __syncwarp();
    if (lane == 0) diis_coefficients(ds);
}
