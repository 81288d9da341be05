/*
 * Spectral basis for the learned search's proposals (no counterpart in the
 * reference): the k leading eigenvectors of A^T A for a small integer
 * matrix A (rows x cols, cols <= 64), by block subspace iteration with a
 * Rayleigh-Ritz step (a standard method: orthonormalise G Q, repeat until
 * G Q stays in span Q, then diagonalise Q^T G Q).
 *
 * Signs: each vector's largest-magnitude component is made positive.  The
 * proposals only depend on the spanned directions (a labeling and its
 * negation have the same value); the proposal network's output quality
 * was checked unchanged against LAPACK's eigenvectors.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "ld_internal.h"

#define SB_MAXC 64
#define SB_MAXK 8

/* dot product of two length-n vectors (four partial sums) */
static double sb_dot(const double *x, const double *y, int n) {
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    int i = 0;
    for (; i + 4 <= n; i += 4) {
        s0 += x[i] * y[i];
        s1 += x[i + 1] * y[i + 1];
        s2 += x[i + 2] * y[i + 2];
        s3 += x[i + 3] * y[i + 3];
    }
    for (; i < n; i++) s0 += x[i] * y[i];
    return (s0 + s1) + (s2 + s3);
}

/* modified Gram-Schmidt on the k columns of q (column-major: column j is
 * q + j*m); a column that vanishes is replaced by a unit vector orthogonal
 * to the others */
static void sb_orthonormalise(double *q, int m, int k) {
    for (int j = 0; j < k; j++) {
        double *qj = q + (size_t)j * m;
        for (int pass = 0; pass < 2; pass++)
            for (int i = 0; i < j; i++) {
                const double *qi = q + (size_t)i * m;
                const double dot = sb_dot(qi, qj, m);
                for (int r = 0; r < m; r++) qj[r] -= dot * qi[r];
            }
        double nrm = sqrt(sb_dot(qj, qj, m));
        if (nrm < 1e-280) {
            for (int e = 0; e < m; e++) {          /* first unit vector not in span */
                for (int r = 0; r < m; r++) qj[r] = r == e ? 1.0 : 0.0;
                for (int i = 0; i < j; i++) {
                    const double *qi = q + (size_t)i * m;
                    const double dot = qi[e];
                    for (int r = 0; r < m; r++) qj[r] -= dot * qi[r];
                }
                nrm = sqrt(sb_dot(qj, qj, m));
                if (nrm > 1e-8) break;
            }
        }
        for (int r = 0; r < m; r++) qj[r] /= nrm;
    }
}

/* cyclic Jacobi on the symmetric k x k matrix h: eigenvalues in w,
 * eigenvectors in the columns of y */
static void sb_jacobi(double *h, int k, double *w, double *y) {
    for (int i = 0; i < k; i++)
        for (int j = 0; j < k; j++) y[i * k + j] = i == j ? 1.0 : 0.0;
    double diag = 0;
    for (int i = 0; i < k; i++) diag += h[i * k + i] * h[i * k + i];
    for (int sweep = 0; sweep < 64; sweep++) {
        double off = 0;
        for (int i = 0; i < k; i++)
            for (int j = i + 1; j < k; j++) off += h[i * k + j] * h[i * k + j];
        if (off <= 1e-32 * diag || off < 1e-280) break;   /* relative: no denormal sweeps */
        for (int p = 0; p < k; p++)
            for (int q = p + 1; q < k; q++) {
                const double apq = h[p * k + q];
                if (fabs(apq) <= 1e-18 * sqrt(diag) || fabs(apq) < 1e-280) continue;
                const double theta = (h[q * k + q] - h[p * k + p]) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int r = 0; r < k; r++) {          /* h <- h J */
                    const double hp = h[r * k + p], hq = h[r * k + q];
                    h[r * k + p] = c * hp - s * hq;
                    h[r * k + q] = s * hp + c * hq;
                }
                for (int r = 0; r < k; r++) {          /* h <- J^T h */
                    const double hp = h[p * k + r], hq = h[q * k + r];
                    h[p * k + r] = c * hp - s * hq;
                    h[q * k + r] = s * hp + c * hq;
                }
                for (int r = 0; r < k; r++) {          /* y <- y J */
                    const double yp = y[r * k + p], yq = y[r * k + q];
                    y[r * k + p] = c * yp - s * yq;
                    y[r * k + q] = s * yp + c * yq;
                }
            }
    }
    for (int i = 0; i < k; i++) w[i] = h[i * k + i];
}

ld_status ld_spectral_basis(const int64_t *a, int32_t rows, int32_t cols, int32_t k, double *out,
                            int32_t *iterations) {
    if (!a || !out || rows < 1 || cols < 1 || k < 1) return ld_fail(LD_ERR_ARG, "bad arguments");
    if (cols > SB_MAXC || k > SB_MAXK) return ld_fail(LD_ERR_LIMIT, "at most %d columns and %d vectors", SB_MAXC, SB_MAXK);
    const int m = cols, kk = k < m ? k : m;
    memset(out, 0, sizeof(double) * (size_t)m * (size_t)k);
    /* G = A^T A is applied as A^T (A Q): about 2 rows x cols x k multiply-adds,
     * with A converted to double once */
    double *ad = (double *)malloc(sizeof(double) * (size_t)rows * (size_t)m);
    if (!ad) return ld_fail(LD_ERR_NOMEM, "out of host memory");
    double scale = 0;                            /* trace(G) >= ||G||_2 */
    for (size_t t = 0; t < (size_t)rows * (size_t)m; t++) {
        ad[t] = (double)a[t];
        scale += ad[t] * ad[t];
    }
    /* column-major blocks: column j of q is q + j*m */
    double q[SB_MAXC * SB_MAXK], z[SB_MAXC * SB_MAXK], yv[SB_MAXK];
    /* z = A^T (A src): per row r, y_j = <a_r, src_j>, then z_j += y_j a_r */
#define SB_APPLY(src)                                                                  \
    do {                                                                               \
        memset(z, 0, sizeof(double) * (size_t)m * (size_t)kk);                         \
        for (int r = 0; r < rows; r++) {                                               \
            const double *ar = ad + (size_t)r * m;                                     \
            for (int j = 0; j < kk; j++) yv[j] = sb_dot(ar, (src) + (size_t)j * m, m); \
            for (int j = 0; j < kk; j++) {                                             \
                double *zj = z + (size_t)j * m;                                        \
                const double yj = yv[j];                                               \
                for (int c = 0; c < m; c++) zj[c] += yj * ar[c];                       \
            }                                                                          \
        }                                                                              \
    } while (0)
    /* a fixed start: G times a deterministic pseudo-random block */
    uint64_t st = 0x9E3779B97F4A7C15ull;
    double r0[SB_MAXC * SB_MAXK];
    for (int i = 0; i < m * kk; i++) {
        st ^= st << 13; st ^= st >> 7; st ^= st << 17;
        r0[i] = (double)(st >> 11) / 9007199254740992.0 - 0.5;
    }
    SB_APPLY(r0);
    /* until G Q stays in span Q (residual below 1e-12 of trace G), or 60
     * iterations: without a spectral gap the leading subspace converges
     * slowly, and an approximate one serves the proposals as well */
    int it = 0;
    for (; it < 60; it++) {
        memcpy(q, z, sizeof(double) * (size_t)m * (size_t)kk);
        sb_orthonormalise(q, m, kk);
        SB_APPLY(q);
        double res = 0;
        for (int j = 0; j < kk; j++) {
            double e[SB_MAXC];
            memcpy(e, z + (size_t)j * m, sizeof(double) * (size_t)m);
            for (int i = 0; i < kk; i++) {
                const double proj = sb_dot(q + (size_t)i * m, z + (size_t)j * m, m);
                for (int r = 0; r < m; r++) e[r] -= proj * q[(size_t)i * m + r];
            }
            res += sb_dot(e, e, m);
        }
        if (scale == 0 || sqrt(res) <= 1e-12 * scale) { it++; break; }
    }
#undef SB_APPLY
    free(ad);
    /* Rayleigh-Ritz: H = Q^T G Q (= Q^T Z), its eigenvectors rotate Q */
    double h[SB_MAXK * SB_MAXK], w[SB_MAXK], y[SB_MAXK * SB_MAXK];
    for (int i = 0; i < kk; i++)
        for (int j = 0; j < kk; j++) h[i * kk + j] = sb_dot(q + (size_t)i * m, z + (size_t)j * m, m);
    for (int i = 0; i < kk; i++)                 /* symmetrise rounding */
        for (int j = i + 1; j < kk; j++) h[i * kk + j] = h[j * kk + i] = 0.5 * (h[i * kk + j] + h[j * kk + i]);
    sb_jacobi(h, kk, w, y);
    int order[SB_MAXK];
    for (int i = 0; i < kk; i++) order[i] = i;
    for (int i = 0; i < kk; i++)                 /* descending eigenvalue */
        for (int j = i + 1; j < kk; j++)
            if (w[order[j]] > w[order[i]]) { const int t = order[i]; order[i] = order[j]; order[j] = t; }
    for (int j = 0; j < kk; j++) {
        const int src = order[j];
        double best = 0;   /* the largest-magnitude component, made positive */
        for (int r = 0; r < m; r++) {
            double s = 0;
            for (int i = 0; i < kk; i++) s += q[(size_t)i * m + r] * y[i * kk + src];
            out[(size_t)r * k + j] = s;
            if (fabs(s) > fabs(best)) best = s;
        }
        if (best < 0)
            for (int r = 0; r < m; r++) out[(size_t)r * k + j] = -out[(size_t)r * k + j];
    }
    if (iterations) *iterations = it;
    return LD_OK;
}
