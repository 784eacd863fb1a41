/*
 * linalg.c -- small dense FP64 kernels of the oracle (TEST INFRASTRUCTURE ONLY).
 *
 * The reference calls LAPACK/BLAS (utils.h:22-55): dpotrf_('L'), dpocon_('L'),
 * dpotrs_('L'), dnrm2_, and its own utils_norm1 (utils.cpp:36-52).  LAPACK
 * is absent here and unpinned by the reference; these are restatements of the
 * published algorithms:
 *  - Cholesky, column-oriented unblocked form (LAPACK dpotf2 semantics:
 *    info = j+1 at the first non-positive or NaN pivot);
 *  - reciprocal condition estimate with Hager's method as refined by Higham
 *    (N. J. Higham, "FORTRAN codes for estimating the one-norm of a real or
 *    complex matrix", ACM TOMS 14(4), 1988, Algorithm 4.1 -- the algorithm
 *    behind LAPACK dlacn2/dpocon), applied to A^-1 = L^-T L^-1.
 * H is held row-major n x n; the factor L occupies the lower triangle.
 */
#include "oracle.h"
#include <math.h>
#include <string.h>

int orc_cholesky(int n, double *a)
{
    for (int j = 0; j < n; j++) {
        double ajj = a[j * n + j];
        for (int k = 0; k < j; k++)
            ajj -= a[j * n + k] * a[j * n + k];
        if (ajj <= 0.0 || isnan(ajj)) {
            a[j * n + j] = ajj;
            return j + 1;
        }
        ajj = sqrt(ajj);
        a[j * n + j] = ajj;
        double r = 1.0 / ajj;
        for (int i = j + 1; i < n; i++) {
            double s = a[i * n + j];
            for (int k = 0; k < j; k++)
                s -= a[i * n + k] * a[j * n + k];
            a[i * n + j] = s * r;
        }
    }
    return 0;
}

/* x <- (L L^T)^-1 x */
void orc_chol_solve(int n, const double *l, double *x)
{
    for (int i = 0; i < n; i++) {
        double s = x[i];
        for (int k = 0; k < i; k++)
            s -= l[i * n + k] * x[k];
        x[i] = s / l[i * n + i];
    }
    for (int i = n - 1; i >= 0; i--) {
        double s = x[i];
        for (int k = i + 1; k < n; k++)
            s -= l[k * n + i] * x[k];
        x[i] = s / l[i * n + i];
    }
}

double orc_nrm2(int n, const double *x)
{
    double s = 0.0;
    for (int i = 0; i < n; i++)
        s += x[i] * x[i];
    return sqrt(s);
}

/* utils.cpp:36-52: maximum absolute row sum. */
double orc_norm1(int n, const double *a)
{
    double best = 0.0;
    for (int i = 0; i < n; i++) {
        double t = 0.0;
        for (int j = 0; j < n; j++)
            t += fabs(a[i * n + j]);
        if (t > best)
            best = t;
    }
    return best;
}

static double asum(int n, const double *x)
{
    double s = 0.0;
    for (int i = 0; i < n; i++)
        s += fabs(x[i]);
    return s;
}

static int iamax(int n, const double *x)
{
    int j = 0;
    double b = fabs(x[0]);
    for (int i = 1; i < n; i++)
        if (fabs(x[i]) > b) {
            b = fabs(x[i]);
            j = i;
        }
    return j;
}

/* Estimate of ||A^-1||_1 for SPD A = L L^T (A^-1 is symmetric, so the
 * "transpose" products of the estimator are the same solve). */
static double inv_norm1_estimate(int n, const double *l, double *x, double *v, int *isgn)
{
    const int itmax = 5;
    double est;
    for (int i = 0; i < n; i++)
        x[i] = 1.0 / n;
    orc_chol_solve(n, l, x);
    if (n == 1) {
        v[0] = x[0];
        return fabs(v[0]);
    }
    est = asum(n, x);
    for (int i = 0; i < n; i++) {
        x[i] = (x[i] >= 0.0) ? 1.0 : -1.0;
        isgn[i] = (int)x[i];
    }
    orc_chol_solve(n, l, x);
    int j = iamax(n, x);
    int iter = 2;
    for (;;) {
        for (int i = 0; i < n; i++)
            x[i] = 0.0;
        x[j] = 1.0;
        orc_chol_solve(n, l, x);
        for (int i = 0; i < n; i++)
            v[i] = x[i];
        double estold = est;
        est = asum(n, v);
        int same = 1;
        for (int i = 0; i < n; i++) {
            int s = (x[i] >= 0.0) ? 1 : -1;
            if (s != isgn[i]) {
                same = 0;
                break;
            }
        }
        if (same || est <= estold)
            break;
        for (int i = 0; i < n; i++) {
            x[i] = (x[i] >= 0.0) ? 1.0 : -1.0;
            isgn[i] = (int)x[i];
        }
        orc_chol_solve(n, l, x);
        int jlast = j;
        j = iamax(n, x);
        if (x[jlast] != fabs(x[j]) && iter < itmax) {
            iter++;
            continue;
        }
        break;
    }
    /* alternative estimate */
    double altsgn = 1.0;
    for (int i = 0; i < n; i++) {
        x[i] = altsgn * (1.0 + (double)i / (double)(n - 1));
        altsgn = -altsgn;
    }
    orc_chol_solve(n, l, x);
    double temp = 2.0 * (asum(n, x) / (3.0 * n));
    if (temp > est)
        est = temp;
    return est;
}

/* dpocon('L') semantics: rcond = (1/||A^-1||_1)/anorm, 0 when degenerate. */
double orc_rcond(int n, const double *l, double anorm, double *work, int *iwork)
{
    if (n == 0)
        return 1.0;
    if (anorm == 0.0)
        return 0.0;
    double ainv = inv_norm1_estimate(n, l, work, work + n, iwork);
    if (ainv != 0.0)
        return (1.0 / ainv) / anorm;
    return 0.0;
}
