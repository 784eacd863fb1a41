/*
 * setup.c -- angular set-up of the oracle (TEST INFRASTRUCTURE ONLY).
 *
 * Restates momopt_init.cpp:88-259: Gauss-Legendre quadrature in mu, 2Q
 * azimuths, the z-even real spherical-harmonic basis with the Condon-Shortley
 * phase, and the Gaunt-like product table obtained by a QR least-squares fit
 * of p_i p_j onto the degree-2N extended basis.
 *
 * The reference takes these from GSL (utils.cpp:55-60 glfixed table,
 * momopt_init.cpp:203-209 gsl_sf_legendre_sphPlm, :233-243 QR); GSL is not
 * present and not version-pinned, so the published algorithms are restated:
 *  - Gauss-Legendre by Newton iteration on the three-term recurrence
 *    (Golub & Welsch style nodes; any correct method gives the same nodes to
 *    rounding), ascending order as GSL's glfixed_point reports them;
 *  - normalised P_l^m by the standard stable recurrence in l;
 *  - Householder QR least squares (Golub & Van Loan, Alg. 5.3.2).
 */
#include "oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

const double ORC_REGULARIZATIONS[ORC_NUM_REG] = {0.0, 1e-3, 1e-2, 1e-1, 5e-1};

void orc_gauss_legendre(int n, double *x, double *w)
{
    int m = (n + 1) / 2;
    for (int i = 0; i < m; i++) {
        double z = cos(M_PI * (i + 0.75) / (n + 0.5));
        double pp = 0.0;
        for (int it = 0; it < 100; it++) {
            double p1 = 1.0, p2 = 0.0;
            for (int j = 1; j <= n; j++) {
                double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
            }
            pp = n * (z * p1 - p2) / (z * z - 1.0);
            double z1 = z;
            z = z1 - p1 / pp;
            if (fabs(z - z1) <= 1e-16 * fabs(z) + 1e-300 && it > 2)
                break;
        }
        /* recompute derivative at the final node for the weight */
        {
            double p1 = 1.0, p2 = 0.0;
            for (int j = 1; j <= n; j++) {
                double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
            }
            pp = n * (z * p1 - p2) / (z * z - 1.0);
        }
        double wi = 2.0 / ((1.0 - z * z) * pp * pp);
        /* z is the i-th largest positive node; store ascending */
        x[i] = -z;
        w[i] = wi;
        x[n - 1 - i] = z;
        w[n - 1 - i] = wi;
    }
    if (n % 2 == 1)
        x[n / 2] = 0.0;
}

double orc_sphPlm(int l, int m, double x)
{
    if (m < 0 || m > l)
        return 0.0;
    double s = sqrt((1.0 - x) * (1.0 + x));
    double pmm = sqrt(1.0 / (4.0 * M_PI));
    for (int k = 1; k <= m; k++)
        pmm *= -s * sqrt((2.0 * k + 1.0) / (2.0 * k));
    if (l == m)
        return pmm;
    double pm1 = x * sqrt(2.0 * m + 3.0) * pmm;
    if (l == m + 1)
        return pm1;
    double plm2 = pmm, plm1 = pm1, pl = 0.0;
    for (int ll = m + 2; ll <= l; ll++) {
        double a = sqrt((4.0 * ll * ll - 1.0) / ((double)ll * ll - (double)m * m));
        double b = sqrt((4.0 * (ll - 1.0) * (ll - 1.0) - 1.0) /
                        ((ll - 1.0) * (ll - 1.0) - (double)m * m));
        pl = a * (x * plm1 - plm2 / b);
        plm2 = plm1;
        plm1 = pl;
    }
    return pl;
}

/* Householder QR of A (rows x cols, row-major, rows >= cols), in place:
 * R in the upper triangle, v_k below the diagonal with v_k[k]=1 implied,
 * tau[k] the reflector scale. */
void orc_householder_qr(int rows, int cols, double *A, double *tau)
{
    for (int k = 0; k < cols; k++) {
        double norm = 0.0;
        for (int i = k; i < rows; i++)
            norm += A[i * cols + k] * A[i * cols + k];
        norm = sqrt(norm);
        if (norm == 0.0) {
            tau[k] = 0.0;
            continue;
        }
        double akk = A[k * cols + k];
        double beta = (akk >= 0) ? -norm : norm;
        double v0 = akk - beta;
        for (int i = k + 1; i < rows; i++)
            A[i * cols + k] /= v0;
        tau[k] = (beta - akk) / beta;
        A[k * cols + k] = beta;
        for (int j = k + 1; j < cols; j++) {
            double s = A[k * cols + j];
            for (int i = k + 1; i < rows; i++)
                s += A[i * cols + k] * A[i * cols + j];
            s *= tau[k];
            A[k * cols + j] -= s;
            for (int i = k + 1; i < rows; i++)
                A[i * cols + j] -= s * A[i * cols + k];
        }
    }
}

/* min ||A beta - b|| given the factorisation above; b is overwritten. */
void orc_householder_lssolve(int rows, int cols, const double *QR, const double *tau,
                                double *b, double *beta)
{
    for (int k = 0; k < cols; k++) {
        double s = b[k];
        for (int i = k + 1; i < rows; i++)
            s += QR[i * cols + k] * b[i];
        s *= tau[k];
        b[k] -= s;
        for (int i = k + 1; i < rows; i++)
            b[i] -= s * QR[i * cols + k];
    }
    for (int k = cols - 1; k >= 0; k--) {
        double s = b[k];
        for (int j = k + 1; j < cols; j++)
            s -= QR[k * cols + j] * beta[j];
        beta[k] = s / QR[k * cols + k];
    }
}

int orc_setup_create(int order, int Q, int useGaunt, orc_setup *s)
{
    memset(s, 0, sizeof(*s));
    if (order < 0 || Q < 2)
        return ORC_ERR_INPUT;
    s->order = order;
    s->Q = Q;
    s->useGaunt = useGaunt;
    /* momopt_init.cpp:88-93 */
    s->nq = Q * Q;
    s->n = (order + 1) * (order + 2) / 2;
    s->n2 = s->n;
    if (useGaunt == 1)
        s->n2 = (2 * order + 1) * (2 * order + 2) / 2;
    int nq = s->nq, n2 = s->n2;
    s->w = (double *)malloc(sizeof(double) * nq);
    s->xi = (double *)malloc(sizeof(double) * nq);
    s->eta = (double *)malloc(sizeof(double) * nq);
    s->p = (double *)malloc(sizeof(double) * nq * n2);

    double *glw = (double *)malloc(sizeof(double) * Q);
    double *glx = (double *)malloc(sizeof(double) * Q);
    orc_gauss_legendre(Q, glx, glw);

    /* momopt_init.cpp:168-217 */
    for (int q1 = 0; q1 < Q / 2; q1++) {
        double wTemp = 2.0 * M_PI / Q * glw[q1];
        for (int q2 = 0; q2 < 2 * Q; q2++) {
            double mu = glx[q1];
            double phi = (q2 + 0.5) * M_PI / Q;
            int q = 2 * q1 * Q + q2;
            s->w[q] = wTemp;
            s->xi[q] = sqrt(1.0 - mu * mu) * cos(phi);
            s->eta[q] = sqrt(1.0 - mu * mu) * sin(phi);
            int N = order + 1;
            if (useGaunt == 1)
                N = 2 * order + 1;
            int k = 0;
            for (int nn = 0; nn < N; nn++) {
                for (int m = -nn; m <= nn; m++) {
                    if ((m + nn) % 2 != 0)
                        continue;
                    double sh;
                    if (m < 0)
                        sh = M_SQRT2 * sin(m * phi) * orc_sphPlm(nn, -m, mu);
                    else if (m > 0)
                        sh = M_SQRT2 * cos(m * phi) * orc_sphPlm(nn, m, mu);
                    else
                        sh = orc_sphPlm(nn, 0, mu);
                    s->p[q * n2 + k] = sh;
                    k++;
                }
            }
        }
    }
    free(glw);
    free(glx);

    /* momopt_init.cpp:221-259: least-squares fit of p_i p_j on the extended
     * basis; keep |beta| > 10e-10. */
    if (useGaunt == 1) {
        int n = s->n;
        double *A = (double *)malloc(sizeof(double) * nq * n2);
        double *tau = (double *)malloc(sizeof(double) * n2);
        double *b = (double *)malloc(sizeof(double) * nq);
        double *beta = (double *)malloc(sizeof(double) * n2);
        memcpy(A, s->p, sizeof(double) * nq * n2);
        orc_householder_qr(nq, n2, A, tau);
        int cap = n * n * n2;
        s->gaunt.n = n;
        s->gaunt.off = (int *)malloc(sizeof(int) * (n * n + 1));
        s->gaunt.idx = (int *)malloc(sizeof(int) * cap);
        s->gaunt.val = (double *)malloc(sizeof(double) * cap);
        int nnz = 0;
        for (int i = 0; i < n; i++) {
            for (int j = 0; j < n; j++) {
                for (int q = 0; q < nq; q++)
                    b[q] = s->p[q * n2 + i] * s->p[q * n2 + j];
                orc_householder_lssolve(nq, n2, A, tau, b, beta);
                s->gaunt.off[i * n + j] = nnz;
                for (int k = 0; k < n2; k++) {
                    if (fabs(beta[k]) > 10e-10) {
                        s->gaunt.idx[nnz] = k;
                        s->gaunt.val[nnz] = beta[k];
                        nnz++;
                    }
                }
            }
        }
        s->gaunt.off[n * n] = nnz;
        free(A);
        free(tau);
        free(b);
        free(beta);
    }
    return ORC_OK;
}

void orc_setup_free(orc_setup *s)
{
    free(s->w);
    free(s->xi);
    free(s->eta);
    free(s->p);
    free(s->gaunt.off);
    free(s->gaunt.idx);
    free(s->gaunt.val);
    memset(s, 0, sizeof(*s));
}
