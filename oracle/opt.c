/*
 * opt.c -- per-cell dual Newton solve of the oracle (TEST INFRASTRUCTURE ONLY).
 *
 * Restates, operation for operation where it matters for rounding:
 *   opt/opt.cpp:27-46     isotropicAlpha
 *   opt/opt.cpp:82-148    opt (Mn / PPn scaling wrapper)
 *   opt/opt.cpp:154-343   optScaled (Newton loop, regularisation ladder)
 *   opt/fobj.cpp:37-236   solveHMn / solveHPPn
 *   opt/fobj.cpp:255-428  fobjMn / fobjPPn
 *   opt/linesearch.cpp:21-99  backtracking Armijo line search
 * Differences from the reference: errors are returned instead of abort(), and
 * per-call scratch is a stack buffer instead of malloc.
 */
#include "oracle.h"
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#define ORC_NMAX 64
#define ORC_N2MAX 256

int orc_cholesky(int n, double *a);
void orc_chol_solve(int n, const double *l, double *x);
double orc_nrm2(int n, const double *x);
double orc_norm1(int n, const double *a);
double orc_rcond(int n, const double *l, double anorm, double *work, int *iwork);

/* opt.cpp:99-126 (commented out in the reference): the modified-CFL bound
 * on the error of the Newton step. */
static double modcfl(int n, const double *da, int momentType)
{
    double da_1 = 0;
    for (int i = 0; i < n; i++)
        da_1 = da_1 + fabs(da[i]);
    int pnOrder = (int)floor(sqrt((double)n)) + 1;
    double m_inf = sqrt((2 * pnOrder + 1) / (2 * M_PI));
    if (momentType == ORC_MN)
        return exp(2.0 * da_1 * m_inf);
    return 1.0 + 2.0 * da_1 * m_inf;
}

/* opt.cpp:27-46 */
static void isotropic_alpha(int n, double *alpha, int momentType, double delta)
{
    if (momentType == ORC_MN)
        alpha[0] = 2.0 * sqrt(M_PI) * log(0.5 / sqrt(M_PI));
    else
        alpha[0] = 1.0 - 4.0 * delta * M_PI;
    for (int i = 1; i < n; i++)
        alpha[i] = 0.0;
}

/* fobj.cpp:37-129 (Mn) and :137-236 (PPn): lower triangle, then symmetrise,
 * or the Gaunt contraction H_ij = sum_k c_ijk G_k. */
static void solve_h(int momentType, int nm, int np2, int nq, const double *alpha,
                    const double *w, const double *p, double delta, double *h, int useGaunt,
                    const orc_gaunt *gt, double *gExt)
{
    for (int k = 0; k < np2; k++)
        gExt[k] = 0.0;
    for (int i = 0; i < nm * nm; i++)
        h[i] = 0.0;
    for (int q = 0; q < nq; q++) {
        const double *pq = p + (size_t)q * np2;
        double temp = 0;
        for (int i = 0; i < nm; i++)
            temp = temp + alpha[i] * pq[i];
        if (momentType == ORC_MN) {
            temp = exp(temp);
            if (useGaunt) {
                for (int k = 0; k < np2; k++)
                    gExt[k] += w[q] * pq[k] * temp;
            } else {
                for (int i = 0; i < nm; i++) {
                    double pi = pq[i];
                    for (int j = 0; j <= i; j++)
                        h[i * nm + j] += w[q] * pi * pq[j] * temp;
                }
            }
        } else {
            temp = 0.5 * temp;
            double temp2 = sqrt(temp * temp + delta);
            double temp3 = temp + temp2;
            if (temp < 0)
                temp3 = -delta / (temp - sqrt(temp * temp + delta));
            double temp4 = 0.5 * w[q] * (temp3 / temp2);
            if (useGaunt) {
                for (int k = 0; k < np2; k++)
                    gExt[k] += pq[k] * temp4;
            } else {
                for (int i = 0; i < nm; i++) {
                    double pi = pq[i];
                    for (int j = 0; j <= i; j++)
                        h[i * nm + j] += pi * pq[j] * temp4;
                }
            }
        }
    }
    if (useGaunt) {
        for (int i = 0; i < nm; i++)
            for (int j = i; j < nm; j++) {
                double hij = 0.0;
                int index = i * nm + j;
                for (int e = gt->off[index]; e < gt->off[index + 1]; e++)
                    hij += gt->val[e] * gExt[gt->idx[e]];
                h[i * nm + j] = h[j * nm + i] = hij;
            }
    } else {
        for (int i = 0; i < nm; i++)
            for (int j = i + 1; j < nm; j++)
                h[i * nm + j] = h[j * nm + i];
    }
}

double orc_fobj(int momentType, int nm, int np2, int nq, const double *alpha,
                const double *u, const double *w, const double *p, double delta,
                double *g, double *h, int useGaunt, const orc_gaunt *gt, double *gExt)
{
    double f = 0;
    if (momentType == ORC_MN) {
        /* fobj.cpp:255-335 */
        if (h != NULL) {
            solve_h(ORC_MN, nm, np2, nq, alpha, w, p, delta, h, useGaunt, gt, gExt);
            if (g != NULL)
                for (int i = 0; i < nm; i++)
                    g[i] = h[i] / p[0] - u[i];
            f = h[0] / (p[0] * p[0]);
            for (int i = 0; i < nm; i++)
                f = f - alpha[i] * u[i];
            return f;
        }
        if (g != NULL)
            for (int i = 0; i < nm; i++)
                g[i] = 0.0;
        for (int q = 0; q < nq; q++) {
            const double *pq = p + (size_t)q * np2;
            double temp = 0;
            for (int i = 0; i < nm; i++)
                temp = temp + alpha[i] * pq[i];
            temp = exp(temp);
            if (g != NULL)
                for (int i = 0; i < nm; i++)
                    g[i] += w[q] * pq[i] * temp;
            f = f + w[q] * temp;
        }
        if (g != NULL)
            for (int i = 0; i < nm; i++)
                g[i] = g[i] - u[i];
        for (int i = 0; i < nm; i++)
            f = f - alpha[i] * u[i];
        return f;
    }
    /* fobj.cpp:355-428 */
    if (g != NULL)
        for (int i = 0; i < nm; i++)
            g[i] = 0.0;
    for (int q = 0; q < nq; q++) {
        const double *pq = p + (size_t)q * np2;
        double temp = 0;
        for (int i = 0; i < nm; i++)
            temp = temp + alpha[i] * pq[i];
        temp = 0.5 * temp;
        double temp2 = sqrt(temp * temp + delta);
        double temp3 = temp + temp2;
        if (temp < 0)
            temp3 = -delta / (temp - sqrt(temp * temp + delta));
        f = f + w[q] * (temp * (temp3)-0.5 * delta + delta * log(temp3));
        if (g != NULL) {
            double temp4 = w[q] * (temp3);
            for (int i = 0; i < nm; i++)
                g[i] += pq[i] * temp4;
        }
    }
    if (h != NULL)
        solve_h(ORC_PPN, nm, np2, nq, alpha, w, p, delta, h, useGaunt, gt, gExt);
    for (int i = 0; i < nm; i++) {
        f = f - alpha[i] * u[i];
        if (g != NULL)
            g[i] = g[i] - u[i];
    }
    return f;
}

/* linesearch.cpp:21-99 */
static double linesearch(int n1, int n2, int nq, double *alpha, const double *d, double f,
                         const double *g, const double *u, const double *w, const double *p,
                         double ppnDelta, int momentType, double *gExt)
{
    double t = 1.0;
    double alphaOld[ORC_NMAX];
    for (int i = 0; i < n1; i++)
        alphaOld[i] = alpha[i];
    const double delta = 1e-3;
    const double beta = .5;
    double maxFactor = 0;
    for (int i = 0; i < n1; i++) {
        double temp = fabs(d[i]) / (fabs(alphaOld[i]) + 1e-100);
        if (temp > maxFactor)
            maxFactor = temp;
    }
    while (t * maxFactor > DBL_EPSILON / 2) {
        for (int i = 0; i < n1; i++)
            alpha[i] = alphaOld[i] + t * d[i];
        double fNew = orc_fobj(momentType, n1, n2, nq, alpha, u, w, p, ppnDelta, NULL, NULL, 0,
                               NULL, gExt);
        double temp = 0.0;
        for (int i = 0; i < n1; i++)
            temp += g[i] * d[i];
        if (fNew <= f + delta * t * temp)
            return t;
        t = beta * t;
    }
    for (int i = 0; i < n1; i++)
        alpha[i] = alphaOld[i];
    return 0.0;
}

/* opt.cpp:154-343 */
static int opt_scaled(int nm, int nm2, int nq, double *u, double *alpha, const double *w,
                      const double *p, orc_options *o, const orc_gaunt *gt, orc_outs *outs)
{
    double f = 0;
    double d[ORC_NMAX], g[ORC_NMAX], uOriginal[ORC_NMAX], alpha0[ORC_NMAX];
    double h[ORC_NMAX * ORC_NMAX], chol[ORC_NMAX * ORC_NMAX];
    double gExt[ORC_N2MAX];
    double work[3 * ORC_NMAX];
    int iwork[ORC_NMAX];
    int maxIter = o->maxIter;
    double tolRel = o->tolRel;
    double r = 0.0;
    double condHMax = o->condHMax;
    int regIndex = 0;
    int status = ORC_OK;

    for (int i = 0; i < nm; i++)
        uOriginal[i] = u[i];
    double rtol = orc_nrm2(nm, u) * tolRel;
    int iter = 0, totalIter = 0;
    double t = 1;
    double err = 0.0;
    for (int i = 0; i < nm; i++)
        alpha0[i] = alpha[i];

    while (1) {
        iter = iter + 1;
        totalIter = totalIter + 1;
        f = orc_fobj(o->momentType, nm, nm2, nq, alpha, u, w, p, o->deltaPPn, g, h, o->useGaunt,
                     gt, gExt);
        memcpy(chol, h, sizeof(double) * nm * nm);
        int error = orc_cholesky(nm, chol);
        double norm = orc_norm1(nm, h);
        double rc = orc_rcond(nm, chol, norm, work, iwork);
        double condest = 1.0 / rc;

        if (iter >= maxIter || error != 0 || t == 0 || condest > condHMax) {
            if (regIndex < ORC_NUM_REG - 1) {
                regIndex++;
                r = ORC_REGULARIZATIONS[regIndex];
                u[0] = 1.0;
                for (int i = 1; i < nm; i++)
                    u[i] = uOriginal[i] * (1.0 - r);
            } else {
                status = ORC_ERR_MAXREG;
                break;
            }
            isotropic_alpha(nm, alpha0, o->momentType, o->deltaPPn);
            rtol = orc_nrm2(nm, u) * tolRel;
            memcpy(alpha, alpha0, nm * sizeof(double));
            iter = 0;
            t = 1;
            if (regIndex == ORC_NUM_REG - 1)
                maxIter = 10 * maxIter;
            continue;
        }
        for (int i = 0; i < nm; i++)
            d[i] = g[i];
        orc_chol_solve(nm, chol, d);
        for (int i = 0; i < nm; i++)
            d[i] = -d[i];
        err = orc_nrm2(nm, g);
        int gammaOk = 1;
        if (o->tolGamma > 0)
            gammaOk = modcfl(nm, d, o->momentType) <= o->tolGamma;
        if (err <= rtol && gammaOk) {
            if (o->momentType == ORC_MN) {
                double u0 = u[0] + g[0];
                for (int i = 0; i < nm; i++) {
                    u[i] += g[i];
                    u[i] /= u0;
                }
                alpha[0] -= log(u0) * 2.0 * sqrt(M_PI);
            }
            break;
        }
        t = linesearch(nm, nm2, nq, alpha, d, f, g, u, w, p, o->deltaPPn, o->momentType, gExt);
    }
    if (outs != NULL) {
        outs->iter = totalIter;
        outs->normG = err;
        outs->r = r;
    }
    return status;
}

/* opt.cpp:82-148 */
int orc_opt(int nm, int nm2, int nq, double *u, double *alpha, orc_options options,
            const double *w, const double *p, const orc_gaunt *g, orc_outs *outs)
{
    if (nm > ORC_NMAX || nm2 > ORC_N2MAX)
        return ORC_ERR_INPUT;
    int status;
    if (options.momentType == ORC_MN) {
        double u0 = u[0];
        if (u0 <= 0)
            return ORC_ERR_U0;
        double alphaScale = log(u0) * 2.0 * sqrt(M_PI);
        alpha[0] = alpha[0] - alphaScale;
        for (int i = 0; i < nm; i++)
            u[i] = u[i] / u0;
        status = opt_scaled(nm, nm2, nq, u, alpha, w, p, &options, g, outs);
        for (int i = 0; i < nm; i++)
            u[i] = u[i] * u0;
        alpha[0] = alpha[0] + alphaScale;
    } else if (options.momentType == ORC_PPN) {
        double u0 = u[0];
        if (u0 <= 0)
            return ORC_ERR_U0;
        for (int i = 0; i < nm; i++) {
            alpha[i] = alpha[i] / u0;
            u[i] = u[i] / u0;
        }
        options.deltaPPn = options.deltaPPn / (u0 * u0);
        status = opt_scaled(nm, nm2, nq, u, alpha, w, p, &options, g, outs);
        for (int i = 0; i < nm; i++) {
            alpha[i] = alpha[i] * u0;
            u[i] = u[i] * u0;
        }
    } else {
        return ORC_ERR_INPUT;
    }
    return status;
}

int orc_opt_batch(const orc_setup *s, orc_options opts, int count, double *u, double *alpha,
                  int *iters, double *regs, int *status)
{
    int worst = ORC_OK;
#pragma omp parallel for schedule(dynamic, 1)
    for (int c = 0; c < count; c++) {
        orc_outs outs = {0.0, 0, 0.0};
        int st = orc_opt(s->n, s->n2, s->nq, u + (size_t)c * s->n, alpha + (size_t)c * s->n, opts,
                         s->w, s->p, &s->gaunt, &outs);
        if (iters)
            iters[c] = outs.iter;
        if (regs)
            regs[c] = outs.r;
        if (status)
            status[c] = st;
        if (st != ORC_OK) {
#pragma omp critical
            worst = st;
        }
    }
    return worst;
}
