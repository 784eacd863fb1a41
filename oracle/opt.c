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


/* ---------------------------------------------------------------------- */
/* Change-of-basis Newton: opt/optcb.cpp (MOMOPT_OPTIMIZATION_TYPE 1).     */
/* The per-cell basis P2M (lower triangular, row-major here; the reference  */
/* keeps it column-major for BLAS) and the multipliers alphaP in that basis */
/* persist between calls.  The BLAS operations optcb.cpp calls are          */
/* restated as row-major lower-triangular loops below.                      */

/* x <- A^-1 x (dtrsv L,N,N) */
static void trsv_l(int n, const double *a, double *x)
{
    for (int i = 0; i < n; i++) {
        double s = x[i];
        for (int k = 0; k < i; k++)
            s -= a[i * n + k] * x[k];
        x[i] = s / a[i * n + i];
    }
}

/* x <- A^-T x (dtrsv L,T,N) */
static void trsv_lt(int n, const double *a, double *x)
{
    for (int i = n - 1; i >= 0; i--) {
        double s = x[i];
        for (int k = i + 1; k < n; k++)
            s -= a[k * n + i] * x[k];
        x[i] = s / a[i * n + i];
    }
}

/* x <- A x (dtrmv L,N,N) */
static void trmv_l(int n, const double *a, double *x)
{
    for (int i = n - 1; i >= 0; i--) {
        double s = 0.0;
        for (int k = 0; k <= i; k++)
            s += a[i * n + k] * x[k];
        x[i] = s;
    }
}

/* x <- A^T x (dtrmv L,T,N) */
static void trmv_lt(int n, const double *a, double *x)
{
    for (int i = 0; i < n; i++) {
        double s = 0.0;
        for (int k = i; k < n; k++)
            s += a[k * n + i] * x[k];
        x[i] = s;
    }
}

/* B <- B A for lower-triangular B and A (dtrmm R,L,N,N) */
static void trmm_rl(int n, double *b, const double *a)
{
    double row[ORC_NMAX];
    for (int i = 0; i < n; i++) {
        for (int j = 0; j <= i; j++) {
            double s = 0.0;
            for (int k = j; k <= i; k++)
                s += b[i * n + k] * a[k * n + j];
            row[j] = s;
        }
        for (int j = 0; j <= i; j++)
            b[i * n + j] = row[j];
    }
}

static void set_identity(int n, double *a)
{
    memset(a, 0, sizeof(double) * (size_t)n * (size_t)n);
    for (int i = 0; i < n; i++)
        a[i * n + i] = 1.0;
}

/* pP <- P2M^-1 p for every quadrature point (dtrsm L,L,N,N on the nm x nq
 * block whose columns are the points' basis vectors); p has row stride np. */
static void basis_to_p(int nm, int nq, const double *T, const double *p, int np, double *pP)
{
    for (int q = 0; q < nq; q++) {
        double *x = pP + (size_t)q * nm;
        for (int k = 0; k < nm; k++)
            x[k] = p[(size_t)q * np + k];
        trsv_l(nm, T, x);
    }
}

/* optcb.cpp:156-415 */
static int optcb_scaled(int nm, int nq, double *u, double *P2M, double *alphaP, double *alphaM,
                        const double *w, const double *p, int np, orc_options *o, orc_outs *outs)
{
    double f = 0.0;
    double alphaP0[ORC_NMAX], dP[ORC_NMAX], gP[ORC_NMAX], uP[ORC_NMAX], gM[ORC_NMAX];
    double chol[ORC_NMAX * ORC_NMAX], hP[ORC_NMAX * ORC_NMAX], P2Min[ORC_NMAX * ORC_NMAX];
    double work[3 * ORC_NMAX];
    double gExt[ORC_N2MAX];
    int iwork[ORC_NMAX];
    double *pP = (double *)malloc(sizeof(double) * (size_t)nq * nm);
    if (!pP)
        return ORC_ERR_INPUT;
    int status = ORC_OK;
    memcpy(alphaP0, alphaP, sizeof(double) * nm);
    memcpy(P2Min, P2M, sizeof(double) * (size_t)nm * (size_t)nm);
    basis_to_p(nm, nq, P2Min, p, np, pP);
    int maxIter = o->maxIter;
    const double tolRel = o->tolRel;
    double r = 0.0;
    const double condHMax = o->condHMax;
    int regIndex = 0;
    memcpy(uP, u, sizeof(double) * nm);
    trsv_l(nm, P2M, uP);
    double rtol = orc_nrm2(nm, u) * tolRel;
    int iter = 0, totalIter = 0;
    double t = 1.0, err = 0.0;
    int hitMaxRegularization = 0;

    while (1) {
        iter = iter + 1;
        totalIter = totalIter + 1;
        f = orc_fobj(o->momentType, nm, nm, nq, alphaP, uP, w, pP, o->deltaPPn, gP, hP, 0, NULL,
                     gExt);
        memcpy(chol, hP, sizeof(double) * (size_t)nm * (size_t)nm);
        int error = orc_cholesky(nm, chol);
        double norm = orc_norm1(nm, hP);
        double condest = 1.0 / orc_rcond(nm, chol, norm, work, iwork);

        /* a bad Hessian at the very first evaluation: isotropic alpha and the
         * standard basis (optcb.cpp:247-265) */
        if (totalIter == 1 && (error != 0 || condest > condHMax)) {
            isotropic_alpha(nm, alphaP0, o->momentType, o->deltaPPn);
            set_identity(nm, P2M);
            set_identity(nm, P2Min);
            memcpy(alphaP, alphaP0, sizeof(double) * nm);
            memcpy(uP, u, sizeof(double) * nm);
            for (int q = 0; q < nq; q++)
                for (int k = 0; k < nm; k++)
                    pP[(size_t)q * nm + k] = p[(size_t)q * np + k];
            rtol = orc_nrm2(nm, u) * tolRel;
            iter = 0;
            t = 1.0;
            continue;
        }

        /* optcb.cpp:268-318 */
        if (iter >= maxIter || error != 0 || t == 0 || condest > condHMax) {
            if (regIndex < ORC_NUM_REG - 1) {
                regIndex++;
                r = ORC_REGULARIZATIONS[regIndex];
                uP[0] = 1.0;
                for (int i = 1; i < nm; i++)
                    uP[i] = u[i] * (1.0 - r);
            } else {
                if (hitMaxRegularization) {
                    status = ORC_ERR_MAXREG;   /* "This should never happen." */
                    break;
                }
                isotropic_alpha(nm, alphaP0, o->momentType, o->deltaPPn);
                set_identity(nm, P2Min);
                memcpy(uP, u, sizeof(double) * nm);
                regIndex = 0;   /* r keeps its last value, as optcb.cpp:288-296 */
                hitMaxRegularization = 1;
                maxIter = o->maxIter;
            }
            rtol = orc_nrm2(nm, uP) * tolRel;
            memcpy(alphaP, alphaP0, sizeof(double) * nm);
            memcpy(P2M, P2Min, sizeof(double) * (size_t)nm * (size_t)nm);
            trsv_l(nm, P2M, uP);
            basis_to_p(nm, nq, P2Min, p, np, pP);
            iter = 0;
            t = 1.0;
            if (regIndex == ORC_NUM_REG - 1)
                maxIter = 10 * maxIter;
            continue;
        }

        /* change of basis by the Cholesky factor L of hP (optcb.cpp:321-332) */
        trsv_l(nm, chol, gP);
        for (int q = 0; q < nq; q++)
            trsv_l(nm, chol, pP + (size_t)q * nm);
        trmm_rl(nm, P2M, chol);
        trmv_lt(nm, chol, alphaP);
        trsv_l(nm, chol, uP);
        for (int i = 0; i < nm; i++)
            dP[i] = -gP[i];
        /* the gradient in the moment basis measures the error (:340-344) */
        memcpy(gM, gP, sizeof(double) * nm);
        trmv_l(nm, P2M, gM);
        err = orc_nrm2(nm, gM);
        if (err <= rtol) {
            memcpy(alphaM, alphaP, sizeof(double) * nm);
            trsv_lt(nm, P2M, alphaM);
            u[0] = 1.0;
            for (int i = 1; i < nm; i++)
                u[i] = u[i] * (1.0 - r);
            break;
        }
        t = linesearch(nm, nm, nq, alphaP, dP, f, gP, uP, w, pP, o->deltaPPn, o->momentType, gExt);
    }
    if (outs != NULL) {
        outs->iter = totalIter;
        outs->normG = err;
        outs->r = r;
    }
    free(pP);
    return status;
}

/* The reference's cond(): the product of the largest absolute row sums of
 * the two arrays as it stores them (column-major, so of the columns of the
 * matrices here) (optbfgs.cpp:515-545). */
static double bfgs_cond(int n, const double *h, const double *hInv)
{
    double n1 = 0.0, n2 = 0.0;
    for (int j = 0; j < n; j++) {
        double s1 = 0.0, s2 = 0.0;
        for (int i = 0; i < n; i++) {
            s1 += fabs(h[i * n + j]);
            s2 += fabs(hInv[i * n + j]);
        }
        if (s1 > n1)
            n1 = s1;
        if (s2 > n2)
            n2 = s2;
    }
    return n1 * n2;
}

/* y <- c A x (dgemv N with beta 0: columns of A scaled by c x_j, in order) */
static void gemv_n(int n, double c, const double *a, const double *x, double *y)
{
    for (int i = 0; i < n; i++)
        y[i] = 0.0;
    for (int j = 0; j < n; j++) {
        const double s = c * x[j];
        for (int i = 0; i < n; i++)
            y[i] += s * a[i * n + j];
    }
}

/* A <- A + c x y^T (dger) */
static void ger(int n, double c, const double *x, const double *y, double *a)
{
    for (int j = 0; j < n; j++) {
        const double s = c * y[j];
        for (int i = 0; i < n; i++)
            a[i * n + j] += x[i] * s;
    }
}

static double dot(int n, const double *x, const double *y)
{
    double s = 0.0;
    for (int i = 0; i < n; i++)
        s += x[i] * y[i];
    return s;
}

/* optbfgs.cpp:163-512.  The outer loop is optcb's Newton iteration in the
 * change of basis; after each basis change up to maxBfgsIter quasi-Newton
 * steps run on BFGS approximations of H and H^-1 in the new basis (both
 * start at the identity), while cond(H) cond(H^-1) < condHMaxBfgs.  Only
 * the outer iterations are counted. */
static int optbfgs_scaled(int nm, int nq, double *u, double *P2M, const double *alphaPin,
                          double *alphaP, double *alphaM, const double *w, const double *p, int np,
                          orc_options *o, orc_outs *outs)
{
    double f = 0.0;
    double alphaP0[ORC_NMAX], dP[ORC_NMAX], gP[ORC_NMAX], uP[ORC_NMAX], gM[ORC_NMAX];
    double gOldP[ORC_NMAX], alphaOldP[ORC_NMAX], gDiff[ORC_NMAX], alphaDiff[ORC_NMAX];
    double tmp[ORC_NMAX];
    double chol[ORC_NMAX * ORC_NMAX], hP[ORC_NMAX * ORC_NMAX], hInvP[ORC_NMAX * ORC_NMAX];
    double P2Min[ORC_NMAX * ORC_NMAX];
    double work[3 * ORC_NMAX];
    double gExt[ORC_N2MAX];
    int iwork[ORC_NMAX];
    double *pP = (double *)malloc(sizeof(double) * (size_t)nq * nm);
    if (!pP)
        return ORC_ERR_INPUT;
    int status = ORC_OK;
    memcpy(alphaP0, alphaPin, sizeof(double) * nm);
    memcpy(P2Min, P2M, sizeof(double) * (size_t)nm * (size_t)nm);
    basis_to_p(nm, nq, P2Min, p, np, pP);
    int maxIter = o->maxIter;
    const double tolRel = o->tolRel;
    double r = 0.0;
    const double condHMax = o->condHMax;
    int regIndex = 0;
    memcpy(uP, u, sizeof(double) * nm);
    trsv_l(nm, P2M, uP);
    double rtol = orc_nrm2(nm, u) * tolRel;
    int iter = 0, totalIter = 0;
    double t = 1.0, err = 0.0;
    int hitMaxRegularization = 0;
    memcpy(alphaP, alphaP0, sizeof(double) * nm);

    while (1) {
        iter = iter + 1;
        totalIter = totalIter + 1;
        f = orc_fobj(o->momentType, nm, nm, nq, alphaP, uP, w, pP, o->deltaPPn, gP, hP, 0, NULL,
                     gExt);
        memcpy(chol, hP, sizeof(double) * (size_t)nm * (size_t)nm);
        int error = orc_cholesky(nm, chol);
        double norm = orc_norm1(nm, hP);
        double condest = 1.0 / orc_rcond(nm, chol, norm, work, iwork);

        /* optbfgs.cpp:280-300: first evaluation with a bad Hessian */
        if (totalIter == 1 && (error != 0 || condest > condHMax)) {
            isotropic_alpha(nm, alphaP0, o->momentType, o->deltaPPn);
            set_identity(nm, P2M);
            set_identity(nm, P2Min);
            memcpy(alphaP, alphaP0, sizeof(double) * nm);
            memcpy(uP, u, sizeof(double) * nm);
            for (int q = 0; q < nq; q++)
                for (int k = 0; k < nm; k++)
                    pP[(size_t)q * nm + k] = p[(size_t)q * np + k];
            rtol = orc_nrm2(nm, u) * tolRel;
            iter = 0;
            t = 1.0;
            continue;
        }

        /* optbfgs.cpp:303-348 */
        if (iter >= maxIter || error != 0 || t == 0 || condest > condHMax) {
            if (regIndex < ORC_NUM_REG - 1) {
                regIndex++;
                r = ORC_REGULARIZATIONS[regIndex];
                uP[0] = 1.0;
                for (int i = 1; i < nm; i++)
                    uP[i] = u[i] * (1.0 - r);
            } else {
                if (hitMaxRegularization) {
                    status = ORC_ERR_MAXREG;
                    break;
                }
                isotropic_alpha(nm, alphaP0, o->momentType, o->deltaPPn);
                set_identity(nm, P2Min);
                memcpy(uP, u, sizeof(double) * nm);
                regIndex = 0;
                hitMaxRegularization = 1;
                maxIter = o->maxIter;
            }
            rtol = orc_nrm2(nm, uP) * tolRel;
            memcpy(alphaP, alphaP0, sizeof(double) * nm);
            memcpy(P2M, P2Min, sizeof(double) * (size_t)nm * (size_t)nm);
            trsv_l(nm, P2M, uP);
            basis_to_p(nm, nq, P2M, p, np, pP);
            iter = 0;
            t = 1.0;
            if (regIndex == ORC_NUM_REG - 1)
                maxIter = 10 * maxIter;
            continue;
        }

        /* optbfgs.cpp:351-364: change of basis by L, H and H^-1 become I */
        trsv_l(nm, chol, gP);
        for (int q = 0; q < nq; q++)
            trsv_l(nm, chol, pP + (size_t)q * nm);
        trmm_rl(nm, P2M, chol);
        trmv_lt(nm, chol, alphaP);
        trsv_l(nm, chol, uP);
        set_identity(nm, hP);
        set_identity(nm, hInvP);

        int solved = 0, iterTempBfgs = 0;
        while (bfgs_cond(nm, hP, hInvP) < o->condHMaxBfgs && iterTempBfgs < o->maxBfgsIter) {
            iterTempBfgs++;
            gemv_n(nm, -1.0, hInvP, gP, dP);
            memcpy(gM, gP, sizeof(double) * nm);
            trmv_l(nm, P2M, gM);
            err = orc_nrm2(nm, gM);
            if (err <= rtol) {
                memcpy(alphaM, alphaP, sizeof(double) * nm);
                trsv_lt(nm, P2M, alphaM);
                u[0] = 1.0;
                for (int i = 1; i < nm; i++)
                    u[i] = u[i] * (1.0 - r);
                solved = 1;
                break;
            }
            memcpy(alphaOldP, alphaP, sizeof(double) * nm);
            memcpy(gOldP, gP, sizeof(double) * nm);
            t = linesearch(nm, nm, nq, alphaP, dP, f, gP, uP, w, pP, o->deltaPPn, o->momentType, gExt);
            f = orc_fobj(o->momentType, nm, nm, nq, alphaP, uP, w, pP, o->deltaPPn, gP, NULL, 0, NULL,
                         gExt);
            for (int i = 0; i < nm; i++) {
                gDiff[i] = gP[i] - gOldP[i];
                alphaDiff[i] = alphaP[i] - alphaOldP[i];
            }
            /* H += g g^T / (a.g) - (H a)(H a)^T / (a.H a)   (optbfgs.cpp:455-466);
             * a failed line search (a = 0) divides by zero, and the NaN in
             * cond() ends the loop, as in the reference */
            double coef = 1.0 / dot(nm, alphaDiff, gDiff);
            ger(nm, coef, gDiff, gDiff, hP);
            gemv_n(nm, 1.0, hP, alphaDiff, tmp);
            coef = -1.0 / dot(nm, alphaDiff, tmp);
            ger(nm, coef, tmp, tmp, hP);
            /* H^-1 update (optbfgs.cpp:469-485) */
            gemv_n(nm, 1.0, hInvP, gDiff, tmp);
            const double gHg = dot(nm, gDiff, tmp);
            const double ag = dot(nm, alphaDiff, gDiff);
            coef = (gHg + ag) / (ag * ag);
            ger(nm, coef, alphaDiff, alphaDiff, hInvP);
            coef = -1.0 / ag;
            ger(nm, coef, tmp, alphaDiff, hInvP);
            ger(nm, coef, alphaDiff, tmp, hInvP);
        }
        if (solved)
            break;
    }
    if (outs != NULL) {
        outs->iter = totalIter;
        outs->normG = err;
        outs->r = r;
    }
    free(pP);
    return status;
}

/* optbfgs.cpp:90-154: scaling wrapper (optScaled iterates on alphaP from a
 * copy of the input) */
int orc_optbfgs(int nm, int nq, double *u, double *P2M, double *alphaP, double *alphaM,
                orc_options options, const double *w, const double *p, int np, orc_outs *outs)
{
    if (nm > ORC_NMAX)
        return ORC_ERR_INPUT;
    const double u0 = u[0];
    if (u0 <= 0)
        return ORC_ERR_U0;
    if (options.maxBfgsIter < 1)
        return ORC_ERR_INPUT;   /* no step would ever be taken */
    double alphaPin[ORC_NMAX];
    memcpy(alphaPin, alphaP, sizeof(double) * nm);
    int status;
    if (options.momentType == ORC_MN) {
        const double alphaScale = log(u0) * 2.0 * sqrt(M_PI);
        for (int i = 0; i < nm; i++)
            u[i] = u[i] / u0;
        status = optbfgs_scaled(nm, nq, u, P2M, alphaPin, alphaP, alphaM, w, p, np, &options, outs);
        for (int i = 0; i < nm; i++)
            u[i] = u[i] * u0;
        alphaM[0] = alphaM[0] + alphaScale;
    } else if (options.momentType == ORC_PPN) {
        options.deltaPPn = options.deltaPPn / (u0 * u0);
        for (int i = 0; i < nm; i++)
            u[i] = u[i] / u0;
        status = optbfgs_scaled(nm, nq, u, P2M, alphaPin, alphaP, alphaM, w, p, np, &options, outs);
        for (int i = 0; i < nm; i++) {
            alphaM[i] = alphaM[i] * u0;
            u[i] = u[i] * u0;
        }
    } else {
        return ORC_ERR_INPUT;
    }
    return status;
}

/* optcb.cpp:87-153: scaling wrapper */
int orc_optcb(int nm, int nq, double *u, double *P2M, double *alphaP, double *alphaM,
              orc_options options, const double *w, const double *p, int np, orc_outs *outs)
{
    if (nm > ORC_NMAX)
        return ORC_ERR_INPUT;
    const double u0 = u[0];
    if (u0 <= 0)
        return ORC_ERR_U0;
    int status;
    if (options.momentType == ORC_MN) {
        const double alphaScale = log(u0) * 2.0 * sqrt(M_PI);
        for (int i = 0; i < nm; i++)
            u[i] = u[i] / u0;
        status = optcb_scaled(nm, nq, u, P2M, alphaP, alphaM, w, p, np, &options, outs);
        for (int i = 0; i < nm; i++)
            u[i] = u[i] * u0;
        alphaM[0] = alphaM[0] + alphaScale;
    } else if (options.momentType == ORC_PPN) {
        options.deltaPPn = options.deltaPPn / (u0 * u0);
        for (int i = 0; i < nm; i++)
            u[i] = u[i] / u0;
        status = optcb_scaled(nm, nq, u, P2M, alphaP, alphaM, w, p, np, &options, outs);
        for (int i = 0; i < nm; i++) {
            alphaM[i] = alphaM[i] * u0;
            u[i] = u[i] * u0;
        }
    } else {
        return ORC_ERR_INPUT;
    }
    return status;
}

/* momopt_init.cpp:146-157: alphaP isotropic and the P2M block with its first
 * nm entries (column-major: the first column) set to one -- singular, so a
 * cell's first solve takes the first-evaluation reset to the standard basis. */
void orc_optcb_init(int nm, int momentType, double delta, double *P2M, double *alphaP)
{
    memset(P2M, 0, sizeof(double) * (size_t)nm * (size_t)nm);
    for (int k = 0; k < nm; k++)
        P2M[k * nm + 0] = 1.0;
    isotropic_alpha(nm, alphaP, momentType, delta);
}

int orc_optcb_batch(const orc_setup *s, orc_options opts, int optType, int count, double *u,
                    double *P2M, double *alphaP, double *alpha, int *iters, double *regs, int *status)
{
    const int n = s->n;
    int worst = ORC_OK;
#pragma omp parallel for schedule(dynamic, 1)
    for (int c = 0; c < count; c++) {
        orc_outs outs = {0.0, 0, 0.0};
        int st = (optType == 2 ? orc_optbfgs : orc_optcb)(n, s->nq, u + (size_t)c * n, P2M + (size_t)c * n * n,
                                                          alphaP + (size_t)c * n, alpha + (size_t)c * n, opts,
                                                          s->w, s->p, s->n2, &outs);
        if (iters)
            iters[c] = outs.iter;
        if (regs)
            regs[c] = outs.r;
        status[c] = st;
        if (st != ORC_OK) {
#pragma omp critical
            worst = st;
        }
    }
    return worst;
}
