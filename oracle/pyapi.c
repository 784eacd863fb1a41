/*
 * pyapi.c -- flat entry points of the oracle for ctypes callers
 * (TEST INFRASTRUCTURE ONLY: tests/, smoke() and the bench's CPU baseline).
 */
#include "oracle.h"
#include <stdlib.h>
#include <string.h>

/* Batched opt() with a freshly built angular set-up. */
int orc_batch(int order, int Q, int useGaunt, int momentType, int maxIter, double tol,
              double condHMax, double deltaPPn, double tolGamma, int count, double *u,
              double *alpha, int *iters, double *regs, int *status)
{
    orc_setup s;
    int st = orc_setup_create(order, Q, useGaunt, &s);
    if (st)
        return st;
    orc_options o;
    o.momentType = momentType;
    o.maxIter = maxIter;
    o.tolRel = tol;
    o.condHMax = condHMax;
    o.deltaPPn = deltaPPn;
    o.useGaunt = useGaunt;
    o.tolGamma = tolGamma;
    st = orc_opt_batch(&s, o, count, u, alpha, iters, regs, status);
    orc_setup_free(&s);
    return st;
}

/* Batched change-of-basis opt (optType 1: optcb.cpp, 2: optbfgs.cpp) with
 * per-vector P2M and alphaP state, in place. */
int orc_batch_cb(int order, int Q, int momentType, int optType, int maxIter, double tol,
                 double condHMax, double deltaPPn, int maxBfgsIter, double condHMaxBfgs, int count,
                 double *u, double *P2M, double *alphaP, double *alpha, int *iters, double *regs,
                 int *status)
{
    orc_setup s;
    int st = orc_setup_create(order, Q, 0, &s);
    if (st)
        return st;
    orc_options o;
    memset(&o, 0, sizeof(o));
    o.momentType = momentType;
    o.maxIter = maxIter;
    o.tolRel = tol;
    o.condHMax = condHMax;
    o.deltaPPn = deltaPPn;
    o.maxBfgsIter = maxBfgsIter;
    o.condHMaxBfgs = condHMaxBfgs;
    st = orc_optcb_batch(&s, o, optType, count, u, P2M, alphaP, alpha, iters, regs, status);
    orc_setup_free(&s);
    return st;
}

/* The reference's initial change-of-basis state for count cells. */
void orc_cb_init(int n, int momentType, double delta, int count, double *P2M, double *alphaP)
{
    for (int c = 0; c < count; c++)
        orc_optcb_init(n, momentType, delta, P2M + (size_t)c * n * n, alphaP + (size_t)c * n);
}

/* Angular set-up copied into caller buffers (sizes from orc_setup_dims). */
int orc_setup_dims(int order, int Q, int useGaunt, int *n, int *n2, int *nq, int *nnz)
{
    orc_setup s;
    int st = orc_setup_create(order, Q, useGaunt, &s);
    if (st)
        return st;
    *n = s.n;
    *n2 = s.n2;
    *nq = s.nq;
    *nnz = useGaunt ? s.gaunt.off[s.n * s.n] : 0;
    orc_setup_free(&s);
    return 0;
}

int orc_setup_copy(int order, int Q, int useGaunt, double *w, double *xi, double *eta, double *p,
                   int *off, int *idx, double *val)
{
    orc_setup s;
    int st = orc_setup_create(order, Q, useGaunt, &s);
    if (st)
        return st;
    memcpy(w, s.w, sizeof(double) * s.nq);
    memcpy(xi, s.xi, sizeof(double) * s.nq);
    memcpy(eta, s.eta, sizeof(double) * s.nq);
    memcpy(p, s.p, sizeof(double) * s.nq * s.n2);
    if (useGaunt) {
        int nnz = s.gaunt.off[s.n * s.n];
        memcpy(off, s.gaunt.off, sizeof(int) * (s.n * s.n + 1));
        memcpy(idx, s.gaunt.idx, sizeof(int) * nnz);
        memcpy(val, s.gaunt.val, sizeof(double) * nnz);
    }
    orc_setup_free(&s);
    return 0;
}

/* Whole-grid solver handle (one node), or node `node` of numNodes. */
void *orc_solver_open_node(const char *deckPath, int node, int numNodes)
{
    orc_deck d;
    if (orc_deck_read(deckPath, &d))
        return NULL;
    orc_solver *s = (orc_solver *)malloc(sizeof(orc_solver));
    if (orc_solver_create_node(&d, node, numNodes, s)) {
        free(s);
        return NULL;
    }
    return s;
}

void *orc_solver_open(const char *deckPath) { return orc_solver_open_node(deckPath, 0, 1); }

void orc_solver_node_info(void *h, int *info, double *origin)
{
    orc_solver *s = (orc_solver *)h;
    info[0] = s->node;
    info[1] = s->numNodesX;
    info[2] = s->numNodesY;
    info[3] = s->nodeX;
    info[4] = s->nodeY;
    info[5] = s->gX[2] - s->gX[1] + 1;
    info[6] = s->gY[2] - s->gY[1] + 1;
    origin[0] = s->initX;
    origin[1] = s->initY;
}

void orc_solver_save_old_h(void *h) { orc_solver_save_old((orc_solver *)h); }
void orc_solver_pre_exchange_h(void *h) { orc_solver_pre_exchange((orc_solver *)h); }
int orc_solver_run_h(void *h, const char *dir, int maxSteps) { return orc_solver_run((orc_solver *)h, dir, maxSteps); }
int orc_solver_stage_exchanged_h(void *h, double dt) { return orc_solver_stage_exchanged((orc_solver *)h, dt); }
void orc_solver_average_h(void *h) { orc_solver_average((orc_solver *)h); }
long long orc_solver_halo_count_h(void *h, int side) { return orc_solver_halo_count((orc_solver *)h, side); }
void orc_solver_halo_h(void *h, int side, int pack, double *buf) { orc_solver_halo((orc_solver *)h, side, pack, buf); }
int orc_solver_output_h(void *h, double time, const char *dir) { return orc_solver_output((orc_solver *)h, time, dir); }

void orc_solver_dims(void *h, int *NX, int *NY, int *n, double *maxDt, double *dx, double *dy)
{
    orc_solver *s = (orc_solver *)h;
    *NX = s->NX;
    *NY = s->NY;
    *n = s->set.n;
    *maxDt = s->maxDt;
    *dx = s->dx;
    *dy = s->dy;
}

/* Runs the time loop of main.cpp but stops after nsteps (no outputs). */
int orc_solver_steps(void *h, int nsteps)
{
    orc_solver *s = (orc_solver *)h;
    for (int k = 0; k < nsteps; k++) {
        int st = orc_solver_update(s, s->maxDt);
        if (st)
            return st;
    }
    return 0;
}

int orc_solver_step_dt(void *h, double dt) { return orc_solver_update((orc_solver *)h, dt); }

void orc_solver_state(void *h, double *moments, double *alpha)
{
    orc_solver *s = (orc_solver *)h;
    size_t bytes = sizeof(double) * (size_t)s->NX * s->NY * s->set.n;
    if (moments)
        memcpy(moments, s->moments, bytes);
    if (alpha) {
        if (s->alpha)
            memcpy(alpha, s->alpha, bytes);
        else
            memset(alpha, 0, bytes);   /* SOLVER moment has no multipliers */
    }
}

void orc_solver_set_state(void *h, const double *moments, const double *alpha)
{
    orc_solver *s = (orc_solver *)h;
    size_t bytes = sizeof(double) * (size_t)s->NX * s->NY * s->set.n;
    if (moments)
        memcpy(s->moments, moments, bytes);
    if (alpha && s->alpha)
        memcpy(s->alpha, alpha, bytes);
}

void orc_solver_stats(void *h, int *maxIter, double *iterMean, long long *numSolves, int *hist)
{
    orc_solver *s = (orc_solver *)h;
    *maxIter = s->stats.maxIter;
    *iterMean = s->stats.iterMean;
    *numSolves = s->stats.numDualSolves;
    for (int i = 0; i < ORC_NUM_REG; i++)
        hist[i] = s->stats.histReg[i];
}

void orc_solver_close(void *h)
{
    if (!h)
        return;
    orc_solver_free((orc_solver *)h);
    free(h);
}

int orc_solver_stage(orc_solver *s, double dt);
int orc_solver_stage_h(void *h, double dt) { return orc_solver_stage((orc_solver *)h, dt); }
long long orc_solver_err_cell(void *h) { return ((orc_solver *)h)->errCell; }

void orc_solver_last_iters(void *h, int *iters)
{
    orc_solver *s = (orc_solver *)h;
    if (s->lastIters)
        memcpy(iters, s->lastIters, sizeof(int) * (size_t)s->NX * s->NY);
    else
        memset(iters, 0, sizeof(int) * (size_t)s->NX * s->NY);
}
