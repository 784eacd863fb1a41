/*
 * solver.c -- whole-grid momopt solver of the oracle (TEST INFRASTRUCTURE ONLY).
 *
 * Restates:
 *   input_deck_reader.cpp:17-159   deck parsing and case-insensitive lookup
 *   main.cpp:67-83, 139-155        deck keys and grid geometry (one node)
 *   main.cpp:257-372               Solver::initializeGrid (IC, sigma fields)
 *   momopt/momopt_init.cpp:51-160  MomOptSolver::init (deck keys, maxDt, IC moments/alpha)
 *   momopt/momopt_update.cpp:38-382 computeAnsatz, minmod, slopefit, solveFlux,
 *                                  solveOptimization, update (Heun RK2)
 *   momopt/momopt_boundaries.cpp:190-223 duplicateBoundaries (periodic IC only,
 *                                  comm.cpp:149-154)
 *   momopt/momopt_output.cpp:21-77 .pn / .opt writers
 *   main.cpp:204-230               time loop
 *   moment/moment_init.cpp:53-298, moment_update.cpp:23-247
 *                                  the linear Pn/FPn solver (SOLVER moment):
 *                                  flux operators, filters, flux, update
 * Layout is the reference's: I2D(i,j) = i*NY + j, I3D(i,j,k) = (i*NY+j)*n + k.
 */
#include "oracle.h"
#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#define ORC_NMAX_PN 512   /* moments per cell of the linear solver (order <= 30) */
#define MIN(a, b) (((a) < (b)) ? (a) : (b))
#define MAX(a, b) (((a) > (b)) ? (a) : (b))
#define SIGN(a, b) ((b) >= 0.0 ? fabs(a) : -fabs(a))

/* ---------------- deck (input_deck_reader.cpp) ---------------- */
#define VLEN 128
typedef struct {
    char key[VLEN];
    char value[VLEN];
} kv_t;

typedef struct {
    kv_t *items;
    int n, cap;
} kvlist;

static void lower_copy(const char *in, char *out)
{
    int i;
    for (i = 0; in[i] != 0 && i < VLEN - 1; i++)
        out[i] = (char)tolower((unsigned char)in[i]);
    out[i] = 0;
}

static int kv_get(const kvlist *l, const char *key, char *value)
{
    char k1[VLEN], k2[VLEN];
    lower_copy(key, k2);
    for (int i = 0; i < l->n; i++) {
        lower_copy(l->items[i].key, k1);
        if (strcmp(k1, k2) == 0) {
            lower_copy(l->items[i].value, value);
            return 1;
        }
    }
    return 0;
}

static int kv_int(const kvlist *l, const char *key, int *v)
{
    char s[VLEN];
    if (!kv_get(l, key, s))
        return 0;
    *v = atoi(s);
    return 1;
}

static int kv_dbl(const kvlist *l, const char *key, double *v)
{
    char s[VLEN];
    if (!kv_get(l, key, s))
        return 0;
    *v = atof(s);
    return 1;
}

int orc_deck_read(const char *path, orc_deck *d)
{
    FILE *f = fopen(path, "r");
    if (!f)
        return ORC_ERR_INPUT;
    kvlist l = {NULL, 0, 0};
    char line[500];
    kv_t kv;
    memset(&kv, 0, sizeof(kv));
    while (fgets(line, sizeof(line), f)) {
        char *nl = strchr(line, '\n');
        if (nl)
            nl[0] = 0;
        char *c = strchr(line, '#');
        if (c)
            c[0] = 0;
        char *pch = strtok(line, " \t");
        if (pch == NULL)
            continue;
        strncpy(kv.key, pch, VLEN - 1);
        pch = strtok(NULL, " ");
        if (pch != NULL)
            strncpy(kv.value, pch, VLEN - 1);
        pch = strtok(NULL, " ");
        if (pch == NULL) {
            if (l.n == l.cap) {
                l.cap = l.cap ? 2 * l.cap : 64;
                l.items = (kv_t *)realloc(l.items, sizeof(kv_t) * l.cap);
            }
            l.items[l.n++] = kv;
        }
    }
    fclose(f);
    memset(d, 0, sizeof(*d));
    int ok = 1;
    char solver[VLEN];
    ok &= kv_get(&l, "SOLVER", solver);
    ok &= kv_int(&l, "NUM_CELLS_X", &d->numCellsX);
    ok &= kv_int(&l, "NUM_CELLS_Y", &d->numCellsY);
    ok &= kv_dbl(&l, "A_X", &d->ax);
    ok &= kv_dbl(&l, "B_X", &d->bx);
    ok &= kv_dbl(&l, "A_Y", &d->ay);
    ok &= kv_dbl(&l, "B_Y", &d->by);
    ok &= kv_dbl(&l, "T_FINAL", &d->tFinal);
    ok &= kv_dbl(&l, "OUT_DELTA_T", &d->outDeltaT);
    ok &= kv_dbl(&l, "GAUSSIAN_SIGMA", &d->gaussianSigma);
    ok &= kv_dbl(&l, "FLOOR", &d->floor_);
    ok &= kv_int(&l, "INIT_COND", &d->initCond);
    ok &= kv_dbl(&l, "SIGMA", &d->sigma);
    ok &= kv_int(&l, "NUM_MPI_PARTITIONS_X", &d->nodesX);
    ok &= kv_int(&l, "NUM_MPI_PARTITIONS_Y", &d->nodesY);
    ok &= kv_get(&l, "SOLVER", solver);
    if (ok && strcmp(solver, "moment") == 0) {
        /* moment_init.cpp:57-61 */
        d->isMoment = 1;
        ok &= kv_int(&l, "MOMENT_MOMENT_ORDER", &d->pnOrder);
        ok &= kv_int(&l, "MOMENT_QUAD_ORDER", &d->pnQuadOrder);
        ok &= kv_int(&l, "MOMENT_FILTER_TYPE", &d->pnFilterType);
        ok &= kv_dbl(&l, "MOMENT_FILTER_TUNE", &d->pnFilterTune);
        ok &= kv_dbl(&l, "MOMENT_CFL_FACTOR", &d->pnCflFactor);
        free(l.items);
        return ok ? ORC_OK : ORC_ERR_INPUT;
    }
    ok &= kv_int(&l, "MOMOPT_MOMENT_ORDER", &d->momentOrder);
    ok &= kv_int(&l, "MOMOPT_QUAD_ORDER", &d->quadOrder);
    ok &= kv_dbl(&l, "MOMOPT_CFL_FACTOR", &d->cflFactor);
    ok &= kv_dbl(&l, "MOMOPT_TOL", &d->tol);
    ok &= kv_dbl(&l, "MOMOPT_COND_H_MAX", &d->condHMax);
    ok &= kv_dbl(&l, "MOMOPT_COND_H_MAX_BFGS", &d->condHMaxBfgs);
    ok &= kv_int(&l, "MOMOPT_MAX_ITER", &d->maxIter);
    ok &= kv_int(&l, "MOMOPT_MAX_BFGS_ITER", &d->maxBfgsIter);
    ok &= kv_int(&l, "MOMOPT_USE_GAUNT", &d->useGaunt);
    ok &= kv_dbl(&l, "MOMOPT_THETA", &d->theta);
    ok &= kv_dbl(&l, "MOMOPT_DELTA_PPN", &d->deltaPPn);
    ok &= kv_int(&l, "MOMOPT_MOMENT_TYPE", &d->momentType);
    ok &= kv_int(&l, "MOMOPT_OPTIMIZATION_TYPE", &d->optType);
    if (!kv_dbl(&l, "MOMOPT_TOL_GAMMA", &d->tolGamma))
        d->tolGamma = 0.0;
    free(l.items);
    if (!ok || strcmp(solver, "momopt") != 0)
        return ORC_ERR_INPUT;
    return ORC_OK;
}

/* ---------------- grid and init ---------------- */
#define I2D(i, j) ((i) * s->NY + (j))
#define I3D(i, j, k) (((size_t)(i) * s->NY + (j)) * n + (k))

static int moment_init(orc_solver *s);

int orc_solver_create(const orc_deck *d, orc_solver *s) { return orc_solver_create_node(d, 0, 1, s); }

int orc_solver_create_node(const orc_deck *d, int node, int numNodes, orc_solver *s)
{
    memset(s, 0, sizeof(*s));
    s->deck = *d;
    if (!d->isMoment &&
        (d->optType < 0 || d->optType > 2 || (d->momentType != ORC_MN && d->momentType != ORC_PPN)))
        return ORC_ERR_INPUT;
    const int ng = 2;
    int sizeX = d->numCellsX, sizeY = d->numCellsY;
    s->dx = (d->bx - d->ax) / sizeX;
    s->dy = (d->by - d->ay) / sizeY;
    double dx = s->dx, dy = s->dy;
    double initX = d->ax, initY = d->ay;
    s->node = 0;
    s->numNodes = 1;
    s->numNodesX = s->numNodesY = 1;
    if (numNodes > 1) {
        /* main.cpp:157-193 */
        const int nX = d->nodesX, nY = d->nodesY;
        if (nX < 1 || nY < 1 || d->numCellsX < nX || d->numCellsY < nY || nX * nY != numNodes || node < 0 ||
            node >= numNodes)
            return ORC_ERR_INPUT;
        s->node = node;
        s->numNodes = numNodes;
        s->numNodesX = nX;
        s->numNodesY = nY;
        s->nodeX = node / nY;
        s->nodeY = node % nY;
        sizeX = d->numCellsX / nX;
        if (s->nodeX < d->numCellsX % nX) {
            sizeX++;
            initX = d->ax + dx * sizeX * s->nodeX;
        } else {
            initX = d->bx - dx * sizeX * (nX - s->nodeX);
        }
        sizeY = d->numCellsY / nY;
        if (s->nodeY < d->numCellsY % nY) {
            sizeY++;
            initY = d->ay + dy * sizeY * s->nodeY;
        } else {
            initY = d->by - dy * sizeY * (nY - s->nodeY);
        }
    }
    s->initX = initX;
    s->initY = initY;
    /* main.cpp:261-269 */
    s->gX[0] = 0;
    s->gX[1] = ng;
    s->gX[2] = ng + sizeX - 1;
    s->gX[3] = 2 * ng + sizeX - 1;
    s->gY[0] = 0;
    s->gY[1] = ng;
    s->gY[2] = ng + sizeY - 1;
    s->gY[3] = 2 * ng + sizeY - 1;
    s->NX = s->gX[3] - s->gX[0] + 1;
    s->NY = s->gY[3] - s->gY[0] + 1;
    size_t C = (size_t)s->NX * s->NY;
    s->initialGrid = (double *)malloc(sizeof(double) * C);
    s->sigmaT = (double *)malloc(sizeof(double) * C);
    s->sigmaS = (double *)malloc(sizeof(double) * C);
    /* main.cpp:282-371 */
    for (int i = s->gX[0]; i <= s->gX[3]; i++) {
        for (int j = s->gY[0]; j <= s->gY[3]; j++) {
            double x_i = initX + (i - s->gX[1]) * dx + dx / 2.0;
            double y_j = initY + (j - s->gY[1]) * dy + dy / 2.0;
            if (i < s->gX[1] || i > s->gX[2] || j < s->gY[1] || j > s->gY[2]) {
                s->initialGrid[I2D(i, j)] = d->floor_;
                s->sigmaT[I2D(i, j)] = d->sigma;
                s->sigmaS[I2D(i, j)] = d->sigma;
            } else if (d->initCond == 0 && d->gaussianSigma == 0.0) {
                s->initialGrid[I2D(i, j)] = d->floor_;
                /* the node at the centre of the partition holds the delta */
                if (s->nodeX == (s->numNodesX - 1) / 2 && s->nodeY == (s->numNodesY - 1) / 2) {
                    int hitX = (s->numNodesX % 2 != 0 && i == (sizeX + ng) / 2) ||
                               (s->numNodesX % 2 == 0 && i == s->gX[2]);
                    int hitY = (s->numNodesY % 2 != 0 && j == (sizeY + ng) / 2) ||
                               (s->numNodesY % 2 == 0 && j == s->gY[2]);
                    if (hitX && hitY)
                        s->initialGrid[I2D(i, j)] = 1.0 / (dx * dy);
                }
                s->sigmaT[I2D(i, j)] = d->sigma;
                s->sigmaS[I2D(i, j)] = d->sigma;
            } else if (d->initCond == 0) {
                double s2 = d->gaussianSigma * d->gaussianSigma;
                double gf = 1.0 / (2.0 * M_PI * s2) * exp(-(x_i * x_i + y_j * y_j) / (2.0 * s2));
                s->initialGrid[I2D(i, j)] = MAX(gf, d->floor_);
                s->sigmaT[I2D(i, j)] = d->sigma;
                s->sigmaS[I2D(i, j)] = d->sigma;
            } else if (d->initCond == 1) {
                s->initialGrid[I2D(i, j)] = d->floor_;
                s->sigmaT[I2D(i, j)] = 1.0;
                s->sigmaS[I2D(i, j)] = 1.0;
                if ((fabs(x_i - 2.0) < 0.5 && fabs(y_j - 2.0) < 0.5) ||
                    (fabs(x_i - 2.0) < 0.5 && fabs(y_j - 0.0) < 0.5) ||
                    (fabs(x_i - 2.0) < 0.5 && fabs(y_j + 2.0) < 0.5) ||
                    (fabs(x_i - 1.0) < 0.5 && fabs(y_j - 1.0) < 0.5) ||
                    (fabs(x_i - 1.0) < 0.5 && fabs(y_j + 1.0) < 0.5) ||
                    (fabs(x_i - 0.0) < 0.5 && fabs(y_j + 2.0) < 0.5) ||
                    (fabs(x_i + 1.0) < 0.5 && fabs(y_j - 1.0) < 0.5) ||
                    (fabs(x_i + 1.0) < 0.5 && fabs(y_j + 1.0) < 0.5) ||
                    (fabs(x_i + 2.0) < 0.5 && fabs(y_j - 2.0) < 0.5) ||
                    (fabs(x_i + 2.0) < 0.5 && fabs(y_j - 0.0) < 0.5) ||
                    (fabs(x_i + 2.0) < 0.5 && fabs(y_j + 2.0) < 0.5)) {
                    s->sigmaT[I2D(i, j)] = 10.0;
                    s->sigmaS[I2D(i, j)] = 0.0;
                }
            } else if (d->initCond == 2) {
                s->sigmaT[I2D(i, j)] = d->sigma;
                s->sigmaS[I2D(i, j)] = d->sigma;
                s->initialGrid[I2D(i, j)] = 1 + sin(2 * M_PI * x_i) * cos(2 * M_PI * y_j);
            }
        }
    }
    if (d->isMoment)
        return moment_init(s);
    /* momopt_init.cpp:72 */
    s->maxDt = d->cflFactor * (2.0 / (2.0 + d->theta)) * (dx * dy) / (dx + dy);
    int st = orc_setup_create(d->momentOrder, d->quadOrder, d->useGaunt, &s->set);
    if (st)
        return st;
    int n = s->set.n;
    s->moments = (double *)malloc(sizeof(double) * C * n);
    s->alpha = (double *)malloc(sizeof(double) * C * n);
    s->flux = (double *)calloc(C * n, sizeof(double));
    s->momentsOld = (double *)calloc(C * n, sizeof(double));
    s->ansatzGrid = (double *)malloc(sizeof(double) * C);
    s->lastIters = (int *)calloc(C, sizeof(int));
    if (d->optType == 1 || d->optType == 2) {
        /* momopt_init.cpp:114-157 */
        s->alphaP = (double *)malloc(sizeof(double) * C * n);
        s->P2M = (double *)malloc(sizeof(double) * C * n * n);
        for (size_t c = 0; c < C; c++)
            orc_optcb_init(n, d->momentType, d->deltaPPn, s->P2M + c * n * n, s->alphaP + c * n);
    }
    /* momopt_init.cpp:120-143 */
    for (int i = s->gX[0]; i <= s->gX[3]; i++)
        for (int j = s->gY[0]; j <= s->gY[3]; j++) {
            s->moments[I3D(i, j, 0)] = s->initialGrid[I2D(i, j)] * 2.0 * sqrt(M_PI);
            for (int k = 1; k < n; k++)
                s->moments[I3D(i, j, k)] = 0.0;
            for (int k = 1; k < n; k++)
                s->alpha[I3D(i, j, k)] = 0.0;
            if (d->momentType == ORC_MN)
                s->alpha[I3D(i, j, 0)] =
                    2.0 * sqrt(M_PI) * log(s->moments[I3D(i, j, 0)] / (2.0 * sqrt(M_PI)));
            else
                s->alpha[I3D(i, j, 0)] =
                    s->moments[I3D(i, j, 0)] - 4.0 * d->deltaPPn * M_PI / s->moments[I3D(i, j, 0)];
        }
    memset(&s->stats, 0, sizeof(s->stats));
    s->status = ORC_OK;
    s->errCell = -1;
    return ORC_OK;
}

void orc_solver_free(orc_solver *s)
{
    free(s->initialGrid);
    free(s->sigmaT);
    free(s->sigmaS);
    free(s->moments);
    free(s->alpha);
    free(s->flux);
    free(s->momentsOld);
    free(s->ansatzGrid);
    free(s->lastIters);
    free(s->alphaP);
    free(s->P2M);
    free(s->pnOps);
    free(s->pnFilter);
    orc_setup_free(&s->set);
    memset(s, 0, sizeof(*s));
}

/* momopt_boundaries.cpp:190-223 */
static void duplicate_boundaries(orc_solver *s)
{
    int n = s->set.n;
    int x0 = s->gX[0], x1 = s->gX[1], x2 = s->gX[2] + 1 - 2, x3 = s->gX[3] + 1 - 2;
    int y0 = s->gY[0], y1 = s->gY[1], y2 = s->gY[2] + 1 - 2, y3 = s->gY[3] + 1 - 2;
    for (int i = 0; i < 2; i++)
        for (int j = s->gY[1]; j <= s->gY[2]; j++)
            for (int k = 0; k < n; k++) {
                s->moments[I3D(x0 + i, j, k)] = s->moments[I3D(x2 + i, j, k)];
                s->moments[I3D(x3 + i, j, k)] = s->moments[I3D(x1 + i, j, k)];
            }
    for (int i = s->gX[1]; i <= s->gX[2]; i++)
        for (int j = 0; j < 2; j++)
            for (int k = 0; k < n; k++) {
                s->moments[I3D(i, y0 + j, k)] = s->moments[I3D(i, y2 + j, k)];
                s->moments[I3D(i, y3 + j, k)] = s->moments[I3D(i, y1 + j, k)];
            }
}

/* momopt_update.cpp:208-277 */
static void solve_optimization(orc_solver *s)
{
    const orc_deck *d = &s->deck;
    int n = s->set.n;
    size_t C = (size_t)s->NX * s->NY;
    orc_options o;
    o.momentType = d->momentType;
    o.maxIter = d->maxIter;
    o.tolRel = d->tol;
    o.condHMax = d->condHMax;
    o.deltaPPn = d->deltaPPn;
    o.useGaunt = (d->useGaunt == 1);
    o.tolGamma = d->tolGamma;
    o.maxBfgsIter = d->maxBfgsIter;
    o.condHMaxBfgs = d->condHMaxBfgs;
#pragma omp parallel for schedule(dynamic, 1)
    for (long index = 0; index < (long)C; index++) {
        orc_outs outs = {0.0, 0, 0.0};
        int st;
        if (d->optType == 2)
            st = orc_optbfgs(n, s->set.nq, &s->moments[(size_t)index * n], &s->P2M[(size_t)index * n * n],
                             &s->alphaP[(size_t)index * n], &s->alpha[(size_t)index * n], o, s->set.w,
                             s->set.p, s->set.n2, &outs);
        else if (d->optType == 1)
            st = orc_optcb(n, s->set.nq, &s->moments[(size_t)index * n], &s->P2M[(size_t)index * n * n],
                           &s->alphaP[(size_t)index * n], &s->alpha[(size_t)index * n], o, s->set.w,
                           s->set.p, s->set.n2, &outs);
        else
            st = orc_opt(n, s->set.n2, s->set.nq, &s->moments[(size_t)index * n],
                         &s->alpha[(size_t)index * n], o, s->set.w, s->set.p, &s->set.gaunt, &outs);
        s->lastIters[index] = outs.iter;
#pragma omp critical
        {
            if (st != ORC_OK && s->status == ORC_OK) {
                s->status = st;
                s->errCell = index;
            }
            if (outs.iter > s->stats.maxIter)
                s->stats.maxIter = outs.iter;
            for (int r = 0; r < ORC_NUM_REG; r++)
                if (fabs(outs.r - ORC_REGULARIZATIONS[r]) < 1e-10)
                    s->stats.histReg[r]++;
            s->stats.iterMean = (s->stats.numDualSolves * s->stats.iterMean + outs.iter) /
                                (s->stats.numDualSolves + 1.0);
            s->stats.numDualSolves++;
        }
    }
}

/* momopt_update.cpp:38-69 */
static double compute_ansatz(const orc_solver *s, const double *alpha, int q)
{
    int n = s->set.n, n2 = s->set.n2;
    double kinetic = 0.0;
    for (int k = 0; k < n; k++)
        kinetic += alpha[k] * s->set.p[(size_t)q * n2 + k];
    if (s->deck.momentType == ORC_MN)
        return exp(kinetic);
    double dl = s->deck.deltaPPn;
    if (kinetic > 0)
        return 0.5 * kinetic + 0.5 * sqrt(kinetic * kinetic + 4 * dl);
    return -dl / (0.5 * kinetic - 0.5 * sqrt(kinetic * kinetic + 4 * dl));
}

/* momopt_update.cpp:77-90 */
static double minmod(double x, double y)
{
    return SIGN(1.0, x) * MAX(0.0, MIN(fabs(x), y * SIGN(1.0, x)));
}

static double slopefit(double left, double center, double right, double theta)
{
    return minmod(theta * (right - center), minmod(0.5 * (right - left), theta * (center - left)));
}

/* momopt_update.cpp:96-202 */
static void solve_flux(orc_solver *s, double dx, double dy)
{
    int n = s->set.n, n2 = s->set.n2, nq = s->set.nq;
    int numY = s->NY;
    long numGridPoints = (long)s->NX * s->NY;
    double theta = s->deck.theta;
    double *ag = s->ansatzGrid;
    for (int i = s->gX[1]; i <= s->gX[2]; i++)
        for (int j = s->gY[1]; j <= s->gY[2]; j++)
            for (int k = 0; k < n; k++)
                s->flux[I3D(i, j, k)] = 0.0;
    for (int q = 0; q < nq; q++) {
#pragma omp parallel for schedule(static)
        for (long index = 0; index < numGridPoints; index++)
            ag[index] = compute_ansatz(s, &s->alpha[(size_t)index * n], q);
        double xi = s->set.xi[q], eta = s->set.eta[q], w = s->set.w[q];
        const double *pq = &s->set.p[(size_t)q * n2];
#pragma omp parallel for schedule(static)
        for (long index = 0; index < numGridPoints; index++) {
            int i = (int)(index / numY);
            int j = (int)(index % numY);
            if (i < s->gX[1] || i > s->gX[2] || j < s->gY[1] || j > s->gY[2])
                continue;
            double flux1 = 0, flux2 = 0, flux3 = 0, flux4 = 0;
            if (xi > 0) {
                double k1 = ag[(i - 2) * numY + j], k2 = ag[(i - 1) * numY + j];
                double k3 = ag[i * numY + j], k4 = ag[(i + 1) * numY + j];
                flux1 = k3 + 0.5 * slopefit(k2, k3, k4, theta) - k2 - 0.5 * slopefit(k1, k2, k3, theta);
                flux1 = flux1 * xi * w;
            }
            if (xi < 0) {
                double k1 = ag[(i - 1) * numY + j], k2 = ag[i * numY + j];
                double k3 = ag[(i + 1) * numY + j], k4 = ag[(i + 2) * numY + j];
                flux2 = k3 - 0.5 * slopefit(k2, k3, k4, theta) - k2 + 0.5 * slopefit(k1, k2, k3, theta);
                flux2 = flux2 * xi * w;
            }
            if (eta > 0) {
                double k1 = ag[i * numY + (j - 2)], k2 = ag[i * numY + (j - 1)];
                double k3 = ag[i * numY + j], k4 = ag[i * numY + (j + 1)];
                flux3 = k3 + 0.5 * slopefit(k2, k3, k4, theta) - k2 - 0.5 * slopefit(k1, k2, k3, theta);
                flux3 = flux3 * eta * w;
            }
            if (eta < 0) {
                double k1 = ag[i * numY + (j - 1)], k2 = ag[i * numY + j];
                double k3 = ag[i * numY + (j + 1)], k4 = ag[i * numY + (j + 2)];
                flux4 = k3 - 0.5 * slopefit(k2, k3, k4, theta) - k2 + 0.5 * slopefit(k1, k2, k3, theta);
                flux4 = flux4 * eta * w;
            }
            for (int k = 0; k < n; k++)
                s->flux[I3D(i, j, k)] += pq[k] * ((flux1 + flux2) / dx + (flux3 + flux4) / dy);
        }
    }
}

/* momopt_update.cpp:316-336 / :344-364 */
static void euler_collide(orc_solver *s, double dt, double dx, double dy)
{
    int n = s->set.n;
    for (int i = s->gX[1]; i <= s->gX[2]; i++)
        for (int j = s->gY[1]; j <= s->gY[2]; j++) {
            s->moments[I3D(i, j, 0)] =
                s->moments[I3D(i, j, 0)] *
                    (1.0 + dt * s->sigmaS[I2D(i, j)] - dt * s->sigmaT[I2D(i, j)]) -
                dt * s->flux[I3D(i, j, 0)];
            for (int k = 1; k < n; k++)
                s->moments[I3D(i, j, k)] =
                    s->moments[I3D(i, j, k)] * (1.0 - dt * s->sigmaT[I2D(i, j)]) -
                    dt * s->flux[I3D(i, j, k)];
            if (s->deck.initCond == 1) {
                double x_i = s->initX + (i - s->gX[1]) * dx;
                double y_j = s->initY + (j - s->gY[1]) * dy;
                if (fabs(x_i) < 0.5 && fabs(y_j) < 0.5)
                    s->moments[I3D(i, j, 0)] = s->moments[I3D(i, j, 0)] + dt * 2.0 * sqrt(M_PI);
            }
        }
}

/* ---------------- SOLVER moment: the linear Pn / FPn solver ---------------- */

static double filter_sspline(double x) { return 1.0 / (1.0 + x * x * x * x); }

static double filter_lanczos(double x)
{
    if (x < .0000001)
        return 1.0;
    return sin(x) / x;
}

/* moment_init.cpp:53-297: maxDt, initial moments, the degree-N basis on the
 * momopt quadrature, the upwind flux operators and the filter factors */
static int moment_init(orc_solver *s)
{
    const orc_deck *d = &s->deck;
    const double dx = s->dx, dy = s->dy;
    s->maxDt = d->pnCflFactor * 0.5 * MIN(dx, dy);
    if ((d->pnOrder + 1) * (d->pnOrder + 2) / 2 > ORC_NMAX_PN)
        return ORC_ERR_INPUT;
    int st = orc_setup_create(d->pnOrder, d->pnQuadOrder, 0, &s->set);
    if (st)
        return st;
    const int n = s->set.n, nq = s->set.nq;
    const size_t C = (size_t)s->NX * s->NY;
    s->moments = (double *)malloc(sizeof(double) * C * n);
    s->flux = (double *)calloc(C * n, sizeof(double));
    s->momentsOld = (double *)calloc(C * n, sizeof(double));
    for (int i = s->gX[0]; i <= s->gX[3]; i++)
        for (int j = s->gY[0]; j <= s->gY[3]; j++) {
            s->moments[I3D(i, j, 0)] = s->initialGrid[I2D(i, j)] * 2.0 * sqrt(M_PI);
            for (int k = 1; k < n; k++)
                s->moments[I3D(i, j, k)] = 0.0;
        }
    /* moment_init.cpp:186-222: quadrature sums split by the sign of xi, eta */
    s->pnOps = (double *)calloc((size_t)4 * n * n, sizeof(double));
    double *xp = s->pnOps, *xm = xp + n * n, *ep = xm + n * n, *em = ep + n * n;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
            for (int q = 0; q < nq; q++) {
                const double mi = s->set.p[(size_t)q * s->set.n2 + i];
                const double mj = s->set.p[(size_t)q * s->set.n2 + j];
                const double vx = s->set.xi[q] * mi * mj * s->set.w[q];
                const double ve = s->set.eta[q] * mi * mj * s->set.w[q];
                if (s->set.xi[q] > 0)
                    xp[i * n + j] += vx;
                else
                    xm[i * n + j] += vx;
                if (s->set.eta[q] > 0)
                    ep[i * n + j] += ve;
                else
                    em[i * n + j] += ve;
            }
    /* moment_init.cpp:225-289 */
    s->pnFilter = (double *)malloc(sizeof(double) * n);
    const double N = d->pnOrder;
    int nm = 0;
    for (int l = 0; l <= d->pnOrder; l++)
        for (int m = -l; m <= l; m++) {
            if ((m + l) % 2 != 0)
                continue;
            double f = 1.0;
            if (d->pnFilterType == 1) {
                const double omega = d->pnFilterTune, L = 1.0, sigt = 1.0;
                const double a = omega / (N * N) / (sigt * L + N) / (sigt * L + N);
                f = 1.0 / (1.0 + a * l * l * (l + 1) * (l + 1));
            } else if (d->pnFilterType == 2) {
                const double sp = -d->pnFilterTune * s->maxDt / log(filter_sspline(N / (N + 1)));
                f = pow(filter_sspline(l / (N + 1)), sp);
            } else if (d->pnFilterType == 3) {
                const double sp = -d->pnFilterTune * s->maxDt / log(filter_lanczos(N / (N + 1)));
                f = pow(filter_lanczos(l / (N + 1)), sp);
            }
            s->pnFilter[nm++] = f;
        }
    memset(&s->stats, 0, sizeof(s->stats));
    s->status = ORC_OK;
    s->errCell = -1;
    return ORC_OK;
}

/* moment_update.cpp:23-40 */
static void moment_scale(orc_solver *s)
{
    const int n = s->set.n;
    for (int i = s->gX[1]; i <= s->gX[2]; i++)
        for (int j = s->gY[1]; j <= s->gY[2]; j++)
            for (int k = 0; k < n; k++)
                s->moments[I3D(i, j, k)] = s->moments[I3D(i, j, k)] * s->pnFilter[k];
}

/* y = A^T x for the n x n operator a (dgemv T on the array the reference
 * fills row by row); y += when acc */
static void op_t(int n, const double *a, const double *x, double *y, int acc)
{
    for (int j = 0; j < n; j++) {
        double t = 0.0;
        for (int i = 0; i < n; i++)
            t += a[(size_t)j * n + i] * x[i];
        y[j] = acc ? y[j] + t : t;
    }
}

/* moment_update.cpp:49-162 */
static void moment_flux(orc_solver *s, double dx, double dy)
{
    const int n = s->set.n;
    const double *xp = s->pnOps, *xm = xp + n * n, *ep = xm + n * n, *em = ep + n * n;
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = s->gX[1]; i <= s->gX[2]; i++) {
        double t[ORC_NMAX_PN], ew[ORC_NMAX_PN], ns[ORC_NMAX_PN];
        for (int j = s->gY[1]; j <= s->gY[2]; j++) {
            const double *m = s->moments;
            for (int k = 0; k < n; k++)
                t[k] = 0.25 * m[I3D(i + 1, j, k)] + 0.75 * m[I3D(i, j, k)] - 1.25 * m[I3D(i - 1, j, k)] +
                       0.25 * m[I3D(i - 2, j, k)];
            op_t(n, xp, t, ew, 0);
            for (int k = 0; k < n; k++)
                t[k] = -0.25 * m[I3D(i + 2, j, k)] + 1.25 * m[I3D(i + 1, j, k)] - 0.75 * m[I3D(i, j, k)] -
                       0.25 * m[I3D(i - 1, j, k)];
            op_t(n, xm, t, ew, 1);
            for (int k = 0; k < n; k++)
                t[k] = 0.25 * m[I3D(i, j + 1, k)] + 0.75 * m[I3D(i, j, k)] - 1.25 * m[I3D(i, j - 1, k)] +
                       0.25 * m[I3D(i, j - 2, k)];
            op_t(n, ep, t, ns, 0);
            for (int k = 0; k < n; k++)
                t[k] = -0.25 * m[I3D(i, j + 2, k)] + 1.25 * m[I3D(i, j + 1, k)] - 0.75 * m[I3D(i, j, k)] -
                       0.25 * m[I3D(i, j - 1, k)];
            op_t(n, em, t, ns, 1);
            for (int k = 0; k < n; k++)
                s->flux[I3D(i, j, k)] = 1.0 / dx * ew[k] + 1.0 / dy * ns[k];
        }
    }
}

/* momopt_update.cpp:283-382 (SOLVER momopt), moment_update.cpp:169-247
 * (SOLVER moment) */
int orc_solver_update(orc_solver *s, double dt)
{
    if (s->deck.isMoment) {
        orc_solver_save_old(s);
        for (int stage = 0; stage < 2; stage++) {
            orc_solver_pre_exchange(s);
            if (s->deck.initCond == 2)
                duplicate_boundaries(s);
            moment_flux(s, s->dx, s->dy);
            euler_collide(s, dt, s->dx, s->dy);
        }
        orc_solver_average(s);
        return ORC_OK;
    }
    int n = s->set.n;
    double dx = s->dx, dy = s->dy;
    for (int i = s->gX[1]; i <= s->gX[2]; i++)
        for (int j = s->gY[1]; j <= s->gY[2]; j++)
            for (int k = 0; k < n; k++)
                s->momentsOld[I3D(i, j, k)] = s->moments[I3D(i, j, k)];
    for (int stage = 0; stage < 2; stage++) {
        if (s->deck.initCond == 2)
            duplicate_boundaries(s);
        solve_optimization(s);
        if (s->status != ORC_OK)
            return s->status;
        solve_flux(s, dx, dy);
        euler_collide(s, dt, dx, dy);
    }
    for (int i = s->gX[1]; i <= s->gX[2]; i++)
        for (int j = s->gY[1]; j <= s->gY[2]; j++)
            for (int k = 0; k < n; k++)
                s->moments[I3D(i, j, k)] = 0.5 * (s->moments[I3D(i, j, k)] + s->momentsOld[I3D(i, j, k)]);
    return ORC_OK;
}

/* momopt_output.cpp:21-77 */
int orc_solver_output(orc_solver *s, double time, const char *dir)
{
    char fn[1024];
    int n = s->set.n;
    snprintf(fn, sizeof(fn), "%s/out_%.3f_%d.pn", dir ? dir : ".", time, s->node);
    FILE *f = fopen(fn, "wb");
    if (!f)
        return ORC_ERR_INPUT;
    int64_t t64 = s->gX[2] - s->gX[1] + 1;
    fwrite(&t64, sizeof(int64_t), 1, f);
    t64 = s->gY[2] - s->gY[1] + 1;
    fwrite(&t64, sizeof(int64_t), 1, f);
    fwrite(&s->deck.ax, sizeof(double), 1, f);
    fwrite(&s->deck.ay, sizeof(double), 1, f);
    fwrite(&s->deck.bx, sizeof(double), 1, f);
    fwrite(&s->deck.by, sizeof(double), 1, f);
    t64 = n;
    fwrite(&t64, sizeof(int64_t), 1, f);
    for (int i = s->gX[1]; i <= s->gX[2]; i++)
        for (int j = s->gY[1]; j <= s->gY[2]; j++)
            fwrite(&s->moments[I3D(i, j, 0)], sizeof(double), n, f);
    fclose(f);
    if (s->deck.isMoment)
        return ORC_OK;   /* moment_output.cpp writes the .pn file only */
    snprintf(fn, sizeof(fn), "%s/out_%.3f_%d.opt", dir ? dir : ".", time, s->node);
    f = fopen(fn, "w");
    if (!f)
        return ORC_ERR_INPUT;
    fprintf(f, "Max number of iterations: %d\n", s->stats.maxIter);
    fprintf(f, "Mean number of iterations: %f\n", s->stats.iterMean);
    fprintf(f, "Number of optimizations: %d\n", (int)s->stats.numDualSolves);
    fprintf(f, "Regularizations Histogram\n");
    for (int i = 0; i < ORC_NUM_REG; i++)
        fprintf(f, "r = %.3e   %d\n", ORC_REGULARIZATIONS[i], s->stats.histReg[i]);
    fclose(f);
    return ORC_OK;
}

/* main.cpp:204-230 */
int orc_solver_run(orc_solver *s, const char *dir, int nsteps_max)
{
    double t = 0;
    double dt = s->maxDt;
    double tFinal = s->deck.tFinal, outDeltaT = s->deck.outDeltaT;
    int steps = 0;
    int st = orc_solver_output(s, t, dir);
    if (st)
        return st;
    for (double tOut = MIN(t + outDeltaT, tFinal); tOut <= tFinal;
         tOut = MIN(tOut + outDeltaT, tFinal)) {
        dt = s->maxDt;
        while (t < tOut) {
            t += dt;
            if (t > tOut) {
                dt = tOut - (t - dt);
                t = tOut;
            }
            st = orc_solver_update(s, dt);
            if (st)
                return st;
            steps++;
            if (nsteps_max >= 0 && steps >= nsteps_max)
                return ORC_OK;
        }
        st = orc_solver_output(s, t, dir);
        if (st)
            return st;
        if (tOut > tFinal - 1e-12 * tFinal)
            break;
    }
    return ORC_OK;
}

/* One RK stage without the Heun average (diagnostics for the tests). */
int orc_solver_stage(orc_solver *s, double dt)
{
    if (s->deck.initCond == 2)
        duplicate_boundaries(s);
    solve_optimization(s);
    if (s->status != ORC_OK)
        return s->status;
    solve_flux(s, s->dx, s->dy);
    euler_collide(s, dt, s->dx, s->dy);
    return ORC_OK;
}

/* ---------------- a node of a partitioned grid ---------------- */

/* momopt_update.cpp:299-308 */
void orc_solver_save_old(orc_solver *s)
{
    int n = s->set.n;
    for (int i = s->gX[1]; i <= s->gX[2]; i++)
        for (int j = s->gY[1]; j <= s->gY[2]; j++)
            for (int k = 0; k < n; k++)
                s->momentsOld[I3D(i, j, k)] = s->moments[I3D(i, j, k)];
}

void orc_solver_pre_exchange(orc_solver *s)
{
    if (s->deck.isMoment && s->deck.pnFilterType != 0)
        moment_scale(s);
}

/* momopt_update.cpp:311-336 (moment_update.cpp:180-203) with the ghosts
 * already exchanged */
int orc_solver_stage_exchanged(orc_solver *s, double dt)
{
    if (s->deck.isMoment) {
        moment_flux(s, s->dx, s->dy);
        euler_collide(s, dt, s->dx, s->dy);
        return ORC_OK;
    }
    solve_optimization(s);
    if (s->status != ORC_OK)
        return s->status;
    solve_flux(s, s->dx, s->dy);
    euler_collide(s, dt, s->dx, s->dy);
    return ORC_OK;
}

/* momopt_update.cpp:367-377 */
void orc_solver_average(orc_solver *s)
{
    int n = s->set.n;
    for (int i = s->gX[1]; i <= s->gX[2]; i++)
        for (int j = s->gY[1]; j <= s->gY[2]; j++)
            for (int k = 0; k < n; k++)
                s->moments[I3D(i, j, k)] = 0.5 * (s->moments[I3D(i, j, k)] + s->momentsOld[I3D(i, j, k)]);
}

/* momopt_boundaries.cpp:17-27 (the used part of the buffers) */
long long orc_solver_halo_count(const orc_solver *s, int side)
{
    long long sx = s->gX[2] - s->gX[1] + 1, sy = s->gY[2] - s->gY[1] + 1;
    return 2LL * (side < 2 ? sx : sy) * s->set.n;
}

/* momopt_boundaries.cpp:30-188; side 0 north, 1 south, 2 east, 3 west */
void orc_solver_halo(orc_solver *s, int side, int pack, double *buf)
{
    int n = s->set.n;
    const int sx = s->gX[2] - s->gX[1] + 1, sy = s->gY[2] - s->gY[1] + 1;
    for (int g = 0; g < 2; g++) {
        if (side < 2) {
            int j = pack ? (side == 0 ? s->gY[2] + 1 - 2 + g : s->gY[1] + g)
                         : (side == 0 ? s->gY[2] + 1 + g : s->gY[0] + g);
            for (int i = s->gX[1]; i <= s->gX[2]; i++) {
                double *b = buf + ((size_t)(i - s->gX[1]) + (size_t)g * sx) * n;
                double *m = &s->moments[I3D(i, j, 0)];
                if (pack)
                    memcpy(b, m, sizeof(double) * n);
                else
                    memcpy(m, b, sizeof(double) * n);
            }
        } else {
            int i = pack ? (side == 2 ? s->gX[2] + 1 - 2 + g : s->gX[1] + g)
                         : (side == 2 ? s->gX[2] + 1 + g : s->gX[0] + g);
            for (int j = s->gY[1]; j <= s->gY[2]; j++) {
                double *b = buf + ((size_t)(j - s->gY[1]) + (size_t)g * sy) * n;
                double *m = &s->moments[I3D(i, j, 0)];
                if (pack)
                    memcpy(b, m, sizeof(double) * n);
                else
                    memcpy(m, b, sizeof(double) * n);
            }
        }
    }
}
