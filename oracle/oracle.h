/*
 * oracle.h -- CPU restatement of the closures-2d Mn/PPn entropy-closure path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle: a plain-C, FP64 restatement
 * of the reference algorithm, used as the checker by tests/, by
 * __graft_entry__.smoke() and by bench.py's cpu_baseline / reference arm.
 * The product (closures-2d_b200/) never links, loads or calls anything here.
 *
 * Parity pin: the restatement reproduces the reference's eight momopt
 * regression goldens (tests/regression/momopt/{delta,gaussian,lattice,smooth}
 * /{mn,ppn}.pn, copied to tests/golden/) -- see tests/test_oracle_golden.py.
 *
 * Each function cites the reference file:line it follows (paths inside the
 * closures-2d project).  Third-party arithmetic the reference pulls from GSL
 * (Gauss-Legendre table, normalised associated Legendre functions, Householder
 * QR least squares) and LAPACK (dpotrf, dpocon, dpotrs) is restated from the
 * published algorithms; neither library is present here and neither version is
 * pinned by the reference (install.md lists no versions).
 */
#ifndef CLOSURES_ORACLE_H
#define CLOSURES_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* opt/opt.h:34-37 */
enum { ORC_MN = 0, ORC_PPN = 1 };

/* opt/opt.h:39-40 */
#define ORC_NUM_REG 5
extern const double ORC_REGULARIZATIONS[ORC_NUM_REG];

/* Status codes.  The reference aborts the process in these cases
 * (opt.cpp:97-101 "u[0] < 0", opt.cpp:256-261 "Max regularization achieved");
 * the oracle returns them so tests can observe the failure. */
enum { ORC_OK = 0, ORC_ERR_U0 = -1, ORC_ERR_MAXREG = -2, ORC_ERR_INPUT = -3 };

/* opt/opt.h:11-23 (tolAbs is unused by the optimisers). */
typedef struct {
    int momentType;
    int maxIter;
    double tolRel;
    double condHMax;
    double deltaPPn;
    int useGaunt;
    /* Supplementary stopping test gamma = modcfl(d) <= tolGamma, present in
     * the reference as commented-out code (opt.cpp:99-126, :339, :343;
     * tolGamma = 1.1 at momopt_update.cpp:226).  0 disables it, which is the
     * reference's current behaviour; 1.1 reproduces the revision that wrote
     * the delta and lattice regression goldens. */
    double tolGamma;
    /* BFGS only (optbfgs.cpp): quasi-Newton steps per Hessian evaluation and
     * the bound on cond(H) * cond(H^-1) of the BFGS approximations */
    int maxBfgsIter;
    double condHMaxBfgs;
} orc_options;

/* opt/opt.h:25-32 */
typedef struct {
    double r;
    int iter;
    double normG;
} orc_outs;

/* Gaunt table (fobj.h:12-22 HStruct), stored CSR over the n*n (i,j) pairs. */
typedef struct {
    int n;          /* moments */
    int *off;       /* n*n+1 offsets */
    int *idx;       /* extended-moment index k */
    double *val;    /* coefficient */
} orc_gaunt;

/* Angular set-up: momopt_init.cpp:88-259 */
typedef struct {
    int order, Q, useGaunt;
    int n, n2, nq;
    double *w, *xi, *eta;   /* [nq] */
    double *p;              /* [nq*n2] row-major, p[q*n2+k] */
    orc_gaunt gaunt;        /* only when useGaunt */
} orc_setup;

int  orc_setup_create(int order, int Q, int useGaunt, orc_setup *s);
void orc_setup_free(orc_setup *s);

/* Gauss-Legendre nodes (ascending) and weights on [-1,1]; utils.cpp:55-60. */
void orc_gauss_legendre(int n, double *x, double *w);
/* Normalised associated Legendre with Condon-Shortley phase
 * (the quantity gsl_sf_legendre_sphPlm returns). */
double orc_sphPlm(int l, int m, double x);
/* Householder QR of a row-major rows x cols matrix in place, and the least
 * squares solve with it (momopt_init.cpp:233-243 uses GSL's). */
void orc_householder_qr(int rows, int cols, double *A, double *tau);
void orc_householder_lssolve(int rows, int cols, const double *QR, const double *tau, double *b, double *beta);

/* Per-cell operator: opt.cpp:82-148 (in-place on u, alpha). */
int orc_opt(int n, int n2, int nq, double *u, double *alpha, orc_options opts,
            const double *w, const double *p, const orc_gaunt *g, orc_outs *outs);

/* Batched opt over count vectors of n (OpenMP, schedule(dynamic,1)), as the
 * reference's solveOptimization loop (momopt_update.cpp:208-277).
 * status[c] receives the orc_opt return code; iters/regs may be NULL. */
int orc_opt_batch(const orc_setup *s, orc_options opts, int count,
                  double *u, double *alpha, int *iters, double *regs, int *status);

/* Change-of-basis Newton, opt/optcb.cpp (MOMOPT_OPTIMIZATION_TYPE 1).  P2M
 * (nm x nm lower triangular, row-major) and alphaP persist per cell and are
 * updated in place; alphaM receives the multipliers in the moment basis.  p
 * is the basis with row stride np (the setup's n2). */
int orc_optcb(int nm, int nq, double *u, double *P2M, double *alphaP, double *alphaM,
              orc_options opts, const double *w, const double *p, int np, orc_outs *outs);
/* momopt_init.cpp:146-157 initial state of a cell (see opt.c). */
void orc_optcb_init(int nm, int momentType, double delta, double *P2M, double *alphaP);
/* BFGS sub-iterations in the change of basis: opt/optbfgs.cpp (type 2); same
 * per-cell state and initialisation as orc_optcb. */
int orc_optbfgs(int nm, int nq, double *u, double *P2M, double *alphaP, double *alphaM,
                orc_options options, const double *w, const double *p, int np, orc_outs *outs);
/* optType 1: orc_optcb, 2: orc_optbfgs on every vector */
int orc_optcb_batch(const orc_setup *s, orc_options opts, int optType, int count, double *u,
                    double *P2M, double *alphaP, double *alpha, int *iters, double *regs, int *status);

/* f,g,H evaluation (fobj.cpp); g and h may be NULL as in the reference. */
double orc_fobj(int momentType, int n, int n2, int nq, const double *alpha,
                const double *u, const double *w, const double *p, double delta,
                double *g, double *h, int useGaunt, const orc_gaunt *gt, double *gExt);

/* ---------------------------------------------------------------------- */
/* Whole solver: main.cpp + momopt_*.cpp                                  */

typedef struct {
    /* input.deck (main.cpp:67-83) */
    int numCellsX, numCellsY;
    double ax, ay, bx, by, tFinal, outDeltaT, gaussianSigma, floor_, sigma;
    int initCond;
    /* momopt deck (momopt_init.cpp:56-68) */
    int nodesX, nodesY;     /* NUM_MPI_PARTITIONS_X, _Y */
    int momentOrder, quadOrder, useGaunt, momentType, optType, maxIter, maxBfgsIter;
    double cflFactor, tol, condHMax, condHMaxBfgs, theta, deltaPPn;
    double tolGamma;        /* optional key MOMOPT_TOL_GAMMA, default 0 (off) */
    /* SOLVER moment (the linear Pn/FPn solver, moment_init.cpp:53-61) */
    int isMoment;
    int pnOrder, pnQuadOrder, pnFilterType;
    double pnFilterTune, pnCflFactor;
} orc_deck;

typedef struct {
    int maxIter;
    int histReg[ORC_NUM_REG];
    double iterMean;
    int64_t numDualSolves;
} orc_stats;

typedef struct {
    orc_deck deck;
    orc_setup set;
    /* this process's block of the partition (main.cpp:157-193; node 0 of
     * 1 x 1 without MPI) */
    int node, numNodes, nodeX, nodeY, numNodesX, numNodesY;
    double initX, initY;
    int gX[4], gY[4];
    int NX, NY;             /* with ghosts */
    double dx, dy, maxDt;
    double *initialGrid, *sigmaT, *sigmaS;   /* [NX*NY] */
    double *moments, *alpha, *flux, *momentsOld, *ansatzGrid;
    double *alphaP, *P2M;   /* change-of-basis state per cell (optType 1, 2) */
    double *pnOps;          /* SOLVER moment: the flux operators xi+, xi-, eta+, eta- [4][n][n] */
    double *pnFilter;       /* SOLVER moment: filter factor per moment [n] */
    orc_stats stats;
    int *lastIters;         /* per-cell iterations of the last stage */
    int status;             /* first error code seen */
    int64_t errCell;
} orc_solver;

/* Deck parsing with the reference's semantics (input_deck_reader.cpp). */
int orc_deck_read(const char *path, orc_deck *d);
int orc_solver_create(const orc_deck *d, orc_solver *s);
/* node of the deck's NUM_MPI_PARTITIONS_X x _Y partition on numNodes nodes */
int orc_solver_create_node(const orc_deck *d, int node, int numNodes, orc_solver *s);
/* The stages of update() for a node whose ghosts a halo exchange fills
 * (comm.cpp:31-147 in place of the periodic copy): save the interior,
 * one stage without the ghost copy, the Heun average. */
void orc_solver_save_old(orc_solver *s);
/* Work of a stage before its exchange: the moment filter of SOLVER moment
 * (moment_update.cpp:178-179), nothing for momopt. */
void orc_solver_pre_exchange(orc_solver *s);
int orc_solver_stage_exchanged(orc_solver *s, double dt);
void orc_solver_average(orc_solver *s);
/* momopt_boundaries.cpp:17-188: doubles per side (north, south, east,
 * west), and the inner strips packed into / the ghost strips unpacked from
 * buf. */
long long orc_solver_halo_count(const orc_solver *s, int side);
void orc_solver_halo(orc_solver *s, int side, int pack, double *buf);
void orc_solver_free(orc_solver *s);
/* One RK2 step, momopt_update.cpp:283-382.  Returns the status. */
int orc_solver_update(orc_solver *s, double dt);
/* momopt_output.cpp:21-77, files out_<t>_0.{pn,opt} in dir. */
int orc_solver_output(orc_solver *s, double time, const char *dir);
/* main.cpp:204-230 time loop including outputs; nsteps_max<0 = no limit. */
int orc_solver_run(orc_solver *s, const char *dir, int nsteps_max);

#ifdef __cplusplus
}
#endif
#endif
