/*
 * closures_gpu.h -- C ABI of libclosures_gpu.so, the B200 (sm_100a) Mn/PPn
 * entropy-closure path of closures-2d.
 *
 * The library replaces, behind plain pointers and sizes, the reference's
 * momopt hot path:
 *   - MomOptSolver::update        src/momopt/momopt_update.cpp:283-382
 *       (solveOptimization :208-277, solveFlux :96-202, Euler/collision/
 *        source :316-336,:344-364, Heun average :367-377)
 *   - opt() per-cell dual solve   src/momopt/opt/opt.cpp:82-343 with
 *       fobj.cpp:37-428 and linesearch.cpp:21-99
 *   - communicateBoundaries       src/comm.cpp:149-154 (serial: periodic copy,
 *       momopt_boundaries.cpp:190-223), done on the device
 *   - angular set-up              src/momopt/momopt_init.cpp:88-259
 *   - the MomOptSolver state      src/momopt/momopt_solver.h:74-78 (moments,
 *       alpha, flux) lives in device memory owned by the context.
 *
 * Conventions: every int-returning call returns CL_OK (0) or a negative
 * CL_ERR_* code and records a message retrievable with cl_last_error(); the
 * context owns all device memory, one CUDA stream and the captured RK2 graph;
 * the caller owns every host buffer.  A context is used by one host thread at
 * a time.  There is no CPU fallback: without a usable sm_100 device
 * cl_create() fails with CL_ERR_CUDA.
 */
#ifndef CLOSURES_GPU_H
#define CLOSURES_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CL_ABI_VERSION 1

enum {
    CL_OK = 0,
    CL_ERR_ARG = -1,       /* bad argument / unsupported configuration */
    CL_ERR_CUDA = -2,      /* CUDA runtime error or no usable device */
    CL_ERR_U0 = -3,        /* a cell had u0 <= 0 (opt.cpp:97-101 aborts) */
    CL_ERR_MAXREG = -4,    /* regularisation ladder exhausted (opt.cpp:256-261) */
    CL_ERR_TIMEOUT = -5,   /* a bounded device wait gave up */
    CL_ERR_STATE = -6      /* call order / state error */
};

enum { CL_MN = 0, CL_PPN = 1 };            /* opt/opt.h:34-37 */
enum { CL_FP64 = 0, CL_MIXED = 1 };        /* arithmetic of the Hessian assembly */
#define CL_NUM_REG 5                       /* opt/opt.h:39-40 */

/* Message of a return code (CL_OK and every CL_ERR_*; "device error" for
 * anything else).  The texts of CL_ERR_U0 and CL_ERR_MAXREG are the
 * reference's own abort messages (opt.cpp:97-101, opt.cpp:256-261).  Needs
 * no device. */
const char *cl_error_text(int code);

/* Angular discretisation: momopt_init.cpp:88-259.  Arrays are owned by the
 * library and released by cl_angular_free(). */
typedef struct {
    int order;          /* MOMOPT_MOMENT_ORDER N */
    int quad_order;     /* MOMOPT_QUAD_ORDER Q */
    int use_gaunt;      /* MOMOPT_USE_GAUNT */
    int n;              /* (N+1)(N+2)/2 moments */
    int n2;             /* (2N+1)(2N+2)/2 if use_gaunt else n */
    int nq;             /* Q*Q quadrature points */
    double *w, *xi, *eta;   /* [nq] weights (sum 4*pi) and directions */
    double *p;              /* [nq*n2] basis, p[q*n2+k] */
    int gaunt_nnz;
    int *gaunt_off;         /* [n*n+1] CSR over (i,j) pairs, row-major i*n+j */
    int *gaunt_idx;         /* [nnz] extended-moment index */
    double *gaunt_val;      /* [nnz] coefficient (|beta| > 1e-9 kept) */
} cl_angular;

/* Builds the quadrature, the z-even real spherical-harmonic basis (with the
 * Condon-Shortley phase) and, if use_gaunt, the product table, in FP64 on
 * the host.  Replaces MomOptSolver::init's set-up, momopt_init.cpp:88-259
 * (and moment_init.cpp:69-183).  Orders 1..6 with the Gaunt table, 1..9
 * without (the entropy-closure contexts take orders up to 6). */
int cl_angular_create(int order, int quad_order, int use_gaunt, cl_angular *out);
void cl_angular_free(cl_angular *a);

/* Solver options: the MOMOPT_* deck keys read at momopt_init.cpp:56-68. */
typedef struct {
    int moment_type;        /* CL_MN or CL_PPN */
    int opt_type;           /* MOMOPT_OPTIMIZATION_TYPE: 0 Newton (opt.cpp),
                               1 change of basis (optcb.cpp), 2 BFGS
                               sub-iterations in the change of basis
                               (optbfgs.cpp) */
    int max_iter;           /* MOMOPT_MAX_ITER */
    double tol;             /* MOMOPT_TOL (relative gradient tolerance) */
    double cond_h_max;      /* MOMOPT_COND_H_MAX */
    double delta_ppn;       /* MOMOPT_DELTA_PPN */
    double tol_gamma;       /* optional supplementary stopping test
                               modcfl(d) <= tol_gamma, commented out in
                               opt.cpp:99-126; 0 = off */
    int precision;          /* CL_FP64 or CL_MIXED */
    int max_bfgs_iter;      /* MOMOPT_MAX_BFGS_ITER (opt_type 2, >= 1) */
    double cond_h_max_bfgs; /* MOMOPT_COND_H_MAX_BFGS (opt_type 2) */
    int contraction;        /* CL_CONTRACT_PAIRS (default): the quadrature
                               directions phi and phi + pi share one
                               contraction through the degree parity of the
                               basis, in the kinetic flux (Mn and PPn) and in
                               the Newton evaluation where supported (Mn,
                               FP64); CL_CONTRACT_SINGLE: every direction on
                               its own. The same sums in another order. */
} cl_options;
enum { CL_CONTRACT_PAIRS = 0, CL_CONTRACT_SINGLE = 1 };

/* Grid description: Solver fields of solver.h:15-61 for one node. */
typedef struct {
    int nx, ny;             /* interior cells (c_sizeX, c_sizeY) */
    int ghost;              /* must be 2 (MomOptSolver::getNumGhostCells) */
    int init_cond;          /* 0 line source/gaussian, 1 lattice, 2 periodic */
    double init_x, init_y;  /* c_initX, c_initY: least x,y of the interior */
    double theta;           /* MOMOPT_THETA limiter parameter */
} cl_grid;

typedef struct {
    int max_iter;                   /* c_optStats.maxIter */
    double iter_mean;               /* c_optStats.iterMean */
    int64_t num_solves;             /* c_optStats.numDualSolves */
    int64_t hist_reg[CL_NUM_REG];   /* c_optStats.histReg */
    int64_t total_iter;             /* sum of iterations (device counter) */
    int64_t total_trials;           /* line-search function evaluations */
    int64_t fallbacks;              /* predicted starts replaced by the fallback start */
    int64_t screened;               /* solves settled by K1's screening pass at their first
                                       evaluation (counted in the fields above as well) */
    int64_t screen_evals;           /* evaluations run by the screening pass (gradient
                                       columns only; those of unsettled cells are not
                                       counted in total_iter) */
    int64_t flux_tiles;             /* K2+K3 16x16 tiles that ran the kinetic flux (the
                                       others had one alpha over tile and halo: zero flux) */
} cl_stats;

typedef struct cl_ctx cl_ctx;

/* Creates a context holding the state of one grid (ghosts included,
 * (nx+4)*(ny+4) cells, layout I3D(i,j,k) = ((i*(ny+4))+j)*n+k of
 * solver.h:12-13) and uploads the angular set-up, sigma fields and the
 * initial moments/alpha.  Replaces MomOptSolver::init's allocations
 * (momopt_init.cpp:103-160). */
int cl_create(const cl_grid *grid, const cl_options *opts, const cl_angular *ang,
              const double *sigma_t, const double *sigma_s,
              const double *moments, const double *alpha, cl_ctx **out);
void cl_destroy(cl_ctx *ctx);
const char *cl_last_error(const cl_ctx *ctx);
/* Message of the last failure of a call that had no context (cl_create,
 * cl_angular_create). */
const char *cl_global_error(void);

/* One Heun RK2 step (MomOptSolver::update, momopt_update.cpp:283-382) on the
 * device, replayed from a captured CUDA graph.  Blocks until the step is
 * done and reports a device-side error (u0 <= 0, ladder exhausted). */
int cl_step(cl_ctx *ctx, double dt, double dx, double dy);
/* Same step launched kernel by kernel (no graph) with CUDA events on the
 * context's stream; ms[0..3] receive the durations of the stage-1
 * optimisation, stage-1 flux/update, stage-2 optimisation and stage-2
 * flux/update/average kernels. */
int cl_step_timed(cl_ctx *ctx, double dt, double dx, double dy, float *ms);
/* Same, without waiting: errors surface at the next cl_sync(). */
int cl_step_async(cl_ctx *ctx, double dt, double dx, double dy);
int cl_sync(cl_ctx *ctx);

/* One RK stage of the step (stage 1 or 2, in that order; momopt_update.cpp
 * :311-336 and :339-377): optimisation of every cell, flux and the Euler,
 * collision and source update of the interior, stage 2 also the Heun
 * average.  No ghost copy: a node of a partitioned grid fills its ghost
 * strips from its neighbours (cl_halo_*) before each stage, as
 * communicateBoundaries does (comm.cpp:31-147).  Asynchronous on the
 * context's stream; errors surface at the next cl_sync(). */
int cl_stage(cl_ctx *ctx, int stage, double dt, double dx, double dy);
/* Same stage, waited for, with the durations of its optimisation kernel
 * (ms[0]) and flux/update kernel (ms[1]) from CUDA events on the context's
 * stream; reports a device-side error like cl_step. */
int cl_stage_timed(cl_ctx *ctx, int stage, double dt, double dx, double dy, float *ms);
/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work (the halo exchange) with the library's. */
int cl_stream(cl_ctx *ctx, void **stream);

/* Halo of a node's block (momopt_boundaries.cpp:17-188).  Sides: */
enum { CL_NORTH = 0, CL_SOUTH = 1, CL_EAST = 2, CL_WEST = 3 };
/* Doubles per side: north/south 2 * nx * n (the two columns next to the
 * largest / least y over the interior x), east/west 2 * ny * n (the two rows
 * next to the largest / least x over the interior y); corners are not
 * exchanged.  Buffer order [strip][cell][k] as getInnerBoundaries packs. */
int cl_halo_counts(const cl_ctx *ctx, long long counts[4]);
/* getInnerBoundaries: the inner strips into the device buffers bufs[side]
 * (null entries skipped), on the context's stream. */
int cl_halo_pack(cl_ctx *ctx, double *const bufs[4]);
/* setOuterBoundaries: the device buffers into the ghost strips (null
 * entries skipped), on the context's stream. */
int cl_halo_unpack(cl_ctx *ctx, double *const bufs[4]);

/* Copies the full state (all cells, ghosts included) to / from the host. */
int cl_get_state(cl_ctx *ctx, double *moments, double *alpha);
int cl_set_state(cl_ctx *ctx, const double *moments, const double *alpha);
/* One RK2 step (MomOptSolver::update, momopt_update.cpp:279-378) on a state
 * held in host memory, as the reference's solver holds c_moments and c_alpha:
 * moments and alpha ([NX*NY][n], ghosts included) are read, stepped and
 * overwritten with the new state.  The result equals cl_set_state, cl_step,
 * cl_get_state; the copies overlap the kernels (bands of cells go up while
 * earlier bands are solved, the multipliers and the first part of the
 * moments come back under the second-stage flux), which needs page-locked
 * host buffers to take effect.  Blocks until the step is done. */
int cl_step_host(cl_ctx *ctx, double dt, double dx, double dy, double *moments, double *alpha);
/* Cumulative optimisation statistics (momopt_update.cpp:256-275). */
int cl_get_stats(cl_ctx *ctx, cl_stats *s);
/* outs.iter of every cell (ghosts included) in the last optimisation stage. */
int cl_get_last_iterations(cl_ctx *ctx, int *iters);
/* Sets those counts (host [NX*NY]), e.g. with a state put back by
 * cl_set_state, for the selective learned start that reads them. */
int cl_set_last_iterations(cl_ctx *ctx, const int *iters);

/* Autotuner of the launch shapes -- no counterpart in the reference, whose
 * per-cell loop is an OpenMP schedule(dynamic,1) over cells
 * (momopt_update.cpp:208-277, :214).  Candidates, each run on copies of the
 * context's current state (the real state is untouched):
 *   K1 (Newton):  cells per CTA and warps -- 32 cells / 8 warps / one CTA
 *                 per SM, or 16 cells / 4 warps / two CTAs per SM (the
 *                 direction-pair layout) -- and the Hessian tile layout:
 *                 direction pairs (even/odd degree column tiles) or one
 *                 direction at a time, where both exist (Mn, FP64);
 *   K2+K3 (flux): the same two tile layouts.
 * Every candidate is launched once untimed, then timed three times with
 * CUDA events on the context's stream; the median decides.  The choice is
 * applied to the context and cached per (order, quadrature, Gaunt, closure,
 * precision, optimisation type) in the process, and in the file named by
 * the environment variable CL_TUNE_CACHE when set; with use_cache = 1 a
 * cached choice is applied without timing.  Grids below 16384 cells, batch-only
 * contexts and the change-of-basis types keep the default shape (nothing is
 * timed; out->ncand = 0).  Every candidate computes the same per-cell sums:
 * the two K1 launch shapes give bit-identical results, the two tile layouts
 * the same sums in another order. */
#define CL_TUNE_MAX 8
typedef struct {
    int newton_warps;         /* K1 warps per CTA: 8 (32 cells per CTA) or 4 (16) */
    int newton_ctas;          /* K1 persistent CTAs per launch */
    int newton_contraction;   /* K1 Hessian tile layout: CL_CONTRACT_PAIRS or _SINGLE */
    int flux_contraction;     /* K2+K3 tile layout */
    int from_cache;           /* 1: taken from the cache, nothing timed */
    int ncand;                /* candidates timed */
    int cand_kernel[CL_TUNE_MAX];        /* 1: K1, 2: K2+K3 */
    int cand_warps[CL_TUNE_MAX];
    int cand_contraction[CL_TUNE_MAX];
    float cand_ms[CL_TUNE_MAX];          /* median launch time */
    int screen_ctas;          /* CTAs of K1's screening pass (0: no screening pass) */
} cl_tuning;
int cl_tune(cl_ctx *ctx, int use_cache, cl_tuning *out);   /* use_cache 0: always time */
/* The shapes in use (after cl_tune, cl_set_launch_shape or the defaults). */
int cl_get_tuning(cl_ctx *ctx, cl_tuning *out);
/* Forces the shapes (CL_ERR_ARG where the configuration has no such
 * instance): newton_warps 8 or 4, contractions CL_CONTRACT_PAIRS/_SINGLE. */
int cl_set_launch_shape(cl_ctx *ctx, int newton_warps, int newton_contraction, int flux_contraction);
/* The exponent-range test of K1 (on by default; Mn in FP64): an evaluation
 * whose gradient meets the tolerance converges without forming the Hessian
 * when the range of alpha . p over the quadrature bounds the Hessian's
 * condition number below MOMOPT_COND_H_MAX / 4 -- the reference's outcome
 * (opt.cpp:244-306) at that evaluation.  Results are bit-identical with the
 * test on or off; off runs every evaluation through the Hessian. */
int cl_set_range_test(cl_ctx *ctx, int enable);
/* K2+K3's uniform-tile shortcut (on by default): a 16x16 tile whose alpha,
 * halo included, is one value bit for bit has zero flux (every slope and
 * upwind difference of momopt_update.cpp:96-202 is an exact zero) and skips
 * the kinetic flux loop.  Results are the same with it off, up to the sign
 * of zero; off, every tile runs the loop. */
int cl_set_uniform_flux_skip(cl_ctx *ctx, int enable);

/* Batched per-vector operator: the GPU equivalent of calling
 * opt(n, n2, nq, u, alpha, options, w, p, &outs) (opt.cpp:82-148) on `count`
 * vectors, in place on u and alpha (host arrays, [count*n] each, the order of
 * the context's angular set-up).  iters/reg/status (nullable, [count]) receive
 * outs.iter, outs.r and the per-vector status (0, CL_ERR_U0, CL_ERR_MAXREG). */
int cl_solve_batch(cl_ctx *ctx, int count, double *u, double *alpha,
                   int *iters, double *reg, int *status);

/* Same on device pointers (no host copies), on the context's stream. */
int cl_solve_batch_device(cl_ctx *ctx, int count, double *d_u, double *d_alpha,
                          int *d_iters, double *d_reg, int *d_status);
/* Same, starting from d_alpha_start (e.g. cl_mlp_predict's output) where it
 * is finite; d_alpha is then the fallback start, taken once in place of the
 * first regularisation step, so a poor prediction costs iterations but does
 * not change the regularisation the plain start would need. */
int cl_solve_batch_device_start(cl_ctx *ctx, int count, double *d_u, double *d_alpha,
                                const double *d_alpha_start, int *d_iters, double *d_reg,
                                int *d_status);
/* Change-of-basis solves on device pointers: optcb() (optcb.cpp:87-415,
 * the OPT_TYPE_CHANGE_BASIS branch of momopt_update.cpp:240-244) for a
 * context created with opt_type 1, optbfgs() (optbfgs.cpp:90-512, the
 * OPT_TYPE_BFGS branch of momopt_update.cpp:245-248) with opt_type 2.  Each
 * vector carries its basis d_P2M [count][n][n] (row-major, lower triangular) and multipliers
 * d_alphaP [count][n] in that basis, read at the start and written back on
 * convergence; d_alpha receives the multipliers in the moment basis and d_u
 * the regularised input moments, as the reference returns them.  A grid
 * context keeps this state per cell by itself (initialised as
 * momopt_init.cpp:146-157 does). */
int cl_solve_batch_cb_device(cl_ctx *ctx, int count, double *d_u, double *d_P2M, double *d_alphaP,
                             double *d_alpha, int *d_iters, double *d_reg, int *d_status);

/* Mixed-order batch: a solver context for several moment orders at one
 * quadrature order, so vectors of different N share one persistent launch.
 * Device pointers; vectors of order orders[s] are packed in segment s. */
typedef struct cl_multi cl_multi;
int cl_multi_create(int norders, const int *orders, int quad_order, int use_gaunt,
                    const cl_options *opts, cl_multi **out);
void cl_multi_destroy(cl_multi *m);
const char *cl_multi_last_error(const cl_multi *m);
int cl_multi_solve_device(cl_multi *m, const int *counts, double *const *d_u,
                          double *const *d_alpha, int *const *d_iters,
                          double *const *d_reg, int *const *d_status);
int cl_multi_solve_device_start(cl_multi *m, const int *counts, double *const *d_u,
                                double *const *d_alpha, double *const *d_alpha_start,
                                int *const *d_iters, double *const *d_reg,
                                int *const *d_status);
/* ------------------------------------------------------------------------
 * Whole solver behind the reference's Solver interface (solver.h:15-61) for
 * the deck's SOLVER (main.cpp:93-106): momopt (MomOptSolver,
 * momopt_init.cpp:51-272, momopt_update.cpp:283-382, momopt_output.cpp:21-77,
 * files out_<t>_<node>.pn / .opt) or moment (MomentSolver, the linear Pn/FPn
 * solver, moment_init.cpp:53-297, moment_update.cpp:169-247,
 * moment_output.cpp:21-56, file out_<t>_<node>.pn); deck parsing
 * (input_deck_reader.cpp), grid and initial condition (main.cpp:257-372). */
typedef struct cl_solver cl_solver;
typedef struct cl_pn cl_pn;
enum { CL_SOLVER_MOMOPT = 0, CL_SOLVER_MOMENT = 1 };
/* Reads deck_path (input.deck semantics, every key of the solver required as
 * in momopt_init.cpp:56-68 / moment_init.cpp:57-61) and creates the solver;
 * *max_dt receives init()'s return value (momopt_init.cpp:72,
 * moment_init.cpp:65).  Output files go to out_dir. */
int cl_solver_create(const char *deck_path, const char *out_dir, cl_solver **out, double *max_dt);
int cl_solver_kind(const cl_solver *s);                 /* CL_SOLVER_MOMOPT or _MOMENT */
int cl_solver_geometry(cl_solver *s, int *nx, int *ny, int *n, double *dx, double *dy, double *t_final,
                       double *out_delta_t);
int cl_solver_update(cl_solver *s, double dt);          /* Solver::update */
int cl_solver_output(cl_solver *s, double time);        /* Solver::outputData */
/* The state (all cells, ghosts included, [(nx+4)*(ny+4)*n]) to / from the host. */
int cl_solver_get_state(cl_solver *s, double *moments);
int cl_solver_set_state(cl_solver *s, const double *moments);
/* The device context of a momopt solver (null for moment), of a moment
 * solver (null for momopt). */
cl_ctx *cl_solver_context(cl_solver *s);
cl_pn *cl_solver_pn(cl_solver *s);
const char *cl_solver_last_error(const cl_solver *s);
void cl_solver_destroy(cl_solver *s);

/* ------------------------------------------------------------------------
 * The linear Pn / FPn solver (SOLVER moment, src/moment/): moments evolved
 * by upwind flux operators with an optional filter, no optimisation.  The
 * host builds the set-up as MomentSolver::init does (moment_init.cpp:53-297);
 * the context holds the grid state on the device and steps it. */
typedef struct {
    int n;                  /* moments per cell, at most 64 (order <= 9) */
    const double *ops;      /* [4][n][n] c_pnFluxOperatorXiPlus, XiMinus,
                               EtaPlus, EtaMinus, row i column j as
                               moment_init.cpp:186-222 fills them */
    const double *filter;   /* [n] c_momentFilter, or null for
                               MOMENT_FILTER_TYPE 0 (no filtering) */
} cl_pn_setup;
/* Grid as for cl_create; moments [(nx+4)*(ny+4)*n], ghosts included. */
int cl_pn_create(const cl_grid *grid, const cl_pn_setup *setup, const double *sigma_t,
                 const double *sigma_s, const double *moments, cl_pn **out);
void cl_pn_destroy(cl_pn *p);
const char *cl_pn_last_error(const cl_pn *p);
/* MomentSolver::update (moment_update.cpp:169-247): one Heun RK2 step, the
 * periodic ghost copy before each stage for INIT_COND 2; waits. */
int cl_pn_step(cl_pn *p, double dt, double dx, double dy);
/* One stage (1 then 2) without the ghost copy, for a node whose halo is
 * exchanged before each stage (cl_pn_halo_*); asynchronous. */
int cl_pn_stage(cl_pn *p, int stage, double dt, double dx, double dy);
/* Same, waited for; *ms receives its duration (CUDA events). */
int cl_pn_stage_timed(cl_pn *p, int stage, double dt, double dx, double dy, float *ms);
/* Bit s set: the ghost strip of side s holds a neighbour's interior (the
 * filter applies to it as to the interior, moment_update.cpp:178-182);
 * default: all sides for INIT_COND 2, none otherwise. */
int cl_pn_set_exchanged_sides(cl_pn *p, int mask);
int cl_pn_sync(cl_pn *p);
int cl_pn_stream(cl_pn *p, void **stream);
/* All cells; ghost strips that a periodic copy or a halo exchange fills hold
 * the values copied before the step's first stage (they are refilled before
 * every stage, so the interior is the reference's). */
int cl_pn_get_state(cl_pn *p, double *moments);
int cl_pn_set_state(cl_pn *p, const double *moments);
/* One RK2 step (MomentSolver::update, moment_update.cpp:151-247) on a state
 * held in host memory ([NX*NY][n], ghosts included, read and overwritten),
 * equal to cl_pn_set_state, cl_pn_step, cl_pn_get_state.  Bands of rows go
 * up, are stepped and come back while later bands are still going up, which
 * needs page-locked host memory to take effect.  Periodic or partitioned
 * grids run the three calls in turn.  Blocks until the step is done. */
int cl_pn_step_host(cl_pn *p, double dt, double dx, double dy, double *moments);
/* As cl_halo_*, on the state the next stage reads (moment_boundaries.cpp). */
int cl_pn_halo_counts(const cl_pn *p, long long counts[4]);
int cl_pn_halo_pack(cl_pn *p, double *const bufs[4]);
int cl_pn_halo_unpack(cl_pn *p, double *const bufs[4]);
/* A node of the block partition of main.cpp:157-193 (the MPI build): the
 * grid of num_cells_x x num_cells_y cells on [ax,bx] x [ay,by] split into
 * nodes_x x nodes_y blocks, node = node_x * nodes_y + node_y. */
typedef struct {
    int node, nodes_x, nodes_y, node_x, node_y;
    int size_x, size_y;     /* interior cells of the node (c_sizeX, c_sizeY) */
    double init_x, init_y;  /* c_initX, c_initY: least x, y of its interior */
} cl_node;
/* Fails with CL_ERR_ARG as main.cpp:160-169 aborts: more partitions than
 * cells, or num_nodes != nodes_x * nodes_y. */
int cl_partition(int num_cells_x, int num_cells_y, int nodes_x, int nodes_y, int num_nodes, int node,
                 double ax, double ay, double bx, double by, cl_node *out);
/* The solver of one node of the deck's NUM_MPI_PARTITIONS_X x _Y partition
 * (num_nodes processes, this one `node`): its block, initial condition and
 * output files out_<t>_<node>.{pn,opt} as the reference's MPI build writes
 * them.  A node steps with cl_solver_stage after filling its halo. */
int cl_solver_create_node(const char *deck_path, const char *out_dir, int node, int num_nodes,
                          cl_solver **out, double *max_dt);
int cl_solver_node(const cl_solver *s, cl_node *out);
/* One RK stage (1 or 2) of the solver with its dx, dy, without the ghost
 * copy (cl_stage / cl_pn_stage); asynchronous on the solver's stream. */
int cl_solver_stage(cl_solver *s, int stage, double dt);
/* The halo of the solver's node (cl_halo_* / cl_pn_halo_*), the stream its
 * device work runs on, a wait for that work, and the sides whose ghost strips
 * the exchange fills (the linear solver filters them like the interior). */
int cl_solver_halo_counts(cl_solver *s, long long counts[4]);
int cl_solver_halo_pack(cl_solver *s, double *const bufs[4]);
int cl_solver_halo_unpack(cl_solver *s, double *const bufs[4]);
int cl_solver_stream(cl_solver *s, void **stream);
int cl_solver_sync(cl_solver *s);
int cl_solver_set_exchanged_sides(cl_solver *s, int mask);

/* main.cpp:204-230: outputs at t = 0 and every OUT_DELTA_T up to T_FINAL;
 * max_steps >= 0 stops after that many RK2 steps. */
int cl_run_deck(const char *deck_path, const char *out_dir, int max_steps);

/* Batched opt() that allocates no device memory -- this entry point has no
 * counterpart in the reference.  For callers whose device memory is owned by
 * an external allocator or pre-reserved pool and who therefore may not call
 * cudaMalloc/cudaFree (both synchronise the device and fragment the pool):
 * the caller passes device arrays d_u, d_alpha ([count*n], solved in place)
 * and optional d_iters, d_reg, d_status ([count]); the work counter, error
 * word, statistics and the angular set-up (uploaded from `ang` each call)
 * live in one fixed 4 MiB device array that every GPU loading the library
 * holds until exit.  Configurations whose padded basis does not fit are
 * rejected with CL_ERR_ARG (message from cl_noalloc_last_error()); M6 at
 * Q = 40 with the Gaunt table fits.  The first call on a device looks up the
 * array's device address, and the first call of each moment order and
 * Gaunt/no-Gaunt combination loads that kernel instance; with CUDA's lazy
 * module loading that load is where the array and the kernel image are
 * placed in device memory, and it may synchronise the device.  So make one
 * warm-up call per configuration at set-up, before any stream capture; later
 * calls of that configuration allocate nothing.
 * All calls share the array, so calls that overlap on the GPU (several
 * streams or threads at once) race; the call waits for its own work on
 * `stream` (a cudaStream_t, null = legacy default stream) before returning.
 * It contracts one quadrature direction at a time (the CL_CONTRACT_SINGLE
 * sums) whatever opts->contraction holds. */
int cl_solve_batch_noalloc(const cl_angular *ang, const cl_options *opts, int count,
                           double *d_u, double *d_alpha, int *d_iters, double *d_reg,
                           int *d_status, void *stream);
const char *cl_noalloc_last_error(void);

/* ------------------------------------------------------------------------
 * Learned warm start (no counterpart in the reference, which starts every
 * solve from the previous stage's alpha, momopt_update.cpp:236-238).  An MLP
 * n -> width -> width -> width -> n (GELU, BF16 weights and activations,
 * FP32 accumulation on the tensor cores, FP32 Adam) maps u/u0 to the
 * multipliers of the scaled problem; Newton then runs from the prediction to
 * the same tolerance, so the network changes iteration counts only.
 * W_l is [in x out] row-major (y = x W + b); four layers. */
typedef struct cl_mlp cl_mlp;
int cl_mlp_create(int n, int width, int moment_type, double delta_ppn, unsigned long long seed, cl_mlp **out);
void cl_mlp_destroy(cl_mlp *m);
const char *cl_mlp_last_error(const cl_mlp *m);
/* Per-component standardisation of the targets: y = (alpha_scaled - mean) / std. */
int cl_mlp_set_output_scaling(cl_mlp *m, const float *mean, const float *stdv);
/* Adam (lr, betas 0.9/0.999) on device pairs (u, alpha) [count x n] FP64,
 * shuffled minibatches; losses[steps] nullable. */
int cl_mlp_train(cl_mlp *m, const double *d_u, const double *d_alpha, int count, int steps, int batch, float lr,
                 unsigned long long seed, float *losses);
/* alpha <- prediction for device u [count x n]; where it is not finite the
 * given alpha is kept (fallback_kind 0, e.g. the previous stage's) or the
 * isotropic multiplier is taken (fallback_kind 1).  *fallbacks nullable;
 * stream null = the network's own stream. */
int cl_mlp_predict(cl_mlp *m, const double *d_u, double *d_alpha, int count, int fallback_kind, int *fallbacks,
                   void *stream);
/* Predictions only for the vectors whose last solve took at least min_iters
 * iterations (d_iters [count], device); the others get a NaN start (the
 * Newton kernel then starts them from their own multipliers).  The selection
 * stays on the device (no host synchronisation). */
int cl_mlp_predict_selected(cl_mlp *m, const double *d_u, const int *d_iters, int min_iters, double *d_alpha,
                            int count, void *stream);
/* The network's GEMM alone: C [M x N] FP32 = A [M x K] . B [N x K]^T with BF16
 * A and B (device, row-major, K a multiple of 8), on the tensor-memory path
 * (tcgen05.mma kind::f16 with TMA-staged operands) the forward pass uses.
 * Waits for the result. */
int cl_tc_gemm_bf16(const void *d_A, const void *d_B, int M, int N, int K, float *d_C);
/* Loss and gradients of one host batch (gradient checks). */
int cl_mlp_loss_and_grads(cl_mlp *m, const double *u, const double *alpha, int rows, float *loss,
                          float *const *gW, float *const *gb);
int cl_mlp_get_params(cl_mlp *m, float *const *W, float *const *b);
int cl_mlp_set_params(cl_mlp *m, float *const *W, float *const *b);
/* Grid warm start: before each optimisation stage cl_step predicts alpha for
 * every cell from its moments (fallback: the previous stage's alpha).  Pass
 * NULL to return to the reference's plain warm start.  The network must
 * outlive its use by the context. */
int cl_set_warm_start(cl_ctx *ctx, cl_mlp *m);
/* Same, predicting only for the cells whose previous optimisation stage took
 * at least min_prev_iters iterations (the cells the previous-stage start
 * served worst); every other cell keeps the reference's previous-stage
 * start.  min_prev_iters 0 predicts every cell, as cl_set_warm_start. */
int cl_set_warm_start_selective(cl_ctx *ctx, cl_mlp *m, int min_prev_iters);

/* Kernel launches issued by the library since load (for the bench). */
int64_t cl_launch_count(void);
/* Device pointers of the context's state (ghosts included) for callers that
 * keep data resident. */
int cl_device_state(cl_ctx *ctx, double **d_moments, double **d_alpha);
/* Measures the FP64 tensor-core (DMMA m16n8k8) throughput of the current
 * device in TFLOP/s: the roofline denominator of the FP64-bound kernels. */
int cl_fp64_peak(double *tflops);
/* Evaluates the kernels' table-driven exp and the CUDA library exp on the
 * device for n host points (accuracy check of the former against the latter). */
int cl_exp_check(const double *x, int n, double *fast, double *ref);
/* Runs the library's DMMA fragment-layout self check on the device; returns
 * CL_OK when the FP64 tensor-core GEMM matches a host GEMM. */
int cl_selftest(void);

#ifdef __cplusplus
}
#endif
#endif
