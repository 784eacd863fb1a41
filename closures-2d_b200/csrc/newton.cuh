// newton.cuh -- host interface of the persistent dual-Newton kernel (K1).
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"
#include "fexp.cuh"

namespace clb {

// One moment order ("problem") of a launch.  Basis rows are padded to
// nqp = multiple of the q-chunk, columns laid out as
//   [0, nb)              basis p_k, k < n (zero for n <= k < nb)
//   [nb, nb + K2p)       Hessian columns: extended basis (Gaunt) or the
//                        products p_i p_j, j <= i, at column i(i+1)/2 + j
// with row q at basis_row(q, ldP) = q * ldP + 4 * (q / 4): ldP % 16 == 4
// doubles and a gap of 4 doubles after every 4 rows make both MMA fragment
// patterns bank-conflict free, and a chunk of rows is one contiguous block
// (copied to shared memory as is).  The gap after rows 4k..4k+3 holds their
// quadrature weights w[4k..4k+3] (basis_wgap), so a staged chunk carries its
// weights.  The array holds nqp * ldP + nqp doubles.
__host__ __device__ __forceinline__ int basis_row(int q, int ldP) { return q * ldP + 4 * (q >> 2); }
__host__ __device__ __forceinline__ int basis_wgap(int q, int ldP)
{
    return ((q >> 2) * 4 + 4) * ldP + 4 * (q >> 2) + (q & 3);
}

struct NewtonProblem {
    const double *P;
    const double *w;            // [nqp], zero on padded rows
    const int *hoff;            // Gaunt CSR (row j*n+i for j <= i); null without Gaunt
    const int *hidx;
    const double *hval;
    const unsigned short *pairs;  // n(n+1)/2 entries (i << 8) | j, j <= i, column order
    // Gaunt contraction in lane-major chunks (build_gaunt_ell), staged in
    // shared memory when the CTA starts on this problem
    const unsigned short *ellPair, *ellIdx;
    const double *ellVal;
    const int *ellOff;
    int ellChunks, ellRows;
    double p0;                  // p[0] = Y_00 (fobj.cpp:305 divides by it)
    // Converged-evaluation test without the Hessian (Mn, FP64): row 0 of the
    // Gaunt contraction (CSR rows (0, j), j < n, G columns in the layout's
    // order; null without Gaunt), bounds gramLo <= lambda <= gramHi of the
    // quadrature Gram matrix sum_q w_q p(q) p(q)^T of the moment basis
    // (gramLo = 0: the test is off), rangeC[k] = max_q |p_k(q)| (k < n) and
    // rangeC[n + l] = max_q ||(p_k(q))_{deg k = l}|| (l <= maxDeg)
    const int *row0Off;
    const unsigned short *row0Idx;
    const double *row0Val;
    const double *rangeC;
    double gramLo, gramHi;
    int maxDeg;
    int n, nb, K2p, nqp, ldP;
    // direction pairs: the basis stores one direction of each (phi, phi + pi)
    // pair with its columns grouped by degree parity (nbe even basis columns,
    // K2e even Hessian columns, each group padded to 8); binv[j] is the moment
    // of basis column j (-1 padding), pcol[c] the G column of product c
    int paired, nbe, K2e;
    const short *binv;
    const int *pcol;
    int count;                  // vectors to solve
    double *u, *alpha;          // [count][n]; alpha: start (or fallback start) in, solution out
    const double *alphaStart;   // nullable [count][n]: predicted start; alpha is then the
                                // fallback taken (once) before the first regularisation
    // change-of-basis Newton (MOMOPT_OPTIMIZATION_TYPE 1): per-vector basis
    // P2M [count][n][n] (row-major lower triangular) and alphaP [count][n],
    // read at the start and written back on convergence; null otherwise
    double *P2M, *alphaP;
    int *iters;                 // nullable [count]
    double *regs;               // nullable [count]
    int *status;                // nullable [count]
    unsigned int *queue;        // work counter, zero before the launch
    int first;                  // index of the first work item: the launch solves
                                // items first .. first + count - 1 (a band of cells)
    // K1 over a list: the cells to solve are cellList[0 .. *countDev), or
    // cells first .. first + count - 1 when cellList is null or *countDev is
    // negative.  The screening pass appends the cells it leaves at
    // pendList[atomicAdd(pendCount, 1)]; it runs only when *gateCount (cells
    // of the launch whose previous solve took at most one iteration, from
    // `iters`) is at least gateMin, and evaluates only such cells.
    const int *cellList;
    const int *countDev;
    int *pendList;
    int *pendCount;
    const int *gateCount;
    int gateMin;
};

// Cells of [first, first + count) whose previous solve took at most one
// iteration (iters[c] <= 1), added to *out (zero before the launch).
cudaError_t launch_screen_gate(const int *iters, int first, int count, int *out, cudaStream_t stream);
// K1's list, most previous iterations first (iters[c], a counting sort in
// one CTA), so that K1 starts the longest Newton chains first and the short
// ones fill in behind them: the *listCount cells of `list` when the
// screening gate is open (list non-null and *gateCount >= gateMin); else the
// cells first .. first + count - 1 when count <= wholeMax, or *outCount = -1
// (K1 takes the range in cell order); written to out[0 .. *outCount).
cudaError_t launch_order_cells(const int *list, const int *listCount, int first, int count, const int *gateCount,
                               int gateMin, int wholeMax, const int *iters, int *out, int *outCount,
                               cudaStream_t stream);

// Per-slot state in shared memory: slot states, doubles (SC_*) and ints (SI_*).
// S_HELP: an idle slot lent, for one round, to a slot whose line search is
// backtracking (plain Newton, work counter exhausted): it evaluates one of the
// parent's next trial points (SI_CELL = parent slot, SI_ITER = k, the trial
// t / 2^k), so that up to T - 1 halvings of linesearch.cpp:53-81 take one
// round instead of one round each.
enum SlotState { S_IDLE = 0, S_NEW = 1, S_NEWTON = 2, S_TRIAL = 3, S_HELP = 4 };
enum { SC_T = 0, SC_FREF, SC_GD, SC_MAXF, SC_RTOL, SC_U0, SC_ASCALE, SC_DELTA, SC_R, SC_N };
enum { SI_CELL = 0, SI_STATE, SI_ITER, SI_TOTAL, SI_REG, SI_MAXITER, SI_PRED, SI_CB, SI_BFGS, SI_N };

struct NewtonArgs {
    NewtonProblem prob[kMaxProblems];
    int nprob;
    int momentType, maxIter, useGaunt;
    double tolRel, condHMax, deltaPPn, tolGamma;
    // grid mode: copy interior moments to momentsOld before solving them
    // (momopt_update.cpp:298-308); null otherwise
    double *momentsOld;
    int NX, NY;
    DevStats *stats;
    int *err;                   // [0] first error code, [1] its vector index
    // launch layout (doubles unless noted), filled by plan_newton()
    int T, kq, ldv, ldE, ldG, ldh, ntq, doubleBuffer;
    int offAlpha, offAold, offD, offU, offScal, offInt, offFpart, offStat;
    int offP, offE, offEg, offG, offH, offVec;
    int offEllVal, offEllIdx, offEllPair, offEllOff, offExp, offBar;
    ExpConsts ex;               // table-driven exp constants (staged in shared memory)
    int smemBytes;
    int tpw;                    // column tiles per warp (general contractions)
    int ntf;                    // > 0: fused contractions with this many tiles per warp
    int ntExact, nbk;           // single problem on the fused path: its column tiles and
                                // GEMM1 k-steps (selects a specialised instance), else 0
    int mixed;                  // Hessian-only tiles by split TF32 (CL_MIXED); needs ntExact
    int optType;                // 0 Newton (opt.cpp), 1 change of basis (optcb.cpp),
                                // 2 BFGS sub-iterations in the change of basis (optbfgs.cpp)
    int maxBfgsIter;            // optType 2: MOMOPT_MAX_BFGS_ITER
    double condHMaxBfgs;        // optType 2: MOMOPT_COND_H_MAX_BFGS
    int cbStride;               // doubles per slot of cbScratch (kCbSlotDoubles or kBfgsSlotDoubles)
    double *cbScratch;          // optType 1, 2: per-slot working state, [grid][T][cbStride]
    // launch shape, set before plan_newton(): warps per CTA (0 or 8: 32
    // slots, three staged chunks, one CTA per SM; 4: 16 slots, two staged
    // chunks, the Gaunt table read through L1, two CTAs per SM -- fused
    // direction-pair instances only)
    int nw;
    int stageEll;               // filled by plan_newton(): Gaunt table staged in shared memory
};

// Fills the layout fields from the problems' sizes; returns 0, -1 when the
// configuration does not fit in shared memory, -2 when mixed precision is
// asked for a configuration without a specialised instance.
int plan_newton(NewtonArgs &a);
// Sets the kernel's shared-memory attribute (call once, outside capture).
cudaError_t prepare_newton(const NewtonArgs &a);
// A fused instance exists for the direction-pair layout with these counts.
bool newton_pair_supported(int nt, int nbk);
// ... and in the 4-warp launch shape.
bool newton_pair4_supported(int nt, int nbk);
// Screening pass (Mn, FP64, direction pairs; a.prob[0] the gradient-column
// layout of the problem): layout, instance check, shared-memory attribute,
// launch and resident CTAs per SM.
int plan_screen(NewtonArgs &a);
bool screen_supported(int nt, int nbk);
cudaError_t prepare_screen(const NewtonArgs &a);
cudaError_t launch_screen(const NewtonArgs &a, int grid, cudaStream_t stream);
int screen_ctas_per_sm(const NewtonArgs &a);
// Launches the persistent kernel on `stream` over `grid` CTAs.
cudaError_t launch_newton(const NewtonArgs &a, int grid, cudaStream_t stream);
int newton_ctas_per_sm(const NewtonArgs &a);

// Kernel instances, grouped by translation unit.  Each returns true when it
// holds the instance `a` selects and then sets *err to the result of
// running it (mode 0 launch, 1 shared-memory attribute, 2 occupancy).
bool newton_run_generic(const NewtonArgs &a, int grid, cudaStream_t s, int mode, int *occ, cudaError_t *err);
bool newton_run_exact_mn_a(const NewtonArgs &a, int grid, cudaStream_t s, int mode, int *occ, cudaError_t *err);
bool newton_run_exact_pair(const NewtonArgs &a, int grid, cudaStream_t s, int mode, int *occ, cudaError_t *err);
bool newton_run_exact_pair4(const NewtonArgs &a, int grid, cudaStream_t s, int mode, int *occ, cudaError_t *err);
bool newton_run_exact_mn_b(const NewtonArgs &a, int grid, cudaStream_t s, int mode, int *occ, cudaError_t *err);
bool newton_run_exact_ppn_a(const NewtonArgs &a, int grid, cudaStream_t s, int mode, int *occ, cudaError_t *err);
bool newton_run_exact_ppn_b(const NewtonArgs &a, int grid, cudaStream_t s, int mode, int *occ, cudaError_t *err);
bool newton_run_mixed_mn(const NewtonArgs &a, int grid, cudaStream_t s, int mode, int *occ, cudaError_t *err);
bool newton_run_mixed_ppn(const NewtonArgs &a, int grid, cudaStream_t s, int mode, int *occ, cudaError_t *err);

}  // namespace clb
