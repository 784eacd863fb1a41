// newton_kernel.cuh -- persistent dual-Newton kernel for the Mn / PPn entropy
// closure (device code; instantiated by the newton_inst_*.cu units).
//
// One launch solves, for every vector u of every problem, the dual problem of
// opt() (src/momopt/opt/opt.cpp:82-343): minimise <eta*(alpha.m)> - alpha.u by
// Newton's method with the Armijo backtracking line search of
// linesearch.cpp:21-99 and the isotropic-restart regularisation ladder
// r in {0, 1e-3, 1e-2, 1e-1, 0.5} (opt.h:39-40, opt.cpp:244-274).
//
// B200 mapping.  A CTA owns T "slots" (cells in flight).  Each round every
// slot needs one evaluation of f, g and H at its current alpha; the rounds are
// batched contractions over the quadrature on the FP64 tensor cores (DMMA
// m16n8k8):
//   S[T x kq]  = alpha[T x nb] . P[kq x nb]^T            (alpha.m per q)
//   E          = w * exp(S)          (Mn)   or the PPn weights
//   G[T x K]  += E[T x kq] . Phess[kq x K]               (Hessian columns)
// with the basis streamed through shared memory in q-chunks by cp.async.
// Then one warp per slot finishes the Newton logic in FP64: H from G (the
// Gaunt contraction of fobj.cpp:130-144 or the packed products), Cholesky,
// Hager/Higham 1-norm condition estimate (the quantity dpocon returns),
// direction, stopping test, line-search bookkeeping and the ladder.
// Converged slots write u, alpha back and are refilled from a global work
// counter, so vectors needing 1 or 40 iterations share the launch.
//
// Every line-search trial evaluation also carries H: when the trial is
// accepted (the usual case) it is reused as the next Newton iteration's
// evaluation, which the reference recomputes at the same alpha.
#pragma once
#include "newton.cuh"

#include <cfloat>
#include <cmath>

namespace clb {

namespace {


constexpr double kSqrtPi = 1.7724538509055160273;
constexpr double kPi = 3.14159265358979323846;

struct Ctx {
    double *sm;
    int lane, warp, g, t4;
};

__device__ __forceinline__ void record_error(int *err, int code, int idx)
{
    if (atomicCAS(&err[0], 0, code) == 0)
        err[1] = idx;
}

// Cholesky of the symmetric matrix whose row `lane` is h[] (registers), in
// the dot-product (Crout) form by columns: lane i >= j forms
// L_ij = (H_ij - sum_k<j L_ik L_jk) / L_jj.  Row j of L is read back from the
// warp's shared-memory matrix Ls (stride ldl, even) with 16-byte broadcast
// loads: lane i writes L_ij there at step j, and 1/L_jj on the diagonal.
// On return h[k] = L_lane,k for k <= lane.  LAPACK-style info: 0, or j+1 at
// the first non-positive or NaN pivot (dpotrf semantics).
__device__ __forceinline__ int chol_regs(double (&h)[kMaxN], double *Ls, int ldl, int n, int lane)
{
#pragma unroll
    for (int j = 0; j < kMaxN; j++) {
        if (j < n) {
            const double *Lj = Ls + j * ldl;
            double s0 = h[j], s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll
            for (int k = 0; k + 1 < j; k += 2) {
                const double2 l = *reinterpret_cast<const double2 *>(Lj + k);
                if (k & 2) {
                    s2 = fma(-h[k], l.x, s2);
                    s3 = fma(-h[k + 1], l.y, s3);
                } else {
                    s0 = fma(-h[k], l.x, s0);
                    s1 = fma(-h[k + 1], l.y, s1);
                }
            }
            if (j & 1)
                s1 = fma(-h[j - 1], Lj[j - 1], s1);
            const double s = (s0 + s1) + (s2 + s3);
            const double djj = __shfl_sync(0xffffffffu, s, j);
            if (!(djj > 0.0))
                return j + 1;
            const double r = rsqrt(djj);
            if (lane == j) {
                h[j] = djj * r;
                Ls[j * ldl + j] = r;
            } else if (lane > j && lane < n) {
                h[j] = s * r;
                Ls[lane * ldl + j] = h[j];
            }
            __syncwarp();
        }
    }
    return 0;
}

// Column `lane` of L^-1 into v[]: Linv_ic = -(sum_{k=c}^{i-1} L_ik Linv_kc) / L_ii,
// rows in order, row i of L and 1/L_ii read from Ls as left by chol_regs.
__device__ __forceinline__ void invert_regs(const double *Ls, int ldl, double (&v)[kMaxN], int n, int lane)
{
#pragma unroll
    for (int i = 0; i < kMaxN; i++) {
        v[i] = 0.0;
        if (i < n) {
            const double *Li = Ls + i * ldl;
            double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
#pragma unroll
            for (int k = 0; k + 1 < i; k += 2) {
                const double2 l = *reinterpret_cast<const double2 *>(Li + k);
                if (k & 2) {
                    a2 = fma(l.x, v[k], a2);
                    a3 = fma(l.y, v[k + 1], a3);
                } else {
                    a0 = fma(l.x, v[k], a0);
                    a1 = fma(l.y, v[k + 1], a1);
                }
            }
            if (i & 1)
                a1 = fma(Li[i - 1], v[i - 1], a1);
            const double rinv = Li[i];
            if (lane == i)
                v[i] = rinv;
            else if (lane < i)
                v[i] = -((a0 + a1) + (a2 + a3)) * rinv;
        }
    }
}

// Rigorous upper bound of ||L^-1||_inf ||L^-1||_1 from the comparison matrix
// M(L) (|L_ii| on the diagonal, -|L_ik| below): |L^-1| <= M(L)^-1 entrywise,
// so ||L^-1||_inf <= ||M(L)^-1 e||_inf and ||L^-1||_1 <= ||M(L)^-T e||_inf.
// The two substitutions (nonnegative terms only) run interleaved; factor rows
// come from h[] (lane i: L_ik) and Ls (1/L_kk on the diagonal, as left by
// chol_regs).  Used where it is tight: Hessians of smooth cells.
__device__ __forceinline__ double cmp_bound(const double (&h)[kMaxN], const double *Ls, int ldl, int n, int lane)
{
    const double rl = (lane < n) ? Ls[lane * ldl + lane] : 0.0;
    double accF = 0.0, accB = 0.0;
#pragma unroll
    for (int s = 0; s < kMaxN; s++) {
        if (s < n) {
            const int kf = s, kb = n - 1 - s;
            const double xf = __shfl_sync(0xffffffffu, (1.0 + accF) * rl, kf);
            const double xb = __shfl_sync(0xffffffffu, (1.0 + accB) * rl, kb);
            if (lane > kf)   // h[k] holds L_lane,k only for k <= lane
                accF = fma(fabs(h[s]), xf, accF);
            if (lane < kb)
                accB = fma(fabs(Ls[kb * ldl + lane]), xb, accB);
        }
    }
    const double x = (lane < n) ? (1.0 + accF) * rl : 0.0, y = (lane < n) ? (1.0 + accB) * rl : 0.0;
    return warp_max(x) * warp_max(y);
}

// z = (L L^T)^-1 x with Linv in Hs; x, z held one element per lane.
__device__ double apply_inv(const double *Hs, int n, int ldh, double *vec, double x, int lane)
{
    __syncwarp();
    vec[lane] = x;
    __syncwarp();
    double y = 0.0;
    if (lane < n)
        for (int k = 0; k <= lane; k++)
            y = fma(Hs[lane * ldh + k], vec[k], y);
    __syncwarp();
    vec[lane] = y;
    __syncwarp();
    double z = 0.0;
    if (lane < n)
        for (int k = lane; k < n; k++)
            z = fma(Hs[k * ldh + lane], vec[k], z);
    return z;
}

__device__ __forceinline__ double sgn1(double x) { return x >= 0.0 ? 1.0 : -1.0; }

// Estimate of ||A^-1||_1 for A = L L^T (Higham 1988, Alg. 4.1, the estimator
// behind LAPACK dlacn2/dpocon); returns rcond = (1/est)/anorm.
__device__ double rcond_warp(const double *Hs, int n, int ldh, double *vec, double anorm, int lane)
{
    const bool act = lane < n;
    if (anorm == 0.0)
        return 0.0;
    double x = act ? 1.0 / n : 0.0;
    x = apply_inv(Hs, n, ldh, vec, x, lane);
    double est;
    if (n == 1) {
        est = fabs(__shfl_sync(0xffffffffu, x, 0));
    } else {
        est = warp_sum(act ? fabs(x) : 0.0);
        double isgn = act ? sgn1(x) : 0.0;
        x = apply_inv(Hs, n, ldh, vec, isgn, lane);
        int j = warp_argmax_first(act ? fabs(x) : -1.0, lane);
        int iter = 2;
        for (;;) {
            x = (lane == j) ? 1.0 : 0.0;
            x = apply_inv(Hs, n, ldh, vec, x, lane);
            double estold = est;
            est = warp_sum(act ? fabs(x) : 0.0);
            bool same = __all_sync(0xffffffffu, !act || sgn1(x) == isgn);
            if (same || est <= estold)
                break;
            isgn = act ? sgn1(x) : 0.0;
            x = apply_inv(Hs, n, ldh, vec, isgn, lane);
            int jlast = j;
            j = warp_argmax_first(act ? fabs(x) : -1.0, lane);
            double xjlast = __shfl_sync(0xffffffffu, x, jlast);
            double xj = __shfl_sync(0xffffffffu, x, j);
            if (xjlast != fabs(xj) && iter < 5) {
                iter++;
                continue;
            }
            break;
        }
        double alt = act ? ((lane & 1) ? -1.0 : 1.0) * (1.0 + (double)lane / (double)(n - 1)) : 0.0;
        alt = apply_inv(Hs, n, ldh, vec, alt, lane);
        double temp = 2.0 * (warp_sum(act ? fabs(alt) : 0.0) / (3.0 * n));
        if (temp > est)
            est = temp;
    }
    if (est != 0.0)
        return (1.0 / est) / anorm;
    return 0.0;
}

struct Layout {
    double *alpha, *aold, *d, *u, *scal, *fpart, *P, *E, *Eg, *G, *H, *vec;
    int *ints;
    unsigned long long *stat;
    double *ellVal;
    unsigned short *ellIdx, *ellPair;
    int *ellOff;
    double *exptab;
    unsigned long long *bar;   // three mbarriers of the staged basis chunks
};

__device__ __forceinline__ Layout make_layout(double *sm, const NewtonArgs &a)
{
    Layout L;
    L.alpha = sm + a.offAlpha;
    L.aold = sm + a.offAold;
    L.d = sm + a.offD;
    L.u = sm + a.offU;
    L.scal = sm + a.offScal;
    L.ints = (int *)(sm + a.offInt);
    L.fpart = sm + a.offFpart;
    L.stat = (unsigned long long *)(sm + a.offStat);
    L.P = sm + a.offP;
    L.E = sm + a.offE;
    L.Eg = sm + a.offEg;
    L.G = sm + a.offG;
    L.H = sm + a.offH;
    L.vec = sm + a.offVec;
    L.ellVal = sm + a.offEllVal;
    L.ellIdx = (unsigned short *)(sm + a.offEllIdx);
    L.ellPair = (unsigned short *)(sm + a.offEllPair);
    L.ellOff = (int *)(sm + a.offEllOff);
    L.exptab = sm + a.offExp;
    L.bar = (unsigned long long *)(sm + a.offBar);
    return L;
}

// Writes the finished slot's results (scaled back) and updates CTA stats.
__device__ void finish_slot(const NewtonArgs &a, const NewtonProblem &pb, Layout &L, int s,
                            double ui, double ai, int status, int lane)
{
    int cell = L.ints[s * SI_N + SI_CELL];
    int n = pb.n;
    if (lane < n) {
        pb.u[(size_t)cell * n + lane] = ui;
        pb.alpha[(size_t)cell * n + lane] = ai;
    }
    if (lane == 0) {
        int total = L.ints[s * SI_N + SI_TOTAL];
        int reg = L.ints[s * SI_N + SI_REG];
        if (pb.iters)
            pb.iters[cell] = total;
        if (pb.regs)
            pb.regs[cell] = kRegularizations[reg];
        if (pb.status)
            pb.status[cell] = status;
        if (status == 0) {
            atomicAdd(&L.stat[reg], 1ull);
            atomicAdd(&L.stat[kNumReg], (unsigned long long)total);
            atomicAdd(&L.stat[kNumReg + 1], 1ull);
            atomicMax((int *)&L.stat[kStatU64], total);
        } else {
            record_error(a.err, status, cell);
        }
        L.ints[s * SI_N + SI_STATE] = S_IDLE;
    }
}

// Loads and scales a newly assigned vector (opt.cpp:82-148 entry half).
__device__ void init_slot(const NewtonArgs &a, const NewtonProblem &pb, Layout &L, int s, int lane,
                          int ldv)
{
    const int n = pb.n;
    const int cell = L.ints[s * SI_N + SI_CELL];
    double ui = 0.0, ai = 0.0;
    int pred = 0;
    if (lane < n) {
        ui = pb.u[(size_t)cell * n + lane];
        ai = pb.alpha[(size_t)cell * n + lane];
    }
    if (pb.alphaStart != nullptr) {
        double ap = (lane < n) ? pb.alphaStart[(size_t)cell * n + lane] : 0.0;
        if (__all_sync(0xffffffffu, isfinite(ap))) {
            ai = ap;
            pred = 1;
        }
    }
    if (a.momentsOld != nullptr && lane < n) {
        int i = cell / a.NY, j = cell % a.NY;
        if (i >= 2 && i < a.NX - 2 && j >= 2 && j < a.NY - 2)
            a.momentsOld[(size_t)cell * n + lane] = ui;
    }
    const double u0 = __shfl_sync(0xffffffffu, ui, 0);
    if (!(u0 > 0.0)) {
        // opt.cpp:97-101 aborts; leave the vector untouched and report.
        if (lane == 0) {
            L.ints[s * SI_N + SI_TOTAL] = 0;
            L.ints[s * SI_N + SI_REG] = 0;
        }
        __syncwarp();
        finish_slot(a, pb, L, s, ui, ai, -3, lane);
        return;
    }
    double *sc = L.scal + s * SC_N;
    double delta = a.deltaPPn;
    if (a.momentType == 0) {
        double ascale = log(u0) * 2.0 * kSqrtPi;
        if (lane == 0)
            ai = ai - ascale;
        ui = ui / u0;
        if (lane == 0)
            sc[SC_ASCALE] = ascale;
    } else {
        ai = ai / u0;
        ui = ui / u0;
        delta = delta / (u0 * u0);
    }
    if (lane < ldv) {
        L.u[s * ldv + lane] = (lane < n) ? ui : 0.0;
        L.alpha[s * ldv + lane] = (lane < n) ? ai : 0.0;
    }
    double rtol = sqrt(warp_sum(ui * ui)) * a.tolRel;
    if (lane == 0) {
        sc[SC_T] = 1.0;
        sc[SC_RTOL] = rtol;
        sc[SC_U0] = u0;
        sc[SC_DELTA] = delta;
        int *si = L.ints + s * SI_N;
        si[SI_ITER] = 0;
        si[SI_TOTAL] = 0;
        si[SI_REG] = 0;
        si[SI_MAXITER] = a.maxIter;
        si[SI_PRED] = pred;
        si[SI_STATE] = S_NEWTON;
    }
}

// Isotropic restart with the next regularisation (opt.cpp:244-274).
__device__ void regularize(const NewtonArgs &a, const NewtonProblem &pb, Layout &L, int s, int lane,
                           int ldv, double ui, double ai)
{
    const int n = pb.n;
    int *si = L.ints + s * SI_N;
    double *sc = L.scal + s * SC_N;
    int reg = si[SI_REG];
    if (si[SI_PRED] == 1) {
        // The predicted start failed (the solve would regularise): restart
        // once from the fallback start with the same u, as plain Newton.
        const int cell = si[SI_CELL];
        double af = (lane < n) ? pb.alpha[(size_t)cell * n + lane] : 0.0;
        const double u0 = sc[SC_U0];
        if (a.momentType == 0) {
            if (lane == 0)
                af = af - sc[SC_ASCALE];
        } else {
            af = af / u0;
        }
        if (lane < n)
            L.alpha[s * ldv + lane] = af;
        __syncwarp();
        if (lane == 0) {
            si[SI_PRED] = 2;
            si[SI_ITER] = 0;
            sc[SC_T] = 1.0;
            si[SI_STATE] = S_NEWTON;
            atomicAdd(&L.stat[kNumReg + 3], 1ull);
        }
        return;
    }
    if (reg >= kNumReg - 1) {
        // opt.cpp:256-261 aborts; report and return the unscaled state.
        double u0 = sc[SC_U0];
        if (a.momentType == 0) {
            ui *= u0;
            if (lane == 0)
                ai += sc[SC_ASCALE];
        } else {
            ui *= u0;
            ai *= u0;
        }
        __syncwarp();
        finish_slot(a, pb, L, s, ui, ai, -4, lane);
        return;
    }
    reg++;
    const double r = kRegularizations[reg];
    const int cell = si[SI_CELL];
    const double u0 = sc[SC_U0];
    double unew = 0.0;
    if (lane < n) {
        double uorig = pb.u[(size_t)cell * n + lane] / u0;   // scaled original (unchanged in memory)
        unew = (lane == 0) ? 1.0 : uorig * (1.0 - r);
        L.u[s * ldv + lane] = unew;
        double a0 = (a.momentType == 0) ? 2.0 * kSqrtPi * log(0.5 / kSqrtPi)
                                        : 1.0 - 4.0 * sc[SC_DELTA] * kPi;
        L.alpha[s * ldv + lane] = (lane == 0) ? a0 : 0.0;
    }
    double rtol = sqrt(warp_sum(unew * unew)) * a.tolRel;
    __syncwarp();
    if (lane == 0) {
        si[SI_REG] = reg;
        si[SI_ITER] = 0;
        sc[SC_T] = 1.0;
        sc[SC_RTOL] = rtol;
        if (reg == kNumReg - 1)
            si[SI_MAXITER] = 10 * si[SI_MAXITER];
        si[SI_STATE] = S_NEWTON;
    }
}

__device__ double modcfl(double di, int n, int lane, int momentType)
{
    double da1 = warp_sum(lane < n ? fabs(di) : 0.0);
    int pnOrder = (int)floor(sqrt((double)n)) + 1;
    double minf = sqrt((2 * pnOrder + 1) / (2 * kPi));
    return momentType == 0 ? exp(2.0 * da1 * minf) : 1.0 + 2.0 * da1 * minf;
}

// Converged (opt.cpp:293-306): Mn write-back of the realised moments, then
// opt()'s rescaling (:107-109, :133-138), and the slot is finished.
__device__ void converge(const NewtonArgs &a, const NewtonProblem &pb, Layout &L, int s, double ui, double ai,
                         double gi, int lane)
{
    const double *sc = L.scal + s * SC_N;
    double uo = ui, ao = ai;
    const double u0 = sc[SC_U0];
    if (a.momentType == 0) {
        double u0w = __shfl_sync(0xffffffffu, ui + gi, 0);
        uo = (ui + gi) / u0w;
        if (lane == 0)
            ao = ai - log(u0w) * 2.0 * kSqrtPi;
        uo = uo * u0;
        if (lane == 0)
            ao = ao + sc[SC_ASCALE];
    } else {
        ao = ai * u0;
        uo = ui * u0;
    }
    __syncwarp();
    finish_slot(a, pb, L, s, uo, ao, 0, lane);
}

// The slot's symmetric H (row stride ldh) from its contraction results Gs:
// the Gaunt sums H_ij = sum_k c_ijk G_k from the ELL table in shared memory
// (fobj.cpp:129-155), or the packed products p_i p_j (fobj.cpp:37-129).
__device__ __forceinline__ void hessian_from_contractions(const NewtonArgs &a, const NewtonProblem &pb,
                                                         const Layout &L, const double *Gs, double *Hs,
                                                         int lane)
{
    const int n = pb.n, ldh = a.ldh;
    const int npairs = n * (n + 1) / 2;
    if (a.useGaunt) {
        for (int c = 0; c < pb.ellChunks; c++) {
            const unsigned short pr = L.ellPair[c * 32 + lane];
            const int e1 = L.ellOff[c + 1];
            int e = L.ellOff[c];
            double v = 0.0;
            // loads of four entries issued ahead of their (in-order) sum
            for (; e + 4 <= e1; e += 4) {
                const int i0 = L.ellIdx[e * 32 + lane], i1 = L.ellIdx[(e + 1) * 32 + lane];
                const int i2 = L.ellIdx[(e + 2) * 32 + lane], i3 = L.ellIdx[(e + 3) * 32 + lane];
                const double w0 = L.ellVal[e * 32 + lane], w1 = L.ellVal[(e + 1) * 32 + lane];
                const double w2 = L.ellVal[(e + 2) * 32 + lane], w3 = L.ellVal[(e + 3) * 32 + lane];
                const double g0 = Gs[i0], g1 = Gs[i1], g2 = Gs[i2], g3 = Gs[i3];
                v += w0 * g0;
                v += w1 * g1;
                v += w2 * g2;
                v += w3 * g3;
            }
            for (; e < e1; e++)
                v += L.ellVal[e * 32 + lane] * Gs[L.ellIdx[e * 32 + lane]];
            if (pr != 0xFFFF) {
                int i = pr >> 8, j = pr & 255;
                Hs[i * ldh + j] = v;
                Hs[j * ldh + i] = v;
            }
        }
    } else {
        for (int pi = lane; pi < npairs; pi += 32) {
            unsigned short pr = pb.pairs[pi];
            int i = pr >> 8, j = pr & 255;
            double v = Gs[pb.pcol ? pb.pcol[pi] : pi];
            Hs[i * ldh + j] = v;
            Hs[j * ldh + i] = v;
        }
    }
}

// A helper slot's trial point: the parent's alpha_old + t_k d with t_k the
// parent's t halved k times, formed as the backtracking loop forms it.
__device__ void init_helper(const NewtonProblem &pb, Layout &L, int s, int lane, int ldv)
{
    const int par = L.ints[s * SI_N + SI_CELL], k = L.ints[s * SI_N + SI_ITER];
    double t = L.scal[par * SC_N + SC_T];
    for (int i = 0; i < k; i++)
        t = 0.5 * t;
    if (lane < ldv)
        L.alpha[s * ldv + lane] =
            (lane < pb.n) ? L.aold[par * ldv + lane] + t * L.d[par * ldv + lane] : 0.0;
    if (lane == 0)
        L.scal[s * SC_N + SC_DELTA] = L.scal[par * SC_N + SC_DELTA];
}

// The helper of slot s with index k (-1: none); slots are at most 32.
__device__ __forceinline__ int find_helper(const Layout &L, int T, int s, int k, int lane)
{
    const int *hi = L.ints + lane * SI_N;
    const unsigned m =
        __ballot_sync(0xffffffffu, lane < T && hi[SI_STATE] == S_HELP && hi[SI_CELL] == s && hi[SI_ITER] == k);
    return m ? __ffs(m) - 1 : -1;
}

__device__ __forceinline__ void release_helpers(Layout &L, int T, int s, int lane)
{
    __syncwarp();
    int *hi = L.ints + lane * SI_N;
    if (lane < T && hi[SI_STATE] == S_HELP && hi[SI_CELL] == s)
        hi[SI_STATE] = S_IDLE;
    __syncwarp();
}

// Sufficient condition, at a Mn evaluation, for the reference's condition
// test (opt.cpp:244-261: dpotrf succeeds and anorm / rcond from dpocon is at
// most MOMOPT_COND_H_MAX) to pass.  With the exponents s_q = alpha . p(q) in
// [lo, hi] over the quadrature, x^T H x = sum_q w_q e^{s_q} (p(q) . x)^2 lies
// between e^lo and e^hi times x^T M x, M = sum_q w_q p(q) p(q)^T with
// gramLo <= lambda(M) <= gramHi, so cond_2(H) <= e^(hi - lo) gramHi / gramLo,
// and the 1-norm condition number whose estimate (a lower bound) dpocon
// returns is at most n cond_2(H).  p_0 is constant, so
// |s_q - alpha_0 p_0| <= min(sum_k>=1 |alpha_k| c_k,
// sum_l>=1 ||alpha of degree l|| d_l) (c_k = max_q |p_k(q)|, d_l the largest
// norm over q of the degree-l basis values; Cauchy-Schwarz per degree),
// which bounds hi - lo by twice that.  The rounding of the computed H
// (quadrature and Gaunt sums: about 1e-10 e^hi in the 2-norm) is covered by
// the 1e-9 e^hi gramHi taken off the smallest eigenvalue, and a factor 4
// covers the estimate's own rounding.  Such an H is far from Cholesky
// breakdown (n eps cond_2(H) << 1).  `ai`: lane k's alpha_k.
__device__ __forceinline__ bool exponent_range_bound(const NewtonArgs &a, const NewtonProblem &pb, double ai,
                                                     int lane)
{
    const int n = pb.n, maxDeg = pb.maxDeg;
    const double b1 = warp_sum((lane >= 1 && lane < n) ? fabs(ai) * pb.rangeC[lane] : 0.0);
    // lane l (1 <= l <= maxDeg) sums alpha_k^2 over degree l's moments
    // k = l (l + 1) / 2 .. l (l + 1) / 2 + l
    const double sq = (lane < n) ? ai * ai : 0.0;
    const int base = lane * (lane + 1) / 2;
    double gl = 0.0;
    for (int j = 0; j <= maxDeg; j++) {
        const double v = __shfl_sync(0xffffffffu, sq, min(base + j, 31));
        if (j <= lane && base + j < n)
            gl += v;
    }
    const double b2 = warp_sum((lane >= 1 && lane <= maxDeg) ? sqrt(gl) * pb.rangeC[n + lane] : 0.0);
    const double span = 2.0 * fmin(b1, b2) * (1.0 + 1e-12);
    if (!(span <= 40.0))
        return false;
    const double ratio = exp(span);
    const double lmin = pb.gramLo - 1e-9 * ratio * pb.gramHi;
    if (!(lmin > 0.0))
        return false;
    return (double)n * ratio * pb.gramHi * (1.0 + 1e-9) <= 0.25 * a.condHMax * lmin;
}

// H_0,lane (lane < n) from the contraction results: the row-0 entries of the
// Gaunt table in its order (the sums of the full contraction without its zero
// padding), or the product column (lane, 0).
__device__ __forceinline__ double hessian_row0(const NewtonArgs &a, const NewtonProblem &pb, const double *Gs,
                                               int lane)
{
    double h0 = 0.0;
    if (a.useGaunt) {
        const int e1 = pb.row0Off[lane + 1];
        for (int e = pb.row0Off[lane]; e < e1; e++)
            h0 = fma(pb.row0Val[e], Gs[pb.row0Idx[e]], h0);
    } else {
        h0 = Gs[pb.pcol ? pb.pcol[lane] : lane];
    }
    return h0;
}

// Newton logic for one slot after its evaluation (warp-wide).  `range`: the
// evaluation is Mn in FP64 (the exponent-range test applies).
__device__ void slot_logic(const NewtonArgs &a, const NewtonProblem &pb, Layout &L, int s, int lane,
                           int warp, bool range)
{
    const int n = pb.n;
    const int ldv = a.ldv, ldG = a.ldG, ldh = a.ldh;
    const bool act = lane < n;
    int *si = L.ints + s * SI_N;
    double *sc = L.scal + s * SC_N;
    double *Hs = L.H + warp * (kMaxN * ldh);
    double *vec = L.vec + warp * 64;
    const double *Gs = L.G + s * ldG;

    const double ui = act ? L.u[s * ldv + lane] : 0.0;
    const double ai = act ? L.alpha[s * ldv + lane] : 0.0;
    const double au = warp_sum(ai * ui);
    double fpart = 0.0;
    for (int k = 0; k < a.ntq; k++)
        fpart += L.fpart[s * a.ntq + k];
    const double fsum = fpart - au;                  // no-Hessian f (linesearch's fobj)

    int state = si[SI_STATE];
    if (state == S_TRIAL) {
        if (lane == 0)
            atomicAdd(&L.stat[kNumReg + 2], 1ull);
        double t = sc[SC_T];
        if (!(fsum <= sc[SC_FREF] + 1e-3 * t * sc[SC_GD])) {
            t = 0.5 * t;
            double ao = act ? L.aold[s * ldv + lane] : 0.0;
            // the next trial points, evaluated this round by helper slots:
            // take them in the backtracking order, stopping where the loop
            // of linesearch.cpp:53-81 would stop
            for (int k = 1; t * sc[SC_MAXF] > DBL_EPSILON / 2; k++) {
                const int h = find_helper(L, a.T, s, k, lane);
                if (h < 0)
                    break;
                const double ah = act ? L.alpha[h * ldv + lane] : 0.0;
                double fp = 0.0;
                for (int q = 0; q < a.ntq; q++)
                    fp += L.fpart[h * a.ntq + q];
                const double fh = fp - warp_sum(ah * ui);
                if (fh <= sc[SC_FREF] + 1e-3 * t * sc[SC_GD]) {
                    // accepted at t: the slot moves to this trial point, and
                    // the next round's evaluation of it (bit for bit the
                    // helper's) is taken, and counted, as the accepted trial
                    if (act)
                        L.alpha[s * ldv + lane] = ah;
                    __syncwarp();
                    if (lane == 0)
                        sc[SC_T] = t;
                    release_helpers(L, a.T, s, lane);
                    return;
                }
                if (lane == 0)
                    atomicAdd(&L.stat[kNumReg + 2], 1ull);
                t = 0.5 * t;
            }
            release_helpers(L, a.T, s, lane);
            if (t * sc[SC_MAXF] > DBL_EPSILON / 2) {
                if (act)
                    L.alpha[s * ldv + lane] = ao + t * L.d[s * ldv + lane];
                __syncwarp();
                if (lane == 0)
                    sc[SC_T] = t;
                return;
            }
            // backtracked all the way (linesearch.cpp:84-98): alpha restored,
            // the next iteration regularises because t == 0.
            __syncwarp();
            if (lane == 0) {
                si[SI_ITER] += 1;
                si[SI_TOTAL] += 1;
            }
            __syncwarp();
            regularize(a, pb, L, s, lane, ldv, ui, ao);
            return;
        }
        // accepted: this evaluation is the next Newton iteration's (opt.cpp:262-274)
    }

    // one Newton iteration (opt.cpp:258-368)
    const int iter = si[SI_ITER] + 1;
    __syncwarp();
    if (lane == 0) {
        si[SI_ITER] = iter;
        si[SI_TOTAL] += 1;
    }
    // the stopping test applies (no gamma test, iterations left, the last
    // line search moved)
    const bool stopTest = !(a.tolGamma > 0.0) && iter < si[SI_MAXITER] && sc[SC_T] != 0.0;
    if (range && a.momentType == 0 && pb.gramLo > 0.0 && stopTest) {
        // Converged with the condition test passing by the exponent range:
        // the gradient needs row 0 of H only (the same sums, in the same
        // order, as the full contraction), and the reference's outcome is
        // convergence at this iteration.  A finite gradient implies finite
        // G (G_0 is a sum of positive terms), so the full contraction's
        // zero-padded entries would add exact zeros.
        const double g0 = act ? hessian_row0(a, pb, Gs, lane) / pb.p0 - ui : 0.0;
        if (sqrt(warp_sum(g0 * g0)) <= sc[SC_RTOL] && exponent_range_bound(a, pb, ai, lane)) {
            converge(a, pb, L, s, ui, ai, g0, lane);
            return;
        }
    }

    // H from the contraction results
    hessian_from_contractions(a, pb, L, Gs, Hs, lane);
    __syncwarp();
    double gi;
    if (a.momentType == 0)
        gi = act ? Hs[lane] / pb.p0 - ui : 0.0;     // fobj.cpp:303-306
    else
        gi = act ? Gs[pb.K2p + lane] - ui : 0.0;    // fobj.cpp:427-431 / :445-452
    const double fH = (a.momentType == 0) ? Hs[0] / (pb.p0 * pb.p0) - au : fsum;

    // row `lane` of H in registers; utils_norm1 = max absolute row sum
    double h[kMaxN], v[kMaxN];
    double rowsum = 0.0;
#pragma unroll
    for (int k = 0; k < kMaxN; k++) {
        h[k] = (act && k < n) ? Hs[lane * ldh + k] : 0.0;
        rowsum += fabs(h[k]);
    }
    const double anorm = warp_max(rowsum);
    // Converged at this evaluation with no regularisation due (most cells of
    // a time step, which start at the previous step's multipliers).  The
    // reference still factors H and estimates its condition number before
    // its stopping test; a rigorous bound that shows cond <= MOMOPT_COND_H_MAX
    // (factor-2 margin for rounding) fixes the same outcome, and neither the
    // inverse nor the direction is needed (without the gamma test).
    //  tier 0: H strictly diagonally dominant with positive diagonal:
    //          ||H^-1||_1 = ||H^-1||_inf <= 1 / min_i (H_ii - sum_j!=i |H_ij|)
    //          (Varah 1975); such H is SPD and its Cholesky factorisation
    //          cannot break down, so the factorisation is not needed either;
    //  tier 1: after the factorisation, the comparison-matrix bound.
    const double err = sqrt(warp_sum(gi * gi));
    const bool convTest = err <= sc[SC_RTOL] && stopTest;
    if (convTest) {
        const double dom = act ? 2.0 * Hs[lane * ldh + lane] - rowsum : DBL_MAX;
        const double delta = -warp_max(-dom);
        if (delta > 0.0 && anorm <= 0.5 * a.condHMax * delta) {
            converge(a, pb, L, s, ui, ai, gi, lane);
            return;
        }
    }
    __syncwarp();
    int info = chol_regs(h, Hs, ldh, n, lane);
    if (info == 0 && convTest && anorm * cmp_bound(h, Hs, ldh, n, lane) <= 0.5 * a.condHMax) {
        converge(a, pb, L, s, ui, ai, gi, lane);
        return;
    }
    double condest = 0.0;
    if (info == 0) {
        // column `lane` of L^-1 in v[], rows of L^-1 in Hs
        invert_regs(Hs, ldh, v, n, lane);
        __syncwarp();
        double colsum = 0.0;
#pragma unroll
        for (int i = 0; i < kMaxN; i++) {
            if (i < n && act)
                Hs[i * ldh + lane] = v[i];
            colsum += fabs(v[i]);
        }
        __syncwarp();
        double rs = 0.0;   // unrolled: the loads issue together, the sum keeps its order
#pragma unroll
        for (int c = 0; c < kMaxN; c++)
            if (act && c <= lane)
                rs += fabs(Hs[lane * ldh + c]);
        // ||A^-1||_1 <= ||L^-1||_1 ||L^-1||_inf, and the Higham estimate never
        // exceeds ||A^-1||_1: when the bound already shows cond <= COND_H_MAX
        // (with a factor-2 margin for rounding) the estimate cannot trigger
        // regularisation and is not needed.
        const double bound = anorm * warp_max(colsum) * warp_max(rs);
        if (!(bound <= 0.5 * a.condHMax)) {
            double rc = rcond_warp(Hs, n, ldh, vec, anorm, lane);
            condest = 1.0 / rc;
        }
    }
    if (iter >= si[SI_MAXITER] || info != 0 || sc[SC_T] == 0.0 || condest > a.condHMax) {
        __syncwarp();
        regularize(a, pb, L, s, lane, ldv, ui, ai);
        return;
    }
    // d = -L^-T (L^-1 g): rows of L^-1 from Hs, columns from registers
    __syncwarp();
    vec[lane] = gi;
    __syncwarp();
    double y = 0.0;
#pragma unroll
    for (int c = 0; c < kMaxN; c++)
        if (act && c <= lane)
            y = fma(Hs[lane * ldh + c], vec[c], y);
    __syncwarp();
    vec[32 + lane] = y;
    __syncwarp();
    double z = 0.0;
#pragma unroll
    for (int i = 0; i < kMaxN; i += 2) {
        if (i < n) {
            const double2 yi = *reinterpret_cast<const double2 *>(vec + 32 + i);
            z = fma(v[i], yi.x, z);
            if (i + 1 < n)
                z = fma(v[i + 1], yi.y, z);
        }
    }
    const double di = act ? -z : 0.0;
    bool gammaOk = true;
    if (a.tolGamma > 0.0)
        gammaOk = modcfl(di, n, lane, a.momentType) <= a.tolGamma;
    if (err <= sc[SC_RTOL] && gammaOk) {
        converge(a, pb, L, s, ui, ai, gi, lane);
        return;
    }
    // line search set-up (linesearch.cpp:21-52)
    const double gd = warp_sum(gi * di);
    const double maxf = warp_max(act ? fabs(di) / (fabs(ai) + 1e-100) : 0.0);
    if (act) {
        L.aold[s * ldv + lane] = ai;
        L.d[s * ldv + lane] = di;
    }
    if (1.0 * maxf > DBL_EPSILON / 2) {
        if (act)
            L.alpha[s * ldv + lane] = ai + 1.0 * di;
        __syncwarp();
        if (lane == 0) {
            sc[SC_T] = 1.0;
            sc[SC_FREF] = fH;
            sc[SC_GD] = gd;
            sc[SC_MAXF] = maxf;
            si[SI_STATE] = S_TRIAL;
        }
        return;
    }
    // zero-length search: linesearch returns 0 without evaluating
    __syncwarp();
    if (lane == 0) {
        sc[SC_T] = 0.0;
        si[SI_ITER] += 1;
        si[SI_TOTAL] += 1;
    }
    __syncwarp();
    regularize(a, pb, L, s, lane, ldv, ui, ai);
}

// ---------------------------------------------------------------------------
// Change-of-basis Newton (MOMOPT_OPTIMIZATION_TYPE 1, opt/optcb.cpp:156-415).
// Each vector carries a lower-triangular basis T (P2M) and multipliers alphaP
// in that basis.  Exponents and f do not depend on the basis (alphaP.pP_q =
// alphaM.p_q with alphaM = T^-T alphaP), so phase A evaluates at alphaM with
// the shared basis as for plain Newton; phase B forms the Hessian in the
// working basis, H_P = T^-1 H_M T^-T, and the gradient g_P = T^-1 g_M by two
// triangular solves, factors H_P = L L^T, takes the reference's decisions on
// it (first-evaluation reset, regularisation), and changes the basis
// T <- T L, alphaP <- L^T alphaP, g_P <- L^-1 g_P, so the Newton step in the
// new basis is d_P = -g_P (the moment-basis step is (T L)^-T d_P).  The
// working state of a slot (T, L^-1, alphaP, the line search's alphaM and
// step) lives in global scratch, L1/L2-resident, so shared memory stays as for
// plain Newton; the vector's stored basis and alphaP are the start of every
// regularisation restart and are written back on convergence.
enum { CB_START_STD = 1, CB_HIT_MAX = 2 };

__device__ __forceinline__ double *cb_slot(const NewtonArgs &a, int s)
{
    return a.cbScratch + ((size_t)blockIdx.x * a.T + s) * a.cbStride;
}
__device__ __forceinline__ double *cb_basis(const NewtonArgs &a, int s) { return cb_slot(a, s); }
__device__ __forceinline__ double *cb_linv(const NewtonArgs &a, int s) { return cb_slot(a, s) + kMaxN * kMaxN; }
__device__ __forceinline__ double *cb_ap(const NewtonArgs &a, int s) { return cb_slot(a, s) + 2 * kMaxN * kMaxN; }
__device__ __forceinline__ double *cb_am(const NewtonArgs &a, int s) { return cb_ap(a, s) + kMaxN; }
__device__ __forceinline__ double *cb_dm(const NewtonArgs &a, int s) { return cb_ap(a, s) + 2 * kMaxN; }
__device__ __forceinline__ double *cb_rdiag(const NewtonArgs &a, int s) { return cb_ap(a, s) + 3 * kMaxN; }

// x = T^-T y (lane i holds y_i, returns x_i): backward substitution with the
// reciprocal diagonal, x_i = (y_i - sum_{k>i} T_ki x_k) / T_ii.
__device__ double cb_solve_t(const double *Tg, double y, int n, int lane)
{
    const double rl = (lane < n) ? 1.0 / Tg[lane * kMaxN + lane] : 0.0;
    double acc = 0.0, x = 0.0;
    for (int i = n - 1; i >= 0; i--) {
        const double xi = __shfl_sync(0xffffffffu, (y - acc) * rl, i);
        if (lane == i)
            x = xi;
        if (lane < i)
            acc = fma(Tg[i * kMaxN + lane], xi, acc);
    }
    return (lane < n) ? x : 0.0;
}

// Columns held per lane (lane j: m[i] = M_ij) replaced by those of T^-1 M:
// forward substitution by rows, row i of T (stride kMaxN) read by every lane
// (one broadcast), rd[i] = 1/T_ii.
__device__ __forceinline__ void cb_trsv_cols(const double *Tg, const double *rd, double (&m)[kMaxN], int n)
{
#pragma unroll
    for (int i = 0; i < kMaxN; i++) {
        if (i < n) {
            const double *Ti = Tg + i * kMaxN;
            double a0 = m[i], a1 = 0.0, a2 = 0.0, a3 = 0.0;
#pragma unroll
            for (int k = 0; k + 1 < i; k += 2) {
                const double2 l = *reinterpret_cast<const double2 *>(Ti + k);
                if (k & 2) {
                    a2 = fma(-l.x, m[k], a2);
                    a3 = fma(-l.y, m[k + 1], a3);
                } else {
                    a0 = fma(-l.x, m[k], a0);
                    a1 = fma(-l.y, m[k + 1], a1);
                }
            }
            if (i & 1)
                a1 = fma(-Ti[i - 1], m[i - 1], a1);
            m[i] = ((a0 + a1) + (a2 + a3)) * rd[i];
        }
    }
}

// alphaM = T^-T alphaP for the slot (working basis), into L.alpha.
__device__ void cb_set_alpha_m(const NewtonArgs &a, const NewtonProblem &pb, Layout &L, int s, int lane)
{
    const int n = pb.n, ldv = a.ldv;
    const double ap = (lane < n) ? cb_ap(a, s)[lane] : 0.0;
    const double am = cb_solve_t(cb_basis(a, s), ap, n, lane);
    __syncwarp();
    if (lane < n)
        L.alpha[s * ldv + lane] = am;
    __syncwarp();
}

// Working basis <- the vector's stored basis, or the identity after a
// restart in the standard basis; alphaP likewise (optcb.cpp:247-318).
__device__ void cb_restart_state(const NewtonArgs &a, const NewtonProblem &pb, Layout &L, int s, int lane)
{
    const int n = pb.n, ldv = a.ldv;
    const int cell = L.ints[s * SI_N + SI_CELL];
    const bool std_ = (L.ints[s * SI_N + SI_CB] & CB_START_STD) != 0;
    double *Tg = cb_basis(a, s);
    const double *T0 = pb.P2M + (size_t)cell * n * n;
    for (int i = 0; i < n; i++)
        if (lane < n)
            Tg[i * kMaxN + lane] = std_ ? (i == lane ? 1.0 : 0.0) : T0[i * n + lane];
    if (lane < n)
        cb_rdiag(a, s)[lane] = std_ ? 1.0 : 1.0 / T0[lane * n + lane];
    double ap;
    if (std_) {
        const double a0 = (a.momentType == 0) ? 2.0 * kSqrtPi * log(0.5 / kSqrtPi)
                                              : 1.0 - 4.0 * L.scal[s * SC_N + SC_DELTA] * kPi;
        ap = (lane == 0) ? a0 : 0.0;
    } else {
        ap = (lane < n) ? pb.alphaP[(size_t)cell * n + lane] : 0.0;
    }
    if (lane < n)
        cb_ap(a, s)[lane] = ap;
    __syncwarp();
    cb_set_alpha_m(a, pb, L, s, lane);
}

// Loads a newly assigned vector (optcb.cpp:87-153 entry half, :170-188).
__device__ void init_slot_cb(const NewtonArgs &a, const NewtonProblem &pb, Layout &L, int s, int lane, int ldv)
{
    const int n = pb.n;
    const int cell = L.ints[s * SI_N + SI_CELL];
    double ui = (lane < n) ? pb.u[(size_t)cell * n + lane] : 0.0;
    if (a.momentsOld != nullptr && lane < n) {
        int i = cell / a.NY, j = cell % a.NY;
        if (i >= 2 && i < a.NX - 2 && j >= 2 && j < a.NY - 2)
            a.momentsOld[(size_t)cell * n + lane] = ui;
    }
    const double u0 = __shfl_sync(0xffffffffu, ui, 0);
    if (!(u0 > 0.0)) {
        if (lane == 0) {
            L.ints[s * SI_N + SI_TOTAL] = 0;
            L.ints[s * SI_N + SI_REG] = 0;
        }
        __syncwarp();
        finish_slot(a, pb, L, s, ui, (lane < n) ? pb.alpha[(size_t)cell * n + lane] : 0.0, -3, lane);
        return;
    }
    double *sc = L.scal + s * SC_N;
    double delta = a.deltaPPn;
    if (a.momentType == 0) {
        if (lane == 0)
            sc[SC_ASCALE] = log(u0) * 2.0 * kSqrtPi;
    } else {
        delta = delta / (u0 * u0);
    }
    ui = ui / u0;
    if (lane < ldv)
        L.u[s * ldv + lane] = (lane < n) ? ui : 0.0;
    const double rtol = sqrt(warp_sum(ui * ui)) * a.tolRel;
    if (lane == 0) {
        sc[SC_T] = 1.0;
        sc[SC_RTOL] = rtol;
        sc[SC_U0] = u0;
        sc[SC_DELTA] = delta;
        sc[SC_R] = 0.0;
        int *si = L.ints + s * SI_N;
        si[SI_ITER] = 0;
        si[SI_TOTAL] = 0;
        si[SI_REG] = 0;
        si[SI_MAXITER] = a.maxIter;
        si[SI_PRED] = 0;
        si[SI_CB] = 0;
        si[SI_BFGS] = 0;
        si[SI_STATE] = S_NEWTON;
    }
    __syncwarp();
    cb_restart_state(a, pb, L, s, lane);
}

// Regularisation restart of the change-of-basis solve (optcb.cpp:268-318).
__device__ void cb_regularize(const NewtonArgs &a, const NewtonProblem &pb, Layout &L, int s, int lane)
{
    const int n = pb.n, ldv = a.ldv;
    int *si = L.ints + s * SI_N;
    double *sc = L.scal + s * SC_N;
    const int cell = si[SI_CELL];
    const double u0 = sc[SC_U0];
    int reg = si[SI_REG], flags = si[SI_CB];
    double r = sc[SC_R];
    const double us = (lane < n) ? pb.u[(size_t)cell * n + lane] / u0 : 0.0;   // scaled original
    double unew;
    int maxIter = si[SI_MAXITER];
    if (reg < kNumReg - 1) {
        reg++;
        r = kRegularizations[reg];
        unew = (lane == 0) ? 1.0 : us * (1.0 - r);
    } else {
        if (flags & CB_HIT_MAX) {
            // "This should never happen." -- the reference aborts
            double uo = us * u0, ao = (lane < n) ? L.alpha[s * ldv + lane] : 0.0;
            if (a.momentType == 0) {
                if (lane == 0)
                    ao += sc[SC_ASCALE];
            } else {
                ao *= u0;
            }
            __syncwarp();
            finish_slot(a, pb, L, s, uo, ao, -4, lane);
            return;
        }
        flags |= CB_HIT_MAX | CB_START_STD;
        unew = us;
        reg = 0;   // r keeps its value (optcb.cpp:288-296)
        maxIter = a.maxIter;
    }
    if (reg == kNumReg - 1)
        maxIter = 10 * maxIter;
    if (lane < n)
        L.u[s * ldv + lane] = unew;
    const double rtol = sqrt(warp_sum(lane < n ? unew * unew : 0.0)) * a.tolRel;
    __syncwarp();
    if (lane == 0) {
        si[SI_REG] = reg;
        si[SI_CB] = flags;
        si[SI_ITER] = 0;
        si[SI_MAXITER] = maxIter;
        sc[SC_R] = r;
        sc[SC_T] = 1.0;
        sc[SC_RTOL] = rtol;
        si[SI_STATE] = S_NEWTON;
    }
    __syncwarp();
    cb_restart_state(a, pb, L, s, lane);
}

// Converged: the regularised input moments and alphaM are returned (no
// moment write-back, optcb.cpp:347-360 and the wrapper's rescaling), the
// vector's basis and alphaP are stored.
__device__ void cb_converge(const NewtonArgs &a, const NewtonProblem &pb, Layout &L, int s, int lane)
{
    const int n = pb.n, ldv = a.ldv;
    int *si = L.ints + s * SI_N;
    const double *sc = L.scal + s * SC_N;
    const int cell = si[SI_CELL];
    const double u0 = sc[SC_U0], r = sc[SC_R];
    const double us = (lane < n) ? pb.u[(size_t)cell * n + lane] / u0 : 0.0;
    double uo = ((lane == 0) ? 1.0 : us * (1.0 - r)) * u0;
    double ao = (lane < n) ? L.alpha[s * ldv + lane] : 0.0;
    if (a.momentType == 0) {
        if (lane == 0)
            ao += sc[SC_ASCALE];
    } else {
        ao *= u0;
    }
    const double *Tg = cb_basis(a, s);
    double *T0 = pb.P2M + (size_t)cell * n * n;
    for (int i = 0; i < n; i++)
        if (lane < n)
            T0[i * n + lane] = Tg[i * kMaxN + lane];
    if (lane < n)
        pb.alphaP[(size_t)cell * n + lane] = cb_ap(a, s)[lane];
    // the histogram bin of r (after a restart in the standard basis the
    // level index is 0 while r keeps its last value, as in the reference)
    int bin = 0;
    for (int k = 0; k < kNumReg; k++)
        if (fabs(r - kRegularizations[k]) < 1e-10)
            bin = k;
    __syncwarp();
    if (lane == 0)
        si[SI_REG] = bin;
    __syncwarp();
    finish_slot(a, pb, L, s, uo, ao, 0, lane);
}

// ---------------------------------------------------------------------------
// BFGS sub-iterations (MOMOPT_OPTIMIZATION_TYPE 2, opt/optbfgs.cpp:163-512).
// The outer iteration is the change-of-basis Newton iteration above; after
// each basis change H and H^-1 in the new basis start at the identity and up
// to MOMOPT_MAX_BFGS_ITER quasi-Newton steps d_P = -H^-1 g_P follow, each
// with the Armijo line search, while cond(H) cond(H^-1) (the reference's
// cond(): largest absolute column sums of the matrices) stays below
// MOMOPT_COND_H_MAX_BFGS.  Only the outer iterations count as iterations.
// Every line-search evaluation carries f, g and H_M, so when the BFGS loop
// ends at an accepted point the outer iteration runs on that evaluation (the
// reference re-evaluates at the same point).  H and H^-1 live in the slot's
// scratch, column j at j * kMaxN, lane i updating row i.
__device__ __forceinline__ double *bfgs_h(const NewtonArgs &a, int s) { return cb_slot(a, s) + kCbSlotDoubles; }
__device__ __forceinline__ double *bfgs_hinv(const NewtonArgs &a, int s) { return bfgs_h(a, s) + kMaxN * kMaxN; }
__device__ __forceinline__ double *bfgs_gold(const NewtonArgs &a, int s) { return bfgs_h(a, s) + 2 * kMaxN * kMaxN; }

// x = T^-1 y (lane i holds y_i, returns x_i): forward substitution with the
// reciprocal diagonal rd.
__device__ double cb_solve_l(const double *Tg, const double *rd, double y, int n, int lane)
{
    const double rl = (lane < n) ? rd[lane] : 0.0;
    double acc = 0.0, x = 0.0;
    for (int i = 0; i < n; i++) {
        const double xi = __shfl_sync(0xffffffffu, (y - acc) * rl, i);
        if (lane == i)
            x = xi;
        if (lane > i && lane < n)
            acc = fma(Tg[lane * kMaxN + i], xi, acc);
    }
    return (lane < n) ? x : 0.0;
}

// H = H^-1 = I after a change of basis (optbfgs.cpp:363-364).
__device__ void bfgs_reset(const NewtonArgs &a, int s, int n, int lane)
{
    double *Hp = bfgs_h(a, s), *Hi = bfgs_hinv(a, s);
    if (lane < n)
        for (int j = 0; j < n; j++) {
            Hp[j * kMaxN + lane] = (j == lane) ? 1.0 : 0.0;
            Hi[j * kMaxN + lane] = (j == lane) ? 1.0 : 0.0;
        }
    __syncwarp();
}

// cond(H) cond(H^-1) as optbfgs.cpp:515-545 computes it; NaN when an update
// divided by zero (a step that did not move alpha), which ends the loop as
// the reference's comparison with NaN does.
__device__ double bfgs_cond(const NewtonArgs &a, int s, int n, int lane)
{
    __syncwarp();
    const double *Hp = bfgs_h(a, s), *Hi = bfgs_hinv(a, s);
    double s1 = 0.0, s2 = 0.0;
    if (lane < n)
        for (int j = 0; j < n; j++) {
            s1 += fabs(Hp[lane * kMaxN + j]);
            s2 += fabs(Hi[lane * kMaxN + j]);
        }
    const bool nan = __any_sync(0xffffffffu, isnan(s1) || isnan(s2));
    const double c = warp_max(s1) * warp_max(s2);
    return nan ? __longlong_as_double(0x7ff8000000000000ll) : c;
}

// The BFGS updates of H and H^-1 with the step ad = alphaDiff and the
// gradient change gd = gDiff (optbfgs.cpp:455-485, the dger/dgemv sequence
// element by element in the same order).
__device__ void bfgs_update(const NewtonArgs &a, int s, int n, int lane, double ad, double gd)
{
    const bool act = lane < n;
    double *Hp = bfgs_h(a, s), *Hi = bfgs_hinv(a, s);
    const double ag = warp_sum(ad * gd);
    const double c1 = 1.0 / ag;
    for (int j = 0; j < n; j++) {
        const double gj = __shfl_sync(0xffffffffu, gd, j);
        if (act)
            Hp[j * kMaxN + lane] += gd * (c1 * gj);
    }
    double t1 = 0.0;
    for (int j = 0; j < n; j++) {
        const double aj = __shfl_sync(0xffffffffu, ad, j);
        if (act)
            t1 = fma(aj, Hp[j * kMaxN + lane], t1);
    }
    const double c2 = -1.0 / warp_sum(ad * t1);
    double t2 = 0.0;
    for (int j = 0; j < n; j++) {
        const double tj = __shfl_sync(0xffffffffu, t1, j);
        const double gj = __shfl_sync(0xffffffffu, gd, j);
        if (act) {
            Hp[j * kMaxN + lane] += t1 * (c2 * tj);
            t2 = fma(gj, Hi[j * kMaxN + lane], t2);
        }
    }
    const double gHg = warp_sum(gd * t2);
    const double c3 = (gHg + ag) / (ag * ag), c4 = -1.0 / ag;
    for (int j = 0; j < n; j++) {
        const double aj = __shfl_sync(0xffffffffu, ad, j);
        const double tj = __shfl_sync(0xffffffffu, t2, j);
        if (act) {
            double h = Hi[j * kMaxN + lane];
            h += ad * (c3 * aj);
            h += t2 * (c4 * aj);
            h += ad * (c4 * tj);
            Hi[j * kMaxN + lane] = h;
        }
    }
}

// One pass of the BFGS loop body at alphaP with gradient gp (working basis),
// f and the moment-basis gradient norm err (optbfgs.cpp:371-445): the
// direction, the stopping test, and the line search set-up.
__device__ void bfgs_step(const NewtonArgs &a, const NewtonProblem &pb, Layout &L, int s, int lane, double gp,
                          double f, double err)
{
    const int n = pb.n, ldv = a.ldv;
    const bool act = lane < n;
    int *si = L.ints + s * SI_N;
    double *sc = L.scal + s * SC_N;
    double *APs = cb_ap(a, s), *AMs = cb_am(a, s), *DMs = cb_dm(a, s);
    const double *Hi = bfgs_hinv(a, s);
    __syncwarp();
    if (lane == 0)
        si[SI_BFGS] += 1;
    double dp = 0.0;
    for (int j = 0; j < n; j++) {
        const double gj = __shfl_sync(0xffffffffu, gp, j);
        if (act)
            dp = fma(-gj, Hi[j * kMaxN + lane], dp);
    }
    if (err <= sc[SC_RTOL]) {
        cb_converge(a, pb, L, s, lane);
        return;
    }
    const double ap = act ? APs[lane] : 0.0;
    const double am = act ? L.alpha[s * ldv + lane] : 0.0;
    const double gd = warp_sum(gp * dp);
    const double maxf = warp_max(act ? fabs(dp) / (fabs(ap) + 1e-100) : 0.0);
    if (1.0 * maxf > DBL_EPSILON / 2) {
        const double dmv = cb_solve_t(cb_basis(a, s), dp, n, lane);   // moment-basis step T^-T d_P
        if (act) {
            L.aold[s * ldv + lane] = ap;
            L.d[s * ldv + lane] = dp;
            bfgs_gold(a, s)[lane] = gp;
            AMs[lane] = am;
            DMs[lane] = dmv;
            L.alpha[s * ldv + lane] = am + dmv;
        }
        __syncwarp();
        if (lane == 0) {
            sc[SC_T] = 1.0;
            sc[SC_FREF] = f;
            sc[SC_GD] = gd;
            sc[SC_MAXF] = maxf;
            si[SI_STATE] = S_TRIAL;
        }
        return;
    }
    // no step possible: the line search returns 0 and the next outer
    // iteration regularises
    __syncwarp();
    if (lane == 0) {
        sc[SC_T] = 0.0;
        si[SI_ITER] += 1;
        si[SI_TOTAL] += 1;
    }
    __syncwarp();
    cb_regularize(a, pb, L, s, lane);
}

// After an accepted line search: the gradient at the new point in the
// working basis, the BFGS updates, and the loop test.  Returns false when the
// loop ends (the outer iteration then runs on this evaluation).
__device__ bool bfgs_after_step(const NewtonArgs &a, const NewtonProblem &pb, Layout &L, int s, int lane,
                                double gm, double f)
{
    const int n = pb.n, ldv = a.ldv;
    const bool act = lane < n;
    const int *si = L.ints + s * SI_N;
    const double gp = cb_solve_l(cb_basis(a, s), cb_rdiag(a, s), gm, n, lane);
    const double ad = act ? cb_ap(a, s)[lane] - L.aold[s * ldv + lane] : 0.0;
    const double gdf = act ? gp - bfgs_gold(a, s)[lane] : 0.0;
    bfgs_update(a, s, n, lane, ad, gdf);
    const double c = bfgs_cond(a, s, n, lane);
    if (c < a.condHMaxBfgs && si[SI_BFGS] < a.maxBfgsIter) {
        bfgs_step(a, pb, L, s, lane, gp, f, sqrt(warp_sum(gm * gm)));
        return true;
    }
    return false;
}

// Newton logic of one change-of-basis slot after its evaluation.
__device__ void slot_logic_cb(const NewtonArgs &a, const NewtonProblem &pb, Layout &L, int s, int lane, int warp)
{
    const int n = pb.n;
    const int ldv = a.ldv, ldG = a.ldG, ldh = a.ldh;
    const bool act = lane < n;
    int *si = L.ints + s * SI_N;
    double *sc = L.scal + s * SC_N;
    double *Hs = L.H + warp * (kMaxN * ldh);
    double *Wi = cb_linv(a, s);   // rows of L^-1, stride kMaxN
    double *APs = cb_ap(a, s), *AMs = cb_am(a, s), *DMs = cb_dm(a, s);
    double *vec = L.vec + warp * 64;
    const double *Gs = L.G + s * ldG;

    // H_M in the moment basis (Gaunt sums or products)
    hessian_from_contractions(a, pb, L, Gs, Hs, lane);
    __syncwarp();
    const double ui = act ? L.u[s * ldv + lane] : 0.0;
    const double am = act ? L.alpha[s * ldv + lane] : 0.0;
    double gi;
    if (a.momentType == 0)
        gi = act ? Hs[lane] / pb.p0 - ui : 0.0;
    else
        gi = act ? Gs[pb.K2p + lane] - ui : 0.0;
    const double au = warp_sum(am * ui);
    double fpart = 0.0;
    for (int k = 0; k < a.ntq; k++)
        fpart += L.fpart[s * a.ntq + k];
    const double fsum = fpart - au;
    const double fH = (a.momentType == 0) ? Hs[0] / (pb.p0 * pb.p0) - au : fsum;

    if (si[SI_STATE] == S_TRIAL) {
        if (lane == 0)
            atomicAdd(&L.stat[kNumReg + 2], 1ull);
        double t = sc[SC_T];
        if (!(fsum <= sc[SC_FREF] + 1e-3 * t * sc[SC_GD])) {
            t = 0.5 * t;
            if (t * sc[SC_MAXF] > DBL_EPSILON / 2) {
                if (act)
                    L.alpha[s * ldv + lane] = AMs[lane] + t * DMs[lane];
                __syncwarp();
                if (lane == 0)
                    sc[SC_T] = t;
                return;
            }
            // backtracked all the way: restored alpha, the next iteration
            // regularises because t == 0
            if (act) {
                APs[lane] = L.aold[s * ldv + lane];
                L.alpha[s * ldv + lane] = AMs[lane];
            }
            __syncwarp();
            if (lane == 0) {
                si[SI_ITER] += 1;
                si[SI_TOTAL] += 1;
            }
            __syncwarp();
            cb_regularize(a, pb, L, s, lane);
            return;
        }
        // accepted: alphaP <- alphaP + t d_P; this evaluation is the next
        // outer iteration's, or (BFGS) the next quasi-Newton step's
        if (act)
            APs[lane] = L.aold[s * ldv + lane] + t * L.d[s * ldv + lane];
        __syncwarp();
        if (a.optType == 2 && bfgs_after_step(a, pb, L, s, lane, gi, fsum))
            return;
    }

    const int iter = si[SI_ITER] + 1;
    const int total = si[SI_TOTAL] + 1;
    __syncwarp();
    if (lane == 0) {
        si[SI_ITER] = iter;
        si[SI_TOTAL] = total;
    }
    const double err = sqrt(warp_sum(gi * gi));   // the moment-basis gradient (:340-344)

    double *Tg = cb_basis(a, s);
    const double *rd = cb_rdiag(a, s);
    vec[lane] = gi;
    __syncwarp();
    // X = T^-1 [H_M | g_M]: lane j < n a column of H_M, lane n the gradient
    double m[kMaxN];
#pragma unroll
    for (int k = 0; k < kMaxN; k++)
        m[k] = (k < n) ? (act ? Hs[lane * ldh + k] : (lane == n ? vec[k] : 0.0)) : 0.0;
    cb_trsv_cols(Tg, rd, m, n);
    __syncwarp();
#pragma unroll
    for (int k = 0; k < kMaxN; k++) {
        if (k < n) {
            if (act)
                Hs[k * ldh + lane] = m[k];
            else if (lane == n)
                vec[32 + k] = m[k];   // g_P
        }
    }
    __syncwarp();
    // H_P = T^-1 X^T: lane j takes row j of X (a column of X^T)
#pragma unroll
    for (int k = 0; k < kMaxN; k++)
        m[k] = (act && k < n) ? Hs[lane * ldh + k] : 0.0;
    cb_trsv_cols(Tg, rd, m, n);
    double rowsum = 0.0;
#pragma unroll
    for (int k = 0; k < kMaxN; k++)
        rowsum += (k < n) ? fabs(m[k]) : 0.0;
    const double anorm = warp_max(act ? rowsum : 0.0);
    __syncwarp();
    int info = chol_regs(m, Hs, ldh, n, lane);
    double condest = 0.0;
    double v[kMaxN];
    if (info == 0) {
        invert_regs(Hs, ldh, v, n, lane);
        __syncwarp();
        double colsum = 0.0;
#pragma unroll
        for (int i = 0; i < kMaxN; i++) {
            if (i < n && act)
                Wi[i * kMaxN + lane] = v[i];   // rows of L^-1
            colsum += fabs(v[i]);
        }
        __syncwarp();
        double rs = 0.0;
        if (act)
            for (int c = 0; c <= lane; c++)
                rs += fabs(Wi[lane * kMaxN + c]);
        const double bound = anorm * warp_max(colsum) * warp_max(rs);
        if (!(bound <= 0.5 * a.condHMax)) {
            const double rc = rcond_warp(Wi, n, kMaxN, vec, anorm, lane);
            condest = 1.0 / rc;
        }
    }
    // a bad Hessian at the very first evaluation: isotropic alpha and the
    // standard basis (optcb.cpp:247-265)
    if (total == 1 && (info != 0 || condest > a.condHMax)) {
        __syncwarp();
        if (lane == 0) {
            si[SI_CB] |= CB_START_STD;
            si[SI_ITER] = 0;
            sc[SC_T] = 1.0;
            si[SI_STATE] = S_NEWTON;
        }
        __syncwarp();
        cb_restart_state(a, pb, L, s, lane);
        return;
    }
    if (iter >= si[SI_MAXITER] || info != 0 || sc[SC_T] == 0.0 || condest > a.condHMax) {
        __syncwarp();
        cb_regularize(a, pb, L, s, lane);
        return;
    }

    // change of basis by L (optcb.cpp:321-332)
    double gpn = 0.0;   // L^-1 g_P
    if (act)
        for (int k = 0; k <= lane; k++)
            gpn = fma(Wi[lane * kMaxN + k], vec[32 + k], gpn);
    // alphaP <- L^T alphaP: lane j sums L_kj alphaP_k over k >= j
    double apn = 0.0;
    if (act) {
        apn = (1.0 / Hs[lane * ldh + lane]) * APs[lane];
        for (int k = lane + 1; k < n; k++)
            apn = fma(Hs[k * ldh + lane], APs[k], apn);
    }
    // T <- T L: lane i forms row i
    {
        double t[kMaxN], tn[kMaxN];
#pragma unroll
        for (int k = 0; k < kMaxN; k++) {
            t[k] = (act && k <= lane) ? Tg[lane * kMaxN + k] : 0.0;
            tn[k] = 0.0;
        }
#pragma unroll
        for (int k = 0; k < kMaxN; k++) {
            if (k < n) {
                const double *Lk = Hs + k * ldh;
                const double lkk = 1.0 / Lk[k];
#pragma unroll
                for (int j = 0; j < kMaxN; j++)
                    if (j <= k)
                        tn[j] = fma(t[k], (j == k) ? lkk : Lk[j], tn[j]);
            }
        }
        __syncwarp();
        double tdiag = 1.0;
#pragma unroll
        for (int k = 0; k < kMaxN; k++) {
            if (act && k <= lane)
                Tg[lane * kMaxN + k] = tn[k];
            if (k == lane)
                tdiag = tn[k];
        }
        if (act)
            cb_rdiag(a, s)[lane] = 1.0 / tdiag;
    }
    __syncwarp();
    if (act)
        APs[lane] = apn;
    __syncwarp();
    if (a.optType == 2) {
        // BFGS loop from H = H^-1 = I, where cond = 1 (optbfgs.cpp:363-371)
        bfgs_reset(a, s, n, lane);
        if (lane == 0)
            si[SI_BFGS] = 0;
        if (1.0 < a.condHMaxBfgs && 0 < a.maxBfgsIter) {
            bfgs_step(a, pb, L, s, lane, gpn, fH, err);
        } else {
            __syncwarp();
            if (lane == 0)
                si[SI_STATE] = S_NEWTON;   // no step: evaluate again
        }
        return;
    }
    if (err <= sc[SC_RTOL]) {
        cb_converge(a, pb, L, s, lane);
        return;
    }
    // line search set-up in the new basis (linesearch.cpp:21-52 with d_P = -g_P)
    const double dp = act ? -gpn : 0.0;
    const double gd = warp_sum(gpn * dp);
    const double maxf = warp_max(act ? fabs(dp) / (fabs(apn) + 1e-100) : 0.0);
    if (1.0 * maxf > DBL_EPSILON / 2) {
        const double dmv = cb_solve_t(Tg, dp, n, lane);   // moment-basis step (T L)^-T d_P
        if (act) {
            L.aold[s * ldv + lane] = apn;
            L.d[s * ldv + lane] = dp;
            AMs[lane] = am;
            DMs[lane] = dmv;
            L.alpha[s * ldv + lane] = am + dmv;
        }
        __syncwarp();
        if (lane == 0) {
            sc[SC_T] = 1.0;
            sc[SC_FREF] = fH;
            sc[SC_GD] = gd;
            sc[SC_MAXF] = maxf;
            si[SI_STATE] = S_TRIAL;
        }
        return;
    }
    __syncwarp();
    if (lane == 0) {
        sc[SC_T] = 0.0;
        si[SI_ITER] += 1;
        si[SI_TOTAL] += 1;
    }
    __syncwarp();
    cb_regularize(a, pb, L, s, lane);
}

// Fused evaluation contractions (used when every problem's G has at most NTF
// column tiles of 8).  Warp w owns slot rows mt = w % 2 (16 slots) and the
// q-group qg = w / 2 (8 of the chunk's 32 quadrature rows): it forms
// S = alpha . P^T for its 16 x 8 block,
// the weights E = w exp(S) in the accumulator layout, and uses them directly
// as the A operand of G += E . Phess.  The A fragment's k-slots t and t+4 are
// taken as quadrature rows 2t and 2t+1 (the rows the accumulator of S gives
// this lane), and the B fragment is read from the same two rows, so E never
// goes through shared memory.  Chunks keep the basis_row layout of the
// global array, under which both fragment patterns (rows g, and rows 2t,
// 2t + 1) are free of bank conflicts.  The four q-group
// partial sums of G are added in q-group order at the end.  Three chunk
// buffers keep one chunk in flight while two are read.
constexpr unsigned long long kWaitNs = 2000000000ull;   // bound on any wait for a staged chunk

// PAIR (Mn, FP64): the chunk's rows are one direction q of each (phi,
// phi + pi) pair and the columns are grouped by degree parity.  GEMM1 forms
// the even and odd half sums S_e, S_o of alpha . p(q); the pair's exponents
// are S_e + S_o (direction q) and S_e - S_o (its partner, whose basis values
// are p(q) with the odd ones negated), and GEMM2 takes their weighted sum as
// the A operand of the even column tiles and their difference for the odd
// ones.  Each MMA so serves two directions.
//
// NW (warps per CTA) sets the launch shape: NW = 8 runs T = 32 slots (two
// 16-slot m-tiles, q-group = warp / 2) with three chunk buffers, one CTA per
// SM; NW = 4 runs T = 16 slots (one m-tile, q-group = warp) with two chunk
// buffers, small enough for two CTAs per SM, so that one CTA's phase B runs
// while the other's phase A keeps the tensor pipe busy.  Each slot's sums
// are the same MMAs in the same order in both shapes.
template <int NTF, int PPN, int NT, int NBK, int MIX, int PAIR = 0, int NW = 8>
__device__ __forceinline__ bool phase_a_fused(const NewtonArgs &a, const NewtonProblem &pb, Layout &L, int tid,
                                              int lane, int warp, unsigned &mbPhase)
{
    static_assert(!PAIR || (PPN == 0 && MIX == 0), "direction pairs: Mn in FP64");
    static_assert(NW == 8 || NW == 4, "launch shapes: 8 warps (32 slots) or 4 warps (16 slots)");
    constexpr int MT = NW / 4;                  // 16-slot m-tiles: T = 16 MT
    constexpr int DEPTH = (NW == 8) ? 3 : 2;    // staged chunk buffers
    const int g = lane >> 2, t4 = lane & 3;
    const int kq = a.kq, ldv = a.ldv, ldG = a.ldG;
    const int nb = pb.nb, ldP = pb.ldP, K2p = pb.K2p;
    // NT > 0: the problem's column tiles and GEMM1 k-steps are compile-time
    // constants (straight-line code); NT == 0: runtime counts up to NTF
    constexpr int NTL = (NT > 0) ? NT : NTF;
    constexpr int KSL = (NBK > 0) ? NBK : 4;
    const int NTH = (NT > 0) ? NT - (PPN ? NBK : 0) : K2p / 8;
    const int NT2 = (NT > 0) ? NT : NTH + (PPN ? nb / 8 : 0);
    const int nchunks = pb.nqp / kq;
    const int chunkDoubles = kq * ldP + kq;   // rows of a chunk, gaps included (basis_row)
    const int mt = (int)((unsigned)warp % MT), qg = (int)((unsigned)warp / MT);
    const int r0 = mt * 16 + g, r1 = r0 + 8;
    const double dl0 = L.scal[r0 * SC_N + SC_DELTA], dl1 = L.scal[r1 * SC_N + SC_DELTA];
    const double *A0 = L.alpha + r0 * ldv + t4, *A1 = L.alpha + r1 * ldv + t4;
    // Mixed precision (MIX, exact tile counts only): the Hessian-only tiles
    // -- Mn: tiles >= NBK (columns past the n that give f and g); PPn: the
    // Hessian tiles -- accumulate split-TF32 products in FP32; the rest FP64.
    static_assert(!MIX || NT > 0, "mixed precision runs the exact-count instances");
    auto lowp = [&](int nt) { return MIX && (PPN ? nt < NTH : nt >= NBK); };
    double acc[NTL][4];
    float acc32[MIX ? NTL : 1][4];
#pragma unroll
    for (int j = 0; j < NTL; j++)
        acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0;
#pragma unroll
    for (int j = 0; j < (MIX ? NTL : 1); j++)
        acc32[j][0] = acc32[j][1] = acc32[j][2] = acc32[j][3] = 0.0f;
    double facc0 = 0.0, facc1 = 0.0;
    const double invL = a.ex.invL, L1 = a.ex.L1, L2 = a.ex.L2;

    // Chunk c into buffer `buf`: one bulk copy of the contiguous block
    // (chunkDoubles is even, the block starts 16-byte aligned), issued by
    // thread 0 with its byte count expected on the buffer's mbarrier.
    const unsigned chunkBytes = (unsigned)chunkDoubles * 8u;
    unsigned pending = 0;   // buffers with a copy issued and not yet waited for
    auto load_chunk = [&](int c, int buf) {
        if (tid == 0) {
            mbar_expect_tx(&L.bar[buf], chunkBytes);
            bulk_copy_g2s(L.P + buf * chunkDoubles, pb.P + (size_t)c * chunkDoubles, chunkBytes, &L.bar[buf]);
        }
        pending |= 1u << buf;
    };
    auto wait_chunk = [&](int buf) -> bool {
        const bool ok = mbar_wait_bounded(&L.bar[buf], (mbPhase >> buf) & 1u, kWaitNs);
        mbPhase ^= 1u << buf;
        pending &= ~(1u << buf);
        return ok;
    };
    // after a timeout: wait (bounded) for the copies still in flight so that
    // none lands in shared memory after the CTA has exited
    auto abandon = [&]() {
        if (tid == 0)
            record_error(a.err, -5, -1);
        for (int b = 0; b < DEPTH; b++)
            if (pending & (1u << b))
                wait_chunk(b);
        return false;
    };
    const int qa = qg * 8 + g;                 // GEMM1 B rows
    const int qb = qg * 8 + 2 * t4;            // GEMM2 B rows qb, qb + 1
    const int offA = basis_row(qa, ldP);
    const int wOff = basis_wgap(qb, ldP);   // weights of rows qb, qb + 1
    const int offB = basis_row(qb, ldP) + g;   // rows qb and qb + 1 share the gap

    // PAIR: the moment of this lane's A columns in each k-step (-1: padding)
    int kb0[PAIR ? KSL : 1], kb1[PAIR ? KSL : 1];
    if constexpr (PAIR) {
#pragma unroll
        for (int ks = 0; ks < KSL; ks++) {
            kb0[ks] = pb.binv[ks * 8 + t4];
            kb1[ks] = pb.binv[ks * 8 + t4 + 4];
        }
    }
    const int nbe = pb.nbe, K2e = pb.K2e;
    // S block of chunk c (the staged copy at Pb); PAIR: even half sums in
    // cs, odd ones in co
    auto gemm1 = [&](const double *Pb, double (&cs)[4], double (&co)[4]) {
        cs[0] = cs[1] = cs[2] = cs[3] = 0.0;
        co[0] = co[1] = co[2] = co[3] = 0.0;
        const double *B1 = Pb + offA;
#pragma unroll
        for (int ks = 0; ks < KSL; ks++) {
            if constexpr (PAIR) {
                const double *Ar0 = L.alpha + r0 * ldv, *Ar1 = L.alpha + r1 * ldv;
                const int k0 = kb0[ks], k1 = kb1[ks];
                const double x0 = (k0 >= 0) ? Ar0[k0] : 0.0, x1 = (k0 >= 0) ? Ar1[k0] : 0.0;
                const double x2 = (k1 >= 0) ? Ar0[k1] : 0.0, x3 = (k1 >= 0) ? Ar1[k1] : 0.0;
                if (ks * 8 < nbe)
                    dmma16x8x8(cs, x0, x1, x2, x3, B1[ks * 8 + t4], B1[ks * 8 + t4 + 4]);
                else
                    dmma16x8x8(co, x0, x1, x2, x3, B1[ks * 8 + t4], B1[ks * 8 + t4 + 4]);
            } else if (NBK > 0 || ks * 8 < nb) {
                dmma16x8x8(cs, A0[ks * 8], A1[ks * 8], A0[ks * 8 + 4], A1[ks * 8 + 4], B1[ks * 8 + t4],
                           B1[ks * 8 + t4 + 4]);
            }
        }
    };
    // e[h]: Hessian weights, eg[h]: PPn gradient weights; h = 0..3 is
    // (slot r0, row qb), (r0, qb + 1), (r1, qb), (r1, qb + 1) of chunk c
    // PAIR: e receives the pair sums of the weights (even tiles) and eg the
    // differences (odd tiles)
    auto weights = [&](const double *Pc, const double (&cs)[4], const double (&co)[4], double (&e)[4],
                       double (&eg)[4]) {
        const double w0 = Pc[wOff], w1 = Pc[wOff + 1];   // staged with the chunk
        if constexpr (PAIR) {
            double sv[8], x[8];
#pragma unroll
            for (int h = 0; h < 4; h++) {
                sv[h] = cs[h] + co[h];
                sv[4 + h] = cs[h] - co[h];
            }
            fast_exp_n<8>(x, sv, L.exptab, invL, L1, L2);
#pragma unroll
            for (int h = 0; h < 4; h++) {
                const double ww = (h & 1) ? w1 : w0;
                x[h] *= ww;
                x[4 + h] *= ww;
            }
            facc0 += (x[0] + x[1]) + (x[4] + x[5]);
            facc1 += (x[2] + x[3]) + (x[6] + x[7]);
#pragma unroll
            for (int h = 0; h < 4; h++) {
                e[h] = x[h] + x[4 + h];
                eg[h] = x[h] - x[4 + h];
            }
        } else if constexpr (PPN == 0) {
            fast_exp_n<4>(e, cs, L.exptab, invL, L1, L2);
            e[0] *= w0;
            e[1] *= w1;
            e[2] *= w0;
            e[3] *= w1;
            facc0 += e[0] + e[1];
            facc1 += e[2] + e[3];
            eg[0] = eg[1] = eg[2] = eg[3] = 0.0;
        } else {
            // fobj.cpp:408-434 and :196-210 (PPn)
#pragma unroll
            for (int h = 0; h < 4; h++) {
                const double dl = (h < 2) ? dl0 : dl1;
                const double ww = (h & 1) ? w1 : w0;
                const double k = 0.5 * cs[h];
                const double s2 = sqrt(k * k + dl);
                double G = k + s2;
                if (k < 0)
                    G = -dl / (k - sqrt(k * k + dl));
                e[h] = 0.5 * ww * (G / s2);
                eg[h] = ww * G;
                const double ft = ww * (k * G - 0.5 * dl + dl * log(G));
                if (h < 2)
                    facc0 += ft;
                else
                    facc1 += ft;
            }
        }
    };

    // Software pipeline over three staged chunks: iteration c accumulates
    // G with chunk c's weights while it forms S and the weights of chunk
    // c + 1, and the copy of chunk c + 2 is in flight.
    load_chunk(0, 0);
    if (nchunks > 1)
        load_chunk(1, 1);
    if (__syncthreads_or(!wait_chunk(0)))
        return abandon();
    double e[4], eg[4];
    {
        double cs[4], co[4];
        gemm1(L.P, cs, co);
        weights(L.P, cs, co, e, eg);
    }
    // G += E . Phess for the chunk staged at Pc (E: weights held in e, eg)
    auto gemm2 = [&](const double *Pc) {
        const double *B2 = Pc + offB;
        unsigned ah[4], al[4];   // the Hessian weights split into TF32 head and tail
        if constexpr (MIX) {
#pragma unroll
            for (int h = 0; h < 4; h++)
                tf32_split((float)e[h], ah[h], al[h]);
        }
#pragma unroll
        for (int nt = 0; nt < NTL; nt++) {
            if (NT > 0 || nt < NT2) {
                const bool hess = (PPN == 0) || nt < NTH;
                const int col = hess ? nb + nt * 8 : (nt - NTH) * 8;
                if (lowp(nt)) {
                    unsigned bh0, bl0, bh1, bl1;
                    tf32_split((float)B2[col], bh0, bl0);
                    tf32_split((float)B2[col + ldP], bh1, bl1);
                    tmma16x8x8(acc32[nt], al[0], al[2], al[1], al[3], bh0, bh1);
                    tmma16x8x8(acc32[nt], ah[0], ah[2], ah[1], ah[3], bl0, bl1);
                    tmma16x8x8(acc32[nt], ah[0], ah[2], ah[1], ah[3], bh0, bh1);
                } else {
                    // PAIR: even column tiles take the sums, odd ones the differences
                    const bool useE = PAIR ? (nt * 8 < K2e) : hess;
                    const double x0 = useE ? e[0] : eg[0], x1 = useE ? e[1] : eg[1];
                    const double x2 = useE ? e[2] : eg[2], x3 = useE ? e[3] : eg[3];
                    dmma16x8x8(acc[nt], x0, x2, x1, x3, B2[col], B2[col + ldP]);
                }
            }
        }
    };
    int bc = 0;   // buffer of chunk c
    if constexpr (DEPTH == 3) {
        for (int c = 0; c + 1 < nchunks; c++) {
            const int bn = (bc == 2) ? 0 : bc + 1, bf = (bn == 2) ? 0 : bn + 1;
            const bool okWait = wait_chunk(bn);
            // chunk c + 1 visible to all; every warp is done with chunk c - 1 (buffer bf)
            if (__syncthreads_or(!okWait))
                return abandon();
            if (c + 2 < nchunks)
                load_chunk(c + 2, bf);
            double cs[4], co[4];
            gemm1(L.P + bn * chunkDoubles, cs, co);
            gemm2(L.P + bc * chunkDoubles);
            weights(L.P + bn * chunkDoubles, cs, co, e, eg);
            bc = bn;
        }
    } else {
        // two buffers: chunk c + 2 goes into chunk c's buffer once every
        // warp has finished its GEMM2 on chunk c
        for (int c = 0; c + 1 < nchunks; c++) {
            const int bn = bc ^ 1;
            const bool okWait = wait_chunk(bn);
            if (__syncthreads_or(!okWait))
                return abandon();
            double cs[4], co[4];
            gemm1(L.P + bn * chunkDoubles, cs, co);
            gemm2(L.P + bc * chunkDoubles);
            weights(L.P + bn * chunkDoubles, cs, co, e, eg);
            if (c + 2 < nchunks) {
                __syncthreads();
                load_chunk(c + 2, bc);
            }
            bc = bn;
        }
    }
    gemm2(L.P + bc * chunkDoubles);   // the last chunk (waited for by the last iteration)
    if constexpr (MIX) {
#pragma unroll
        for (int nt = 0; nt < NTL; nt++)
            if (lowp(nt))
                for (int h = 0; h < 4; h++)
                    acc[nt][h] = (double)acc32[nt][h];
    }
    __syncthreads();   // the G region overlaps the staged basis
#pragma unroll 1
    for (int step = 0; step < 4; step++) {
        if (qg == step) {
#pragma unroll
            for (int nt = 0; nt < NTL; nt++) {
                if (NT > 0 || nt < NT2) {
                    double *G0 = L.G + r0 * ldG + nt * 8 + 2 * t4;
                    if (step == 0) {
                        G0[0] = acc[nt][0];
                        G0[1] = acc[nt][1];
                        G0[8 * ldG] = acc[nt][2];
                        G0[8 * ldG + 1] = acc[nt][3];
                    } else {
                        G0[0] += acc[nt][0];
                        G0[1] += acc[nt][1];
                        G0[8 * ldG] += acc[nt][2];
                        G0[8 * ldG + 1] += acc[nt][3];
                    }
                }
            }
        }
        __syncthreads();
    }
    facc0 += __shfl_xor_sync(0xffffffffu, facc0, 1);
    facc0 += __shfl_xor_sync(0xffffffffu, facc0, 2);
    facc1 += __shfl_xor_sync(0xffffffffu, facc1, 1);
    facc1 += __shfl_xor_sync(0xffffffffu, facc1, 2);
    if (t4 == 0) {
        L.fpart[r0 * a.ntq + qg] = facc0;
        L.fpart[r1 * a.ntq + qg] = facc1;
    }
    __syncthreads();
    return true;
}

template <int TPW, int NTF, int PPN, int NT, int NBK, int MIX, int PAIR = 0, int NW = 8>
__global__ void __launch_bounds__(NW * 32, NW == 8 ? 1 : 2) newton_kernel(const __grid_constant__ NewtonArgs a)
{
    static_assert(NW == 8 || NTF > 0, "the 4-warp shape runs the fused contractions only");
    constexpr int kThreads = NW * 32, kWarps = NW;
    extern __shared__ __align__(16) double sm[];
    __shared__ int ctl[4];   // [0] problem, [1] done, [2] exhausted, [3] next slot of phase B
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t4 = lane & 3;
    const int T = a.T, MT = a.T / 16, kq = a.kq, ldv = a.ldv, ldE = a.ldE, ldG = a.ldG;
    Layout L = make_layout(sm, a);

    for (int i = tid; i < 4 * T * ldv; i += kThreads)
        L.alpha[i] = 0.0;   // alpha, aold, d, u are contiguous
    for (int i = tid; i < T * SI_N; i += kThreads)
        L.ints[i] = (i % SI_N == SI_STATE) ? S_IDLE : 0;
    for (int i = tid; i <= kStatU64; i += kThreads)
        L.stat[i] = 0ull;
    for (int i = tid; i < 64; i += kThreads)
        L.exptab[i] = a.ex.tab[i];
    for (int i = tid; i < T * SC_N; i += kThreads)
        L.scal[i] = 0.0;
    if (tid == 0) {
        ctl[0] = 0;
        ctl[1] = 0;
        ctl[2] = 0;
    }
    if (tid == 0) {
        for (int b = 0; b < 3; b++)
            mbar_init(&L.bar[b], 1);
        mbar_init_fence();
    }
    __syncthreads();
    int loadedProb = -1;
    unsigned mbPhase = 0;   // parity of the next phase of each chunk mbarrier

    for (;;) {
        // ---- refill idle slots from the work counter of the current problem
        if (tid == 0) {
            int p = ctl[0];
            int nIdle = 0, nActive = 0;
            for (int s = 0; s < T; s++) {
                if (L.ints[s * SI_N + SI_STATE] == S_HELP)   // helpers serve one round
                    L.ints[s * SI_N + SI_STATE] = S_IDLE;
                if (L.ints[s * SI_N + SI_STATE] == S_IDLE)
                    nIdle++;
                else
                    nActive++;
            }
            bool exhausted = ctl[2] != 0;
            while (nIdle > 0) {
                if (exhausted) {
                    if (nActive == 0 && p + 1 < a.nprob) {
                        p++;
                        exhausted = false;
                        continue;
                    }
                    break;
                }
                const NewtonProblem &pb = a.prob[p];
                const bool list = pb.cellList && *pb.countDev >= 0;
                const int count = list ? *pb.countDev : pb.count;
                unsigned base = atomicAdd(pb.queue, (unsigned)nIdle);
                if (base >= (unsigned)count) {
                    exhausted = true;
                    continue;
                }
                int take = min(nIdle, count - (int)base);
                int c = 0;
                for (int s = 0; s < T && c < take; s++) {
                    if (L.ints[s * SI_N + SI_STATE] == S_IDLE) {
                        L.ints[s * SI_N + SI_CELL] = list ? pb.cellList[(int)base + c] : pb.first + (int)base + c;
                        L.ints[s * SI_N + SI_STATE] = S_NEW;
                        c++;
                    }
                }
                nIdle -= take;
                nActive += take;
                if (nIdle > 0)
                    exhausted = true;
            }
            // idle slots once the work counter is exhausted: lend them to
            // slots whose line search is backtracking (plain Newton)
            if (a.optType == 0 && exhausted && nIdle > 0) {
                for (int s = 0; s < T && nIdle > 0; s++) {
                    if (L.ints[s * SI_N + SI_STATE] != S_TRIAL || !(L.scal[s * SC_N + SC_T] < 1.0))
                        continue;
                    int k = 0;
                    for (int h = 0; h < T && nIdle > 0; h++) {
                        if (L.ints[h * SI_N + SI_STATE] == S_IDLE) {
                            L.ints[h * SI_N + SI_STATE] = S_HELP;
                            L.ints[h * SI_N + SI_CELL] = s;
                            L.ints[h * SI_N + SI_ITER] = ++k;
                            nIdle--;
                        }
                    }
                }
            }
            ctl[0] = p;
            ctl[2] = exhausted ? 1 : 0;
            ctl[1] = (nActive == 0) ? 1 : 0;
            ctl[3] = 0;
        }
        __syncthreads();
        if (ctl[1])
            break;
        const NewtonProblem &pb = a.prob[ctl[0]];
        if (ctl[0] != loadedProb) {
            // stage this order's Gaunt contraction table in shared memory
            // (or read it from global memory through L1 where the launch
            // shape leaves no room for it)
            loadedProb = ctl[0];
            // (a compile-time choice: the 8-warp shape's table pointers stay
            // shared-memory pointers, which the loads in phase B rely on)
            if constexpr (NW != 8) {
                if (a.useGaunt) {
                    L.ellVal = const_cast<double *>(pb.ellVal);
                    L.ellIdx = const_cast<unsigned short *>(pb.ellIdx);
                    L.ellPair = const_cast<unsigned short *>(pb.ellPair);
                    L.ellOff = const_cast<int *>(pb.ellOff);
                }
            } else if (a.useGaunt) {
                for (int i = tid; i < pb.ellRows * 32; i += kThreads) {
                    L.ellVal[i] = pb.ellVal[i];
                    L.ellIdx[i] = pb.ellIdx[i];
                }
                for (int i = tid; i < pb.ellChunks * 32; i += kThreads)
                    L.ellPair[i] = pb.ellPair[i];
                for (int i = tid; i <= pb.ellChunks; i += kThreads)
                    L.ellOff[i] = pb.ellOff[i];
            }
        }
        for (int s = warp; s < T; s += kWarps) {
            const int st = L.ints[s * SI_N + SI_STATE];
            if (st == S_NEW)
                (a.optType != 0) ? init_slot_cb(a, pb, L, s, lane, ldv) : init_slot(a, pb, L, s, lane, ldv);
            else if (st == S_HELP)
                init_helper(pb, L, s, lane, ldv);
        }
        __syncthreads();

        // ---- phase A: evaluation contractions over the quadrature
        if constexpr (NTF > 0) {
            if (!phase_a_fused<NTF, PPN, NT, NBK, MIX, PAIR, NW>(a, pb, L, tid, lane, warp, mbPhase))
                return;   // a staged chunk never arrived (error recorded)
        } else {
        const int nb = pb.nb, ldP = pb.ldP, K2p = pb.K2p;
        const int NTH = K2p / 8;
        const int NT2 = NTH + (a.momentType == 1 ? nb / 8 : 0);
        const int ntiles2 = MT * NT2;
        const int nchunks = pb.nqp / kq;
        const int chunkDoubles = kq * ldP + kq;   // rows of a chunk, gaps included (basis_row)
        const int mt1 = warp % MT, ntq = warp / MT;
        double acc[TPW][4];
#pragma unroll
        for (int j = 0; j < TPW; j++)
            acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0;
        double facc0 = 0.0, facc1 = 0.0;
        const int r0 = mt1 * 16 + g, r1 = r0 + 8;
        const double dl0 = L.scal[r0 * SC_N + SC_DELTA], dl1 = L.scal[r1 * SC_N + SC_DELTA];

        auto load_chunk = [&](int c, int buf) {
            const double *src = pb.P + (size_t)c * chunkDoubles;
            double *dst = L.P + buf * chunkDoubles;
            for (int i = tid; i < chunkDoubles / 2; i += kThreads)
                cp_async16(dst + 2 * i, src + 2 * i);
            cp_async_commit();
        };
        if (a.doubleBuffer)
            load_chunk(0, 0);
        for (int c = 0; c < nchunks; c++) {
            int buf = a.doubleBuffer ? (c & 1) : 0;
            if (a.doubleBuffer) {
                if (c + 1 < nchunks) {
                    load_chunk(c + 1, buf ^ 1);
                    cp_async_wait<1>();
                } else {
                    cp_async_wait<0>();
                }
            } else {
                load_chunk(c, 0);
                cp_async_wait<0>();
            }
            __syncthreads();
            const double *Pb = L.P + buf * chunkDoubles;
            // GEMM1: S = alpha . P^T for this warp's 16 x 8 tile
            {
                double cs[4] = {0.0, 0.0, 0.0, 0.0};
                const double *A0 = L.alpha + r0 * ldv, *A1 = L.alpha + r1 * ldv;
                const double *B = Pb + basis_row(ntq * 8 + g, ldP);
                for (int k0 = 0; k0 < nb; k0 += 8)
                    dmma16x8x8(cs, A0[k0 + t4], A1[k0 + t4], A0[k0 + t4 + 4], A1[k0 + t4 + 4],
                               B[k0 + t4], B[k0 + t4 + 4]);
                const int ql = ntq * 8 + 2 * t4;
                const int qg = c * kq + ql;
                const double w0 = __ldg(&pb.w[qg]), w1 = __ldg(&pb.w[qg + 1]);
                if (a.momentType == 0) {
                    const double invL = a.ex.invL, L1 = a.ex.L1, L2 = a.ex.L2;
                    double ex4[4];
                    fast_exp_n<4>(ex4, cs, L.exptab, invL, L1, L2);
                    double e0 = w0 * ex4[0], e1 = w1 * ex4[1], e2 = w0 * ex4[2], e3 = w1 * ex4[3];
                    L.E[r0 * ldE + ql] = e0;
                    L.E[r0 * ldE + ql + 1] = e1;
                    L.E[r1 * ldE + ql] = e2;
                    L.E[r1 * ldE + ql + 1] = e3;
                    facc0 += e0 + e1;
                    facc1 += e2 + e3;
                } else {
                    // fobj.cpp:408-434 and :196-210 (PPn)
                    double wv[2] = {w0, w1};
#pragma unroll
                    for (int h = 0; h < 4; h++) {
                        double dl = (h < 2) ? dl0 : dl1;
                        double ww = wv[h & 1];
                        double k = 0.5 * cs[h];
                        double s2 = sqrt(k * k + dl);
                        double G = k + s2;
                        if (k < 0)
                            G = -dl / (k - sqrt(k * k + dl));
                        double eh = 0.5 * ww * (G / s2);
                        double eg = ww * G;
                        double ft = ww * (k * G - 0.5 * dl + dl * log(G));
                        int row = (h < 2) ? r0 : r1;
                        L.E[row * ldE + ql + (h & 1)] = eh;
                        L.Eg[row * ldE + ql + (h & 1)] = eg;
                        if (h < 2)
                            facc0 += ft;
                        else
                            facc1 += ft;
                    }
                }
            }
            __syncthreads();
            // GEMM2: G += E . Phess (and Eg . P for the PPn gradient)
            for (int k0 = 0; k0 < kq; k0 += 8) {
#pragma unroll
                for (int j = 0; j < TPW; j++) {
                    int ti = warp + kWarps * j;
                    if (ti < ntiles2) {
                        int mt2 = ti % MT, nt2 = ti / MT;
                        const double *Ab = (nt2 < NTH) ? L.E : L.Eg;
                        int col = (nt2 < NTH) ? nb + nt2 * 8 : (nt2 - NTH) * 8;
                        const double *A0 = Ab + (mt2 * 16 + g) * ldE + k0 + t4;
                        const double *A1 = A0 + 8 * ldE;
                        const double *B0 = Pb + basis_row(k0 + t4, ldP) + col + g;
                        // row k0 + t4 + 4 is 4 * ldP + 4 doubles further (one gap)
                        dmma16x8x8(acc[j], A0[0], A1[0], A0[4], A1[4], B0[0], B0[4 * ldP + 4]);
                    }
                }
            }
            __syncthreads();
        }
        // dump accumulators and f partial sums
#pragma unroll
        for (int j = 0; j < TPW; j++) {
            int ti = warp + kWarps * j;
            if (ti < ntiles2) {
                int mt2 = ti % MT, nt2 = ti / MT;
                double *G0 = L.G + (mt2 * 16 + g) * ldG + nt2 * 8 + 2 * t4;
                G0[0] = acc[j][0];
                G0[1] = acc[j][1];
                G0[8 * ldG] = acc[j][2];
                G0[8 * ldG + 1] = acc[j][3];
            }
        }
        facc0 += __shfl_xor_sync(0xffffffffu, facc0, 1);
        facc0 += __shfl_xor_sync(0xffffffffu, facc0, 2);
        facc1 += __shfl_xor_sync(0xffffffffu, facc1, 1);
        facc1 += __shfl_xor_sync(0xffffffffu, facc1, 2);
        if (t4 == 0) {
            L.fpart[r0 * a.ntq + ntq] = facc0;
            L.fpart[r1 * a.ntq + ntq] = facc1;
        }
        __syncthreads();
        }

        // ---- phase B: per-slot Newton logic, one warp per slot.  Warps take
        // the slots from a shared counter, so a warp that drew a cell needing
        // the full Newton step (factorisation, inverse, condition estimate)
        // does not also hold back cells that converged at this evaluation;
        // a slot's logic touches only its own state and its helpers'.
        for (;;) {
            int s = 0;
            if (lane == 0)
                s = atomicAdd(&ctl[3], 1);
            s = __shfl_sync(0xffffffffu, s, 0);
            if (s >= T)
                break;
            int st = L.ints[s * SI_N + SI_STATE];
            if (st == S_NEWTON || st == S_TRIAL) {
                if (a.optType != 0)
                    slot_logic_cb(a, pb, L, s, lane, warp);
                else
                    slot_logic(a, pb, L, s, lane, warp, PPN == 0 && MIX == 0);
            }
        }
        if constexpr (NTF > 0)
            fence_proxy_async_smem();   // this round's shared-memory writes before the next bulk copies
        __syncthreads();
    }

    // flush CTA statistics (hist, totalIter, numSolves, trials are contiguous)
    if (tid < kStatU64) {
        unsigned long long v = L.stat[tid];
        if (v)
            atomicAdd(&a.stats->hist[0] + tid, v);
    } else if (tid == kStatU64) {
        atomicMax(&a.stats->maxIter, *(int *)&L.stat[kStatU64]);
    }
}

// ---------------------------------------------------------------------------
// Screening pass (Mn, FP64, direction pairs): the first evaluation of every
// cell of a launch, with the gradient columns of G only (the first n Gaunt or
// product columns, laid out as in the full layout's parity groups, so each
// sum is the full evaluation's bit for bit).  A cell whose first Newton
// iteration converges with the condition test decided by the exponent-range
// bound (the outcome of opt.cpp:244-306 at that evaluation) is finished here
// as K1 would finish it; every other cell is appended to pb.pendList, and K1
// solves those from their starts (the screening evaluation is not counted).
// Without the Hessian columns, the Newton state and the Gaunt table, a CTA
// of 8 warps fits twice per SM.
__device__ void screen_logic(const NewtonArgs &a, const NewtonProblem &pb, Layout &L, int s, int lane)
{
    const int n = pb.n, ldv = a.ldv;
    const bool act = lane < n;
    int *si = L.ints + s * SI_N;
    const double *sc = L.scal + s * SC_N;
    const double ui = act ? L.u[s * ldv + lane] : 0.0;
    const double ai = act ? L.alpha[s * ldv + lane] : 0.0;
    bool conv = false;
    if (lane == 0)
        atomicAdd(&L.stat[kNumReg + 5], 1ull);
    // slot_logic's stopping-test conditions at iteration 1 (t = 1)
    if (!(a.tolGamma > 0.0) && 1 < si[SI_MAXITER]) {
        const double g0 = act ? hessian_row0(a, pb, L.G + s * a.ldG, lane) / pb.p0 - ui : 0.0;
        conv = sqrt(warp_sum(g0 * g0)) <= sc[SC_RTOL] && exponent_range_bound(a, pb, ai, lane);
        if (conv) {
            __syncwarp();
            if (lane == 0) {
                si[SI_ITER] = 1;
                si[SI_TOTAL] = 1;
            }
            __syncwarp();
            converge(a, pb, L, s, ui, ai, g0, lane);
            if (lane == 0)
                atomicAdd(&L.stat[kNumReg + 4], 1ull);
        }
    }
    if (!conv && lane == 0) {
        pb.pendList[atomicAdd(pb.pendCount, 1)] = si[SI_CELL];
        si[SI_STATE] = S_IDLE;
    }
}

template <int NT, int NBK>
__global__ void __launch_bounds__(256, 2) screen_kernel(const __grid_constant__ NewtonArgs a)
{
    constexpr int kThreads = 256, kWarps = 8;
    extern __shared__ __align__(16) double sm[];
    __shared__ int ctl[4];   // [0] done, [1] next slot of the test, [2] slots claimed, [3] counter exhausted
    __shared__ int repValid, repHits;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int T = a.T, ldv = a.ldv;
    const NewtonProblem &pb = a.prob[0];
    const int n = pb.n;
    Layout L = make_layout(sm, a);
    // The representative: the start (u, alpha) of a cell this CTA settled,
    // as loaded, and the results written for it.  A later cell whose start
    // is the same, bit for bit, takes those results without an evaluation
    // (the first evaluation is a function of the start alone; not with
    // predicted starts, which enter it too).  Floor cells that no
    // perturbation has reached share one start.
    double *repIn = L.Eg, *repOut = L.Eg + 2 * ldv;   // [2][ldv] each: u, alpha
    double *rawU = L.aold, *rawA = L.d;               // per slot: the start as loaded
    const bool dedup = pb.alphaStart == nullptr;
    for (int i = tid; i < 4 * T * ldv; i += kThreads)
        L.alpha[i] = 0.0;
    for (int i = tid; i < T * SI_N; i += kThreads)
        L.ints[i] = (i % SI_N == SI_STATE) ? S_IDLE : 0;
    for (int i = tid; i <= kStatU64; i += kThreads)
        L.stat[i] = 0ull;
    for (int i = tid; i < 64; i += kThreads)
        L.exptab[i] = a.ex.tab[i];
    for (int i = tid; i < T * SC_N; i += kThreads)
        L.scal[i] = 0.0;
    if (tid == 0) {
        for (int b = 0; b < 3; b++)
            mbar_init(&L.bar[b], 1);
        mbar_init_fence();
        repValid = 0;
    }
    __syncthreads();
    unsigned mbPhase = 0;
    if (pb.gateCount && *pb.gateCount < pb.gateMin)
        return;   // most cells iterate: K1 solves them all, in one pass
    for (;;) {
        if (tid == 0) {
            ctl[2] = 0;
            ctl[3] = 0;
            repHits = 0;
        }
        __syncthreads();
        // Refill, kBatch candidates per warp at a time (their loads in
        // flight together): cells whose previous solve took more than one
        // iteration go straight to K1's list, copies of the representative
        // are finished here, the rest take slots (a cell drawn after the
        // slots ran out goes to the list).
        constexpr int kBatch = 4;
        for (;;) {
            int base = -1;
            if (lane == 0 && *(volatile int *)&ctl[2] < T && !*(volatile int *)&ctl[3]) {
                const unsigned item = atomicAdd(pb.queue, (unsigned)kBatch);
                if (item < (unsigned)pb.count)
                    base = (int)item;
                else
                    ctl[3] = 1;
            }
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base < 0)
                break;
            const int cnt = min(kBatch, pb.count - base);
            double ub[kBatch], ab[kBatch];
#pragma unroll
            for (int b = 0; b < kBatch; b++) {
                const size_t at = (size_t)(pb.first + base + b) * n + lane;
                ub[b] = (b < cnt && lane < n) ? pb.u[at] : 0.0;
                ab[b] = (b < cnt && lane < n) ? pb.alpha[at] : 0.0;
            }
            const int itb = (lane < cnt && pb.iters) ? pb.iters[pb.first + base + lane] : 0;
#pragma unroll
            for (int b = 0; b < kBatch; b++) {
                if (b >= cnt)
                    break;
                const int cell = pb.first + base + b;
                const double uk = ub[b], ak = ab[b];
                if (__shfl_sync(0xffffffffu, itb, b) > 1) {
                    if (lane == 0)
                        pb.pendList[atomicAdd(pb.pendCount, 1)] = cell;
                    continue;
                }
                if (dedup && *(volatile int *)&repValid) {
                    const bool same = lane >= n ||
                                      (__double_as_longlong(uk) == __double_as_longlong(repIn[lane]) &&
                                       __double_as_longlong(ak) == __double_as_longlong(repIn[ldv + lane]));
                    if (__all_sync(0xffffffffu, same)) {
                        if (lane < n) {
                            pb.u[(size_t)cell * n + lane] = repOut[lane];
                            pb.alpha[(size_t)cell * n + lane] = repOut[ldv + lane];
                            if (a.momentsOld != nullptr) {
                                const int i = cell / a.NY, j = cell % a.NY;
                                if (i >= 2 && i < a.NX - 2 && j >= 2 && j < a.NY - 2)
                                    a.momentsOld[(size_t)cell * n + lane] = uk;
                            }
                        }
                        if (lane == 0) {
                            // finish_slot's records of a first-iteration convergence
                            if (pb.iters)
                                pb.iters[cell] = 1;
                            if (pb.regs)
                                pb.regs[cell] = kRegularizations[0];
                            if (pb.status)
                                pb.status[cell] = 0;
                            atomicAdd(&L.stat[0], 1ull);
                            atomicAdd(&L.stat[kNumReg], 1ull);
                            atomicAdd(&L.stat[kNumReg + 1], 1ull);
                            atomicMax((int *)&L.stat[kStatU64], 1);
                            atomicAdd(&L.stat[kNumReg + 4], 1ull);
                            atomicAdd(&repHits, 1);
                        }
                        continue;
                    }
                }
                int s = 0;
                if (lane == 0)
                    s = atomicAdd(&ctl[2], 1);
                s = __shfl_sync(0xffffffffu, s, 0);
                if (s < T) {
                    if (lane < ldv) {
                        rawU[s * ldv + lane] = uk;
                        rawA[s * ldv + lane] = ak;
                    }
                    if (lane == 0) {
                        L.ints[s * SI_N + SI_CELL] = cell;
                        L.ints[s * SI_N + SI_STATE] = S_NEW;
                    }
                } else if (lane == 0) {
                    pb.pendList[atomicAdd(pb.pendCount, 1)] = cell;
                }
            }
        }
        __syncthreads();
        const int filled = min(ctl[2], T);
        if (tid == 0) {
            for (int s = filled; s < T; s++)
                L.ints[s * SI_N + SI_STATE] = S_IDLE;
            ctl[0] = (filled == 0);
            ctl[1] = 0;
        }
        __syncthreads();
        if (ctl[0])
            break;
        for (int s = warp; s < T; s += kWarps)
            if (L.ints[s * SI_N + SI_STATE] == S_NEW)
                init_slot(a, pb, L, s, lane, ldv);
        __syncthreads();
        if (!phase_a_fused<8, 0, NT, NBK, 0, 1, 8>(a, pb, L, tid, lane, warp, mbPhase))
            return;   // a staged chunk never arrived (error recorded)
        for (;;) {
            int s = 0;
            if (lane == 0)
                s = atomicAdd(&ctl[1], 1);
            s = __shfl_sync(0xffffffffu, s, 0);
            if (s >= T)
                break;
            if (L.ints[s * SI_N + SI_STATE] == S_NEWTON)
                screen_logic(a, pb, L, s, lane);
        }
        fence_proxy_async_smem();   // this round's shared-memory writes before the next bulk copies
        __syncthreads();
        // a new representative when the current one found no copy this
        // round: the first slot settled here (SI_ITER = 1)
        if (dedup && warp == 0 && repHits == 0) {
            const unsigned m = __ballot_sync(0xffffffffu, lane < filled && L.ints[lane * SI_N + SI_ITER] == 1);
            if (m) {
                const int s = __ffs(m) - 1, cell = L.ints[s * SI_N + SI_CELL];
                if (lane < ldv) {
                    repIn[lane] = rawU[s * ldv + lane];
                    repIn[ldv + lane] = rawA[s * ldv + lane];
                    repOut[lane] = (lane < n) ? pb.u[(size_t)cell * n + lane] : 0.0;
                    repOut[ldv + lane] = (lane < n) ? pb.alpha[(size_t)cell * n + lane] : 0.0;
                }
                __syncwarp();
                if (lane == 0)
                    repValid = 1;
            }
        }
    }
    if (tid < kStatU64) {
        unsigned long long v = L.stat[tid];
        if (v)
            atomicAdd(&a.stats->hist[0] + tid, v);
    } else if (tid == kStatU64) {
        atomicMax(&a.stats->maxIter, *(int *)&L.stat[kStatU64]);
    }
}

__global__ void screen_gate_kernel(const int *iters, int first, int count, int *out)
{
    int v = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
        v += (iters[first + i] <= 1) ? 1 : 0;
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, m);
    if ((threadIdx.x & 31) == 0 && v)
        atomicAdd(out, v);
}

template <int NT, int NBK>
cudaError_t screen_run(const NewtonArgs &a, int grid, cudaStream_t stream, int mode, int *occ)
{
    auto *k = screen_kernel<NT, NBK>;
    if (mode == 1)
        return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, a.smemBytes);
    if (mode == 2) {
        int b = 0;
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k, 256, a.smemBytes);
        *occ = b < 1 ? 1 : b;
        return e;
    }
    k<<<grid, 256, a.smemBytes, stream>>>(a);
    return cudaGetLastError();
}

// One kernel instance: mode 0 launches it, 1 sets its shared-memory limit,
// 2 writes its resident CTAs per SM to *occ.
template <int TPW, int NTF, int PPN, int NT, int NBK, int MIX = 0, int PAIR = 0, int NW = 8>
cudaError_t newton_run(const NewtonArgs &a, int grid, cudaStream_t stream, int mode, int *occ)
{
    auto *k = newton_kernel<TPW, NTF, PPN, NT, NBK, MIX, PAIR, NW>;
    if (mode == 1)
        return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, a.smemBytes);
    if (mode == 2) {
        int b = 0;
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k, NW * 32, a.smemBytes);
        *occ = b < 1 ? 1 : b;
        return e;
    }
    k<<<grid, NW * 32, a.smemBytes, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace
}  // namespace clb
