// capi.cu -- implementation of the C ABI declared in include/closures_gpu.h.
//
// Owns the device state of one grid (moments, alpha, saved moments, sigma
// fields), the device copies of the angular set-up in the layouts the
// kernels want, one stream and the captured RK2 graph.
#include "closures_gpu.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cstdlib>
#include <map>
#include <mutex>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../host/angular.h"
#include "common.cuh"
#include "flux.cuh"
#include "newton.cuh"

using namespace clb;

static std::atomic<long long> g_launches{0};
int clb_mlp_reserve_for(cl_mlp *m, size_t rows);
static thread_local std::string g_global_err;

#define CUDA_TRY(ctx, call)                                                                    \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            (ctx)->err = std::string(#call) + ": " + cudaGetErrorString(e_);                   \
            return CL_ERR_CUDA;                                                                \
        }                                                                                      \
    } while (0)

namespace {

int round_up(int x, int m) { return (x + m - 1) / m * m; }

// cl_step_host: bands of cells whose upload and first-stage solve overlap
constexpr int kHostBands = 4;

// Device copy of one moment order's angular data in the kernels' layouts.
struct DeviceBasis {
    int n = 0, n2 = 0, nq = 0, nb = 0, K2p = 0, nqp = 0, ldP = 0, ldPf = 0, useGaunt = 0;
    // flux layout: nqpF rows of Pf (directions, or one direction of each
    // pair with fluxPaired), nbF columns (nbeF even-degree ones first when
    // paired); xi, eta, cxw, cyw in chunk order, 16 directions per chunk
    int nqpF = 0, nbF = 0, nbeF = 0, fluxPaired = 0;
    short *fbinv = nullptr;                        // [nbF] moment of each flux column (paired)
    // direction pairs (Newton layout): basis and Hessian columns grouped by
    // degree parity, even group first (nbe, K2e columns, multiples of 8)
    int paired = 0, nbe = 0, K2e = 0;
    short *binv = nullptr;                         // [nb] moment of each basis column, -1 padding
    int *pcol = nullptr;                           // [n(n+1)/2] G column of each product (no Gaunt)
    double p0 = 0;
    double *P = nullptr, *w = nullptr;            // Newton layout
    double *Pf = nullptr, *xi = nullptr, *eta = nullptr, *cxw = nullptr, *cyw = nullptr;  // flux
    int *hoff = nullptr, *hidx = nullptr;
    double *hval = nullptr;
    unsigned short *pairs = nullptr;
    unsigned short *ellPair = nullptr, *ellIdx = nullptr;
    double *ellVal = nullptr;
    int *ellOff = nullptr;
    int ellChunks = 0, ellRows = 0;
    // row 0 of the Gaunt contraction (CSR rows (0, j), layout columns) and
    // the eigenvalue bounds of the quadrature Gram matrix of the moment basis
    int *r0off = nullptr;
    unsigned short *r0idx = nullptr;
    double *r0val = nullptr;
    double *rangeC = nullptr;   // max_q |p_k(q)|, then max_q of each degree's norm
    double gramLo = 0, gramHi = 0;
    int maxDeg = 0;
    // screening layout (paired): the basis columns and the gradient columns
    // of G only (the first n Gaunt or product columns in the parity groups)
    double *Ps = nullptr;
    int ldPs = 0, K2ps = 0, K2es = 0;
    unsigned short *r0idxS = nullptr;   // row-0 Gaunt entries in the screening columns
    int *pcolS = nullptr;               // products (k, 0) in the screening columns
    int screenOk = 0;

    void release()
    {
        cudaFree(P);
        cudaFree(w);
        cudaFree(Pf);
        cudaFree(xi);
        cudaFree(eta);
        cudaFree(cxw);
        cudaFree(cyw);
        cudaFree(hoff);
        cudaFree(hidx);
        cudaFree(hval);
        cudaFree(pairs);
        cudaFree(ellPair);
        cudaFree(ellIdx);
        cudaFree(ellVal);
        cudaFree(ellOff);
        cudaFree(binv);
        cudaFree(pcol);
        cudaFree(fbinv);
        cudaFree(r0off);
        cudaFree(r0idx);
        cudaFree(r0val);
        cudaFree(rangeC);
        cudaFree(Ps);
        cudaFree(r0idxS);
        cudaFree(pcolS);
        *this = DeviceBasis();
    }
};

template <class T>
cudaError_t upload(T **dst, const std::vector<T> &src)
{
    cudaError_t e = cudaMalloc((void **)dst, sizeof(T) * (src.empty() ? 1 : src.size()));
    if (e != cudaSuccess)
        return e;
    if (!src.empty())
        e = cudaMemcpy(*dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice);
    return e;
}

// Degree of each z-even harmonic in the basis order (degree l has l + 1).
static void harmonic_degrees(int count, std::vector<int> &deg)
{
    deg.resize(count);
    int k = 0;
    for (int l = 0; k < count; l++)
        for (int m = 0; m <= l && k < count; m++)
            deg[k++] = l;
}

// Columns of one group layout: even-parity entries first, then odd, each
// group padded to a multiple of 8; col[i] = position of entry i.
static void parity_columns(const std::vector<int> &deg, int paired, std::vector<int> &col, int &evenCols,
                           int &total)
{
    const int cnt = (int)deg.size();
    col.resize(cnt);
    if (!paired) {
        for (int i = 0; i < cnt; i++)
            col[i] = i;
        evenCols = 0;
        total = round_up(cnt, 8);
        return;
    }
    int ne = 0;
    for (int i = 0; i < cnt; i++)
        ne += (deg[i] % 2 == 0);
    evenCols = round_up(ne, 8);
    int ie = 0, io = 0;
    for (int i = 0; i < cnt; i++)
        col[i] = (deg[i] % 2 == 0) ? ie++ : evenCols + io++;
    total = evenCols + round_up(cnt - ne, 8);
}

// n, n2, nq, w, xi, eta, p[nq*n2], Gaunt CSR -> device layouts.
//
// Newton layout with `paired`: the directions phi and phi + pi of one
// Gauss-Legendre level (q and q + Q in the reference's order, momopt_init.cpp
// :181-186) have the same weight and basis values equal up to the degree
// parity, p_l(q + Q) = (-1)^l p_l(q) (for the Gaunt basis and for products
// likewise).  Only the first direction of each pair is stored, with the
// columns grouped by parity, and the kernel evaluates both directions from
// the two half sums alpha_even . p_even +- alpha_odd . p_odd.
cudaError_t build_device_basis(DeviceBasis &B, int n, int n2, int nq, int useGaunt, const double *w,
                               const double *xi, const double *eta, const double *p, const int *goff,
                               const int *gidx, const double *gval, int gnnz, int paired = 0,
                               int fluxPaired = 0)
{
    B.n = n;
    B.n2 = n2;
    B.nq = nq;
    B.useGaunt = useGaunt;
    const int Q = (int)std::lround(std::sqrt((double)nq));
    if (Q * Q != nq || Q % 2 != 0)
        paired = fluxPaired = 0;
    B.paired = paired;
    const int K2 = useGaunt ? n2 : n * (n + 1) / 2;
    std::vector<unsigned short> prod(n * (n + 1) / 2);
    product_columns(n, prod.data());
    std::vector<int> degB, degH, colB, colH;
    harmonic_degrees(n, degB);
    if (useGaunt) {
        harmonic_degrees(n2, degH);
    } else {
        degH.resize(K2);
        for (int c = 0; c < K2; c++)
            degH[c] = degB[prod[c] >> 8] + degB[prod[c] & 255];
    }
    parity_columns(degB, paired, colB, B.nbe, B.nb);
    parity_columns(degH, paired, colH, B.K2e, B.K2p);
    const int rows = paired ? nq / 2 : nq;
    B.nqp = round_up(rows, 32);
    int ldP = B.nb + B.K2p;
    while (ldP % 16 != 4)
        ldP++;
    B.ldP = ldP;
    B.p0 = p[0];
    std::vector<double> P((size_t)B.nqp * ldP + B.nqp, 0.0), W(B.nqp, 0.0);
    for (int r = 0; r < rows; r++) {
        const int q = paired ? (r / Q) * 2 * Q + r % Q : r;
        const double *pq = p + (size_t)q * n2;
        double *row = &P[(size_t)basis_row(r, ldP)];
        for (int k = 0; k < n; k++)
            row[colB[k]] = pq[k];
        if (useGaunt) {
            for (int k = 0; k < n2; k++)
                row[B.nb + colH[k]] = pq[k];
        } else {
            for (int c = 0; c < K2; c++)
                row[B.nb + colH[c]] = pq[prod[c] >> 8] * pq[prod[c] & 255];
        }
        W[r] = w[q];
        P[(size_t)basis_wgap(r, ldP)] = w[q];
    }
    // Flux layout.  A chunk holds 16 directions: 16 rows of Pf, or with
    // fluxPaired 8 rows (pairs r) whose directions are q(r) and q(r) + Q,
    // the chunk's directions 0..7 and 8..15.  The partner's xi, eta and
    // weights are its own values (the upwind branch and the flux weight are
    // per direction); only the basis row is shared.
    std::vector<int> colF;
    parity_columns(degB, fluxPaired, colF, B.nbeF, B.nbF);
    B.fluxPaired = fluxPaired;
    B.ldPf = B.nbF + 4;
    const int fchunks = fluxPaired ? (nq / 2 + 7) / 8 : (nq + 15) / 16;
    const int frows = fluxPaired ? 8 : 16;
    B.nqpF = fchunks * frows;
    std::vector<double> Pf((size_t)B.nqpF * B.ldPf, 0.0), XI(fchunks * 16, 0.0), ET(fchunks * 16, 0.0),
        CX(fchunks * 16, 0.0), CY(fchunks * 16, 0.0);
    for (int r = 0; r < (fluxPaired ? nq / 2 : nq); r++) {
        const int q = fluxPaired ? (r / Q) * 2 * Q + r % Q : r;
        const double *pq = p + (size_t)q * n2;
        for (int k = 0; k < n; k++)
            Pf[(size_t)r * B.ldPf + colF[k]] = pq[k];
        for (int h = 0; h < (fluxPaired ? 2 : 1); h++) {
            const int qq = q + h * Q;
            const int d = fluxPaired ? (r / 8) * 16 + h * 8 + r % 8 : r;
            XI[d] = xi[qq];
            ET[d] = eta[qq];
            CX[d] = xi[qq] * w[qq];
            CY[d] = eta[qq] * w[qq];
        }
    }
    std::vector<unsigned short> &pairs = prod;
    // Gram matrix M = sum_q w_q p(q) p(q)^T of the moment basis: Gershgorin
    // bounds of its eigenvalues, widened by 1e-12 of the largest diagonal
    // entry for the rounding of the sums (gramLo = 0 when not positive)
    {
        std::vector<double> M((size_t)n * n, 0.0);
        for (int q = 0; q < nq; q++) {
            const double *pq = p + (size_t)q * n2;
            for (int i = 0; i < n; i++)
                for (int j = 0; j < n; j++)
                    M[(size_t)i * n + j] += w[q] * pq[i] * pq[j];
        }
        double lo = 0.0, hi = 0.0, dmax = 0.0;
        for (int i = 0; i < n; i++) {
            double r = 0.0;
            for (int j = 0; j < n; j++)
                if (j != i)
                    r += std::fabs(M[(size_t)i * n + j]);
            const double d = M[(size_t)i * n + i];
            lo = (i == 0) ? d - r : std::min(lo, d - r);
            hi = std::max(hi, d + r);
            dmax = std::max(dmax, std::fabs(d));
        }
        lo -= 1e-12 * dmax;
        hi += 1e-12 * dmax;
        B.gramLo = lo > 0.0 ? lo : 0.0;
        B.gramHi = hi;
    }
    // bounds of |alpha . p(q) - alpha_0 p_0| from the coefficients: the
    // largest |p_k(q)| and the largest norm of each degree's values over q,
    // rounded up by 1e-12
    B.maxDeg = degB[n - 1];
    std::vector<double> rangeC(n + B.maxDeg + 1, 0.0);
    for (int q = 0; q < nq; q++) {
        const double *pq = p + (size_t)q * n2;
        std::vector<double> sq(B.maxDeg + 1, 0.0);
        for (int k = 0; k < n; k++) {
            rangeC[k] = std::max(rangeC[k], std::fabs(pq[k]));
            sq[degB[k]] += pq[k] * pq[k];
        }
        for (int l = 0; l <= B.maxDeg; l++)
            rangeC[n + l] = std::max(rangeC[n + l], std::sqrt(sq[l]));
    }
    for (auto &x : rangeC)
        x *= 1.0 + 1e-12;
    cudaError_t e;
    if ((e = upload(&B.rangeC, rangeC)) != cudaSuccess) return e;
    if ((e = upload(&B.P, P)) != cudaSuccess) return e;
    if ((e = upload(&B.w, W)) != cudaSuccess) return e;
    if ((e = upload(&B.Pf, Pf)) != cudaSuccess) return e;
    if ((e = upload(&B.xi, XI)) != cudaSuccess) return e;
    if ((e = upload(&B.eta, ET)) != cudaSuccess) return e;
    if ((e = upload(&B.cxw, CX)) != cudaSuccess) return e;
    if ((e = upload(&B.cyw, CY)) != cudaSuccess) return e;
    if ((e = upload(&B.pairs, pairs)) != cudaSuccess) return e;
    if (paired) {
        std::vector<short> binv(B.nb, (short)-1);
        for (int k = 0; k < n; k++)
            binv[colB[k]] = (short)k;
        if ((e = upload(&B.binv, binv)) != cudaSuccess) return e;
        if (!useGaunt) {
            std::vector<int> pcol(colH.begin(), colH.end());
            if ((e = upload(&B.pcol, pcol)) != cudaSuccess) return e;
        }
    }
    if (fluxPaired) {
        std::vector<short> fbinv(B.nbF, (short)-1);
        for (int k = 0; k < n; k++)
            fbinv[colF[k]] = (short)k;
        if ((e = upload(&B.fbinv, fbinv)) != cudaSuccess) return e;
    }
    if (useGaunt) {
        std::vector<int> off(goff, goff + n * n + 1), idx(gidx, gidx + gnnz);
        std::vector<double> val(gval, gval + gnnz);
        if ((e = upload(&B.hoff, off)) != cudaSuccess) return e;
        if ((e = upload(&B.hidx, idx)) != cudaSuccess) return e;
        if ((e = upload(&B.hval, val)) != cudaSuccess) return e;
        const int chunks = gaunt_ell_chunks(n), maxRows = 32 * chunks * 64;
        std::vector<unsigned short> epair(chunks * 32), eidx((size_t)maxRows * 32);
        std::vector<double> eval((size_t)maxRows * 32);
        std::vector<int> eoff(chunks + 1);
        int rows2 = build_gaunt_ell(n, goff, gidx, gval, epair.data(), eidx.data(), eval.data(), eoff.data(),
                                    maxRows);
        if (rows2 < 0)
            return cudaErrorInvalidValue;
        eidx.resize((size_t)rows2 * 32);
        eval.resize((size_t)rows2 * 32);
        for (auto &x : eidx)   // G columns in the layout's order
            x = (unsigned short)colH[x];
        B.ellChunks = chunks;
        B.ellRows = rows2;
        // pairs (0, j) are the Gaunt table's rows j = 0 .. n-1 (row i n + j, i <= j)
        std::vector<int> r0off(n + 1);
        std::vector<unsigned short> r0idx;
        std::vector<double> r0val;
        for (int j = 0; j <= n; j++)
            r0off[j] = goff[j] - goff[0];
        for (int k = goff[0]; k < goff[n]; k++) {
            r0idx.push_back((unsigned short)colH[gidx[k]]);
            r0val.push_back(gval[k]);
        }
        if ((e = upload(&B.r0off, r0off)) != cudaSuccess) return e;
        if ((e = upload(&B.r0idx, r0idx)) != cudaSuccess) return e;
        if ((e = upload(&B.r0val, r0val)) != cudaSuccess) return e;
        if ((e = upload(&B.ellPair, epair)) != cudaSuccess) return e;
        if ((e = upload(&B.ellIdx, eidx)) != cudaSuccess) return e;
        if ((e = upload(&B.ellVal, eval)) != cudaSuccess) return e;
        if ((e = upload(&B.ellOff, eoff)) != cudaSuccess) return e;
    }
    if (paired) {
        // Screening layout: the gradient needs G columns k < n (Gaunt) or the
        // products (k, 0) (both of degree deg k).  In the full layout they are
        // the first entries of their parity group, so here they keep their
        // positions within the group (and within their 8-column tile), the
        // odd group starting at K2es.
        int ne = 0;
        for (int k = 0; k < n; k++)
            ne += (degB[k] % 2 == 0);
        B.K2es = round_up(ne, 8);
        B.K2ps = B.K2es + round_up(n - ne, 8);
        std::vector<int> colS(n);
        bool ok = true;
        for (int k = 0; k < n; k++) {
            colS[k] = (degB[k] % 2 == 0) ? colH[k] : colH[k] - B.K2e + B.K2es;
            ok = ok && (degH[k] == degB[k]) && colS[k] >= 0 && colS[k] < B.K2ps;
        }
        int ldPs = B.nb + B.K2ps;
        while (ldPs % 16 != 4)
            ldPs++;
        B.ldPs = ldPs;
        std::vector<double> Ps((size_t)B.nqp * ldPs + B.nqp, 0.0);
        for (int r = 0; r < rows; r++) {
            const int q = (r / Q) * 2 * Q + r % Q;
            const double *pq = p + (size_t)q * n2;
            double *row = &Ps[(size_t)basis_row(r, ldPs)];
            for (int k = 0; k < n; k++)
                row[colB[k]] = pq[k];
            for (int k = 0; k < n; k++)
                row[B.nb + colS[k]] = useGaunt ? pq[k] : pq[prod[k] >> 8] * pq[prod[k] & 255];
            Ps[(size_t)basis_wgap(r, ldPs)] = w[q];
        }
        if ((e = upload(&B.Ps, Ps)) != cudaSuccess) return e;
        if (useGaunt) {
            std::vector<unsigned short> r0s;
            for (int k = goff[0]; k < goff[n]; k++) {
                ok = ok && gidx[k] < n;
                r0s.push_back((unsigned short)(gidx[k] < n ? colS[gidx[k]] : 0));
            }
            if ((e = upload(&B.r0idxS, r0s)) != cudaSuccess) return e;
        } else {
            if ((e = upload(&B.pcolS, colS)) != cudaSuccess) return e;
        }
        B.screenOk = ok ? 1 : 0;
    }
    return cudaSuccess;
}

// Direction-pair layout counts: column tiles and k-steps of the fused
// evaluation (the exact-instance key), without building anything.
static void paired_counts(int n, int n2, int useGaunt, int &nt, int &nbk)
{
    std::vector<int> degB, degH, col;
    std::vector<unsigned short> prod(n * (n + 1) / 2);
    product_columns(n, prod.data());
    harmonic_degrees(n, degB);
    if (useGaunt) {
        harmonic_degrees(n2, degH);
    } else {
        degH.resize(prod.size());
        for (size_t c = 0; c < prod.size(); c++)
            degH[c] = degB[prod[c] >> 8] + degB[prod[c] & 255];
    }
    int even = 0, nb = 0, k2 = 0;
    parity_columns(degB, 1, col, even, nb);
    parity_columns(degH, 1, col, even, k2);
    nt = k2 / 8;
    nbk = nb / 8;
}

NewtonProblem make_problem(const DeviceBasis &B)
{
    NewtonProblem pb;
    memset(&pb, 0, sizeof(pb));
    pb.P = B.P;
    pb.w = B.w;
    pb.hoff = B.hoff;
    pb.hidx = B.hidx;
    pb.hval = B.hval;
    pb.pairs = B.pairs;
    pb.ellPair = B.ellPair;
    pb.ellIdx = B.ellIdx;
    pb.ellVal = B.ellVal;
    pb.ellOff = B.ellOff;
    pb.ellChunks = B.ellChunks;
    pb.ellRows = B.ellRows;
    pb.p0 = B.p0;
    pb.row0Off = B.r0off;
    pb.row0Idx = B.r0idx;
    pb.row0Val = B.r0val;
    pb.rangeC = B.rangeC;
    pb.maxDeg = B.maxDeg;
    pb.gramLo = (B.useGaunt && !B.r0off) ? 0.0 : B.gramLo;
    pb.gramHi = B.gramHi;
    pb.n = B.n;
    pb.nb = B.nb;
    pb.K2p = B.K2p;
    pb.nqp = B.nqp;
    pb.ldP = B.ldP;
    pb.paired = B.paired;
    pb.nbe = B.nbe;
    pb.K2e = B.K2e;
    pb.binv = B.binv;
    pb.pcol = B.pcol;
    return pb;
}

// The screening pass's view of the basis: the gradient-column layout.
static NewtonProblem make_screen_problem(const DeviceBasis &B)
{
    NewtonProblem pb = make_problem(B);
    pb.P = B.Ps;
    pb.ldP = B.ldPs;
    pb.K2p = B.K2ps;
    pb.K2e = B.K2es;
    pb.row0Idx = B.r0idxS;
    pb.pcol = B.pcolS;
    pb.ellPair = pb.ellIdx = nullptr;
    pb.ellVal = nullptr;
    pb.ellOff = nullptr;
    pb.ellChunks = pb.ellRows = 0;
    return pb;
}

int check_options(const cl_options *o, std::string &err)
{
    if (!o) {
        err = "null options";
        return CL_ERR_ARG;
    }
    if (o->opt_type < 0 || o->opt_type > 2) {
        err = "MOMOPT_OPTIMIZATION_TYPE " + std::to_string(o->opt_type) + " out of range";
        return CL_ERR_ARG;
    }
    if (o->opt_type == 2 && o->max_bfgs_iter < 1) {
        // optbfgs.cpp would never take a step and end in "Max regularization
        // achieved."
        err = "MOMOPT_MAX_BFGS_ITER must be >= 1";
        return CL_ERR_ARG;
    }
    if (o->moment_type != CL_MN && o->moment_type != CL_PPN) {
        err = "moment type out of range";
        return CL_ERR_ARG;
    }
    if (o->contraction != CL_CONTRACT_PAIRS && o->contraction != CL_CONTRACT_SINGLE) {
        err = "contraction must be CL_CONTRACT_PAIRS or CL_CONTRACT_SINGLE";
        return CL_ERR_ARG;
    }
    if (o->precision != CL_FP64 && o->precision != CL_MIXED) {
        err = "precision must be CL_FP64 or CL_MIXED";
        return CL_ERR_ARG;
    }
    if (o->max_iter < 1) {
        err = "MOMOPT_MAX_ITER must be >= 1";
        return CL_ERR_ARG;
    }
    return CL_OK;
}

void fill_newton_options(NewtonArgs &a, const cl_options &o, int useGaunt)
{
    a.momentType = o.moment_type;
    a.maxIter = o.max_iter;
    a.useGaunt = useGaunt;
    a.tolRel = o.tol;
    a.condHMax = o.cond_h_max;
    a.deltaPPn = o.delta_ppn;
    a.mixed = o.precision == CL_MIXED;
    a.optType = o.opt_type;
    a.tolGamma = o.tol_gamma;
    a.maxBfgsIter = o.max_bfgs_iter;
    a.condHMaxBfgs = o.cond_h_max_bfgs;
    a.cbStride = (o.opt_type == 2) ? kBfgsSlotDoubles : kCbSlotDoubles;
}

int sm_count()
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

const char *error_text(int code) { return cl_error_text(code); }

}  // namespace

struct cl_ctx {
    cudaStream_t stream = nullptr;
    cl_grid grid;
    cl_options opt;
    int n = 0, NX = 0, NY = 0;
    long long C = 0;
    DeviceBasis B;
    double *dMom = nullptr, *dAlpha = nullptr, *dOld = nullptr, *dSigT = nullptr, *dSigS = nullptr;
    unsigned int *dQueue = nullptr;   // [4 + kHostBands]: stage 1, stage 2, batch, spare, bands
    DevStats *dStats = nullptr;
    int *dErr = nullptr;
    int *hErr = nullptr;              // pinned [2]
    int *dIters = nullptr;            // [C] iterations of each cell in the last stage
    cl_mlp *warm = nullptr;           // learned warm start (null: previous stage's alpha)
    int warmMinIters = 0;             // > 0: predict only cells whose previous stage took this many iterations
    double *dAlphaPred = nullptr;     // [C][n] predicted starts when warm is set
    double *dP2M = nullptr, *dAlphaP = nullptr;   // change-of-basis state per cell (opt type 1)
    double *dCbScratch = nullptr;     // working basis per Newton slot (opt type 1)
    NewtonArgs nargs;
    FluxArgs fargs;
    int nCtas = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    double gdt = 0, gdx = 0, gdy = 0;
    int graphKernels = 0;
    // cl_step_host: copy stream and its events (created on first use)
    cudaStream_t copyStream = nullptr;
    cudaEvent_t evStart = nullptr, evK1 = nullptr, evFlux = nullptr, evBand[8] = {};
    // batch scratch (grow only)
    double *bU = nullptr, *bA = nullptr, *bR = nullptr;
    int *bI = nullptr, *bS = nullptr;
    long long bCap = 0;
    // autotuner: the other contraction layout (built on first use) and the
    // host angular data it is built from; which basis each kernel reads
    DeviceBasis B2;
    int newtonB2 = 0, fluxB2 = 0;
    int rangeTest = 1;   // K1's exponent-range test (cl_set_range_test)
    // screening pass before K1 in grid stages (Mn, FP64, direction pairs):
    // its arguments, CTAs, the list of cells left for K1 and, per stage or
    // band, the list length and the screening work counter
    NewtonArgs sargs;
    int screen = 0, nCtasScreen = 0;
    int *dPend = nullptr, *dPend2 = nullptr, *dPendCount = nullptr, *dGate = nullptr, *dOrderCount = nullptr;
    unsigned int *dScreenQ = nullptr;
    int angN = 0, angN2 = 0, angNq = 0, angGaunt = 0, angNnz = 0;
    std::vector<double> aw, axi, aeta, ap, agval;
    std::vector<int> agoff, agidx;
    cl_tuning tuning{};
    std::string err;
};

extern "C" {

static void update_screen(cl_ctx *ctx);

const char *cl_global_error(void) { return g_global_err.c_str(); }

const char *cl_error_text(int code)
{
    switch (code) {
    case CL_OK:
        return "no error";
    case CL_ERR_ARG:
        return "bad argument or unsupported configuration";
    case CL_ERR_CUDA:
        return "CUDA error or no usable device";
    case CL_ERR_U0:
        return "u[0] < 0";
    case CL_ERR_MAXREG:
        return "Max regularization achieved.";
    case CL_ERR_TIMEOUT:
        return "device wait timed out";
    case CL_ERR_STATE:
        return "call order or state error";
    default:
        return "device error";
    }
}

int cl_angular_create(int order, int quad_order, int use_gaunt, cl_angular *out)
{
    if (!out) {
        g_global_err = "null output";
        return CL_ERR_ARG;
    }
    memset(out, 0, sizeof(*out));
    Angular A;
    if (build_angular(order, quad_order, use_gaunt, A) != 0) {
        g_global_err = "unsupported order/quadrature (order 1..6 with the Gaunt table, 1..9 without; Q >= 2 even)";
        return CL_ERR_ARG;
    }
    out->order = A.order;
    out->quad_order = A.Q;
    out->use_gaunt = A.useGaunt;
    out->n = A.n;
    out->n2 = A.n2;
    out->nq = A.nq;
    auto dup = [](const std::vector<double> &v) {
        double *p = (double *)malloc(sizeof(double) * (v.size() ? v.size() : 1));
        if (!v.empty())
            memcpy(p, v.data(), sizeof(double) * v.size());
        return p;
    };
    out->w = dup(A.w);
    out->xi = dup(A.xi);
    out->eta = dup(A.eta);
    out->p = dup(A.p);
    out->gaunt_nnz = (int)A.gidx.size();
    if (A.useGaunt) {
        out->gaunt_off = (int *)malloc(sizeof(int) * A.goff.size());
        memcpy(out->gaunt_off, A.goff.data(), sizeof(int) * A.goff.size());
        out->gaunt_idx = (int *)malloc(sizeof(int) * (A.gidx.size() + 1));
        memcpy(out->gaunt_idx, A.gidx.data(), sizeof(int) * A.gidx.size());
        out->gaunt_val = dup(A.gval);
    }
    return CL_OK;
}

void cl_angular_free(cl_angular *a)
{
    if (!a)
        return;
    free(a->w);
    free(a->xi);
    free(a->eta);
    free(a->p);
    free(a->gaunt_off);
    free(a->gaunt_idx);
    free(a->gaunt_val);
    memset(a, 0, sizeof(*a));
}

const char *cl_last_error(const cl_ctx *ctx) { return ctx ? ctx->err.c_str() : g_global_err.c_str(); }

int64_t cl_launch_count(void) { return (int64_t)g_launches.load(); }

static int ctx_fail(cl_ctx *ctx, int code)
{
    g_global_err = ctx->err;
    cl_destroy(ctx);
    return code;
}

int cl_create(const cl_grid *grid, const cl_options *opts, const cl_angular *ang, const double *sigma_t,
              const double *sigma_s, const double *moments, const double *alpha, cl_ctx **out)
{
    if (!out || !grid || !ang || !sigma_t || !sigma_s || !moments || !alpha) {
        g_global_err = "null argument";
        return CL_ERR_ARG;
    }
    *out = nullptr;
    std::string e;
    int rc = check_options(opts, e);
    if (rc) {
        g_global_err = e;
        return rc;
    }
    if (grid->ghost != 2 || grid->nx < 1 || grid->ny < 1) {
        g_global_err = "grid must have nx, ny >= 1 and 2 ghost cells";
        return CL_ERR_ARG;
    }
    if (ang->n < 1 || ang->n > kMaxN || ang->nq < 1 || !ang->p || !ang->w) {
        g_global_err = "angular set-up missing or order > 6";
        return CL_ERR_ARG;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        g_global_err = "no CUDA device (the B200 path has no CPU fallback)";
        return CL_ERR_CUDA;
    }
    cl_ctx *ctx = new cl_ctx();
    ctx->grid = *grid;
    ctx->opt = *opts;
    ctx->n = ang->n;
    ctx->NX = grid->nx + 4;
    ctx->NY = grid->ny + 4;
    ctx->C = (long long)ctx->NX * ctx->NY;
    const size_t C = (size_t)ctx->C, n = (size_t)ctx->n;
    CUDA_TRY(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    // Both optimisation types sum the moment-basis Hessian the way the deck
    // asks (Gaunt table or basis products).  The change-of-basis solve then
    // transforms it to its working basis; optcb.cpp instead transforms the
    // degree-N basis rows and sums products, which is the same Hessian in
    // exact arithmetic.
    const int gauntNewton = ang->use_gaunt;
    // direction pairs where a fused instance takes the paired layout (Mn,
    // FP64, the default contraction)
    int paired = 0;
    if (opts->moment_type == CL_MN && opts->precision == CL_FP64 && opts->contraction == CL_CONTRACT_PAIRS) {
        int pnt = 0, pnbk = 0;
        paired_counts(ang->n, ang->n2, gauntNewton, pnt, pnbk);
        paired = newton_pair_supported(pnt, pnbk) ? 1 : 0;
    }
    // the flux kernel takes direction pairs for either closure
    const int fluxPaired = opts->contraction == CL_CONTRACT_PAIRS ? 1 : 0;
    cudaError_t ce = build_device_basis(ctx->B, ang->n, ang->n2, ang->nq, gauntNewton, ang->w, ang->xi,
                                        ang->eta, ang->p, ang->gaunt_off, ang->gaunt_idx, ang->gaunt_val,
                                        ang->gaunt_nnz, paired, fluxPaired);
    if (ce != cudaSuccess) {
        ctx->err = std::string("basis upload: ") + cudaGetErrorString(ce);
        return ctx_fail(ctx, CL_ERR_CUDA);
    }
    ctx->angN = ang->n;
    ctx->angN2 = ang->n2;
    ctx->angNq = ang->nq;
    ctx->angGaunt = gauntNewton;
    ctx->angNnz = ang->gaunt_nnz;
    ctx->aw.assign(ang->w, ang->w + ang->nq);
    ctx->axi.assign(ang->xi, ang->xi + ang->nq);
    ctx->aeta.assign(ang->eta, ang->eta + ang->nq);
    ctx->ap.assign(ang->p, ang->p + (size_t)ang->nq * ang->n2);
    if (gauntNewton && ang->gaunt_off) {
        ctx->agoff.assign(ang->gaunt_off, ang->gaunt_off + ang->n * ang->n + 1);
        ctx->agidx.assign(ang->gaunt_idx, ang->gaunt_idx + ang->gaunt_nnz);
        ctx->agval.assign(ang->gaunt_val, ang->gaunt_val + ang->gaunt_nnz);
    }
    if (cudaMalloc(&ctx->dMom, C * n * 8) != cudaSuccess || cudaMalloc(&ctx->dAlpha, C * n * 8) != cudaSuccess ||
        cudaMalloc(&ctx->dOld, C * n * 8) != cudaSuccess || cudaMalloc(&ctx->dSigT, C * 8) != cudaSuccess ||
        cudaMalloc(&ctx->dSigS, C * 8) != cudaSuccess || cudaMalloc(&ctx->dQueue, (4 + kHostBands) * sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&ctx->dStats, sizeof(DevStats)) != cudaSuccess || cudaMalloc(&ctx->dErr, 2 * sizeof(int)) != cudaSuccess ||
        cudaMallocHost(&ctx->hErr, 2 * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&ctx->dIters, C * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&ctx->dPend, C * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&ctx->dPend2, C * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&ctx->dPendCount, (4 + kHostBands) * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&ctx->dScreenQ, (4 + kHostBands) * sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&ctx->dGate, (4 + kHostBands) * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&ctx->dOrderCount, (4 + kHostBands) * sizeof(int)) != cudaSuccess) {
        ctx->err = "device allocation failed";
        return ctx_fail(ctx, CL_ERR_CUDA);
    }
    cudaMemcpy(ctx->dMom, moments, C * n * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(ctx->dAlpha, alpha, C * n * 8, cudaMemcpyHostToDevice);
    cudaMemset(ctx->dOld, 0, C * n * 8);
    cudaMemcpy(ctx->dSigT, sigma_t, C * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(ctx->dSigS, sigma_s, C * 8, cudaMemcpyHostToDevice);
    cudaMemset(ctx->dStats, 0, sizeof(DevStats));
    cudaMemset(ctx->dErr, 0, 2 * sizeof(int));
    cudaMemset(ctx->dIters, 0, C * sizeof(int));
    ctx->hErr[0] = ctx->hErr[1] = 0;

    NewtonArgs &a = ctx->nargs;
    memset(&a, 0, sizeof(a));
    a.nprob = 1;
    a.prob[0] = make_problem(ctx->B);
    fill_newton_options(a, *opts, gauntNewton);
    a.stats = ctx->dStats;
    a.err = ctx->dErr;
    a.NX = ctx->NX;
    a.NY = ctx->NY;
    if (opts->opt_type != 0) {
        // momopt_init.cpp:146-157: alphaP isotropic, and the first n entries
        // of each P2M block (its first column, as the reference stores it
        // column-major) set to one -- singular, so each cell's first solve
        // takes the first-evaluation reset to the standard basis
        std::vector<double> hP2M(C * n * n, 0.0), hAP(C * n, 0.0);
        const double a0 = (opts->moment_type == CL_MN) ? 2.0 * std::sqrt(M_PI) * std::log(0.5 / std::sqrt(M_PI))
                                                       : 1.0 - 4.0 * opts->delta_ppn * M_PI;
        for (size_t c = 0; c < C; c++) {
            for (size_t k = 0; k < n; k++)
                hP2M[c * n * n + k * n] = 1.0;
            hAP[c * n] = a0;
        }
        if (upload(&ctx->dP2M, hP2M) != cudaSuccess || upload(&ctx->dAlphaP, hAP) != cudaSuccess) {
            ctx->err = "device allocation failed";
            return ctx_fail(ctx, CL_ERR_CUDA);
        }
        a.prob[0].P2M = ctx->dP2M;
        a.prob[0].alphaP = ctx->dAlphaP;
    }
    int pl = plan_newton(a);
    if (ctx->B.paired && (pl != 0 || a.ntf == 0 || a.ntExact == 0)) {
        // the paired layout only runs fused: keep one direction at a time
        ctx->B.release();
        if ((ce = build_device_basis(ctx->B, ang->n, ang->n2, ang->nq, gauntNewton, ang->w, ang->xi, ang->eta,
                                     ang->p, ang->gaunt_off, ang->gaunt_idx, ang->gaunt_val, ang->gaunt_nnz,
                                     0, fluxPaired)) != cudaSuccess) {
            ctx->err = std::string("basis upload: ") + cudaGetErrorString(ce);
            return ctx_fail(ctx, CL_ERR_CUDA);
        }
        NewtonProblem keep = a.prob[0];
        a.prob[0] = make_problem(ctx->B);
        a.prob[0].P2M = keep.P2M;
        a.prob[0].alphaP = keep.alphaP;
        pl = plan_newton(a);
    }
    if (pl != 0) {
        ctx->err = pl == -2 ? "mixed precision needs a configuration with at most 16 Hessian column tiles"
                            : "Newton kernel layout does not fit in shared memory";
        return ctx_fail(ctx, CL_ERR_ARG);
    }
    if ((ce = prepare_newton(a)) != cudaSuccess) {
        ctx->err = std::string("Newton kernel attributes: ") + cudaGetErrorString(ce);
        return ctx_fail(ctx, CL_ERR_CUDA);
    }
    ctx->nCtas = sm_count() * newton_ctas_per_sm(a);
    if (opts->opt_type != 0) {
        if (cudaMalloc(&ctx->dCbScratch, (size_t)ctx->nCtas * a.T * a.cbStride * sizeof(double)) != cudaSuccess) {
            ctx->err = "device allocation failed";
            return ctx_fail(ctx, CL_ERR_CUDA);
        }
        a.cbScratch = ctx->dCbScratch;
    }

    FluxArgs &f = ctx->fargs;
    memset(&f, 0, sizeof(f));
    f.tilesRun = &ctx->dStats->fluxTiles;
    f.skipUniform = 1;
    f.alpha = ctx->dAlpha;
    f.moments = ctx->dMom;
    f.sigmaT = ctx->dSigT;
    f.sigmaS = ctx->dSigS;
    f.P = ctx->B.Pf;
    f.xi = ctx->B.xi;
    f.eta = ctx->B.eta;
    f.cxw = ctx->B.cxw;
    f.cyw = ctx->B.cyw;
    f.n = ctx->n;
    f.nb = ctx->B.nbF;
    f.paired = ctx->B.fluxPaired;
    f.nbe = ctx->B.nbeF;
    f.binv = ctx->B.fbinv;
    f.ldPf = ctx->B.ldPf;
    f.nqp = ctx->B.nqpF;
    f.NX = ctx->NX;
    f.NY = ctx->NY;
    f.momentType = opts->moment_type;
    f.initCond = grid->init_cond;
    f.theta = grid->theta;
    f.deltaPPn = opts->delta_ppn;
    f.initX = grid->init_x;
    f.initY = grid->init_y;
    if (plan_flux(f) != 0) {
        ctx->err = "flux kernel layout does not fit in shared memory";
        return ctx_fail(ctx, CL_ERR_ARG);
    }
    if ((ce = prepare_flux(f)) != cudaSuccess) {
        ctx->err = std::string("flux kernel attributes: ") + cudaGetErrorString(ce);
        return ctx_fail(ctx, CL_ERR_CUDA);
    }
    if (cudaDeviceSynchronize() != cudaSuccess) {
        ctx->err = std::string("set-up: ") + cudaGetErrorString(cudaGetLastError());
        return ctx_fail(ctx, CL_ERR_CUDA);
    }
    update_screen(ctx);
    ctx->tuning.newton_warps = a.nw;
    ctx->tuning.newton_ctas = ctx->nCtas;
    ctx->tuning.newton_contraction = ctx->B.paired ? CL_CONTRACT_PAIRS : CL_CONTRACT_SINGLE;
    ctx->tuning.flux_contraction = ctx->B.fluxPaired ? CL_CONTRACT_PAIRS : CL_CONTRACT_SINGLE;
    *out = ctx;
    return CL_OK;
}

void cl_destroy(cl_ctx *ctx)
{
    if (!ctx)
        return;
    if (ctx->stream)
        cudaStreamSynchronize(ctx->stream);
    if (ctx->exec)
        cudaGraphExecDestroy(ctx->exec);
    if (ctx->graph)
        cudaGraphDestroy(ctx->graph);
    ctx->B.release();
    ctx->B2.release();
    cudaFree(ctx->dMom);
    cudaFree(ctx->dAlpha);
    cudaFree(ctx->dOld);
    cudaFree(ctx->dPend);
    cudaFree(ctx->dPend2);
    cudaFree(ctx->dPendCount);
    cudaFree(ctx->dScreenQ);
    cudaFree(ctx->dGate);
    cudaFree(ctx->dOrderCount);
    cudaFree(ctx->dSigT);
    cudaFree(ctx->dSigS);
    cudaFree(ctx->dQueue);
    cudaFree(ctx->dStats);
    cudaFree(ctx->dErr);
    cudaFreeHost(ctx->hErr);
    cudaFree(ctx->dIters);
    cudaFree(ctx->dAlphaPred);
    cudaFree(ctx->dP2M);
    cudaFree(ctx->dAlphaP);
    cudaFree(ctx->dCbScratch);
    cudaFree(ctx->bU);
    cudaFree(ctx->bA);
    cudaFree(ctx->bR);
    cudaFree(ctx->bI);
    cudaFree(ctx->bS);
    if (ctx->copyStream) {
        cudaStreamSynchronize(ctx->copyStream);
        cudaStreamDestroy(ctx->copyStream);
    }
    for (cudaEvent_t ev : {ctx->evStart, ctx->evK1, ctx->evFlux})
        if (ev)
            cudaEventDestroy(ev);
    for (cudaEvent_t ev : ctx->evBand)
        if (ev)
            cudaEventDestroy(ev);
    if (ctx->stream)
        cudaStreamDestroy(ctx->stream);
    delete ctx;
}

// The learned starts of a stage on `st`: every cell, or the cells whose
// previous stage took at least warmMinIters iterations.  Returns the kernel
// launches it issued (for the launch count) or -1.
static int enqueue_prediction(cl_ctx *ctx, cudaStream_t st)
{
    const int chunks = (int)((ctx->C + (1 << 18) - 1) >> 18);
    if (ctx->warmMinIters > 0) {
        if (cl_mlp_predict_selected(ctx->warm, ctx->dMom, ctx->dIters, ctx->warmMinIters, ctx->dAlphaPred,
                                    (int)ctx->C, st) != CL_OK)
            return -1;
        return 1 + 6 * chunks;
    }
    if (cl_mlp_predict(ctx->warm, ctx->dMom, ctx->dAlphaPred, (int)ctx->C, 2, nullptr, st) != CL_OK)
        return -1;
    return 2 + 4 * chunks;
}

// Screening before K1 where it applies: Mn, FP64, plain Newton, K1 on the
// direction-pair layout with the exponent-range test on.
static void update_screen(cl_ctx *ctx)
{
    ctx->screen = 0;
    ctx->tuning.screen_ctas = 0;
    const DeviceBasis &B = ctx->newtonB2 ? ctx->B2 : ctx->B;
    const NewtonArgs &k = ctx->nargs;
    if (!ctx->rangeTest || !ctx->dPend || !B.paired || !B.screenOk || k.nprob != 1 || k.momentType != 0 ||
        k.mixed || k.optType != 0 || !(k.prob[0].gramLo > 0.0))
        return;
    NewtonArgs s = k;
    s.prob[0] = make_screen_problem(B);
    if (plan_screen(s) != 0 || prepare_screen(s) != cudaSuccess)
        return;
    ctx->sargs = s;
    ctx->nCtasScreen = sm_count() * screen_ctas_per_sm(s);
    ctx->screen = 1;
    ctx->tuning.screen_ctas = ctx->nCtasScreen;
}

// Fraction of a launch's cells whose previous solve took one iteration, at
// or above which the screening pass runs: then it settles enough cells (most
// of them copies of repeated starts) that K1's time over the rest is not set
// by long Newton chains the easy cells would have run beside.  Measured on
// the M6 pulse's whole run: 0.85 -> 51.6 s, 0.6 -> 46.3 s, 0.45 -> 45.9 s
// (and its window at t = 0.9, 56 % one-iteration cells, 6 % faster screened).
constexpr double kScreenGate = 0.45;

// Whole stages of at most this many cells are ordered for K1 too (gate
// shut, or no screening): one CTA sorts them in a small fraction of the
// stage.  Larger stages keep cell order: sorting 646,416 cells in one CTA
// took about a millisecond per stage and measured 4-6 % slower at t = 0.9 of
// the M6 pulse.
constexpr int kOrderWholeMax = 131072;

// K1 of a grid stage or band (`a` complete; `slot` selects the counters).
// With screening: the gate count and the screening pass over the same
// cells.  Then the order of K1's cells, longest previous Newton chain first
// (the cells the screening left; or the whole range when it is small), and
// K1 over that list.
static cudaError_t launch_stage_newton(cl_ctx *ctx, NewtonArgs &a, int slot, cudaStream_t st, int *nk)
{
    cudaError_t e;
    const NewtonProblem kp = a.prob[0];
    if (kp.iters && ctx->dPend && (ctx->screen || kp.count <= kOrderWholeMax)) {
        int gateMin = 0;
        if (ctx->screen) {
            NewtonArgs s = ctx->sargs;
            NewtonProblem &sp = s.prob[0];
            sp.count = kp.count;
            sp.first = kp.first;
            sp.u = kp.u;
            sp.alpha = kp.alpha;
            sp.iters = kp.iters;
            sp.regs = kp.regs;
            sp.status = kp.status;
            sp.alphaStart = kp.alphaStart;
            sp.queue = ctx->dScreenQ + slot;
            sp.pendList = ctx->dPend + kp.first;
            sp.pendCount = ctx->dPendCount + slot;
            sp.gateCount = ctx->dGate + slot;
            sp.gateMin = gateMin = (int)std::ceil(kScreenGate * kp.count);
            s.momentsOld = a.momentsOld;
            if ((e = cudaMemsetAsync(ctx->dScreenQ + slot, 0, sizeof(unsigned), st)) != cudaSuccess)
                return e;
            if ((e = cudaMemsetAsync(ctx->dPendCount + slot, 0, sizeof(int), st)) != cudaSuccess)
                return e;
            if ((e = cudaMemsetAsync(ctx->dGate + slot, 0, sizeof(int), st)) != cudaSuccess)
                return e;
            if ((e = launch_screen_gate(kp.iters, kp.first, kp.count, ctx->dGate + slot, st)) != cudaSuccess)
                return e;
            if ((e = launch_screen(s, ctx->nCtasScreen, st)) != cudaSuccess)
                return e;
            *nk += 2;
        }
        if ((e = launch_order_cells(ctx->screen ? ctx->dPend + kp.first : nullptr, ctx->dPendCount + slot, kp.first,
                                    kp.count, ctx->screen ? ctx->dGate + slot : nullptr, gateMin, kOrderWholeMax,
                                    kp.iters, ctx->dPend2 + kp.first, ctx->dOrderCount + slot, st)) != cudaSuccess)
            return e;
        *nk += 1;
        a.prob[0].cellList = ctx->dPend2 + kp.first;
        a.prob[0].countDev = ctx->dOrderCount + slot;
    }
    if ((e = launch_newton(a, ctx->nCtas, st)) != cudaSuccess)
        return e;
    *nk += 1;
    return cudaSuccess;
}

// Enqueues RK stage `stage` (0 or 1) on the context's stream: [periodic
// ghost copy], [warm-start prediction], K1, K2+K3 (stage 1 also the Heun
// average).  The stage's work counter must be zero when K1 starts.
static cudaError_t enqueue_stage(cl_ctx *ctx, int stage, double dt, double dx, double dy, bool ghostCopy,
                                 int *nk, cudaEvent_t beforeK1 = nullptr, cudaEvent_t afterK1 = nullptr)
{
    cudaError_t e;
    if (ghostCopy) {
        if ((e = launch_ghost_periodic(ctx->dMom, ctx->n, ctx->NX, ctx->NY, ctx->stream)) != cudaSuccess)
            return e;
        *nk += 2;
    }
    if (ctx->warm) {
        const int k = enqueue_prediction(ctx, ctx->stream);
        if (k < 0)
            return cudaErrorLaunchFailure;
        *nk += k;
    }
    NewtonArgs a = ctx->nargs;
    a.prob[0].count = (int)ctx->C;
    a.prob[0].u = ctx->dMom;
    a.prob[0].alpha = ctx->dAlpha;
    a.prob[0].queue = ctx->dQueue + stage;
    a.prob[0].iters = ctx->dIters;
    a.prob[0].alphaStart = ctx->warm ? ctx->dAlphaPred : nullptr;
    a.momentsOld = (stage == 0) ? ctx->dOld : nullptr;
    if (beforeK1 && (e = cudaEventRecord(beforeK1, ctx->stream)) != cudaSuccess)
        return e;
    if ((e = launch_stage_newton(ctx, a, stage, ctx->stream, nk)) != cudaSuccess)
        return e;
    if (afterK1 && (e = cudaEventRecord(afterK1, ctx->stream)) != cudaSuccess)
        return e;
    FluxArgs f = ctx->fargs;
    f.dt = dt;
    f.dx = dx;
    f.dy = dy;
    f.momentsOld = (stage == 1) ? ctx->dOld : nullptr;
    if ((e = launch_flux(f, ctx->stream)) != cudaSuccess)
        return e;
    *nk += 1;
    return cudaSuccess;
}

// Enqueues one RK2 step on the context's stream (uncaptured form).
static cudaError_t enqueue_step(cl_ctx *ctx, double dt, double dx, double dy, int *kernels)
{
    cudaError_t e;
    int nk = 0;
    const bool periodic = ctx->grid.init_cond == 2;
    if ((e = cudaMemsetAsync(ctx->dQueue, 0, 2 * sizeof(unsigned), ctx->stream)) != cudaSuccess)
        return e;
    for (int stage = 0; stage < 2; stage++)
        if ((e = enqueue_stage(ctx, stage, dt, dx, dy, periodic, &nk)) != cudaSuccess)
            return e;
    if (kernels)
        *kernels = nk;
    return cudaSuccess;
}

static int read_device_error(cl_ctx *ctx)
{
    CUDA_TRY(ctx, cudaMemcpyAsync(ctx->hErr, ctx->dErr, 2 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->hErr[0] != 0) {
        long long cell = ctx->hErr[1];
        char buf[256];
        if (cell < 0)
            snprintf(buf, sizeof(buf), "%s", error_text(ctx->hErr[0]));
        else if (ctx->NY > 0 && cell < ctx->C)
            snprintf(buf, sizeof(buf), "%s (cell i=%lld j=%lld)", error_text(ctx->hErr[0]), cell / ctx->NY,
                     cell % ctx->NY);
        else
            snprintf(buf, sizeof(buf), "%s (vector %lld)", error_text(ctx->hErr[0]), cell);
        ctx->err = buf;
        return ctx->hErr[0];
    }
    return CL_OK;
}

int cl_step_async(cl_ctx *ctx, double dt, double dx, double dy)
{
    if (!ctx)
        return CL_ERR_ARG;
    if (!ctx->exec || dt != ctx->gdt || dx != ctx->gdx || dy != ctx->gdy) {
        if (ctx->exec) {
            cudaGraphExecDestroy(ctx->exec);
            ctx->exec = nullptr;
        }
        if (ctx->graph) {
            cudaGraphDestroy(ctx->graph);
            ctx->graph = nullptr;
        }
        CUDA_TRY(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        int nk = 0;
        cudaError_t e = enqueue_step(ctx, dt, dx, dy, &nk);
        cudaGraph_t gph = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &gph);
        if (e != cudaSuccess || e2 != cudaSuccess) {
            if (gph)
                cudaGraphDestroy(gph);
            ctx->err = std::string("graph capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2);
            return CL_ERR_CUDA;
        }
        ctx->graph = gph;
        CUDA_TRY(ctx, cudaGraphInstantiate(&ctx->exec, ctx->graph, 0));
        ctx->gdt = dt;
        ctx->gdx = dx;
        ctx->gdy = dy;
        ctx->graphKernels = nk;
    }
    CUDA_TRY(ctx, cudaGraphLaunch(ctx->exec, ctx->stream));
    g_launches += ctx->graphKernels;
    return CL_OK;
}

int cl_step_timed(cl_ctx *ctx, double dt, double dx, double dy, float *ms)
{
    if (!ctx || !ms)
        return CL_ERR_ARG;
    cudaEvent_t ev[7];
    for (int i = 0; i < 7; i++)
        CUDA_TRY(ctx, cudaEventCreate(&ev[i]));
    const bool periodic = ctx->grid.init_cond == 2;
    cudaError_t e = cudaMemsetAsync(ctx->dQueue, 0, 2 * sizeof(unsigned), ctx->stream);
    int nk = 0;
    for (int stage = 0; stage < 2 && e == cudaSuccess; stage++) {
        cudaEventRecord(ev[3 * stage], ctx->stream);
        if (periodic) {
            e = launch_ghost_periodic(ctx->dMom, ctx->n, ctx->NX, ctx->NY, ctx->stream);
            nk += 2;
        }
        if (ctx->warm && e == cudaSuccess) {
            const int k = enqueue_prediction(ctx, ctx->stream);
            if (k < 0)
                e = cudaErrorLaunchFailure;
            nk += k < 0 ? 0 : k;
        }
        NewtonArgs a = ctx->nargs;
        a.prob[0].count = (int)ctx->C;
        a.prob[0].u = ctx->dMom;
        a.prob[0].alpha = ctx->dAlpha;
        a.prob[0].queue = ctx->dQueue + stage;
        a.prob[0].iters = ctx->dIters;
        a.prob[0].alphaStart = ctx->warm ? ctx->dAlphaPred : nullptr;
        a.momentsOld = (stage == 0) ? ctx->dOld : nullptr;
        if (e == cudaSuccess)
            e = launch_stage_newton(ctx, a, stage, ctx->stream, &nk);
        cudaEventRecord(ev[3 * stage + 1], ctx->stream);
        FluxArgs f = ctx->fargs;
        f.dt = dt;
        f.dx = dx;
        f.dy = dy;
        f.momentsOld = (stage == 1) ? ctx->dOld : nullptr;
        if (e == cudaSuccess)
            e = launch_flux(f, ctx->stream);
        nk++;
        cudaEventRecord(ev[3 * stage + 2], ctx->stream);
    }
    g_launches += nk;
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess) {
        cudaEventElapsedTime(&ms[0], ev[0], ev[1]);
        cudaEventElapsedTime(&ms[1], ev[1], ev[2]);
        cudaEventElapsedTime(&ms[2], ev[3], ev[4]);
        cudaEventElapsedTime(&ms[3], ev[4], ev[5]);
    }
    for (int i = 0; i < 7; i++)
        cudaEventDestroy(ev[i]);
    if (e != cudaSuccess) {
        ctx->err = std::string("timed step: ") + cudaGetErrorString(e);
        return CL_ERR_CUDA;
    }
    return read_device_error(ctx);
}

int cl_sync(cl_ctx *ctx)
{
    if (!ctx)
        return CL_ERR_ARG;
    return read_device_error(ctx);
}

int cl_stage(cl_ctx *ctx, int stage, double dt, double dx, double dy)
{
    if (!ctx || (stage != 1 && stage != 2))
        return CL_ERR_ARG;
    CUDA_TRY(ctx, cudaMemsetAsync(ctx->dQueue + (stage - 1), 0, sizeof(unsigned), ctx->stream));
    int nk = 0;
    cudaError_t e = enqueue_stage(ctx, stage - 1, dt, dx, dy, false, &nk);
    g_launches += nk;
    if (e != cudaSuccess) {
        ctx->err = std::string("stage: ") + cudaGetErrorString(e);
        return CL_ERR_CUDA;
    }
    return CL_OK;
}

int cl_stage_timed(cl_ctx *ctx, int stage, double dt, double dx, double dy, float *ms)
{
    if (!ctx || !ms || (stage != 1 && stage != 2))
        return CL_ERR_ARG;
    cudaEvent_t ev[3];
    for (int i = 0; i < 3; i++)
        CUDA_TRY(ctx, cudaEventCreate(&ev[i]));
    cudaError_t e = cudaMemsetAsync(ctx->dQueue + (stage - 1), 0, sizeof(unsigned), ctx->stream);
    int nk = 0;
    if (e == cudaSuccess)
        e = enqueue_stage(ctx, stage - 1, dt, dx, dy, false, &nk, ev[0], ev[1]);
    if (e == cudaSuccess)
        e = cudaEventRecord(ev[2], ctx->stream);
    g_launches += nk;
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess) {
        cudaEventElapsedTime(&ms[0], ev[0], ev[1]);
        cudaEventElapsedTime(&ms[1], ev[1], ev[2]);
    }
    for (int i = 0; i < 3; i++)
        cudaEventDestroy(ev[i]);
    if (e != cudaSuccess) {
        ctx->err = std::string("timed stage: ") + cudaGetErrorString(e);
        return CL_ERR_CUDA;
    }
    return read_device_error(ctx);
}

int cl_stream(cl_ctx *ctx, void **stream)
{
    if (!ctx || !stream)
        return CL_ERR_ARG;
    *stream = (void *)ctx->stream;
    return CL_OK;
}

int cl_halo_counts(const cl_ctx *ctx, long long counts[4])
{
    if (!ctx || !counts)
        return CL_ERR_ARG;
    const long long nx = ctx->NX - 4, ny = ctx->NY - 4, n = ctx->n;
    counts[CL_NORTH] = counts[CL_SOUTH] = 2 * nx * n;
    counts[CL_EAST] = counts[CL_WEST] = 2 * ny * n;
    return CL_OK;
}

static int halo(cl_ctx *ctx, double *const bufs[4], int pack)
{
    if (!ctx || !bufs)
        return CL_ERR_ARG;
    HaloBuffers b;
    for (int s = 0; s < 4; s++)
        b.p[s] = bufs[s];
    CUDA_TRY(ctx, launch_halo(ctx->dMom, ctx->n, ctx->NX, ctx->NY, b, pack, ctx->stream));
    g_launches += 1;
    return CL_OK;
}

int cl_halo_pack(cl_ctx *ctx, double *const bufs[4]) { return halo(ctx, bufs, 1); }

int cl_halo_unpack(cl_ctx *ctx, double *const bufs[4]) { return halo(ctx, bufs, 0); }

int cl_step(cl_ctx *ctx, double dt, double dx, double dy)
{
    int rc = cl_step_async(ctx, dt, dx, dy);
    if (rc)
        return rc;
    return cl_sync(ctx);
}

int cl_get_state(cl_ctx *ctx, double *moments, double *alpha)
{
    if (!ctx)
        return CL_ERR_ARG;
    size_t bytes = (size_t)ctx->C * ctx->n * 8;
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (moments)
        CUDA_TRY(ctx, cudaMemcpy(moments, ctx->dMom, bytes, cudaMemcpyDeviceToHost));
    if (alpha)
        CUDA_TRY(ctx, cudaMemcpy(alpha, ctx->dAlpha, bytes, cudaMemcpyDeviceToHost));
    return CL_OK;
}

int cl_set_state(cl_ctx *ctx, const double *moments, const double *alpha)
{
    if (!ctx)
        return CL_ERR_ARG;
    size_t bytes = (size_t)ctx->C * ctx->n * 8;
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (moments)
        CUDA_TRY(ctx, cudaMemcpy(ctx->dMom, moments, bytes, cudaMemcpyHostToDevice));
    if (alpha)
        CUDA_TRY(ctx, cudaMemcpy(ctx->dAlpha, alpha, bytes, cudaMemcpyHostToDevice));
    return CL_OK;
}

// One RK2 step on a state held in host memory, equal to cl_set_state,
// cl_step and cl_get_state (the reference's solver keeps c_moments and
// c_alpha on the host, momopt_update.cpp:279-378).  The copies run on a
// second stream and overlap the kernels: the state goes up in kHostBands
// bands of cells, each band's first-stage solve starting when its band has
// arrived; the multipliers come back while the second-stage flux runs, and
// the first part of the moments while the rest of that flux runs (its tiles
// split in two launches at a whole number of waves).  With a periodic deck
// or a learned warm start, whose first kernels read the whole grid, the
// state goes up in one band.  Page-locked host buffers give the overlap;
// others are still correct.
int cl_step_host(cl_ctx *ctx, double dt, double dx, double dy, double *moments, double *alpha)
{
    if (!ctx || !moments || !alpha)
        return CL_ERR_ARG;
    if (!ctx->copyStream) {
        CUDA_TRY(ctx, cudaStreamCreateWithFlags(&ctx->copyStream, cudaStreamNonBlocking));
        for (cudaEvent_t *ev : {&ctx->evStart, &ctx->evK1, &ctx->evFlux})
            CUDA_TRY(ctx, cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
        for (int b = 0; b < kHostBands; b++)
            CUDA_TRY(ctx, cudaEventCreateWithFlags(&ctx->evBand[b], cudaEventDisableTiming));
    }
    cudaStream_t S = ctx->stream, X = ctx->copyStream;
    const size_t n = (size_t)ctx->n, C = (size_t)ctx->C, rowBytes = (size_t)ctx->NY * n * 8;
    const bool periodic = ctx->grid.init_cond == 2;
    const int bands = (periodic || ctx->warm) ? 1 : kHostBands;
    int nk = 0;
    cudaError_t e = cudaSuccess;
    auto run = [&](cudaError_t r) {
        if (e == cudaSuccess)
            e = r;
    };
    // earlier work on the device state is done before the copies start
    run(cudaEventRecord(ctx->evStart, S));
    run(cudaStreamWaitEvent(X, ctx->evStart, 0));
    run(cudaMemsetAsync(ctx->dQueue, 0, (4 + kHostBands) * sizeof(unsigned), S));
    size_t band0[kHostBands + 1];
    for (int b = 0; b <= bands; b++)
        band0[b] = C * b / bands;
    for (int b = 0; b < bands; b++) {
        const size_t off = band0[b] * n, bytes = (band0[b + 1] - band0[b]) * n * 8;
        run(cudaMemcpyAsync(ctx->dMom + off, moments + off, bytes, cudaMemcpyHostToDevice, X));
        run(cudaMemcpyAsync(ctx->dAlpha + off, alpha + off, bytes, cudaMemcpyHostToDevice, X));
        run(cudaEventRecord(ctx->evBand[b], X));
    }
    for (int stage = 0; stage < 2 && e == cudaSuccess; stage++) {
        if (stage == 0 && bands == 1)
            run(cudaStreamWaitEvent(S, ctx->evBand[0], 0));
        if (periodic) {
            run(launch_ghost_periodic(ctx->dMom, ctx->n, ctx->NX, ctx->NY, S));
            nk += 2;
        }
        if (ctx->warm && e == cudaSuccess) {
            const int k = enqueue_prediction(ctx, S);
            if (k < 0)
                run(cudaErrorLaunchFailure);
            nk += k < 0 ? 0 : k;
        }
        NewtonArgs a = ctx->nargs;
        a.prob[0].u = ctx->dMom;
        a.prob[0].alpha = ctx->dAlpha;
        a.prob[0].iters = ctx->dIters;
        a.prob[0].alphaStart = ctx->warm ? ctx->dAlphaPred : nullptr;
        a.momentsOld = (stage == 0) ? ctx->dOld : nullptr;
        const int parts = (stage == 0) ? bands : 1;
        for (int b = 0; b < parts; b++) {
            if (stage == 0 && bands > 1)
                run(cudaStreamWaitEvent(S, ctx->evBand[b], 0));
            a.prob[0].first = (stage == 0) ? (int)band0[b] : 0;
            a.prob[0].count = (stage == 0) ? (int)(band0[b + 1] - band0[b]) : (int)C;
            a.prob[0].queue = ctx->dQueue + ((stage == 0 && bands > 1) ? 4 + b : stage);
            if (e == cudaSuccess) {
                NewtonArgs ab = a;   // the band's own list and counters
                run(launch_stage_newton(ctx, ab, (stage == 0 && bands > 1) ? 4 + b : stage, S, &nk));
            }
        }
        FluxArgs f = ctx->fargs;
        f.dt = dt;
        f.dx = dx;
        f.dy = dy;
        f.momentsOld = (stage == 1) ? ctx->dOld : nullptr;
        if (stage == 0) {
            if (e == cudaSuccess)
                run(launch_flux(f, S));
            nk++;
            continue;
        }
        // the multipliers are final: read them back under the flux
        run(cudaEventRecord(ctx->evK1, S));
        run(cudaStreamWaitEvent(X, ctx->evK1, 0));
        run(cudaMemcpyAsync(alpha, ctx->dAlpha, C * n * 8, cudaMemcpyDeviceToHost, X));
        // flux in two launches; the cell rows that the first completes go
        // back while the second runs (each tile writes only its own cells)
        const int tiles = f.tilesX * f.tilesY, sms = sm_count();
        int tA = (tiles / 2) / sms * sms;
        const int fullRows = tA / f.tilesY;
        if (tA <= 0 || fullRows <= 0)
            tA = 0;
        size_t rowsA = 0;
        if (tA > 0) {
            if (e == cudaSuccess)
                run(launch_flux_tiles(f, 0, tA, S));
            nk++;
            rowsA = 2 + (size_t)fullRows * flux_tile_rows(f);
            run(cudaEventRecord(ctx->evFlux, S));
            run(cudaStreamWaitEvent(X, ctx->evFlux, 0));
            run(cudaMemcpyAsync(moments, ctx->dMom, rowsA * rowBytes, cudaMemcpyDeviceToHost, X));
        }
        if (e == cudaSuccess)
            run(launch_flux_tiles(f, tA, tiles - tA, S));
        nk++;
        run(cudaMemcpyAsync(moments + rowsA * ctx->NY * n, ctx->dMom + rowsA * ctx->NY * n,
                            C * n * 8 - rowsA * rowBytes, cudaMemcpyDeviceToHost, S));
    }
    g_launches += nk;
    run(cudaStreamSynchronize(X));
    run(cudaStreamSynchronize(S));
    if (e != cudaSuccess) {
        ctx->err = std::string("host-state step: ") + cudaGetErrorString(e);
        return CL_ERR_CUDA;
    }
    return read_device_error(ctx);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Autotuner of the launch shapes (cl_tune): K1 cells per CTA / warps and the
// Hessian tile layout, K2+K3 tile layout.  Candidates run on copies of the
// context's state; the median of three timed launches decides.

static void invalidate_graph(cl_ctx *ctx)
{
    if (ctx->exec) {
        cudaGraphExecDestroy(ctx->exec);
        ctx->exec = nullptr;
    }
    if (ctx->graph) {
        cudaGraphDestroy(ctx->graph);
        ctx->graph = nullptr;
    }
}

// Builds the other contraction layout (both kernels) into ctx->B2 once.
static int ensure_alt_basis(cl_ctx *ctx)
{
    if (ctx->B2.P)
        return CL_OK;
    int paired = 0;
    if (ctx->opt.moment_type == CL_MN && ctx->opt.precision == CL_FP64 && !ctx->B.paired) {
        int pnt = 0, pnbk = 0;
        paired_counts(ctx->angN, ctx->angN2, ctx->angGaunt, pnt, pnbk);
        paired = newton_pair_supported(pnt, pnbk) ? 1 : 0;
    }
    const int fluxPaired = ctx->B.fluxPaired ? 0 : 1;
    cudaError_t e = build_device_basis(ctx->B2, ctx->angN, ctx->angN2, ctx->angNq, ctx->angGaunt, ctx->aw.data(),
                                       ctx->axi.data(), ctx->aeta.data(), ctx->ap.data(),
                                       ctx->agoff.empty() ? nullptr : ctx->agoff.data(),
                                       ctx->agidx.empty() ? nullptr : ctx->agidx.data(),
                                       ctx->agval.empty() ? nullptr : ctx->agval.data(), ctx->angNnz, paired,
                                       fluxPaired);
    if (e != cudaSuccess) {
        ctx->B2.release();
        ctx->err = std::string("tuner basis: ") + cudaGetErrorString(e);
        return CL_ERR_CUDA;
    }
    return CL_OK;
}

// Newton arguments of the context with the basis `B` and `nw` warps per
// CTA; returns false where that shape has no instance.
static bool newton_shape(const cl_ctx *ctx, const DeviceBasis &B, int nw, NewtonArgs &a)
{
    a = ctx->nargs;
    NewtonProblem keep = a.prob[0];
    a.prob[0] = make_problem(B);
    a.prob[0].P2M = keep.P2M;
    a.prob[0].alphaP = keep.alphaP;
    if (!ctx->rangeTest)
        a.prob[0].gramLo = 0.0;
    a.nw = nw;
    if (plan_newton(a) != 0 || a.ntf == 0 || (B.paired && a.ntExact == 0))
        return false;
    return prepare_newton(a) == cudaSuccess;
}

static void flux_basis(FluxArgs &f, const DeviceBasis &B)
{
    f.P = B.Pf;
    f.xi = B.xi;
    f.eta = B.eta;
    f.cxw = B.cxw;
    f.cyw = B.cyw;
    f.nb = B.nbF;
    f.paired = B.fluxPaired;
    f.nbe = B.nbeF;
    f.binv = B.fbinv;
    f.ldPf = B.ldPf;
    f.nqp = B.nqpF;
}

static float median3(float *v)
{
    std::sort(v, v + 3);
    return v[1];
}

struct TuneScratch {
    double *u = nullptr, *a = nullptr;
    int *it = nullptr, *err = nullptr;
    unsigned *q = nullptr;
    DevStats *st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ~TuneScratch()
    {
        cudaFree(u);
        cudaFree(a);
        cudaFree(it);
        cudaFree(err);
        cudaFree(q);
        cudaFree(st);
        if (e0)
            cudaEventDestroy(e0);
        if (e1)
            cudaEventDestroy(e1);
    }
};

// Median K1 time (ms) of `a` (basis B) over the context's state (copies),
// the screening pass included where it applies to B; < 0 if a launch failed
// or reported an error.
static float time_newton(cl_ctx *ctx, NewtonArgs a, const DeviceBasis &B, TuneScratch &S)
{
    const size_t C = (size_t)ctx->C, n = (size_t)ctx->n;
    a.prob[0].count = (int)C;
    a.prob[0].u = S.u;
    a.prob[0].alpha = S.a;
    a.prob[0].iters = S.it;
    a.prob[0].regs = nullptr;
    a.prob[0].status = nullptr;
    a.prob[0].alphaStart = nullptr;
    a.prob[0].queue = S.q;
    a.prob[0].first = 0;
    a.momentsOld = nullptr;
    a.stats = S.st;
    a.err = S.err;
    const int grid = sm_count() * newton_ctas_per_sm(a);
    NewtonArgs sa;
    int sgrid = 0;
    if (ctx->rangeTest && ctx->dPend && B.paired && B.screenOk && a.nprob == 1 && a.momentType == 0 &&
        !a.mixed && a.optType == 0 && a.prob[0].gramLo > 0.0) {
        sa = a;
        sa.prob[0] = make_screen_problem(B);
        if (plan_screen(sa) == 0 && prepare_screen(sa) == cudaSuccess) {
            NewtonProblem &sp = sa.prob[0];
            sp.count = (int)C;
            sp.u = S.u;
            sp.alpha = S.a;
            sp.iters = S.it;
            sp.queue = S.q + 1;
            sp.pendList = ctx->dPend;
            sp.pendCount = (int *)(S.q + 2);
            sp.gateCount = (const int *)(S.q + 3);
            sp.gateMin = (int)std::ceil(kScreenGate * (double)C);
            sgrid = sm_count() * screen_ctas_per_sm(sa);
            a.prob[0].cellList = ctx->dPend2;
            a.prob[0].countDev = (const int *)(S.q + 4);
        }
    }
    float ms[3] = {0, 0, 0};
    cudaStream_t st = ctx->stream;
    for (int r = 0; r < 4; r++) {
        if (cudaMemcpyAsync(S.u, ctx->dMom, C * n * 8, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(S.a, ctx->dAlpha, C * n * 8, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(S.it, ctx->dIters, C * sizeof(int), cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
            cudaMemsetAsync(S.q, 0, 5 * sizeof(unsigned), st) != cudaSuccess ||
            cudaMemsetAsync(S.err, 0, 2 * sizeof(int), st) != cudaSuccess)
            return -1.0f;
        cudaEventRecord(S.e0, st);
        if (sgrid > 0) {
            if (launch_screen_gate(S.it, 0, (int)C, (int *)(S.q + 3), st) != cudaSuccess ||
                launch_screen(sa, sgrid, st) != cudaSuccess ||
                launch_order_cells(ctx->dPend, (const int *)(S.q + 2), 0, (int)C, (const int *)(S.q + 3),
                                   sa.prob[0].gateMin, kOrderWholeMax, S.it, ctx->dPend2, (int *)(S.q + 4),
                                   st) != cudaSuccess)
                return -1.0f;
            g_launches += 3;
        }
        if (launch_newton(a, grid, st) != cudaSuccess)
            return -1.0f;
        g_launches++;
        cudaEventRecord(S.e1, st);
        if (cudaStreamSynchronize(st) != cudaSuccess)
            return -1.0f;
        int herr[2] = {0, 0};
        cudaMemcpy(herr, S.err, sizeof(herr), cudaMemcpyDeviceToHost);
        if (herr[0] != 0)
            return -1.0f;
        if (r > 0)
            cudaEventElapsedTime(&ms[r - 1], S.e0, S.e1);
    }
    return median3(ms);
}

static float time_flux(cl_ctx *ctx, FluxArgs f, TuneScratch &S)
{
    const size_t C = (size_t)ctx->C, n = (size_t)ctx->n;
    f.moments = S.u;
    f.alpha = ctx->dAlpha;
    f.momentsOld = nullptr;
    f.tilesRun = nullptr;
    f.dt = 1e-6;
    f.dx = f.dy = 1.0;
    if (plan_flux(f) != 0 || prepare_flux(f) != cudaSuccess)
        return -1.0f;
    float ms[3] = {0, 0, 0};
    cudaStream_t st = ctx->stream;
    for (int r = 0; r < 4; r++) {
        if (cudaMemcpyAsync(S.u, ctx->dMom, C * n * 8, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            return -1.0f;
        cudaEventRecord(S.e0, st);
        if (launch_flux(f, st) != cudaSuccess)
            return -1.0f;
        g_launches++;
        cudaEventRecord(S.e1, st);
        if (cudaStreamSynchronize(st) != cudaSuccess)
            return -1.0f;
        if (r > 0)
            cudaEventElapsedTime(&ms[r - 1], S.e0, S.e1);
    }
    return median3(ms);
}

// Makes the shapes current: K1 with `nw` warps on the Newton layout
// `ncontr`, K2+K3 on the flux layout `fcontr`.
static int apply_shape(cl_ctx *ctx, int nw, int ncontr, int fcontr)
{
    const int wantNP = ncontr == CL_CONTRACT_PAIRS, wantFP = fcontr == CL_CONTRACT_PAIRS;
    if ((wantNP != ctx->B.paired || wantFP != ctx->B.fluxPaired) && ensure_alt_basis(ctx) != CL_OK)
        return CL_ERR_CUDA;
    const DeviceBasis *bn = (wantNP == ctx->B.paired) ? &ctx->B : (ctx->B2.P && ctx->B2.paired == wantNP) ? &ctx->B2 : nullptr;
    const DeviceBasis *bf = (wantFP == ctx->B.fluxPaired) ? &ctx->B
                            : (ctx->B2.Pf && ctx->B2.fluxPaired == wantFP) ? &ctx->B2 : nullptr;
    if (!bn || !bf) {
        ctx->err = "launch shape: that contraction layout does not exist for this configuration";
        return CL_ERR_ARG;
    }
    NewtonArgs a;
    if (!newton_shape(ctx, *bn, nw, a)) {
        ctx->err = "launch shape: no Newton instance for that shape";
        return CL_ERR_ARG;
    }
    FluxArgs f = ctx->fargs;
    flux_basis(f, *bf);
    if (plan_flux(f) != 0 || prepare_flux(f) != cudaSuccess) {
        ctx->err = "launch shape: flux layout";
        return CL_ERR_ARG;
    }
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->nargs = a;
    ctx->nCtas = sm_count() * newton_ctas_per_sm(a);
    ctx->fargs = f;
    ctx->newtonB2 = (bn == &ctx->B2);
    ctx->fluxB2 = (bf == &ctx->B2);
    if (!ctx->newtonB2 && !ctx->fluxB2)
        ctx->B2.release();
    update_screen(ctx);
    invalidate_graph(ctx);
    ctx->tuning.newton_warps = nw;
    ctx->tuning.newton_ctas = ctx->nCtas;
    ctx->tuning.newton_contraction = ncontr;
    ctx->tuning.flux_contraction = fcontr;
    return CL_OK;
}

// Cache of tuned shapes: key -> (nw, Newton contraction, flux contraction).
static std::mutex g_tune_mutex;
static std::map<std::string, std::array<int, 3>> g_tune_cache;
static bool g_tune_file_read = false;

static std::string tune_key(const cl_ctx *ctx)
{
    char buf[160];
    snprintf(buf, sizeof(buf), "n%d_n2%d_nq%d_gaunt%d_mt%d_prec%d_opt%d", ctx->angN, ctx->angN2, ctx->angNq,
             ctx->angGaunt, ctx->opt.moment_type, ctx->opt.precision, ctx->opt.opt_type);
    return buf;
}

static void tune_cache_load()
{
    if (g_tune_file_read)
        return;
    g_tune_file_read = true;
    const char *path = getenv("CL_TUNE_CACHE");
    if (!path || !*path)
        return;
    FILE *fp = fopen(path, "r");
    if (!fp)
        return;
    char key[160];
    int v[3];
    while (fscanf(fp, "%159s %d %d %d", key, &v[0], &v[1], &v[2]) == 4)
        g_tune_cache[key] = {v[0], v[1], v[2]};
    fclose(fp);
}

static void tune_cache_store(const std::string &key, const std::array<int, 3> &v)
{
    g_tune_cache[key] = v;
    const char *path = getenv("CL_TUNE_CACHE");
    if (!path || !*path)
        return;
    FILE *fp = fopen(path, "a");
    if (!fp)
        return;
    fprintf(fp, "%s %d %d %d\n", key.c_str(), v[0], v[1], v[2]);
    fclose(fp);
}

extern "C" {

int cl_get_tuning(cl_ctx *ctx, cl_tuning *out)
{
    if (!ctx || !out)
        return CL_ERR_ARG;
    *out = ctx->tuning;
    return CL_OK;
}

int cl_set_uniform_flux_skip(cl_ctx *ctx, int enable)
{
    if (!ctx)
        return CL_ERR_ARG;
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->fargs.skipUniform = enable ? 1 : 0;
    invalidate_graph(ctx);
    return CL_OK;
}

int cl_set_range_test(cl_ctx *ctx, int enable)
{
    if (!ctx)
        return CL_ERR_ARG;
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->rangeTest = enable ? 1 : 0;
    ctx->nargs.prob[0].gramLo = enable ? make_problem(ctx->newtonB2 ? ctx->B2 : ctx->B).gramLo : 0.0;
    update_screen(ctx);
    invalidate_graph(ctx);
    return CL_OK;
}

int cl_set_launch_shape(cl_ctx *ctx, int newton_warps, int newton_contraction, int flux_contraction)
{
    if (!ctx || (newton_warps != 8 && newton_warps != 4) ||
        (newton_contraction != CL_CONTRACT_PAIRS && newton_contraction != CL_CONTRACT_SINGLE) ||
        (flux_contraction != CL_CONTRACT_PAIRS && flux_contraction != CL_CONTRACT_SINGLE))
        return CL_ERR_ARG;
    int rc = apply_shape(ctx, newton_warps, newton_contraction, flux_contraction);
    if (rc == CL_OK) {
        ctx->tuning.from_cache = 0;
        ctx->tuning.ncand = 0;
    }
    return rc;
}

int cl_tune(cl_ctx *ctx, int use_cache, cl_tuning *out)
{
    if (!ctx)
        return CL_ERR_ARG;
    const long long kMinCells = 16384;
    if (ctx->C < kMinCells || ctx->nargs.optType != 0) {
        // too small to time meaningfully, or a change-of-basis type: defaults
        if (out)
            *out = ctx->tuning;
        return CL_OK;
    }
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    tune_cache_load();
    const std::string key = tune_key(ctx);
    auto hit = g_tune_cache.find(key);
    if (use_cache && hit != g_tune_cache.end()) {
        int rc = apply_shape(ctx, hit->second[0], hit->second[1], hit->second[2]);
        if (rc != CL_OK)
            return rc;
        ctx->tuning.from_cache = 1;
        ctx->tuning.ncand = 0;
        if (out)
            *out = ctx->tuning;
        return CL_OK;
    }
    int rc = ensure_alt_basis(ctx);
    if (rc != CL_OK)
        return rc;
    const size_t C = (size_t)ctx->C, n = (size_t)ctx->n;
    TuneScratch S;
    if (cudaMalloc(&S.u, C * n * 8) != cudaSuccess || cudaMalloc(&S.a, C * n * 8) != cudaSuccess ||
        cudaMalloc(&S.it, C * sizeof(int)) != cudaSuccess || cudaMalloc(&S.err, 2 * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&S.q, 5 * sizeof(unsigned)) != cudaSuccess || cudaMalloc(&S.st, sizeof(DevStats)) != cudaSuccess ||
        cudaEventCreate(&S.e0) != cudaSuccess || cudaEventCreate(&S.e1) != cudaSuccess) {
        ctx->err = "tuner scratch";
        return CL_ERR_CUDA;
    }
    cl_tuning T = ctx->tuning;
    T.ncand = 0;
    T.from_cache = 0;
    // K1 candidates: each existing Newton layout in each launch shape
    float bestN = 1e30f;
    int bestNw = ctx->tuning.newton_warps, bestNc = ctx->tuning.newton_contraction;
    for (const DeviceBasis *B : {&ctx->B, &ctx->B2}) {
        if (!B->P || (B == &ctx->B2 && B->paired == ctx->B.paired))
            continue;
        for (int nw : {8, 4}) {
            NewtonArgs a;
            if (!newton_shape(ctx, *B, nw, a))
                continue;
            const float ms = time_newton(ctx, a, *B, S);
            if (ms < 0 || T.ncand >= CL_TUNE_MAX)
                continue;
            const int contr = B->paired ? CL_CONTRACT_PAIRS : CL_CONTRACT_SINGLE;
            T.cand_kernel[T.ncand] = 1;
            T.cand_warps[T.ncand] = nw;
            T.cand_contraction[T.ncand] = contr;
            T.cand_ms[T.ncand] = ms;
            T.ncand++;
            if (ms < bestN) {
                bestN = ms;
                bestNw = nw;
                bestNc = contr;
            }
        }
    }
    // K2+K3 candidates: the two flux layouts
    float bestF = 1e30f;
    int bestFc = ctx->tuning.flux_contraction;
    for (const DeviceBasis *B : {&ctx->B, &ctx->B2}) {
        if (!B->Pf || (B == &ctx->B2 && B->fluxPaired == ctx->B.fluxPaired))
            continue;
        FluxArgs f = ctx->fargs;
        flux_basis(f, *B);
        const float ms = time_flux(ctx, f, S);
        if (ms < 0 || T.ncand >= CL_TUNE_MAX)
            continue;
        const int contr = B->fluxPaired ? CL_CONTRACT_PAIRS : CL_CONTRACT_SINGLE;
        T.cand_kernel[T.ncand] = 2;
        T.cand_warps[T.ncand] = 16;
        T.cand_contraction[T.ncand] = contr;
        T.cand_ms[T.ncand] = ms;
        T.ncand++;
        if (ms < bestF) {
            bestF = ms;
            bestFc = contr;
        }
    }
    rc = apply_shape(ctx, bestNw, bestNc, bestFc);
    if (rc != CL_OK)
        return rc;
    T.newton_warps = ctx->tuning.newton_warps;
    T.newton_ctas = ctx->tuning.newton_ctas;
    T.screen_ctas = ctx->tuning.screen_ctas;
    T.newton_contraction = bestNc;
    T.flux_contraction = bestFc;
    ctx->tuning = T;
    tune_cache_store(key, {bestNw, bestNc, bestFc});
    if (out)
        *out = T;
    return CL_OK;
}

}  // extern "C"

extern "C" {

int cl_set_warm_start(cl_ctx *ctx, cl_mlp *m) { return cl_set_warm_start_selective(ctx, m, 0); }

int cl_set_warm_start_selective(cl_ctx *ctx, cl_mlp *m, int min_prev_iters)
{
    if (!ctx || min_prev_iters < 0)
        return CL_ERR_ARG;
    ctx->warmMinIters = m ? min_prev_iters : 0;
    if (m) {
        int rc = clb_mlp_reserve_for(m, (size_t)ctx->C);
        if (rc) {
            ctx->err = "warm-start buffers";
            return rc;
        }
        if (!ctx->dAlphaPred &&
            cudaMalloc(&ctx->dAlphaPred, (size_t)ctx->C * ctx->n * sizeof(double)) != cudaSuccess) {
            ctx->err = "warm-start buffers";
            return CL_ERR_CUDA;
        }
    }
    ctx->warm = m;
    // the captured step changes: re-capture at the next cl_step
    invalidate_graph(ctx);
    return CL_OK;
}

int cl_get_last_iterations(cl_ctx *ctx, int *iters)
{
    if (!ctx || !iters)
        return CL_ERR_ARG;
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    CUDA_TRY(ctx, cudaMemcpy(iters, ctx->dIters, (size_t)ctx->C * sizeof(int), cudaMemcpyDeviceToHost));
    return CL_OK;
}

int cl_set_last_iterations(cl_ctx *ctx, const int *iters)
{
    if (!ctx || !iters)
        return CL_ERR_ARG;
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    CUDA_TRY(ctx, cudaMemcpy(ctx->dIters, iters, (size_t)ctx->C * sizeof(int), cudaMemcpyHostToDevice));
    return CL_OK;
}

int cl_device_state(cl_ctx *ctx, double **d_moments, double **d_alpha)
{
    if (!ctx)
        return CL_ERR_ARG;
    if (d_moments)
        *d_moments = ctx->dMom;
    if (d_alpha)
        *d_alpha = ctx->dAlpha;
    return CL_OK;
}

int cl_get_stats(cl_ctx *ctx, cl_stats *s)
{
    if (!ctx || !s)
        return CL_ERR_ARG;
    DevStats d;
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    CUDA_TRY(ctx, cudaMemcpy(&d, ctx->dStats, sizeof(d), cudaMemcpyDeviceToHost));
    s->max_iter = d.maxIter;
    s->num_solves = (int64_t)d.numSolves;
    s->total_iter = (int64_t)d.totalIter;
    for (int i = 0; i < CL_NUM_REG; i++)
        s->hist_reg[i] = (int64_t)d.hist[i];
    s->iter_mean = d.numSolves ? (double)d.totalIter / (double)d.numSolves : 0.0;
    s->total_trials = (int64_t)d.trials;
    s->fallbacks = (int64_t)d.fallbacks;
    s->screened = (int64_t)d.screened;
    s->screen_evals = (int64_t)d.screenEvals;
    s->flux_tiles = (int64_t)d.fluxTiles;
    return CL_OK;
}

int cl_solve_batch_device(cl_ctx *ctx, int count, double *d_u, double *d_alpha, int *d_iters, double *d_reg,
                          int *d_status)
{
    return cl_solve_batch_device_start(ctx, count, d_u, d_alpha, nullptr, d_iters, d_reg, d_status);
}

int cl_solve_batch_device_start(cl_ctx *ctx, int count, double *d_u, double *d_alpha, const double *d_alpha_start,
                                int *d_iters, double *d_reg, int *d_status)
{
    if (!ctx || count < 0 || (count > 0 && (!d_u || !d_alpha)))
        return CL_ERR_ARG;
    if (ctx->nargs.optType != 0) {
        ctx->err = "change-of-basis contexts solve batches with cl_solve_batch_cb_device";
        return CL_ERR_STATE;
    }
    if (count == 0)
        return CL_OK;
    NewtonArgs a = ctx->nargs;
    a.prob[0].count = count;
    a.prob[0].u = d_u;
    a.prob[0].alpha = d_alpha;
    a.prob[0].iters = d_iters;
    a.prob[0].regs = d_reg;
    a.prob[0].status = d_status;
    a.prob[0].alphaStart = d_alpha_start;
    a.prob[0].queue = ctx->dQueue + 2;
    a.momentsOld = nullptr;
    CUDA_TRY(ctx, cudaMemsetAsync(ctx->dQueue + 2, 0, sizeof(unsigned), ctx->stream));
    CUDA_TRY(ctx, launch_newton(a, ctx->nCtas, ctx->stream));
    g_launches += 1;
    return CL_OK;
}

int cl_solve_batch_cb_device(cl_ctx *ctx, int count, double *d_u, double *d_P2M, double *d_alphaP,
                             double *d_alpha, int *d_iters, double *d_reg, int *d_status)
{
    if (!ctx || count < 0 || (count > 0 && (!d_u || !d_P2M || !d_alphaP || !d_alpha)))
        return CL_ERR_ARG;
    if (ctx->nargs.optType == 0) {
        ctx->err = "the context was not created for MOMOPT_OPTIMIZATION_TYPE 1 or 2";
        return CL_ERR_STATE;
    }
    if (count == 0)
        return CL_OK;
    NewtonArgs a = ctx->nargs;
    a.prob[0].count = count;
    a.prob[0].u = d_u;
    a.prob[0].alpha = d_alpha;
    a.prob[0].P2M = d_P2M;
    a.prob[0].alphaP = d_alphaP;
    a.prob[0].iters = d_iters;
    a.prob[0].regs = d_reg;
    a.prob[0].status = d_status;
    a.prob[0].alphaStart = nullptr;
    a.prob[0].queue = ctx->dQueue + 2;
    a.momentsOld = nullptr;
    CUDA_TRY(ctx, cudaMemsetAsync(ctx->dQueue + 2, 0, sizeof(unsigned), ctx->stream));
    CUDA_TRY(ctx, launch_newton(a, ctx->nCtas, ctx->stream));
    g_launches += 1;
    return CL_OK;
}

int cl_solve_batch(cl_ctx *ctx, int count, double *u, double *alpha, int *iters, double *reg, int *status)
{
    if (!ctx || count < 0 || (count > 0 && (!u || !alpha)))
        return CL_ERR_ARG;
    if (count == 0)
        return CL_OK;
    const size_t n = ctx->n;
    if (count > ctx->bCap) {
        cudaFree(ctx->bU);
        cudaFree(ctx->bA);
        cudaFree(ctx->bR);
        cudaFree(ctx->bI);
        cudaFree(ctx->bS);
        ctx->bU = ctx->bA = ctx->bR = nullptr;
        ctx->bI = ctx->bS = nullptr;
        ctx->bCap = 0;
        CUDA_TRY(ctx, cudaMalloc(&ctx->bU, (size_t)count * n * 8));
        CUDA_TRY(ctx, cudaMalloc(&ctx->bA, (size_t)count * n * 8));
        CUDA_TRY(ctx, cudaMalloc(&ctx->bR, (size_t)count * 8));
        CUDA_TRY(ctx, cudaMalloc(&ctx->bI, (size_t)count * 4));
        CUDA_TRY(ctx, cudaMalloc(&ctx->bS, (size_t)count * 4));
        ctx->bCap = count;
    }
    CUDA_TRY(ctx, cudaMemcpyAsync(ctx->bU, u, (size_t)count * n * 8, cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(ctx->bA, alpha, (size_t)count * n * 8, cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(ctx, cudaMemsetAsync(ctx->dErr, 0, 2 * sizeof(int), ctx->stream));
    int rc = cl_solve_batch_device(ctx, count, ctx->bU, ctx->bA, ctx->bI, ctx->bR, ctx->bS);
    if (rc)
        return rc;
    CUDA_TRY(ctx, cudaMemcpyAsync(u, ctx->bU, (size_t)count * n * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(alpha, ctx->bA, (size_t)count * n * 8, cudaMemcpyDeviceToHost, ctx->stream));
    if (iters)
        CUDA_TRY(ctx, cudaMemcpyAsync(iters, ctx->bI, (size_t)count * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (reg)
        CUDA_TRY(ctx, cudaMemcpyAsync(reg, ctx->bR, (size_t)count * 8, cudaMemcpyDeviceToHost, ctx->stream));
    if (status)
        CUDA_TRY(ctx, cudaMemcpyAsync(status, ctx->bS, (size_t)count * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    rc = read_device_error(ctx);
    cudaMemsetAsync(ctx->dErr, 0, 2 * sizeof(int), ctx->stream);
    return rc;
}

// ---------------------------------------------------------------- multi-order
}  // extern "C"

struct cl_multi {
    cudaStream_t stream = nullptr;
    cl_options opt;
    int nprob = 0;
    DeviceBasis B[kMaxProblems];
    NewtonArgs nargs;
    unsigned int *dQueue = nullptr;
    DevStats *dStats = nullptr;
    int *dErr = nullptr;
    int nCtas = 0;
    std::string err;
};

extern "C" {

const char *cl_multi_last_error(const cl_multi *m) { return m ? m->err.c_str() : g_global_err.c_str(); }

void cl_multi_destroy(cl_multi *m)
{
    if (!m)
        return;
    if (m->stream)
        cudaStreamSynchronize(m->stream);
    for (int p = 0; p < m->nprob; p++)
        m->B[p].release();
    cudaFree(m->dQueue);
    cudaFree(m->dStats);
    cudaFree(m->dErr);
    if (m->stream)
        cudaStreamDestroy(m->stream);
    delete m;
}

int cl_multi_create(int norders, const int *orders, int quad_order, int use_gaunt, const cl_options *opts,
                    cl_multi **out)
{
    if (!out || !orders || norders < 1 || norders > kMaxProblems) {
        g_global_err = "bad order list";
        return CL_ERR_ARG;
    }
    *out = nullptr;
    std::string e;
    int rc = check_options(opts, e);
    if (rc) {
        g_global_err = e;
        return rc;
    }
    if (opts->opt_type != 0) {
        g_global_err = "the change-of-basis solve runs one moment order per context (cl_create)";
        return CL_ERR_ARG;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        g_global_err = "no CUDA device (the B200 path has no CPU fallback)";
        return CL_ERR_CUDA;
    }
    cl_multi *m = new cl_multi();
    m->opt = *opts;
    m->nprob = norders;
    if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) {
        g_global_err = "stream creation failed";
        cl_multi_destroy(m);
        return CL_ERR_CUDA;
    }
    NewtonArgs &a = m->nargs;
    memset(&a, 0, sizeof(a));
    a.nprob = norders;
    for (int p = 0; p < norders; p++) {
        Angular A;
        if (orders[p] > 6 || build_angular(orders[p], quad_order, use_gaunt, A) != 0) {
            g_global_err = "unsupported order (1..6)";
            cl_multi_destroy(m);
            return CL_ERR_ARG;
        }
        cudaError_t ce = build_device_basis(m->B[p], A.n, A.n2, A.nq, A.useGaunt, A.w.data(), A.xi.data(),
                                            A.eta.data(), A.p.data(), A.goff.data(), A.gidx.data(),
                                            A.gval.data(), (int)A.gidx.size());
        if (ce != cudaSuccess) {
            g_global_err = std::string("basis upload: ") + cudaGetErrorString(ce);
            cl_multi_destroy(m);
            return CL_ERR_CUDA;
        }
        a.prob[p] = make_problem(m->B[p]);
    }
    fill_newton_options(a, *opts, use_gaunt ? 1 : 0);
    if (cudaMalloc(&m->dQueue, kMaxProblems * sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&m->dStats, sizeof(DevStats)) != cudaSuccess || cudaMalloc(&m->dErr, 2 * sizeof(int)) != cudaSuccess) {
        g_global_err = "device allocation failed";
        cl_multi_destroy(m);
        return CL_ERR_CUDA;
    }
    cudaMemset(m->dStats, 0, sizeof(DevStats));
    cudaMemset(m->dErr, 0, 2 * sizeof(int));
    a.stats = m->dStats;
    a.err = m->dErr;
    const int pl = plan_newton(a);
    if (pl != 0) {
        g_global_err = pl == -2 ? "mixed precision needs a single moment order per launch"
                                : "Newton kernel layout does not fit in shared memory";
        cl_multi_destroy(m);
        return CL_ERR_ARG;
    }
    if (prepare_newton(a) != cudaSuccess) {
        g_global_err = "Newton kernel attributes";
        cl_multi_destroy(m);
        return CL_ERR_CUDA;
    }
    m->nCtas = sm_count() * newton_ctas_per_sm(a);
    cudaDeviceSynchronize();
    *out = m;
    return CL_OK;
}

int cl_multi_solve_device(cl_multi *m, const int *counts, double *const *d_u, double *const *d_alpha,
                          int *const *d_iters, double *const *d_reg, int *const *d_status)
{
    return cl_multi_solve_device_start(m, counts, d_u, d_alpha, nullptr, d_iters, d_reg, d_status);
}

int cl_multi_solve_device_start(cl_multi *m, const int *counts, double *const *d_u, double *const *d_alpha,
                                double *const *d_alpha_start, int *const *d_iters, double *const *d_reg,
                                int *const *d_status)
{
    if (!m || !counts || !d_u || !d_alpha)
        return CL_ERR_ARG;
    NewtonArgs a = m->nargs;
    for (int p = 0; p < m->nprob; p++) {
        a.prob[p].count = counts[p];
        a.prob[p].u = d_u[p];
        a.prob[p].alpha = d_alpha[p];
        a.prob[p].iters = d_iters ? d_iters[p] : nullptr;
        a.prob[p].regs = d_reg ? d_reg[p] : nullptr;
        a.prob[p].status = d_status ? d_status[p] : nullptr;
        a.prob[p].alphaStart = d_alpha_start ? d_alpha_start[p] : nullptr;
        a.prob[p].queue = m->dQueue + p;
    }
    cudaError_t e = cudaMemsetAsync(m->dQueue, 0, kMaxProblems * sizeof(unsigned), m->stream);
    if (e == cudaSuccess)
        e = launch_newton(a, m->nCtas, m->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(m->stream);
    g_launches += 1;
    if (e != cudaSuccess) {
        m->err = std::string("multi solve: ") + cudaGetErrorString(e);
        return CL_ERR_CUDA;
    }
    int herr[2];
    cudaMemcpy(herr, m->dErr, sizeof(herr), cudaMemcpyDeviceToHost);
    if (herr[0]) {
        m->err = error_text(herr[0]);
        cudaMemset(m->dErr, 0, sizeof(herr));
        return herr[0];
    }
    return CL_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- self check
namespace {
__global__ void dmma_selftest_kernel(const double *A, const double *B, double *C)
{
    // one warp: C[16x8] = A[16x8] . B[8x8] (A row-major, B row-major k x n)
    int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    double c[4] = {0, 0, 0, 0};
    dmma16x8x8(c, A[g * 8 + t], A[(g + 8) * 8 + t], A[g * 8 + t + 4], A[(g + 8) * 8 + t + 4], B[t * 8 + g],
               B[(t + 4) * 8 + g]);
    C[g * 8 + 2 * t] = c[0];
    C[g * 8 + 2 * t + 1] = c[1];
    C[(g + 8) * 8 + 2 * t] = c[2];
    C[(g + 8) * 8 + 2 * t + 1] = c[3];
}
__global__ void tmma_selftest_kernel(const float *A, const float *B, float *C)
{
    // one warp: C[16x8] = A[16x8] . B[8x8] in TF32 (integer-valued inputs: exact)
    int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    float c[4] = {0, 0, 0, 0};
    tmma16x8x8(c, __float_as_uint(A[g * 8 + t]), __float_as_uint(A[(g + 8) * 8 + t]),
               __float_as_uint(A[g * 8 + t + 4]), __float_as_uint(A[(g + 8) * 8 + t + 4]),
               __float_as_uint(B[t * 8 + g]), __float_as_uint(B[(t + 4) * 8 + g]));
    C[g * 8 + 2 * t] = c[0];
    C[g * 8 + 2 * t + 1] = c[1];
    C[(g + 8) * 8 + 2 * t] = c[2];
    C[(g + 8) * 8 + 2 * t + 1] = c[3];
}
}  // namespace

// TF32 fragment layout (the mixed-precision Hessian tiles rely on it).
static int tmma_selftest()
{
    float hA[128], hB[64], hC[128], ref[128];
    for (int i = 0; i < 128; i++)
        hA[i] = (float)((i * 7) % 11 - 5);
    for (int i = 0; i < 64; i++)
        hB[i] = (float)((i * 5) % 9 - 4);
    for (int r = 0; r < 16; r++)
        for (int c = 0; c < 8; c++) {
            float s = 0;
            for (int k = 0; k < 8; k++)
                s += hA[r * 8 + k] * hB[k * 8 + c];
            ref[r * 8 + c] = s;
        }
    float *d = nullptr;
    if (cudaMalloc(&d, sizeof(float) * 320) != cudaSuccess) {
        g_global_err = "selftest allocation failed";
        return CL_ERR_CUDA;
    }
    cudaMemcpy(d, hA, sizeof(hA), cudaMemcpyHostToDevice);
    cudaMemcpy(d + 128, hB, sizeof(hB), cudaMemcpyHostToDevice);
    tmma_selftest_kernel<<<1, 32>>>(d, d + 128, d + 192);
    g_launches += 1;
    cudaError_t e = cudaMemcpy(hC, d + 192, sizeof(hC), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) {
        g_global_err = std::string("selftest: ") + cudaGetErrorString(e);
        return CL_ERR_CUDA;
    }
    for (int i = 0; i < 128; i++)
        if (hC[i] != ref[i]) {
            g_global_err = "TF32 fragment layout mismatch";
            return CL_ERR_STATE;
        }
    return CL_OK;
}

extern "C" int cl_selftest(void)
{
    double hA[128], hB[64], hC[128], ref[128];
    for (int i = 0; i < 128; i++)
        hA[i] = 0.25 * (i % 13) - 1.0 + 1e-3 * i;
    for (int i = 0; i < 64; i++)
        hB[i] = 0.5 * (i % 7) - 1.5 + 1e-4 * i;
    for (int r = 0; r < 16; r++)
        for (int c = 0; c < 8; c++) {
            double s = 0;
            for (int k = 0; k < 8; k++)
                s += hA[r * 8 + k] * hB[k * 8 + c];
            ref[r * 8 + c] = s;
        }
    double *d = nullptr;
    if (cudaMalloc(&d, sizeof(double) * 320) != cudaSuccess) {
        g_global_err = "selftest allocation failed";
        return CL_ERR_CUDA;
    }
    cudaMemcpy(d, hA, sizeof(hA), cudaMemcpyHostToDevice);
    cudaMemcpy(d + 128, hB, sizeof(hB), cudaMemcpyHostToDevice);
    dmma_selftest_kernel<<<1, 32>>>(d, d + 128, d + 192);
    g_launches += 1;
    cudaError_t e = cudaMemcpy(hC, d + 192, sizeof(hC), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) {
        g_global_err = std::string("selftest: ") + cudaGetErrorString(e);
        return CL_ERR_CUDA;
    }
    for (int i = 0; i < 128; i++)
        if (std::fabs(hC[i] - ref[i]) > 1e-12 * (1.0 + std::fabs(ref[i]))) {
            g_global_err = "DMMA fragment layout mismatch";
            return CL_ERR_STATE;
        }
    return tmma_selftest();
}

// Lets the host solver layer report through cl_global_error().
void clb_set_global_error(const char *msg) { g_global_err = msg ? msg : ""; }

// Kernel launches of the other translation units, for cl_launch_count().
void clb_count_launches(long long k) { g_launches += k; }

// ------------------------------------------------------------- FP64 peak
namespace {
// Independent DMMA chains per warp; each m16n8k8 is 1024 FMA = 2048 flops.
__global__ void dmma_peak_kernel(double *out, int iters)
{
    double a0 = 1e-3 * threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3;
    double b0 = 2e-3 * threadIdx.x, b1 = b0 + 1;
    double c[8][4];
#pragma unroll
    for (int u = 0; u < 8; u++)
        c[u][0] = c[u][1] = c[u][2] = c[u][3] = 0.0;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int u = 0; u < 8; u++)
            dmma16x8x8(c[u], a0, a1, a2, a3, b0, b1);
    }
    double s = 0;
#pragma unroll
    for (int u = 0; u < 8; u++)
        s += c[u][0] + c[u][1] + c[u][2] + c[u][3];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}
}  // namespace

extern "C" int cl_fp64_peak(double *tflops)
{
    if (!tflops)
        return CL_ERR_ARG;
    int sms = sm_count();
    if (sms <= 0) {
        g_global_err = "no CUDA device";
        return CL_ERR_CUDA;
    }
    const int blocks = sms * 4, threads = 256, iters = 4000;
    double *d = nullptr;
    if (cudaMalloc(&d, sizeof(double) * blocks * threads) != cudaSuccess) {
        g_global_err = "peak probe allocation failed";
        return CL_ERR_CUDA;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    dmma_peak_kernel<<<blocks, threads>>>(d, 100);
    float best = 1e30f;
    for (int r = 0; r < 3; r++) {
        cudaEventRecord(e0);
        dmma_peak_kernel<<<blocks, threads>>>(d, iters);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        best = ms < best ? ms : best;
    }
    g_launches += 4;
    cudaError_t e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    if (e != cudaSuccess) {
        g_global_err = std::string("peak probe: ") + cudaGetErrorString(e);
        return CL_ERR_CUDA;
    }
    double flops = 2048.0 * 8.0 * iters * (blocks * (threads / 32));
    *tflops = flops / (best * 1e-3) / 1e12;
    return CL_OK;
}

// ---------------------------------------------------------- exp accuracy
namespace {
__global__ void exp_check_kernel(const double *x, int n, double *fast, double *ref, ExpConsts ex)
{
    __shared__ double tab[64];
    for (int i = threadIdx.x; i < 64; i += blockDim.x)
        tab[i] = ex.tab[i];
    __syncthreads();
    // the batched form the kernels use: four consecutive inputs per thread
    int i = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
    if (i + 3 < n) {
        double xv[4] = {x[i], x[i + 1], x[i + 2], x[i + 3]}, yv[4];
        fast_exp_n<4>(yv, xv, tab, ex.invL, ex.L1, ex.L2);
        for (int h = 0; h < 4; h++) {
            fast[i + h] = yv[h];
            ref[i + h] = exp(xv[h]);
        }
    } else {
        for (; i < n; i++) {
            fast[i] = fast_exp(x[i], tab, ex.invL, ex.L1, ex.L2);
            ref[i] = exp(x[i]);
        }
    }
}
}  // namespace

extern "C" int cl_exp_check(const double *x, int n, double *fast, double *ref)
{
    if (!x || !fast || !ref || n <= 0)
        return CL_ERR_ARG;
    double *d = nullptr;
    if (cudaMalloc(&d, sizeof(double) * 3 * (size_t)n) != cudaSuccess) {
        g_global_err = "exp check allocation failed";
        return CL_ERR_CUDA;
    }
    ExpConsts ex;
    exp_consts_init(ex);
    cudaMemcpy(d, x, sizeof(double) * n, cudaMemcpyHostToDevice);
    exp_check_kernel<<<((n + 3) / 4 + 255) / 256, 256>>>(d, n, d + n, d + 2 * (size_t)n, ex);
    g_launches += 1;
    cudaMemcpy(fast, d + n, sizeof(double) * n, cudaMemcpyDeviceToHost);
    cudaError_t e = cudaMemcpy(ref, d + 2 * (size_t)n, sizeof(double) * n, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) {
        g_global_err = std::string("exp check: ") + cudaGetErrorString(e);
        return CL_ERR_CUDA;
    }
    return CL_OK;
}
