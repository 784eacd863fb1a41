// flux.cu -- second-order kinetic flux, Euler/collision/source update and
// Heun average for one RK stage, fused in one kernel.
//
// Replaces MomOptSolver::solveFlux (src/momopt/momopt_update.cpp:96-202) and
// the stage updates (:316-336, :344-364, :367-377).  The reference loops q
// outermost and streams a whole-grid ansatz array once per quadrature point;
// here a CTA owns a 16 x 16 tile of interior cells and, per chunk of 16
// directions:
//   1. ansatz on the tile + 2-cell halo: S = alpha . P^T on the FP64 tensor
//      cores (DMMA), then exp (Mn) or the PPn closure (computeAnsatz :38-69);
//   2. the limited upwind stencil per (cell, q): slopefit / minmod with theta
//      (:77-90), the four upwind branches by sign(xi_q), sign(eta_q)
//      (:145-188), F = (flux1+flux2)/dx + (flux3+flux4)/dy;
//   3. projection flux_k += F . p_qk on the tensor cores.
// The epilogue applies u0*(1+dt sigma_s-dt sigma_t)-dt F0, u_k*(1-dt
// sigma_t)-dt F_k, the lattice source at the cell's lower-left corner
// coordinate, and (stage 2) the average with the saved moments.
#include "flux.cuh"

#include "closures_gpu.h"

namespace clb {

namespace {

constexpr int TX = 16, TY = 16;            // interior tile (x slow, y fast)
constexpr int HX = TX + 4, HY = TY + 4;    // with the 2-cell halo
constexpr int HC = HX * HY;                // 400 halo cells (25 m16 tiles)
constexpr int IC = TX * TY;                // 256 interior cells (16 m16 tiles)
// The stencils never read the 2 x 2 halo corners: the ansatz runs on the
// other 384 halo cells (24 m16 tiles), taken row by row.
constexpr int kAnsatzTiles = (HC - 16) / 16;
__device__ __forceinline__ int halo_cell(int r)
{
    if (r < 2 * TY)
        return (r / TY) * HY + 2 + r % TY;
    r -= 2 * TY;
    if (r < TX * HY)
        return (2 + r / HY) * HY + r % HY;
    r -= TX * HY;
    return (TX + 2 + r / TY) * HY + 2 + r % TY;
}
constexpr int kFluxThreads = 512;          // 16 warps: one interior m-tile each
constexpr int kFluxWarps = kFluxThreads / 32;
constexpr int kQ = 16;                     // directions per chunk
static_assert(kFluxWarps == kQ && TX == 16 && TY == 16, "stencil mapping: one warp per direction, 16 x 16 tile");
constexpr double kSqrtPi = 1.7724538509055160273;

// slopefit(l, c, r, theta) = minmod(theta (r - c), minmod((r - l) / 2,
// theta (c - l))) with minmod(x, y) = SIGN(1,x) MAX(0, MIN(|x|, y SIGN(1,x)))
// (momopt_update.cpp:77-90).  The nested form equals, exactly, sign(a)
// min(|a|, |b|, |c|) when a, b, c share one sign and 0 otherwise (only the
// sign of a zero result can differ); the sign test runs on the integer
// high words.
__device__ __forceinline__ double minmod3(double a, double b, double c)
{
    const double m = fmin(fabs(a), fmin(fabs(b), fabs(c)));
    const int ha = __double2hiint(a), hb = __double2hiint(b), hc = __double2hiint(c);
    return (((ha ^ hb) | (ha ^ hc)) >= 0) ? copysign(m, a) : 0.0;
}

__device__ __forceinline__ double slopefit(double l, double c, double r, double th)
{
    return minmod3(th * (r - c), 0.5 * (r - l), th * (c - l));
}

// The closure of the ansatz (computeAnsatz, momopt_update.cpp:38-69) on K
// kinetic values: exp for Mn, the positive-part closure for PPn.
template <int K>
__device__ __forceinline__ void closure_n(double (&v)[K], const double (&kin)[K], const FluxArgs &f,
                                          const double *sExp)
{
    if (f.momentType == 0) {
        fast_exp_n<K>(v, kin, sExp, f.ex.invL, f.ex.L1, f.ex.L2);
    } else {
        const double dl = f.deltaPPn;
#pragma unroll
        for (int h = 0; h < K; h++) {
            const double x = kin[h];
            if (x > 0)
                v[h] = 0.5 * x + 0.5 * sqrt(x * x + 4 * dl);
            else
                v[h] = -dl / (0.5 * x - 0.5 * sqrt(x * x + 4 * dl));
        }
    }
}

// PAIR = 1: direction pairs.  Directions q and q + Q (phi and phi + pi) have
// the same weight and p_l(q + Q) = (-1)^l p_l(q), so with the basis columns
// grouped by degree parity one MMA chain per parity gives both exponents,
// S(q) = S_even + S_odd and S(q + Q) = S_even - S_odd, and the projection
// takes F(q) + F(q + Q) on the even columns and F(q) - F(q + Q) on the odd
// ones: half the tensor-core work of one direction at a time.  The stencil
// is per direction either way.
template <int PAIR>
__global__ void __launch_bounds__(kFluxThreads, 1) flux_kernel(const __grid_constant__ FluxArgs f)
{
    extern __shared__ __align__(16) double sm[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t4 = lane & 3;
    const int tile = blockIdx.x + f.tileBase;
    const int bx = tile / f.tilesY, by = tile % f.tilesY;
    const int i0 = 2 + bx * TX, j0 = 2 + by * TY;     // first interior cell of the tile
    const int n = f.n, nb = f.nb, ldPf = f.ldPf;
    constexpr int kq = kQ;
    const int ldAl = f.ldAl, ldA = f.ldA, ldF = f.ldF;
    double *sAl = sm + f.offAl;     // [HC][ldAl]
    double *sA = sm + f.offA;       // [kq][ldA] ansatz, q-major
    double *sF = sm + f.offF;       // [kq][ldF] stencil flux, q-major
    double *sP = sm + f.offP;       // [2][kq][ldPf]
    double *sQ = sm + f.offQ;       // [2][4][kq] xi, eta, xi*w, eta*w
    double *sExp = sm + f.offExp;   // fast_exp table
    for (int i = tid; i < 64; i += kFluxThreads)
        sExp[i] = f.ex.tab[i];

    // alpha of the halo region in the basis's column order (zero outside
    // the grid)
    for (int idx = tid; idx < HC * nb; idx += kFluxThreads) {
        int h = idx / nb, c = idx % nb;
        int hi = h / HY, hj = h % HY;
        int i = i0 - 2 + hi, j = j0 - 2 + hj;
        const int k = PAIR ? (int)f.binv[c] : c;
        double v = 0.0;
        if (k >= 0 && k < n && i < f.NX && j < f.NY)
            v = f.alpha[((size_t)i * f.NY + j) * n + k];
        sAl[h * ldAl + c] = v;
    }

    constexpr int kr = PAIR ? kQ / 2 : kQ;   // rows of P per chunk
    const int nchunks = f.nqp / kr;
    auto load_chunk = [&](int c, int buf) {
        const double *src = f.P + (size_t)c * kr * ldPf;
        double *dst = sP + buf * kq * ldPf;
        for (int i = tid; i < kr * ldPf / 2; i += kFluxThreads)
            cp_async16(dst + 2 * i, src + 2 * i);
        double *q = sQ + buf * 4 * kq;
        for (int i = tid; i < kq / 2; i += kFluxThreads) {
            cp_async16(q + 2 * i, f.xi + c * kq + 2 * i);
            cp_async16(q + kq + 2 * i, f.eta + c * kq + 2 * i);
            cp_async16(q + 2 * kq + 2 * i, f.cxw + c * kq + 2 * i);
            cp_async16(q + 3 * kq + 2 * i, f.cyw + c * kq + 2 * i);
        }
        cp_async_commit();
    };

    // projection accumulators: warp owns interior m-tile `warp` (16 cells), all k tiles
    double acc[4][4];
#pragma unroll
    for (int j = 0; j < 4; j++)
        acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0;
    const int NTf = nb / 8;
    const int ntiles1 = kAnsatzTiles * (kq / 8);

    // Per chunk: the stencil, then in one barrier interval the projection of
    // this chunk and the ansatz of the next (they use disjoint buffers), so a
    // chunk takes two CTA barriers and the projection's MMAs interleave with
    // the next ansatz's exponentials across warps.
    auto ansatz = [&](const double *Pb) {
        // 1. ansatz on the halo tile
        if (PAIR) {
            const int nbe = f.nbe;
            for (int mt = warp; mt < kAnsatzTiles; mt += kFluxWarps) {
                double ce[4] = {0.0, 0.0, 0.0, 0.0}, co[4] = {0.0, 0.0, 0.0, 0.0};
                const int c0 = halo_cell(mt * 16 + g), c1 = halo_cell(mt * 16 + g + 8);
                const double *A0 = sAl + c0 * ldAl;
                const double *A1 = sAl + c1 * ldAl;
                const double *B = Pb + g * ldPf;
                for (int k0 = 0; k0 < nbe; k0 += 8)
                    dmma16x8x8(ce, A0[k0 + t4], A1[k0 + t4], A0[k0 + t4 + 4], A1[k0 + t4 + 4], B[k0 + t4],
                               B[k0 + t4 + 4]);
                for (int k0 = nbe; k0 < nb; k0 += 8)
                    dmma16x8x8(co, A0[k0 + t4], A1[k0 + t4], A0[k0 + t4 + 4], A1[k0 + t4 + 4], B[k0 + t4],
                               B[k0 + t4 + 4]);
                double kin[8], v[8];
#pragma unroll
                for (int h = 0; h < 4; h++) {
                    kin[h] = ce[h] + co[h];
                    kin[4 + h] = ce[h] - co[h];
                }
                closure_n<8>(v, kin, f, sExp);
#pragma unroll
                for (int h = 0; h < 4; h++) {
                    int cell = (h & 2) ? c1 : c0;
                    int q = 2 * t4 + (h & 1);
                    sA[q * ldA + cell] = v[h];
                    sA[(q + 8) * ldA + cell] = v[4 + h];
                }
            }
        } else
        for (int ti = warp; ti < ntiles1; ti += kFluxWarps) {
            int mt = ti % kAnsatzTiles, nt = ti / kAnsatzTiles;
            double cs[4] = {0.0, 0.0, 0.0, 0.0};
            const int c0 = halo_cell(mt * 16 + g), c1 = halo_cell(mt * 16 + g + 8);
            const double *A0 = sAl + c0 * ldAl;
            const double *A1 = sAl + c1 * ldAl;
            const double *B = Pb + (nt * 8 + g) * ldPf;
            for (int k0 = 0; k0 < nb; k0 += 8)
                dmma16x8x8(cs, A0[k0 + t4], A1[k0 + t4], A0[k0 + t4 + 4], A1[k0 + t4 + 4], B[k0 + t4],
                           B[k0 + t4 + 4]);
            double v[4];
            closure_n<4>(v, cs, f, sExp);
#pragma unroll
            for (int h = 0; h < 4; h++) {
                int cell = (h & 2) ? c1 : c0;
                int q = nt * 8 + 2 * t4 + (h & 1);
                sA[q * ldA + cell] = v[h];
            }
        }
    };
    auto stencil = [&](const double *Qb) {
        // 2. limited upwind stencil.  Thread (q = warp, column j = lane % 16)
        //    sweeps interior rows ib..ib+7 (ib = 8 * (lane / 16)) down its
        //    column: each slopefit of a cell is formed once and serves the
        //    cell's own face and its neighbour's (x: down the sweep, y: by a
        //    lane shuffle), in the reference's expression
        //    ((k3 +- sf/2) - k2) -+ sf'/2 (:145-188).
        //    The 1/dx, 1/dy of F are folded into xi w / dx and eta w / dy.
        {
            const int q = warp;
            const int j = lane & 15, ib = (lane >> 4) * 8;
            const double *col = sA + q * ldA + (j + 2) + 2 * HY;   // col[i * HY] = ansatz of interior row i
            const double xi = Qb[q], eta = Qb[kq + q];
            const double cxd = Qb[2 * kq + q] / f.dx, cyd = Qb[3 * kq + q] / f.dy;
            const double th = f.theta;
            double fx[8];
            if (xi > 0) {
                // flux1(i) = ((k_i + sf_i / 2) - k_{i-1}) - sf_{i-1} / 2,
                // sf_i = slopefit(k_{i-1}, k_i, k_{i+1})
                double km1 = col[(ib - 1) * HY], k0 = col[ib * HY];
                double sprev = slopefit(col[(ib - 2) * HY], km1, k0, th);
#pragma unroll
                for (int r = 0; r < 8; r++) {
                    const double kp1 = col[(ib + r + 1) * HY];
                    const double sc = slopefit(km1, k0, kp1, th);
                    fx[r] = (((k0 + 0.5 * sc) - km1) - 0.5 * sprev) * cxd;
                    sprev = sc;
                    km1 = k0;
                    k0 = kp1;
                }
            } else {
                // flux2(i) = ((k_{i+1} - sf_{i+1} / 2) - k_i) + sf_i / 2
                double k0 = col[ib * HY], kp1 = col[(ib + 1) * HY];
                double scur = slopefit(col[(ib - 1) * HY], k0, kp1, th);
#pragma unroll
                for (int r = 0; r < 8; r++) {
                    const double kp2 = col[(ib + r + 2) * HY];
                    const double sn = slopefit(k0, kp1, kp2, th);
                    fx[r] = (((kp1 - 0.5 * sn) - k0) + 0.5 * scur) * cxd;
                    scur = sn;
                    k0 = kp1;
                    kp1 = kp2;
                }
            }
            // y direction: lane j forms sf_j of its row and takes sf_{j-1}
            // (eta > 0) or sf_{j+1} (eta < 0) from its neighbour lane; the
            // tile-edge ones (column -1 or 16) of rows ib..ib+7 are formed
            // by lanes 0..7 of each half in one step
            double edge = 0.0;
            if (j < 8) {
                const double *hr = sA + q * ldA + (ib + j + 2) * HY;   // halo row, column c at hr[c + 2]
                edge = (eta > 0) ? slopefit(hr[0], hr[1], hr[2], th) : slopefit(hr[17], hr[18], hr[19], th);
            }
            double *out = sF + q * ldF + ib * TY + j;
#pragma unroll
            for (int r = 0; r < 8; r++) {
                const double *row = col + (ib + r) * HY;
                const double km = row[-1], k0 = row[0], kp = row[1];
                const double sc = slopefit(km, k0, kp, th);
                const double se = __shfl_sync(0xffffffffu, edge, r, 16);
                double fy;
                if (eta > 0) {
                    double sl = __shfl_up_sync(0xffffffffu, sc, 1, 16);
                    if (j == 0)
                        sl = se;
                    fy = ((k0 + 0.5 * sc) - km) - 0.5 * sl;
                } else {
                    double sr = __shfl_down_sync(0xffffffffu, sc, 1, 16);
                    if (j == 15)
                        sr = se;
                    fy = ((kp - 0.5 * sr) - k0) + 0.5 * sc;
                }
                out[r * TY] = fx[r] + fy * cyd;
            }
        }
    };
    auto projection = [&](const double *Pb) {
        // 3. projection on the basis: flux[ic][k] += F[ic][q] p[q][k]
        if (PAIR) {
            // k = the chunk's 8 pairs; rows t4, t4 + 4 of sF and their
            // partners 8 rows further
            const double *A0 = sF + t4 * ldF + warp * 16 + g;
            const double *A8 = A0 + 8 * ldF;
            const double f0 = A0[0], f1 = A0[8], f2 = A0[4 * ldF], f3 = A0[4 * ldF + 8];
            const double p0 = A8[0], p1 = A8[8], p2 = A8[4 * ldF], p3 = A8[4 * ldF + 8];
            const double s0 = f0 + p0, s1 = f1 + p1, s2 = f2 + p2, s3 = f3 + p3;
            const double d0 = f0 - p0, d1 = f1 - p1, d2 = f2 - p2, d3 = f3 - p3;
            const int nbe = f.nbe;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if (j < NTf) {
                    const double *B0 = Pb + t4 * ldPf + j * 8 + g;
                    if (j * 8 < nbe)
                        dmma16x8x8(acc[j], s0, s1, s2, s3, B0[0], B0[4 * ldPf]);
                    else
                        dmma16x8x8(acc[j], d0, d1, d2, d3, B0[0], B0[4 * ldPf]);
                }
            }
        } else
        for (int k0 = 0; k0 < kq; k0 += 8) {
            const double *A0 = sF + (k0 + t4) * ldF + warp * 16 + g;
            double a0 = A0[0], a1 = A0[8], a2 = A0[4 * ldF], a3 = A0[4 * ldF + 8];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if (j < NTf) {
                    const double *B0 = Pb + (k0 + t4) * ldPf + j * 8 + g;
                    dmma16x8x8(acc[j], a0, a1, a2, a3, B0[0], B0[4 * ldPf]);
                }
            }
        }
    };
    load_chunk(0, 0);
    cp_async_wait<0>();
    __syncthreads();
    // A uniform neighbourhood: when every staged alpha of the tile and its
    // halo is the same, bit for bit, every cell has the same ansatz, every
    // slope and upwind difference is an exact zero, and so is the flux of
    // every interior cell (up to the sign of zero).  The chunk loop is then
    // skipped and the update applies zero flux.  Floor cells that no
    // perturbation has reached, still most of the grid early in a pulse run,
    // stay bit-identical to each other.
    bool differs = false;
    for (int idx = tid; idx < HC * nb; idx += kFluxThreads) {
        const int h = idx / nb, c = idx % nb;
        differs |= __double_as_longlong(sAl[h * ldAl + c]) != __double_as_longlong(sAl[c]);
    }
    const int nloop = (__syncthreads_or(differs) || !f.skipUniform) ? nchunks : 0;
    if (tid == 0 && nloop > 0 && f.tilesRun != nullptr)
        atomicAdd(f.tilesRun, 1ull);
    if (nloop > 0)
        ansatz(sP);   // chunk 0, buffer 0
    __syncthreads();
    for (int c = 0; c < nloop; c++) {
        const int buf = c & 1;
        if (c + 1 < nchunks)
            load_chunk(c + 1, buf ^ 1);   // the buffer of chunk c - 1, free since the last barrier
        stencil(sQ + buf * 4 * kq);
        cp_async_wait<0>();
        __syncthreads();   // the stencil flux of chunk c complete; chunk c + 1 staged
        projection(sP + buf * kq * ldPf);
        if (c + 1 < nchunks)
            ansatz(sP + (buf ^ 1) * kq * ldPf);
        __syncthreads();   // the ansatz of chunk c + 1 complete; chunk c's buffers free
    }

    // epilogue: Euler + collision + source (+ Heun average)
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if (j >= NTf)
            continue;
#pragma unroll
        for (int h = 0; h < 4; h++) {
            int ic = warp * 16 + g + ((h & 2) ? 8 : 0);
            int k = j * 8 + 2 * t4 + (h & 1);
            if (PAIR)
                k = f.binv[k];
            int i = i0 + ic / TY, jj = j0 + ic % TY;
            if (k < 0 || k >= n || i >= f.NX - 2 || jj >= f.NY - 2)
                continue;
            size_t cell = (size_t)i * f.NY + jj;
            double st = f.sigmaT[cell], ss = f.sigmaS[cell];
            double u = f.moments[cell * n + k];
            double F = acc[j][h];
            double dt = f.dt;
            double v;
            if (k == 0)
                v = u * (1.0 + dt * ss - dt * st) - dt * F;
            else
                v = u * (1.0 - dt * st) - dt * F;
            if (k == 0 && f.initCond == 1) {
                double x = f.initX + (i - 2) * f.dx;
                double y = f.initY + (jj - 2) * f.dy;
                if (fabs(x) < 0.5 && fabs(y) < 0.5)
                    v = v + dt * 2.0 * kSqrtPi;
            }
            if (f.momentsOld != nullptr)
                v = 0.5 * (v + f.momentsOld[cell * n + k]);
            f.moments[cell * n + k] = v;
        }
    }
}

__global__ void ghost_periodic_kernel(double *m, int n, int NX, int NY)
{
    // momopt_boundaries.cpp:190-223: x strips over interior j, then y strips
    // over interior i (corners untouched).
    const int ny = NY - 4, nx = NX - 4;
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    int totalX = 2 * ny * n, totalY = 2 * nx * n;
    if (idx < totalX) {
        int k = idx % n, r = idx / n;
        int j = 2 + r % ny, i = r / ny;   // i in {0,1}
        m[((size_t)(0 + i) * NY + j) * n + k] = m[((size_t)(NX - 4 + i) * NY + j) * n + k];
        m[((size_t)(NX - 2 + i) * NY + j) * n + k] = m[((size_t)(2 + i) * NY + j) * n + k];
    }
}

__global__ void ghost_periodic_y_kernel(double *m, int n, int NX, int NY)
{
    const int nx = NX - 4;
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    int total = 2 * nx * n;
    if (idx < total) {
        int k = idx % n, r = idx / n;
        int j = r % 2, i = 2 + r / 2;
        m[((size_t)i * NY + 0 + j) * n + k] = m[((size_t)i * NY + NY - 4 + j) * n + k];
        m[((size_t)i * NY + NY - 2 + j) * n + k] = m[((size_t)i * NY + 2 + j) * n + k];
    }
}

// Node halo (momopt_boundaries.cpp:30-188) for all four sides in one launch:
// pack copies the inner strips of the block into bufs[side], unpack the
// buffers into the ghost strips.  North/south: the two columns next to
// y = max / y = min over the interior i, element (j, i - 2, k) at
// (j * nx + i - 2) * n + k; east/west: the two rows next to x = max / x = min
// over the interior j likewise.  Corners are not exchanged.
__global__ void halo_kernel(double *m, int n, int NX, int NY, HaloBuffers b, int pack)
{
    const int nx = NX - 4, ny = NY - 4;
    const long long cntNS = 2LL * nx * n, cntEW = 2LL * ny * n;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int side;
    if (idx < 2 * cntNS) {
        side = idx < cntNS ? CL_NORTH : CL_SOUTH;
        idx -= (side == CL_SOUTH) ? cntNS : 0;
    } else {
        idx -= 2 * cntNS;
        if (idx >= 2 * cntEW)
            return;
        side = idx < cntEW ? CL_EAST : CL_WEST;
        idx -= (side == CL_WEST) ? cntEW : 0;
    }
    double *buf = b.p[side];
    if (buf == nullptr)
        return;
    const int k = (int)(idx % n);
    const long long r = idx / n;
    int i, j;
    if (side == CL_NORTH || side == CL_SOUTH) {
        const int s = (int)(r / nx);
        i = 2 + (int)(r % nx);
        if (pack)
            j = (side == CL_NORTH) ? NY - 4 + s : 2 + s;
        else
            j = (side == CL_NORTH) ? NY - 2 + s : s;
    } else {
        const int s = (int)(r / ny);
        j = 2 + (int)(r % ny);
        if (pack)
            i = (side == CL_EAST) ? NX - 4 + s : 2 + s;
        else
            i = (side == CL_EAST) ? NX - 2 + s : s;
    }
    double *cell = m + ((size_t)i * NY + j) * n + k;
    if (pack)
        buf[idx] = *cell;
    else
        *cell = buf[idx];
}

}  // namespace

cudaError_t launch_halo(double *moments, int n, int NX, int NY, const HaloBuffers &b, int pack,
                        cudaStream_t stream)
{
    const long long total = 4LL * (NX - 4) * n + 4LL * (NY - 4) * n;
    if (total <= 0)
        return cudaSuccess;
    halo_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(moments, n, NX, NY, b, pack);
    return cudaGetLastError();
}

int plan_flux(FluxArgs &f)
{
    if (f.nb > 32 || f.nb % 8 != 0 || (f.paired && f.binv == nullptr))
        return -1;   // the projection accumulators hold four column tiles
    f.kq = kQ;
    f.ldAl = f.nb + 4;
    f.ldA = HC + 2;      // ldA % 8 == 2: conflict-free fragment stores
    f.ldF = IC + 4;      // ldF % 16 == 4
    int off = 0;
    auto take = [&](int nd) {
        int o = off;
        off += (nd + 1) & ~1;
        return o;
    };
    f.offAl = take(HC * f.ldAl);
    f.offA = take(f.kq * f.ldA);
    f.offF = take(f.kq * f.ldF);
    f.offP = take(2 * f.kq * f.ldPf);
    f.offQ = take(2 * 4 * f.kq);
    f.offExp = take(64);
    exp_consts_init(f.ex);
    f.smemBytes = off * 8;
    f.tilesX = (f.NX - 4 + TX - 1) / TX;
    f.tilesY = (f.NY - 4 + TY - 1) / TY;
    return f.smemBytes <= 227 * 1024 - 64 ? 0 : -1;
}

cudaError_t prepare_flux(const FluxArgs &f)
{
    if (f.paired)
        return cudaFuncSetAttribute(flux_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, f.smemBytes);
    return cudaFuncSetAttribute(flux_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, f.smemBytes);
}

cudaError_t launch_flux_tiles(const FluxArgs &f, int first, int count, cudaStream_t stream)
{
    if (first < 0 || count <= 0 || first + count > f.tilesX * f.tilesY)
        return cudaErrorInvalidValue;
    FluxArgs g = f;
    g.tileBase = first;
    if (g.paired)
        flux_kernel<1><<<count, kFluxThreads, g.smemBytes, stream>>>(g);
    else
        flux_kernel<0><<<count, kFluxThreads, g.smemBytes, stream>>>(g);
    return cudaGetLastError();
}

cudaError_t launch_flux(const FluxArgs &f, cudaStream_t stream)
{
    return launch_flux_tiles(f, 0, f.tilesX * f.tilesY, stream);
}

int flux_tile_rows(const FluxArgs &) { return TX; }

cudaError_t launch_ghost_periodic(double *moments, int n, int NX, int NY, cudaStream_t stream)
{
    int totalX = 2 * (NY - 4) * n;
    ghost_periodic_kernel<<<(totalX + 255) / 256, 256, 0, stream>>>(moments, n, NX, NY);
    int totalY = 2 * (NX - 4) * n;
    ghost_periodic_y_kernel<<<(totalY + 255) / 256, 256, 0, stream>>>(moments, n, NX, NY);
    return cudaGetLastError();
}

}  // namespace clb
