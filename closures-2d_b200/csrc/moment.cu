// moment.cu -- the linear Pn / FPn solver (SOLVER moment, src/moment/) on
// the device: the state of one grid, the RK2 step of MomentSolver::update
// (moment_update.cpp:169-247) and the halo of a partitioned grid.
//
// One kernel per RK stage (pn_tile_kernel on the FP64 tensor cores up to
// order 6, pn_stage_kernel above): for each interior cell it applies the moment
// filter to the stencil values as it loads them (moment_update.cpp:23-40
// scales the interior in place before the ghost copy, so ghost strips that
// hold interior copies are filtered too and the physical boundary's are not),
// forms the four one-sided stencil combinations of moment_update.cpp:95-143,
// multiplies them by the upwind flux operators, and applies the Euler,
// collision and lattice-source update (stage 2 also the Heun average).  The
// state ping-pongs between two buffers: stage 1 reads U and writes V, stage
// 2 reads V and writes U, taking the step's start value of its own cell from
// U, so no cell is overwritten while a neighbour still reads it and no copy
// of the old state is needed.
#include "closures_gpu.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "flux.cuh"

using namespace clb;

void clb_set_global_error(const char *msg);
void clb_count_launches(long long k);

namespace {

constexpr int kPnWarps = 8;   // cells in flight per CTA, one warp each
constexpr int kPnMaxN = 64;   // moments per cell (order <= 9)
constexpr int kPnMaxBands = 16;   // row bands of cl_pn_step_host
constexpr double kSqrtPiPn = 1.7724538509055160273;   // sqrt(M_PI) rounded to double

struct PnArgs {
    const double *in;       // state read by this stage, ghosts filled
    const double *old;      // stage 2: the step's start state, else null
    double *out;            // interior written
    const double *opsT;     // [4][n][n] operators transposed: opsT[(o*n+i)*n+k] = op_o[k][i]
    const double *filter;   // [n] or null
    const double *sigT, *sigS;
    int n, NX, NY, initCond;
    int filteredGhosts;     // bit s: ghost strip of side s holds (filtered) interior values
    double dt, rdx, rdy, dx, dy, initX, initY;
    int rowBegin, rowEnd;   // interior rows (x) of this launch; band starts are multiples of kTI
};

__device__ __forceinline__ bool filtered_cell(const PnArgs &a, int i, int j)
{
    if (i >= 2 && i < a.NX - 2 && j >= 2 && j < a.NY - 2)
        return true;
    int side = (j >= a.NY - 2) ? CL_NORTH : (j < 2) ? CL_SOUTH : (i >= a.NX - 2) ? CL_EAST : CL_WEST;
    return (a.filteredGhosts >> side) & 1;
}

// ca a + cb b + cc c + cd d, left to right without contraction, as the
// reference's expressions (moment_update.cpp:97-98 and the three like it)
// evaluate.
__device__ __forceinline__ double stencil4(double ca, double a, double cb, double b, double cc, double c,
                                           double cd, double d)
{
    double s = __dadd_rn(__dmul_rn(ca, a), __dmul_rn(cb, b));
    s = __dadd_rn(s, __dmul_rn(cc, c));
    return __dadd_rn(s, __dmul_rn(cd, d));
}

template <int R>
__global__ void __launch_bounds__(kPnWarps * 32) pn_stage_kernel(PnArgs a)
{
    extern __shared__ double ops[];   // [4][n][n], as opsT
    const int n = a.n;
    for (int e = threadIdx.x; e < 4 * n * n; e += blockDim.x)
        ops[e] = a.opsT[e];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ny = a.NY - 4;
    const long long cells = (long long)(a.rowEnd - a.rowBegin) * ny;
    for (long long c = (long long)blockIdx.x * kPnWarps + warp; c < cells; c += (long long)gridDim.x * kPnWarps) {
        const int i = 2 + a.rowBegin + (int)(c / ny), j = 2 + (int)(c % ny);
        double t[4][R], self[R];
        const size_t NY = a.NY;
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int k = lane + 32 * r;
            const bool act = k < n;
            const double f = (act && a.filter) ? a.filter[k] : 1.0;
            auto ld = [&](int ci, int cj) {
                if (!act)
                    return 0.0;
                const double v = a.in[((size_t)ci * NY + cj) * n + k];
                return (a.filter && filtered_cell(a, ci, cj)) ? __dmul_rn(v, f) : v;
            };
            const double m0 = ld(i, j);
            const double xm2 = ld(i - 2, j), xm1 = ld(i - 1, j), xp1 = ld(i + 1, j), xp2 = ld(i + 2, j);
            const double ym2 = ld(i, j - 2), ym1 = ld(i, j - 1), yp1 = ld(i, j + 1), yp2 = ld(i, j + 2);
            self[r] = m0;
            // moment_update.cpp:95-143: upwind combinations for xi > 0, xi < 0,
            // eta > 0, eta < 0
            t[0][r] = stencil4(0.25, xp1, 0.75, m0, -1.25, xm1, 0.25, xm2);
            t[1][r] = stencil4(-0.25, xp2, 1.25, xp1, -0.75, m0, -0.25, xm1);
            t[2][r] = stencil4(0.25, yp1, 0.75, m0, -1.25, ym1, 0.25, ym2);
            t[3][r] = stencil4(-0.25, yp2, 1.25, yp1, -0.75, m0, -0.25, ym1);
        }
        // y_k = sum_i op[k][i] t_i per operator (dgemv T on the row-filled
        // arrays); east-west = xi+ part + xi- part, likewise north-south
        double part[4][R];
#pragma unroll
        for (int o = 0; o < 4; o++) {
#pragma unroll
            for (int r = 0; r < R; r++)
                part[o][r] = 0.0;
            const double *opo = ops + (size_t)o * n * n;
#pragma unroll
            for (int rs = 0; rs < R; rs++) {
                const int i0 = 32 * rs;
                const int i1 = (n < i0 + 32) ? n : i0 + 32;
                for (int ii = i0; ii < i1; ii++) {
                    const double ti = __shfl_sync(0xffffffffu, t[o][rs], ii - i0);
#pragma unroll
                    for (int r = 0; r < R; r++) {
                        const int k = lane + 32 * r;
                        if (k < n)
                            part[o][r] = fma(opo[(size_t)ii * n + k], ti, part[o][r]);
                    }
                }
            }
        }
        const size_t cell = (size_t)i * NY + j;
        const double sT = a.sigT[cell], sS = a.sigS[cell];
        const double dt = a.dt;
        bool source = false;
        if (a.initCond == 1) {
            // moment_update.cpp:197-199: x_i = c_initX + (i - c_gX[1]) dx
            const double x = __dadd_rn(a.initX, __dmul_rn((double)(i - 2), a.dx));
            const double y = __dadd_rn(a.initY, __dmul_rn((double)(j - 2), a.dy));
            source = fabs(x) < 0.5 && fabs(y) < 0.5;
        }
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int k = lane + 32 * r;
            if (k >= n)
                continue;
            const double ew = __dadd_rn(part[0][r], part[1][r]);
            const double ns = __dadd_rn(part[2][r], part[3][r]);
            const double F = __dadd_rn(__dmul_rn(a.rdx, ew), __dmul_rn(a.rdy, ns));
            double u;
            if (k == 0) {
                // moment_update.cpp:186-187 / :214-215
                const double g = __dsub_rn(__dadd_rn(1.0, __dmul_rn(dt, sS)), __dmul_rn(dt, sT));
                u = __dsub_rn(__dmul_rn(self[r], g), __dmul_rn(dt, F));
                if (source)
                    u = __dadd_rn(u, __dmul_rn(__dmul_rn(dt, 2.0), kSqrtPiPn));
            } else {
                u = __dsub_rn(__dmul_rn(self[r], __dsub_rn(1.0, __dmul_rn(dt, sT))), __dmul_rn(dt, F));
            }
            if (a.old)
                u = __dmul_rn(0.5, __dadd_rn(u, a.old[cell * n + k]));   // moment_update.cpp:237-246
            a.out[cell * n + k] = u;
        }
    }
}

// Orders up to 6 (n <= 32): tensor-core form of the same stage.  A CTA owns a
// tile of kTI x kTJ interior cells; warp w owns row w of it, so the MMA's 16
// rows are 16 cells along j.  The tile with its 2-cell halo is staged in
// shared memory (filtered on load by the rule above, moments zero-padded to
// NP), the four stencil combinations are formed directly as A fragments
// (16 cells x 8 moments), and the operators, staged once per CTA, are the B
// fragments: ew = T_xi+ Op_xi+^T + T_xi- Op_xi-^T (likewise ns) accumulate in
// FP64 tensor-core MMAs.  Cell and operator rows are padded by 4 doubles so
// the fragment loads spread over the banks.
constexpr int kTI = 8, kTJ = 16;

template <int NP>
__global__ void __launch_bounds__(kTI * 32, 2) pn_tile_kernel(PnArgs a)
{
    constexpr int CS = NP + 4;   // doubles per cell in the tile
    constexpr int OS = NP + 4;   // row stride of the staged operators
    constexpr int RW = kTJ + 4;  // cells per tile row with the halo
    constexpr int NT = NP / 8;
    extern __shared__ double sm[];
    double *ops = sm;                        // [4][NP][OS]: ops[(o*NP + i)*OS + k] = op_o[k][i]
    double *tile = ops + 4 * NP * OS;        // [kTI+4][RW][CS]
    const int n = a.n, tid = threadIdx.x;
    for (int e = tid; e < 4 * NP * NP; e += blockDim.x) {
        const int o = e / (NP * NP), r = e % (NP * NP), i = r / NP, k = r % NP;
        ops[(o * NP + i) * OS + k] = (i < n && k < n) ? a.opsT[((size_t)o * n + i) * n + k] : 0.0;
    }
    const int lane = tid & 31, warp = tid >> 5, g = lane >> 2, t = lane & 3;
    const int ny = a.NY - 4;
    const int tilesJ = (ny + kTJ - 1) / kTJ;
    const int tiles = ((a.rowEnd - a.rowBegin + kTI - 1) / kTI) * tilesJ;
    const size_t NY = a.NY;
    for (int tl = blockIdx.x; tl < tiles; tl += gridDim.x) {
        const int i0 = 2 + a.rowBegin + (tl / tilesJ) * kTI, j0 = 2 + (tl % tilesJ) * kTJ;
        __syncthreads();   // the previous tile's readers are done (and the operators staged)
        // staged in batches of 8 loads per thread, all issued before any is used
        constexpr int kTileElems = (kTI + 4) * RW * NP, kStep = kTI * 32, kBatch = 8;
        for (int e0 = tid; e0 < kTileElems; e0 += kBatch * kStep) {
            double v[kBatch];
#pragma unroll
            for (int b = 0; b < kBatch; b++) {
                const int e = e0 + b * kStep;
                const int k = e % NP, cell = e / NP, r = cell / RW, c = cell % RW;
                const int gi = i0 - 2 + r, gj = j0 - 2 + c;
                v[b] = (e < kTileElems && k < n && gi < a.NX && gj < a.NY) ? a.in[((size_t)gi * NY + gj) * n + k]
                                                                          : 0.0;
            }
#pragma unroll
            for (int b = 0; b < kBatch; b++) {
                const int e = e0 + b * kStep;
                if (e >= kTileElems)
                    continue;
                const int k = e % NP, cell = e / NP, r = cell / RW, c = cell % RW;
                double x = v[b];
                if (a.filter && k < n && filtered_cell(a, i0 - 2 + r, j0 - 2 + c))
                    x = __dmul_rn(x, a.filter[k]);
                tile[cell * CS + k] = x;
            }
        }
        __syncthreads();
        const int ii = warp, i = i0 + ii;
        auto T = [&](int r, int c, int m) { return tile[(r * RW + c) * CS + m]; };
        double acc[2][NT][4];
#pragma unroll
        for (int h = 0; h < 2; h++)
#pragma unroll
            for (int kt = 0; kt < NT; kt++)
#pragma unroll
                for (int e = 0; e < 4; e++)
                    acc[h][kt][e] = 0.0;
#pragma unroll
        for (int o = 0; o < 4; o++) {
#pragma unroll 1
            for (int ic = 0; ic < NT; ic++) {
                double av[4];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    // fragment element q: cell g (+8 for q = 1, 3), moment t (+4 for q >= 2)
                    const int c = 2 + g + ((q & 1) ? 8 : 0), m = ic * 8 + t + ((q & 2) ? 4 : 0);
                    const int r = ii + 2;
                    if (o == 0)
                        av[q] = stencil4(0.25, T(r + 1, c, m), 0.75, T(r, c, m), -1.25, T(r - 1, c, m), 0.25,
                                         T(r - 2, c, m));
                    else if (o == 1)
                        av[q] = stencil4(-0.25, T(r + 2, c, m), 1.25, T(r + 1, c, m), -0.75, T(r, c, m), -0.25,
                                         T(r - 1, c, m));
                    else if (o == 2)
                        av[q] = stencil4(0.25, T(r, c + 1, m), 0.75, T(r, c, m), -1.25, T(r, c - 1, m), 0.25,
                                         T(r, c - 2, m));
                    else
                        av[q] = stencil4(-0.25, T(r, c + 2, m), 1.25, T(r, c + 1, m), -0.75, T(r, c, m), -0.25,
                                         T(r, c - 1, m));
                }
                const double *ob = ops + (o * NP + ic * 8 + t) * OS + g;
#pragma unroll
                for (int kt = 0; kt < NT; kt++)
                    dmma16x8x8(acc[o >> 1][kt], av[0], av[1], av[2], av[3], ob[kt * 8], ob[4 * OS + kt * 8]);
            }
        }
        if (i >= 2 + a.rowEnd)
            continue;
        const double dt = a.dt;
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int cj = j0 + g + ((e & 2) ? 8 : 0);
            if (cj >= a.NY - 2)
                continue;
            const size_t cell = (size_t)i * NY + cj;
            const double sT = a.sigT[cell], sS = a.sigS[cell];
            bool source = false;
            if (a.initCond == 1) {
                const double x = __dadd_rn(a.initX, __dmul_rn((double)(i - 2), a.dx));
                const double y = __dadd_rn(a.initY, __dmul_rn((double)(cj - 2), a.dy));
                source = fabs(x) < 0.5 && fabs(y) < 0.5;
            }
            const double *self = tile + ((ii + 2) * RW + (cj - j0 + 2)) * CS;
#pragma unroll
            for (int kt = 0; kt < NT; kt++) {
                const int k = kt * 8 + 2 * t + (e & 1);
                if (k >= n)
                    continue;
                const double F = __dadd_rn(__dmul_rn(a.rdx, acc[0][kt][e]), __dmul_rn(a.rdy, acc[1][kt][e]));
                double u;
                if (k == 0) {
                    const double gm = __dsub_rn(__dadd_rn(1.0, __dmul_rn(dt, sS)), __dmul_rn(dt, sT));
                    u = __dsub_rn(__dmul_rn(self[0], gm), __dmul_rn(dt, F));
                    if (source)
                        u = __dadd_rn(u, __dmul_rn(__dmul_rn(dt, 2.0), kSqrtPiPn));
                } else {
                    u = __dsub_rn(__dmul_rn(self[k], __dsub_rn(1.0, __dmul_rn(dt, sT))), __dmul_rn(dt, F));
                }
                if (a.old)
                    u = __dmul_rn(0.5, __dadd_rn(u, a.old[cell * n + k]));
                a.out[cell * n + k] = u;
            }
        }
    }
}

template <int NP>
size_t pn_tile_smem() { return (size_t)(4 * NP * (NP + 4) + (kTI + 4) * (kTJ + 4) * (NP + 4)) * sizeof(double); }

}  // namespace

struct cl_pn {
    cudaStream_t stream = nullptr;
    cl_grid grid;
    int n = 0, NX = 0, NY = 0;
    long long C = 0;
    double *U = nullptr, *V = nullptr, *cur = nullptr;   // state buffers; cur = read by the next stage
    double *opsT = nullptr, *filter = nullptr, *sigT = nullptr, *sigS = nullptr;
    int exchanged = -1;    // sides whose ghosts hold neighbour values (-1: periodic or none)
    int nCtas = 0;
    std::string err;
    // cl_pn_step_host: upload and readback streams and their events (created on first use)
    cudaStream_t up = nullptr, down = nullptr;
    cudaEvent_t evStart = nullptr, evUp[kPnMaxBands] = {}, evDone[kPnMaxBands] = {};
};

static int pn_fail(cl_pn *p, int rc)
{
    clb_set_global_error(p->err.c_str());
    cl_pn_destroy(p);
    return rc;
}

#define PN_TRY(p, call)                                                                        \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            (p)->err = std::string(#call) + ": " + cudaGetErrorString(e_);                     \
            return CL_ERR_CUDA;                                                                \
        }                                                                                      \
    } while (0)

// One stage over interior rows [rowBegin, rowEnd) (rowEnd < 0: all rows) on
// `stream` (null: the solver's); reads p->cur.
static cudaError_t pn_launch(cl_pn *p, int stage, double dt, double dx, double dy, int rowBegin = 0,
                             int rowEnd = -1, cudaStream_t stream = nullptr)
{
    if (rowEnd < 0)
        rowEnd = p->NX - 4;
    if (!stream)
        stream = p->stream;
    PnArgs a;
    a.rowBegin = rowBegin;
    a.rowEnd = rowEnd;
    a.in = p->cur;
    a.out = (stage == 1) ? p->V : p->U;
    a.old = (stage == 2) ? p->U : nullptr;
    a.opsT = p->opsT;
    a.filter = p->filter;
    a.sigT = p->sigT;
    a.sigS = p->sigS;
    a.n = p->n;
    a.NX = p->NX;
    a.NY = p->NY;
    a.initCond = p->grid.init_cond;
    a.filteredGhosts = (p->exchanged >= 0) ? p->exchanged : (p->grid.init_cond == 2 ? 0xF : 0);
    a.dt = dt;
    a.rdx = 1.0 / dx;
    a.rdy = 1.0 / dy;
    a.dx = dx;
    a.dy = dy;
    a.initX = p->grid.init_x;
    a.initY = p->grid.init_y;
    const int np = (p->n + 7) / 8 * 8;
    const long long rows = rowEnd - rowBegin, ny = p->NY - 4;
    if (rows <= 0)
        return cudaSuccess;
    const long long units = (np <= 32) ? ((rows + kTI - 1) / kTI) * ((ny + kTJ - 1) / kTJ)
                                       : (rows * ny + kPnWarps - 1) / kPnWarps;
    const int ctas = (int)std::max<long long>(1, std::min<long long>(units, p->nCtas));
    switch (np) {
    case 8:
        pn_tile_kernel<8><<<ctas, kTI * 32, pn_tile_smem<8>(), stream>>>(a);
        break;
    case 16:
        pn_tile_kernel<16><<<ctas, kTI * 32, pn_tile_smem<16>(), stream>>>(a);
        break;
    case 24:
        pn_tile_kernel<24><<<ctas, kTI * 32, pn_tile_smem<24>(), stream>>>(a);
        break;
    case 32:
        pn_tile_kernel<32><<<ctas, kTI * 32, pn_tile_smem<32>(), stream>>>(a);
        break;
    default:
        pn_stage_kernel<2><<<ctas, kPnWarps * 32, (size_t)4 * p->n * p->n * sizeof(double), stream>>>(a);
    }
    clb_count_launches(1);
    return cudaGetLastError();
}

extern "C" {

int cl_pn_create(const cl_grid *grid, const cl_pn_setup *setup, const double *sigma_t, const double *sigma_s,
                 const double *moments, cl_pn **out)
{
    if (!out)
        return CL_ERR_ARG;
    *out = nullptr;
    if (!grid || !setup || !setup->ops || !sigma_t || !sigma_s || !moments || grid->nx < 1 || grid->ny < 1 ||
        grid->ghost != 2 || setup->n < 1) {
        clb_set_global_error("cl_pn_create: invalid arguments");
        return CL_ERR_ARG;
    }
    if (setup->n > kPnMaxN) {
        clb_set_global_error("cl_pn_create: more than 64 moments per cell (order > 9)");
        return CL_ERR_ARG;
    }
    int dev = 0, ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1 || cudaGetDevice(&dev) != cudaSuccess) {
        clb_set_global_error("no CUDA device");
        return CL_ERR_CUDA;
    }
    cl_pn *p = new cl_pn();
    p->grid = *grid;
    p->n = setup->n;
    p->NX = grid->nx + 4;
    p->NY = grid->ny + 4;
    p->C = (long long)p->NX * p->NY;
    const size_t C = (size_t)p->C, n = (size_t)p->n;
    if (cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&p->U, C * n * 8) != cudaSuccess || cudaMalloc(&p->V, C * n * 8) != cudaSuccess ||
        cudaMalloc(&p->opsT, 4 * n * n * 8) != cudaSuccess || cudaMalloc(&p->sigT, C * 8) != cudaSuccess ||
        cudaMalloc(&p->sigS, C * 8) != cudaSuccess ||
        (setup->filter && cudaMalloc(&p->filter, n * 8) != cudaSuccess)) {
        p->err = "device allocation failed";
        return pn_fail(p, CL_ERR_CUDA);
    }
    std::vector<double> opsT(4 * n * n);
    for (size_t o = 0; o < 4; o++)
        for (size_t k = 0; k < n; k++)
            for (size_t i = 0; i < n; i++)
                opsT[(o * n + i) * n + k] = setup->ops[(o * n + k) * n + i];
    cudaMemcpy(p->opsT, opsT.data(), 4 * n * n * 8, cudaMemcpyHostToDevice);
    if (setup->filter)
        cudaMemcpy(p->filter, setup->filter, n * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(p->sigT, sigma_t, C * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(p->sigS, sigma_s, C * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(p->U, moments, C * n * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(p->V, moments, C * n * 8, cudaMemcpyHostToDevice);
    p->cur = p->U;
    // the kernel for this n, its shared memory, and the units it loops over
    const int np = (int)(n + 7) / 8 * 8;
    const void *fn = nullptr;
    size_t smem = 0;
    long long units = 0;
    switch (np) {
    case 8: fn = (const void *)pn_tile_kernel<8>; smem = pn_tile_smem<8>(); break;
    case 16: fn = (const void *)pn_tile_kernel<16>; smem = pn_tile_smem<16>(); break;
    case 24: fn = (const void *)pn_tile_kernel<24>; smem = pn_tile_smem<24>(); break;
    case 32: fn = (const void *)pn_tile_kernel<32>; smem = pn_tile_smem<32>(); break;
    default: fn = (const void *)pn_stage_kernel<2>; smem = 4 * n * n * 8;
    }
    const int threads = (np <= 32) ? kTI * 32 : kPnWarps * 32;
    if (np <= 32)
        units = (long long)((grid->nx + kTI - 1) / kTI) * ((grid->ny + kTJ - 1) / kTJ);
    else
        units = ((long long)grid->nx * grid->ny + kPnWarps - 1) / kPnWarps;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int occ = 0;
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, threads, smem);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess || occ < 1 || cudaDeviceSynchronize() != cudaSuccess) {
        p->err = std::string("set-up: ") + cudaGetErrorString(e != cudaSuccess ? e : cudaGetLastError());
        return pn_fail(p, CL_ERR_CUDA);
    }
    p->nCtas = (int)std::max<long long>(1, std::min<long long>(units, (long long)sms * occ));
    *out = p;
    return CL_OK;
}

void cl_pn_destroy(cl_pn *p)
{
    if (!p)
        return;
    if (p->stream)
        cudaStreamSynchronize(p->stream);
    for (cudaStream_t st : {p->up, p->down})
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
    if (p->evStart)
        cudaEventDestroy(p->evStart);
    for (int b = 0; b < kPnMaxBands; b++) {
        if (p->evUp[b])
            cudaEventDestroy(p->evUp[b]);
        if (p->evDone[b])
            cudaEventDestroy(p->evDone[b]);
    }
    cudaFree(p->U);
    cudaFree(p->V);
    cudaFree(p->opsT);
    cudaFree(p->filter);
    cudaFree(p->sigT);
    cudaFree(p->sigS);
    if (p->stream)
        cudaStreamDestroy(p->stream);
    delete p;
}

const char *cl_pn_last_error(const cl_pn *p) { return p ? p->err.c_str() : cl_global_error(); }

int cl_pn_stage(cl_pn *p, int stage, double dt, double dx, double dy)
{
    if (!p || (stage != 1 && stage != 2))
        return CL_ERR_ARG;
    if ((stage == 1) != (p->cur == p->U)) {
        p->err = "stages must alternate 1, 2";
        return CL_ERR_STATE;
    }
    PN_TRY(p, pn_launch(p, stage, dt, dx, dy));
    p->cur = (stage == 1) ? p->V : p->U;
    return CL_OK;
}

int cl_pn_sync(cl_pn *p)
{
    if (!p)
        return CL_ERR_ARG;
    PN_TRY(p, cudaStreamSynchronize(p->stream));
    return CL_OK;
}

int cl_pn_step(cl_pn *p, double dt, double dx, double dy)
{
    if (!p)
        return CL_ERR_ARG;
    for (int stage = 1; stage <= 2; stage++) {
        if (p->grid.init_cond == 2) {
            PN_TRY(p, launch_ghost_periodic(p->cur, p->n, p->NX, p->NY, p->stream));
            clb_count_launches(2);
        }
        int rc = cl_pn_stage(p, stage, dt, dx, dy);
        if (rc)
            return rc;
    }
    return cl_pn_sync(p);
}

int cl_pn_stage_timed(cl_pn *p, int stage, double dt, double dx, double dy, float *ms)
{
    if (!p || !ms)
        return CL_ERR_ARG;
    cudaEvent_t e0, e1;
    PN_TRY(p, cudaEventCreate(&e0));
    PN_TRY(p, cudaEventCreate(&e1));
    cudaEventRecord(e0, p->stream);
    int rc = cl_pn_stage(p, stage, dt, dx, dy);
    cudaEventRecord(e1, p->stream);
    cudaError_t e = cudaEventSynchronize(e1);
    if (rc == CL_OK && e == cudaSuccess)
        cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc)
        return rc;
    PN_TRY(p, e);
    return CL_OK;
}

int cl_pn_stream(cl_pn *p, void **stream)
{
    if (!p || !stream)
        return CL_ERR_ARG;
    *stream = (void *)p->stream;
    return CL_OK;
}

int cl_pn_set_exchanged_sides(cl_pn *p, int mask)
{
    if (!p || mask < 0 || mask > 0xF)
        return CL_ERR_ARG;
    p->exchanged = mask;
    return CL_OK;
}

int cl_pn_get_state(cl_pn *p, double *moments)
{
    if (!p || !moments)
        return CL_ERR_ARG;
    PN_TRY(p, cudaStreamSynchronize(p->stream));
    PN_TRY(p, cudaMemcpy(moments, p->cur, (size_t)p->C * p->n * 8, cudaMemcpyDeviceToHost));
    return CL_OK;
}

int cl_pn_set_state(cl_pn *p, const double *moments)
{
    if (!p || !moments)
        return CL_ERR_ARG;
    PN_TRY(p, cudaStreamSynchronize(p->stream));
    PN_TRY(p, cudaMemcpy(p->U, moments, (size_t)p->C * p->n * 8, cudaMemcpyHostToDevice));
    // the second buffer needs the ghost strips; the device copy is cheaper
    // than a second upload
    PN_TRY(p, cudaMemcpyAsync(p->V, p->U, (size_t)p->C * p->n * 8, cudaMemcpyDeviceToDevice, p->stream));
    p->cur = p->U;
    return CL_OK;
}

// One RK2 step on a state in host memory ([NX*NY][n], ghosts included, read
// and overwritten), equal to cl_pn_set_state, cl_pn_step, cl_pn_get_state.
// The grid goes up in bands of interior rows (multiples of the tile height)
// on one stream and comes back on another; stage 1 of band b runs once band
// b + 1 has arrived (its stencil reaches two rows into it), stage 2 of band
// b after stage 1 of band b + 1, and band b goes back as soon as its stage 2
// is done, while later bands are still going up.  Each band is also copied
// to the second state buffer on the device, whose ghost cells must hold the
// uploaded values.  Periodic and partitioned grids, whose ghost strips are
// refilled from the whole grid, take the three calls one after the other.
int cl_pn_step_host(cl_pn *p, double dt, double dx, double dy, double *moments)
{
    if (!p || !moments)
        return CL_ERR_ARG;
    if (p->grid.init_cond == 2 || p->exchanged > 0) {
        int rc = cl_pn_set_state(p, moments);
        if (rc == CL_OK)
            rc = cl_pn_step(p, dt, dx, dy);
        if (rc == CL_OK)
            rc = cl_pn_get_state(p, moments);
        return rc;
    }
    if (p->cur != p->U) {
        p->err = "a step starts after stage 2";
        return CL_ERR_STATE;
    }
    if (!p->up) {
        PN_TRY(p, cudaStreamCreateWithFlags(&p->up, cudaStreamNonBlocking));
        PN_TRY(p, cudaStreamCreateWithFlags(&p->down, cudaStreamNonBlocking));
        PN_TRY(p, cudaEventCreateWithFlags(&p->evStart, cudaEventDisableTiming));
        for (int b = 0; b < kPnMaxBands; b++) {
            PN_TRY(p, cudaEventCreateWithFlags(&p->evUp[b], cudaEventDisableTiming));
            PN_TRY(p, cudaEventCreateWithFlags(&p->evDone[b], cudaEventDisableTiming));
        }
    }
    const int nx = p->NX - 4;
    // about 12 bands of whole tile rows (the last one takes the remainder)
    const int bandRows = std::max(kTI, (nx + 11) / 12 / kTI * kTI);
    const int bands = std::min(kPnMaxBands, (nx + bandRows - 1) / bandRows);
    int r0[kPnMaxBands + 1];
    for (int b = 0; b < bands; b++)
        r0[b] = b * bandRows;
    r0[bands] = nx;
    const size_t rowBytes = (size_t)p->NY * p->n * 8, rowElems = (size_t)p->NY * p->n;
    // cell rows copied with band b: its interior rows, plus the ghost rows
    // before the first band and after the last
    auto first = [&](int b) { return (size_t)(b == 0 ? 0 : 2 + r0[b]); };
    auto last = [&](int b) { return (size_t)(b == bands - 1 ? p->NX : 2 + r0[b + 1]); };
    cudaError_t e = cudaSuccess;
    auto run = [&](cudaError_t r) {
        if (e == cudaSuccess)
            e = r;
    };
    run(cudaEventRecord(p->evStart, p->stream));
    run(cudaStreamWaitEvent(p->up, p->evStart, 0));
    run(cudaStreamWaitEvent(p->down, p->evStart, 0));
    for (int b = 0; b < bands; b++) {
        const size_t off = first(b) * rowElems, bytes = (last(b) - first(b)) * rowBytes;
        run(cudaMemcpyAsync(p->U + off, moments + off, bytes, cudaMemcpyHostToDevice, p->up));
        run(cudaMemcpyAsync(p->V + off, p->U + off, bytes, cudaMemcpyDeviceToDevice, p->up));
        run(cudaEventRecord(p->evUp[b], p->up));
    }
    auto stage2 = [&](int b) {
        p->cur = p->V;
        run(pn_launch(p, 2, dt, dx, dy, r0[b], r0[b + 1]));
        run(cudaEventRecord(p->evDone[b], p->stream));
        run(cudaStreamWaitEvent(p->down, p->evDone[b], 0));
        const size_t off = first(b) * rowElems, bytes = (last(b) - first(b)) * rowBytes;
        run(cudaMemcpyAsync(moments + off, p->U + off, bytes, cudaMemcpyDeviceToHost, p->down));
    };
    for (int b = 0; b < bands && e == cudaSuccess; b++) {
        run(cudaStreamWaitEvent(p->stream, p->evUp[std::min(b + 1, bands - 1)], 0));
        p->cur = p->U;
        run(pn_launch(p, 1, dt, dx, dy, r0[b], r0[b + 1]));
        if (b > 0)
            stage2(b - 1);
    }
    if (e == cudaSuccess)
        stage2(bands - 1);
    p->cur = p->U;
    run(cudaStreamSynchronize(p->down));
    run(cudaStreamSynchronize(p->up));
    run(cudaStreamSynchronize(p->stream));
    if (e != cudaSuccess) {
        p->err = std::string("host-state step: ") + cudaGetErrorString(e);
        return CL_ERR_CUDA;
    }
    return CL_OK;
}

int cl_pn_halo_counts(const cl_pn *p, long long counts[4])
{
    if (!p || !counts)
        return CL_ERR_ARG;
    const long long nx = p->NX - 4, ny = p->NY - 4, n = p->n;
    counts[CL_NORTH] = counts[CL_SOUTH] = 2 * nx * n;
    counts[CL_EAST] = counts[CL_WEST] = 2 * ny * n;
    return CL_OK;
}

static int pn_halo(cl_pn *p, double *const bufs[4], int pack)
{
    if (!p || !bufs)
        return CL_ERR_ARG;
    HaloBuffers b;
    for (int s = 0; s < 4; s++)
        b.p[s] = bufs[s];
    PN_TRY(p, launch_halo(p->cur, p->n, p->NX, p->NY, b, pack, p->stream));
    clb_count_launches(1);
    return CL_OK;
}

int cl_pn_halo_pack(cl_pn *p, double *const bufs[4]) { return pn_halo(p, bufs, 1); }

int cl_pn_halo_unpack(cl_pn *p, double *const bufs[4]) { return pn_halo(p, bufs, 0); }

}  // extern "C"
