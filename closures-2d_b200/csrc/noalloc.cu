// noalloc.cu -- batched opt() for callers that must not allocate device memory.
//
// Some host applications own every byte of device memory through their own
// allocator or pool and do not allow a library to call cudaMalloc/cudaFree
// (those calls synchronise the device and fragment a pool that was reserved
// up front, e.g. inside a simulation's time loop).  cl_solve_batch_noalloc
// serves them: the caller passes device inputs and outputs, and everything
// else the persistent Newton kernel needs -- work counter, error word,
// statistics, and the angular set-up in the kernel's padded layout -- lives
// in one fixed, file-scope device array of kNoAllocBytes.  That array exists
// on every GPU that loads the library, for the life of the process.
#include "closures_gpu.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <mutex>

#include "../host/angular.h"
#include "common.cuh"
#include "angular.h"
#include "newton.cuh"

using namespace clb;

namespace {

constexpr size_t kNoAllocBytes = 4u << 20;   // 4 MiB per device
constexpr int kMaxDevices = 64;
constexpr size_t kHeaderBytes = 256;         // queue, error word, statistics

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Host-side staging of the same size (static storage, no heap allocation).
static unsigned char g_stage[kNoAllocBytes];
static void *g_scratch_ptr[kMaxDevices];
static std::mutex g_mutex;
static thread_local char g_msg[256];

int fail(int code, const char *msg)
{
    std::snprintf(g_msg, sizeof(g_msg), "%s", msg);
    return code;
}

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
int round8(int x) { return (x + 7) / 8 * 8; }

}  // namespace

extern "C" const char *cl_noalloc_last_error(void) { return g_msg; }

extern "C" int cl_solve_batch_noalloc(const cl_angular *ang, const cl_options *opts, int count, double *d_u,
                                      double *d_alpha, int *d_iters, double *d_reg, int *d_status,
                                      void *stream_ptr)
{
    g_msg[0] = 0;
    if (!ang || !opts || count < 0 || (count > 0 && (!d_u || !d_alpha)))
        return fail(CL_ERR_ARG, "null argument");
    if (opts->opt_type != 0 || (opts->moment_type != CL_MN && opts->moment_type != CL_PPN) ||
        opts->max_iter < 1)
        return fail(CL_ERR_ARG, "unsupported options (optimisation type must be 0)");
    if (ang->n < 1 || ang->n > kMaxN || !ang->p || !ang->w)
        return fail(CL_ERR_ARG, "angular set-up missing or order > 6");
    if (count == 0)
        return CL_OK;
    cudaStream_t stream = (cudaStream_t)stream_ptr;

    // sizes of the kernel layout (same as the context's device basis)
    const int n = ang->n, n2 = ang->n2, nq = ang->nq, gaunt = ang->use_gaunt ? 1 : 0;
    const int nb = round8(n);
    const int K2 = gaunt ? n2 : n * (n + 1) / 2;
    const int K2p = round8(K2);
    const int nqp = (nq + 31) / 32 * 32;
    int ldP = nb + K2p;
    while (ldP % 16 != 4)
        ldP++;
    const int npairs = n * (n + 1) / 2;
    const int nnz = gaunt ? ang->gaunt_nnz : 0;
    size_t off = kHeaderBytes;
    const size_t offP = off;
    off = align_up(off + sizeof(double) * ((size_t)nqp * ldP + nqp), 256);
    const size_t offW = off;
    off = align_up(off + sizeof(double) * (size_t)nqp, 256);
    const size_t offPairs = off;
    off = align_up(off + sizeof(unsigned short) * (size_t)npairs, 256);
    const size_t offHoff = off;
    off = align_up(off + sizeof(int) * (size_t)(gaunt ? n * n + 1 : 1), 256);
    const size_t offHidx = off;
    off = align_up(off + sizeof(int) * (size_t)(nnz ? nnz : 1), 256);
    const size_t offHval = off;
    off = align_up(off + sizeof(double) * (size_t)(nnz ? nnz : 1), 256);
    // Gaunt table in lane-major chunks; rows bounded by the pair count times
    // the longest entry list, which the CSR gives
    const int chunks = gaunt ? gaunt_ell_chunks(n) : 0;
    int maxPer = 0;
    if (gaunt)
        for (int r = 0; r < n * n; r++)
            maxPer = std::max(maxPer, ang->gaunt_off[r + 1] - ang->gaunt_off[r]);
    const int maxRows = chunks * maxPer;
    const size_t offEllPair = off;
    off = align_up(off + sizeof(unsigned short) * (size_t)(chunks * 32 + 1), 256);
    const size_t offEllOff = off;
    off = align_up(off + sizeof(int) * (size_t)(chunks + 1), 256);
    const size_t offEllIdx = off;
    off = align_up(off + sizeof(unsigned short) * (size_t)(maxRows * 32 + 1), 256);
    const size_t offEllVal = off;
    off = align_up(off + sizeof(double) * (size_t)(maxRows * 32 + 1), 256);
    if (off > kNoAllocBytes) {
        char buf[200];
        std::snprintf(buf, sizeof(buf),
                      "configuration needs %zu bytes of fixed scratch, above the %zu-byte maximum "
                      "(reduce the moment order or quadrature, or use cl_solve_batch)",
                      off, kNoAllocBytes);
        return fail(CL_ERR_ARG, buf);
    }

    std::lock_guard<std::mutex> lock(g_mutex);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return fail(CL_ERR_CUDA, "no usable CUDA device");
    // one-time set-up per device: the device address of the fixed array
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(CL_ERR_CUDA, cudaGetErrorString(e));
        g_scratch_ptr[dev] = p;
    }
    unsigned char *base = (unsigned char *)g_scratch_ptr[dev];

    // host staging of the padded basis, pair lists and Gaunt table
    std::memset(g_stage, 0, off);
    double *P = (double *)(g_stage + offP);
    double *W = (double *)(g_stage + offW);
    unsigned short *pairs = (unsigned short *)(g_stage + offPairs);
    product_columns(n, pairs);
    for (int q = 0; q < nq; q++) {
        const double *pq = ang->p + (size_t)q * n2;
        double *row = P + (size_t)basis_row(q, ldP);
        for (int k = 0; k < n; k++)
            row[k] = pq[k];
        if (gaunt) {
            for (int k = 0; k < n2; k++)
                row[nb + k] = pq[k];
        } else {
            for (int c = 0; c < npairs; c++)
                row[nb + c] = pq[pairs[c] >> 8] * pq[pairs[c] & 255];
        }
        W[q] = ang->w[q];
        P[(size_t)basis_wgap(q, ldP)] = ang->w[q];
    }
    int ellRows = 0;
    if (gaunt) {
        std::memcpy(g_stage + offHoff, ang->gaunt_off, sizeof(int) * (n * n + 1));
        if (nnz) {
            std::memcpy(g_stage + offHidx, ang->gaunt_idx, sizeof(int) * nnz);
            std::memcpy(g_stage + offHval, ang->gaunt_val, sizeof(double) * nnz);
        }
        ellRows = build_gaunt_ell(n, ang->gaunt_off, ang->gaunt_idx, ang->gaunt_val,
                                  (unsigned short *)(g_stage + offEllPair), (unsigned short *)(g_stage + offEllIdx),
                                  (double *)(g_stage + offEllVal), (int *)(g_stage + offEllOff), maxRows);
        if (ellRows < 0)
            return fail(CL_ERR_ARG, "Gaunt table layout failed");
    }
    // the header (work counter, error word, statistics) starts at zero each call
    cudaError_t e = cudaMemcpyAsync(base, g_stage, off, cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess)
        return fail(CL_ERR_CUDA, cudaGetErrorString(e));

    NewtonArgs a;
    std::memset(&a, 0, sizeof(a));
    a.nprob = 1;
    NewtonProblem &pb = a.prob[0];
    pb.P = (const double *)(base + offP);
    pb.w = (const double *)(base + offW);
    pb.pairs = (const unsigned short *)(base + offPairs);
    pb.hoff = gaunt ? (const int *)(base + offHoff) : nullptr;
    pb.hidx = gaunt ? (const int *)(base + offHidx) : nullptr;
    pb.hval = gaunt ? (const double *)(base + offHval) : nullptr;
    pb.ellPair = gaunt ? (const unsigned short *)(base + offEllPair) : nullptr;
    pb.ellIdx = gaunt ? (const unsigned short *)(base + offEllIdx) : nullptr;
    pb.ellVal = gaunt ? (const double *)(base + offEllVal) : nullptr;
    pb.ellOff = gaunt ? (const int *)(base + offEllOff) : nullptr;
    pb.ellChunks = chunks;
    pb.ellRows = ellRows;
    pb.p0 = ang->p[0];
    pb.n = n;
    pb.nb = nb;
    pb.K2p = K2p;
    pb.nqp = nqp;
    pb.ldP = ldP;
    pb.count = count;
    pb.u = d_u;
    pb.alpha = d_alpha;
    pb.iters = d_iters;
    pb.regs = d_reg;
    pb.status = d_status;
    pb.queue = (unsigned int *)base;                 // header bytes [0, 16)
    a.err = (int *)(base + 16);                      // header bytes [16, 24)
    a.stats = (DevStats *)(base + 64);               // header bytes [64, 64 + sizeof)
    a.momentType = opts->moment_type;
    a.maxIter = opts->max_iter;
    a.useGaunt = gaunt;
    a.tolRel = opts->tol;
    a.condHMax = opts->cond_h_max;
    a.deltaPPn = opts->delta_ppn;
    a.tolGamma = opts->tol_gamma;
    a.mixed = opts->precision == CL_MIXED;
    const int pl = plan_newton(a);
    if (pl == -2)
        return fail(CL_ERR_ARG, "mixed precision needs a configuration with at most 16 Hessian column tiles");
    if (pl != 0)
        return fail(CL_ERR_ARG, "Newton kernel layout does not fit in shared memory");
    if ((e = prepare_newton(a)) != cudaSuccess)
        return fail(CL_ERR_CUDA, cudaGetErrorString(e));
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if ((e = launch_newton(a, sms * newton_ctas_per_sm(a), stream)) != cudaSuccess)
        return fail(CL_ERR_CUDA, cudaGetErrorString(e));
    int herr[2] = {0, 0};
    e = cudaMemcpyAsync(herr, base + 16, sizeof(herr), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess)
        return fail(CL_ERR_CUDA, cudaGetErrorString(e));
    if (herr[0] != 0) {
        if (herr[1] >= 0)
            std::snprintf(g_msg, sizeof(g_msg), "%s (vector %d)", cl_error_text(herr[0]), herr[1]);
        else
            std::snprintf(g_msg, sizeof(g_msg), "%s", cl_error_text(herr[0]));
        return herr[0];
    }
    return CL_OK;
}
