// mlp.cu -- learned warm start for the dual Newton solve.
//
// A small multilayer perceptron maps the normalised moments u/u0 of a cell to
// the multipliers alpha of the scaled problem (u0 = 1).  Newton then starts
// from the prediction and runs to the same tolerance; where the prediction is
// not finite the caller's fallback multipliers (previous step, or isotropic)
// are used, so the network changes iteration counts, not the converged
// answer.  There is no counterpart in the reference, which starts each solve
// from the previous stage's alpha (momopt_update.cpp:236-238).
//
// Network: n -> W -> W -> W -> n with GELU (exact erf form) between layers,
// BF16 weights and activations feeding tensor-core MMAs (mma.sync m16n8k16,
// BF16 x BF16 -> FP32), FP32 master weights, FP32 Adam.  Outputs are the
// multipliers standardised per component with the training set's mean and
// standard deviation.  Training and inference both run on these kernels.
#include "closures_gpu.h"

#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include "tc_gemm.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

namespace {

constexpr int kLayers = 4;
constexpr int BM = 64, BN = 64, BK = 32, KPAD = 8;
constexpr double kSqrtPi = 1.7724538509055160273;
constexpr double kPi = 3.14159265358979323846;

enum Epi { EPI_F32 = 0, EPI_BIAS_GELU = 1, EPI_BIAS = 2 };

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z)
{
    const float phi = 0.39894228040143268f * __expf(-0.5f * z * z);
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * phi;
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3,
                                         unsigned b0, unsigned b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// C[M x N] = op(A)[M x K] . op(B)[K x N].  A is [M x K] row-major (TA = 0) or
// [K x M] (TA = 1); B is [K x N] row-major (TB = 0) or [N x K] (TB = 1).
// Epilogues: FP32 store; bias + GELU (pre-activation FP32, activation BF16);
// bias (FP32).  Tiles 64 x 64 x 32, four warps of 32 x 32.
// Mdev (nullable): the rows come from a device count, M = min(M, *Mdev - moff)
// (a compacted selection whose size the host does not know); tiles past it
// return at once.
template <int TA, int TB, int EPI>
__global__ void __launch_bounds__(128) gemm_kernel(const __nv_bfloat16 *__restrict__ A,
                                                   const __nv_bfloat16 *__restrict__ B, int M, int N, int K,
                                                   float *__restrict__ C, const float *__restrict__ bias,
                                                   __nv_bfloat16 *__restrict__ Act, const int *Mdev, int moff)
{
    __shared__ __align__(16) __nv_bfloat16 As[BM][BK + KPAD];
    __shared__ __align__(16) __nv_bfloat16 Bs[BN][BK + KPAD];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    if (Mdev) {
        const int rem = *Mdev - moff;
        M = rem < M ? (rem > 0 ? rem : 0) : M;
        if (m0 >= M)
            return;
    }
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
            acc[i][j][0] = acc[i][j][1] = acc[i][j][2] = acc[i][j][3] = 0.0f;
    const __nv_bfloat16 zero = __float2bfloat16(0.0f);
    for (int k0 = 0; k0 < K; k0 += BK) {
        for (int idx = tid; idx < BM * BK; idx += 128) {
            int r = idx / BK, c = idx % BK;
            int m = m0 + r, k = k0 + c;
            __nv_bfloat16 v = zero;
            if (m < M && k < K)
                v = TA ? A[(size_t)k * M + m] : A[(size_t)m * K + k];
            As[r][c] = v;
        }
        for (int idx = tid; idx < BN * BK; idx += 128) {
            int r = idx / BK, c = idx % BK;
            int nn = n0 + r, k = k0 + c;
            __nv_bfloat16 v = zero;
            if (nn < N && k < K)
                v = TB ? B[(size_t)nn * K + k] : B[(size_t)k * N + nn];
            Bs[r][c] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk += 16) {
            unsigned a[2][4], b[4][2];
#pragma unroll
            for (int i = 0; i < 2; i++) {
                int r = wm + i * 16 + g;
                a[i][0] = *reinterpret_cast<const unsigned *>(&As[r][kk + 2 * t]);
                a[i][1] = *reinterpret_cast<const unsigned *>(&As[r + 8][kk + 2 * t]);
                a[i][2] = *reinterpret_cast<const unsigned *>(&As[r][kk + 2 * t + 8]);
                a[i][3] = *reinterpret_cast<const unsigned *>(&As[r + 8][kk + 2 * t + 8]);
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                int c = wn + j * 8 + g;
                b[j][0] = *reinterpret_cast<const unsigned *>(&Bs[c][kk + 2 * t]);
                b[j][1] = *reinterpret_cast<const unsigned *>(&Bs[c][kk + 2 * t + 8]);
            }
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < 4; j++)
                    mma_bf16(acc[i][j], a[i][0], a[i][1], a[i][2], a[i][3], b[j][0], b[j][1]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int h = 0; h < 4; h++) {
                int m = m0 + wm + i * 16 + g + ((h & 2) ? 8 : 0);
                int nn = n0 + wn + j * 8 + 2 * t + (h & 1);
                if (m >= M || nn >= N)
                    continue;
                float v = acc[i][j][h];
                if (EPI == EPI_F32) {
                    C[(size_t)m * N + nn] = v;
                } else if (EPI == EPI_BIAS_GELU) {
                    v += bias[nn];
                    C[(size_t)m * N + nn] = v;
                    Act[(size_t)m * N + nn] = __float2bfloat16(gelu(v));
                } else {
                    C[(size_t)m * N + nn] = v + bias[nn];
                }
            }
}

__global__ void cast_bf16_kernel(const float *x, __nv_bfloat16 *y, size_t n)
{
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < n)
        y[i] = __float2bfloat16(x[i]);
}

// dY = 2 (Y - T) / (B n) for the mean squared error over B x n entries; returns
// per-block partial losses.
__global__ void mse_grad_kernel(const float *Y, const float *T, __nv_bfloat16 *dY, float *dYf, int total, float scale,
                                float *lossPart)
{
    __shared__ float red[256];
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (i < total) {
        float d = Y[i] - T[i];
        l = d * d;
        float gval = 2.0f * d * scale;
        dY[i] = __float2bfloat16(gval);
        dYf[i] = gval;
    }
    red[threadIdx.x] = l;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        lossPart[blockIdx.x] = red[0];
}

// dZ = dA * gelu'(Z)
__global__ void gelu_back_kernel(const float *dA, const float *Z, __nv_bfloat16 *dZ, float *dZf, size_t n)
{
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < n) {
        float v = dA[i] * gelu_grad(Z[i]);
        dZ[i] = __float2bfloat16(v);
        dZf[i] = v;
    }
}

// db[j] = sum_rows dZ[r][j]
__global__ void colsum_kernel(const float *dZ, int rows, int cols, float *db)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < cols) {
        float s = 0.0f;
        for (int r = 0; r < rows; r++)
            s += dZ[(size_t)r * cols + j];
        db[j] = s;
    }
}

// rows perm[0..batch) of (u, alpha) into contiguous minibatch buffers
__global__ void gather_kernel(const double *u, const double *alpha, const int *perm, int batch, int n, double *bu,
                              double *ba)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < batch * n) {
        int r = i / n, k = i % n;
        size_t src = (size_t)perm[r] * n + k;
        bu[i] = u[src];
        ba[i] = alpha[src];
    }
}

__global__ void adam_kernel(float *w, float *m, float *v, const float *g, size_t n, float lr, float b1, float b2,
                            float eps, float c1, float c2)
{
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < n) {
        float gi = g[i];
        float mi = b1 * m[i] + (1.0f - b1) * gi;
        float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// Linear part of the closure near isotropy (Mn): for u/u0 = (1, x_1, ...)
// close to isotropic, exp(alpha.m) ~ e^{alpha0 p0} (1 + sum alpha_k m_k) with
// orthonormal m_k gives alpha_k ~ 4 pi p0 x_k = 2 sqrt(pi) x_k, and alpha_0 the
// isotropic value 2 sqrt(pi) log(1/(2 sqrt(pi))).  The network learns the
// remainder, so near-isotropic cells need only a small correction.
__device__ __forceinline__ double alpha_linear(int k, double x, int momentType)
{
    if (momentType != CL_MN)
        return 0.0;
    return k == 0 ? 2.0 * kSqrtPi * log(0.5 / kSqrtPi) : 2.0 * kSqrtPi * x;
}

// Inputs: x = u/u0 (BF16); targets (alpha_scaled - linear - mean)/std (FP32).
__global__ void prep_kernel(const double *u, const double *alpha, int count, int n, int momentType,
                            const float *mean, const float *stdv, __nv_bfloat16 *X, float *Tgt)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count * n)
        return;
    int c = i / n, k = i % n;
    double u0 = u[(size_t)c * n];
    double x = u[i] / u0;
    X[i] = __float2bfloat16((float)x);
    if (Tgt) {
        double a = alpha[i];
        if (momentType == CL_MN) {
            if (k == 0)
                a -= log(u0) * 2.0 * kSqrtPi;
        } else {
            a /= u0;
        }
        a -= alpha_linear(k, x, momentType);
        Tgt[i] = (float)((a - mean[k]) / stdv[k]);
    }
}

// alpha = unscale(Y * std + mean); non-finite predictions (or u0 <= 0) take
// the fallback multipliers.  fallbackKind: 0 = keep alpha as given (previous
// stage), 1 = isotropic alpha for this u0, 2 = write NaN so that the Newton
// kernel's start falls back to its own multipliers.
// With idx (nullable), row r of Y is cell idx[off + r] (rows past *cnt - off
// are not there).
__global__ void predict_out_kernel(const float *Y, const double *u, double *alpha, int count, int n,
                                   int momentType, double delta, const float *mean, const float *stdv,
                                   int fallbackKind, int *fallbacks, const int *idx = nullptr,
                                   const int *cnt = nullptr, int off = 0)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= count || (idx && off + r >= *cnt))
        return;
    // Y row r; u and alpha rows of cell c (with an index list) or r
    const int c = idx ? idx[off + r] : r;
    const float *Yr = Y + (size_t)r * n;
    double u0 = u[(size_t)c * n];
    bool ok = u0 > 0.0;
    double a[32];
    for (int k = 0; k < n && ok; k++) {
        double x = u[(size_t)c * n + k] / u0;
        double v = (double)Yr[k] * stdv[k] + mean[k] + alpha_linear(k, x, momentType);
        if (!isfinite(v))
            ok = false;
        a[k] = v;
    }
    if (ok) {
        if (momentType == CL_MN)
            a[0] += log(u0) * 2.0 * kSqrtPi;
        else
            for (int k = 0; k < n; k++)
                a[k] *= u0;
        for (int k = 0; k < n; k++)
            alpha[(size_t)c * n + k] = a[k];
        return;
    }
    atomicAdd(fallbacks, 1);
    if (fallbackKind == 2) {
        // mark the start as unusable: the Newton kernel then starts from its
        // fallback multipliers
        alpha[(size_t)c * n] = __longlong_as_double(0x7ff8000000000000ll);
    } else if (fallbackKind == 1 && u0 > 0.0) {
        double a0 = (momentType == CL_MN) ? 2.0 * kSqrtPi * log(u0 / (2.0 * kSqrtPi))
                                          : u0 - 4.0 * delta * kPi / u0;
        alpha[(size_t)c * n] = a0;
        for (int k = 1; k < n; k++)
            alpha[(size_t)c * n + k] = 0.0;
    }
}

template <int TA, int TB, int EPI>
cudaError_t gemm(const __nv_bfloat16 *A, const __nv_bfloat16 *B, int M, int N, int K, float *C, const float *bias,
                 __nv_bfloat16 *Act, cudaStream_t s, const int *Mdev = nullptr, int moff = 0)
{
    dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
    gemm_kernel<TA, TB, EPI><<<grid, 128, 0, s>>>(A, B, M, N, K, C, bias, Act, Mdev, moff);
    return cudaGetLastError();
}

// Cells whose last optimisation took at least minIters iterations are listed
// in idx (count in *cnt, order arbitrary); the others get a NaN start, so the
// Newton kernel starts them from their own (previous-stage) multipliers.
__global__ void select_kernel(const int *iters, int count, int minIters, int *idx, int *cnt, double *alpha, int n)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= count)
        return;
    if (iters[c] >= minIters)
        idx[atomicAdd(cnt, 1)] = c;
    else
        alpha[(size_t)c * n] = __longlong_as_double(0x7ff8000000000000ll);
}

// Inputs x = u/u0 of the listed cells idx[off + r], r < min(rows, *cnt - off).
__global__ void prep_idx_kernel(const double *u, const int *idx, const int *cnt, int off, int rows, int n,
                                __nv_bfloat16 *X)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int r = i / n, k = i % n;
    if (r >= rows || off + r >= *cnt)
        return;
    const size_t c = (size_t)idx[off + r];
    X[i] = __float2bfloat16((float)(u[c * n + k] / u[c * n]));
}

int blocks(size_t n, int t = 256) { return (int)((n + t - 1) / t); }

int round8(int x) { return (x + 7) / 8 * 8; }

// x [rows x n] -> xp [rows x np] with zero columns n..np-1 (a row stride of a
// multiple of 16 bytes, as the tensor-memory GEMM's TMA loads need)
__global__ void pad_cols_kernel(const __nv_bfloat16 *x, int rows, int n, int np, __nv_bfloat16 *xp)
{
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= (size_t)rows * np)
        return;
    const int r = (int)(i / np), k = (int)(i % np);
    xp[i] = k < n ? x[(size_t)r * n + k] : __float2bfloat16(0.0f);
}

// W [K x N] FP32 row-major -> Wt [N x Kp] BF16 (the K-major B operand), zero
// columns K..Kp-1
__global__ void transpose_cast_kernel(const float *W, int K, int N, int Kp, __nv_bfloat16 *Wt)
{
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= (size_t)N * Kp)
        return;
    const int c = (int)(i / Kp), k = (int)(i % Kp);
    Wt[i] = k < K ? __float2bfloat16(W[(size_t)k * N + c]) : __float2bfloat16(0.0f);
}

// The driver's tensor-map encoder, through the runtime's entry-point query
// (no link against the driver library).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

// 2-D map of a row-major BF16 [rows x cols] matrix (cols a multiple of 8,
// base 16-byte aligned) in boxes of boxRows x 64 with the 128 B swizzle;
// reads past the matrix are zero.
bool bf16_map(CUtensorMap *map, const __nv_bfloat16 *base, int rows, int cols, int boxRows)
{
    auto enc = tensor_map_encoder();
    if (!enc || cols % 8 != 0 || ((uintptr_t)base & 15) != 0)
        return false;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
    cuuint32_t box[2] = {(cuuint32_t)clb::tc::BK, (cuuint32_t)boxRows};
    cuuint32_t estr[2] = {1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void *)base, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int sm_count_dev()
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms < 1)
            sms = 1;
    }
    return sms;
}

// The persistent tensor-memory GEMM: one CTA per SM (or per tile, if fewer).
template <int BN, int EPI>
cudaError_t tc_gemm_bn(const CUtensorMap &ma, const CUtensorMap &mb, int M, int N, int K, float *Z, const float *bias,
                       __nv_bfloat16 *Act, const int *Mdev, int moff, int *err, cudaStream_t s)
{
    static bool attr = false;
    auto *k = clb::tc::tc_gemm_persistent_kernel<BN, EPI>;
    const int smem = clb::tc::smem_bytes_persistent(BN);
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess)
            return e;
        attr = true;
    }
    const int tiles = ((N + BN - 1) / BN) * ((M + clb::tc::BM - 1) / clb::tc::BM);
    const int grid = tiles < sm_count_dev() ? tiles : sm_count_dev();
    k<<<grid, 192, smem, s>>>(ma, mb, M, N, K, Z, bias, Act, Mdev, moff, err);
    return cudaGetLastError();
}

// Z (nullable) / Act (nullable) [M x N] = epilogue(A [M x K] . B [N x K]^T):
// the tensor-memory GEMM (tc_gemm.cuh); K a multiple of 8.
template <int EPI>
cudaError_t tc_gemm(const __nv_bfloat16 *A, const __nv_bfloat16 *B, int M, int N, int K, float *Z, const float *bias,
                    __nv_bfloat16 *Act, const int *Mdev, int moff, int *err, cudaStream_t s)
{
    const int bn = N <= 32 ? 32 : (N <= 64 ? 64 : 128);
    CUtensorMap ma, mb;
    if (!bf16_map(&ma, A, M, K, clb::tc::BM) || !bf16_map(&mb, B, N, K, bn))
        return cudaErrorInvalidValue;
    if (bn == 32)
        return tc_gemm_bn<32, EPI>(ma, mb, M, N, K, Z, bias, Act, Mdev, moff, err, s);
    if (bn == 64)
        return tc_gemm_bn<64, EPI>(ma, mb, M, N, K, Z, bias, Act, Mdev, moff, err, s);
    return tc_gemm_bn<128, EPI>(ma, mb, M, N, K, Z, bias, Act, Mdev, moff, err, s);
}

}  // namespace

struct cl_mlp {
    int n = 0, width = 0, momentType = CL_MN;
    double delta = 0;
    int dims[kLayers + 1];
    float *W[kLayers] = {}, *b[kLayers] = {}, *mW[kLayers] = {}, *vW[kLayers] = {}, *mb[kLayers] = {},
          *vb[kLayers] = {}, *gW[kLayers] = {}, *gb[kLayers] = {};
    __nv_bfloat16 *W16[kLayers] = {};
    __nv_bfloat16 *Wt16[kLayers] = {};   // [out x round8(in)] BF16, the K-major operand of the forward GEMMs
    float *mean = nullptr, *stdv = nullptr;  // device [n]
    std::vector<float> hmean, hstd;
    int adamStep = 0;
    // work buffers (grow only)
    size_t cap = 0;
    __nv_bfloat16 *X = nullptr, *Xp = nullptr, *Act[kLayers] = {}, *dZ16 = nullptr;   // Xp: X padded to round8(n)
    int *tcErr = nullptr;       // error word of the tensor-memory GEMM's bounded waits
    bool keepZ = true;          // forward keeps the hidden pre-activations (training)
    float *Z[kLayers] = {}, *T = nullptr, *dA = nullptr, *dZ = nullptr, *loss = nullptr;
    int *fallbacks = nullptr;
    int *sel = nullptr;         // selected cells (+ their count) of cl_mlp_predict_selected
    size_t selCap = 0;
    cudaStream_t stream = nullptr;
    std::string err;
};

static int mlp_reserve(cl_mlp *m, size_t rows)
{
    if (rows <= m->cap)
        return CL_OK;
    cudaFree(m->X);
    cudaFree(m->Xp);
    cudaFree(m->dZ16);
    cudaFree(m->T);
    cudaFree(m->dA);
    cudaFree(m->dZ);
    cudaFree(m->loss);
    for (int l = 0; l < kLayers; l++) {
        cudaFree(m->Act[l]);
        cudaFree(m->Z[l]);
    }
    size_t w = (size_t)(m->width > m->n ? m->width : m->n);
    bool ok = cudaMalloc(&m->X, rows * m->n * sizeof(__nv_bfloat16)) == cudaSuccess &&
              cudaMalloc(&m->Xp, rows * round8(m->n) * sizeof(__nv_bfloat16)) == cudaSuccess &&
              cudaMalloc(&m->dZ16, rows * w * sizeof(__nv_bfloat16)) == cudaSuccess &&
              cudaMalloc(&m->T, rows * m->n * sizeof(float)) == cudaSuccess &&
              cudaMalloc(&m->dA, rows * w * sizeof(float)) == cudaSuccess &&
              cudaMalloc(&m->dZ, rows * w * sizeof(float)) == cudaSuccess &&
              cudaMalloc(&m->loss, (rows * m->n / 256 + 2) * sizeof(float)) == cudaSuccess;
    for (int l = 0; l < kLayers && ok; l++)
        ok = cudaMalloc(&m->Act[l], rows * w * sizeof(__nv_bfloat16)) == cudaSuccess &&
             cudaMalloc(&m->Z[l], rows * w * sizeof(float)) == cudaSuccess;
    if (!ok) {
        m->err = "MLP work buffer allocation failed";
        m->cap = 0;
        return CL_ERR_CUDA;
    }
    m->cap = rows;
    return CL_OK;
}

// forward over `rows` inputs already in m->X (with Mdev: min(rows, *Mdev -
// moff) of them); output pre-activations in Z[3]
//
// The layer GEMMs run on the tensor-memory path (tcgen05, tc_gemm.cuh): the
// input padded to round8(n) columns, the weights as K-major BF16 copies.
static cudaError_t mlp_forward(cl_mlp *m, int rows, const int *Mdev = nullptr, int moff = 0)
{
    const int np = round8(m->n);
    pad_cols_kernel<<<blocks((size_t)rows * np), 256, 0, m->stream>>>(m->X, rows, m->n, np, m->Xp);
    cudaError_t e = cudaGetLastError();
    const __nv_bfloat16 *in = m->Xp;
    for (int l = 0; l < kLayers && e == cudaSuccess; l++) {
        const int K = round8(m->dims[l]), N = m->dims[l + 1];
        if (l < kLayers - 1)
            e = tc_gemm<clb::tc::EPI_BIAS_GELU>(in, m->Wt16[l], rows, N, K, m->keepZ ? m->Z[l] : nullptr, m->b[l],
                                                 m->Act[l], Mdev, moff, m->tcErr, m->stream);
        else
            e = tc_gemm<clb::tc::EPI_BIAS>(in, m->Wt16[l], rows, N, K, m->Z[l], m->b[l], nullptr, Mdev, moff,
                                            m->tcErr, m->stream);
        in = m->Act[l];
    }
    return e;
}

static cudaError_t mlp_sync_weights(cl_mlp *m)
{
    for (int l = 0; l < kLayers; l++) {
        size_t cnt = (size_t)m->dims[l] * m->dims[l + 1];
        cast_bf16_kernel<<<blocks(cnt), 256, 0, m->stream>>>(m->W[l], m->W16[l], cnt);
        const int K = m->dims[l], N = m->dims[l + 1], Kp = round8(K);
        transpose_cast_kernel<<<blocks((size_t)N * Kp), 256, 0, m->stream>>>(m->W[l], K, N, Kp, m->Wt16[l]);
    }
    return cudaGetLastError();
}

// backward of the MSE loss for the batch in X/T; gradients into gW/gb
static cudaError_t mlp_backward(cl_mlp *m, int rows, float *lossOut)
{
    const int n = m->n;
    const int total = rows * n;
    int nb = blocks(total);
    mse_grad_kernel<<<nb, 256, 0, m->stream>>>(m->Z[kLayers - 1], m->T, m->dZ16, m->dZ, total, 1.0f / (float)total,
                                               m->loss);
    cudaError_t e = cudaGetLastError();
    for (int l = kLayers - 1; l >= 0 && e == cudaSuccess; l--) {
        int K = m->dims[l], N = m->dims[l + 1];
        const __nv_bfloat16 *in = (l == 0) ? m->X : m->Act[l - 1];
        // dW_l = in^T . dZ_l   ([K x rows] . [rows x N])
        e = gemm<1, 0, EPI_F32>(in, m->dZ16, K, N, rows, m->gW[l], nullptr, nullptr, m->stream);
        colsum_kernel<<<blocks(N), 256, 0, m->stream>>>(m->dZ, rows, N, m->gb[l]);
        if (l > 0 && e == cudaSuccess) {
            // dA_{l-1} = dZ_l . W_l^T   ([rows x N] . [N x K])
            e = gemm<0, 1, EPI_F32>(m->dZ16, m->W16[l], rows, K, N, m->dA, nullptr, nullptr, m->stream);
            size_t cnt = (size_t)rows * K;
            gelu_back_kernel<<<blocks(cnt), 256, 0, m->stream>>>(m->dA, m->Z[l - 1], m->dZ16, m->dZ, cnt);
        }
    }
    if (lossOut && e == cudaSuccess) {
        std::vector<float> part(nb);
        e = cudaMemcpyAsync(part.data(), m->loss, sizeof(float) * nb, cudaMemcpyDeviceToHost, m->stream);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(m->stream);
        double s = 0;
        for (float p : part)
            s += p;
        *lossOut = (float)(s / total);
    }
    return e;
}

// The tensor-memory GEMM's error word (a bounded wait that gave up), read
// after the stream has been synchronised, and cleared.
static int tc_error(cl_mlp *m)
{
    int h = 0;
    if (cudaMemcpy(&h, m->tcErr, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return CL_ERR_CUDA;
    if (h != 0) {
        cudaMemset(m->tcErr, 0, sizeof(int));
        m->err = "tensor-memory GEMM: a bounded wait timed out";
        return CL_ERR_TIMEOUT;
    }
    return CL_OK;
}

extern "C" {

int cl_mlp_create(int n, int width, int moment_type, double delta_ppn, unsigned long long seed, cl_mlp **out)
{
    if (!out || n < 1 || n > 32 || width < 8 || width > 4096)
        return CL_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
        return CL_ERR_CUDA;
    cl_mlp *m = new cl_mlp();
    m->n = n;
    m->width = width;
    m->momentType = moment_type;
    m->delta = delta_ppn;
    m->dims[0] = n;
    m->dims[1] = m->dims[2] = m->dims[3] = width;
    m->dims[4] = n;
    cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
    std::mt19937_64 rng(seed);
    bool ok = true;
    for (int l = 0; l < kLayers && ok; l++) {
        size_t cnt = (size_t)m->dims[l] * m->dims[l + 1];
        int N = m->dims[l + 1];
        // He-style uniform init scaled by fan-in
        std::uniform_real_distribution<float> U(-1.0f, 1.0f);
        float sc = std::sqrt(3.0f / (float)m->dims[l]);
        std::vector<float> w(cnt), z(cnt, 0.0f), bz(N, 0.0f);
        for (auto &v : w)
            v = U(rng) * sc;
        ok = cudaMalloc(&m->W[l], cnt * 4) == cudaSuccess && cudaMalloc(&m->mW[l], cnt * 4) == cudaSuccess &&
             cudaMalloc(&m->vW[l], cnt * 4) == cudaSuccess && cudaMalloc(&m->gW[l], cnt * 4) == cudaSuccess &&
             cudaMalloc(&m->W16[l], cnt * 2) == cudaSuccess &&
             cudaMalloc(&m->Wt16[l], (size_t)N * round8(m->dims[l]) * 2) == cudaSuccess &&
             cudaMalloc(&m->b[l], N * 4) == cudaSuccess &&
             cudaMalloc(&m->mb[l], N * 4) == cudaSuccess && cudaMalloc(&m->vb[l], N * 4) == cudaSuccess &&
             cudaMalloc(&m->gb[l], N * 4) == cudaSuccess;
        if (ok) {
            cudaMemcpy(m->W[l], w.data(), cnt * 4, cudaMemcpyHostToDevice);
            cudaMemcpy(m->mW[l], z.data(), cnt * 4, cudaMemcpyHostToDevice);
            cudaMemcpy(m->vW[l], z.data(), cnt * 4, cudaMemcpyHostToDevice);
            cudaMemcpy(m->b[l], bz.data(), N * 4, cudaMemcpyHostToDevice);
            cudaMemcpy(m->mb[l], bz.data(), N * 4, cudaMemcpyHostToDevice);
            cudaMemcpy(m->vb[l], bz.data(), N * 4, cudaMemcpyHostToDevice);
        }
    }
    ok = ok && cudaMalloc(&m->mean, n * 4) == cudaSuccess && cudaMalloc(&m->stdv, n * 4) == cudaSuccess &&
         cudaMalloc(&m->fallbacks, sizeof(int)) == cudaSuccess && cudaMalloc(&m->tcErr, sizeof(int)) == cudaSuccess &&
         cudaMemset(m->tcErr, 0, sizeof(int)) == cudaSuccess;
    if (!ok) {
        cl_mlp_destroy(m);
        return CL_ERR_CUDA;
    }
    m->hmean.assign(n, 0.0f);
    m->hstd.assign(n, 1.0f);
    cudaMemcpy(m->mean, m->hmean.data(), n * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(m->stdv, m->hstd.data(), n * 4, cudaMemcpyHostToDevice);
    mlp_sync_weights(m);
    cudaStreamSynchronize(m->stream);
    *out = m;
    return CL_OK;
}

void cl_mlp_destroy(cl_mlp *m)
{
    if (!m)
        return;
    if (m->stream)
        cudaStreamSynchronize(m->stream);
    for (int l = 0; l < kLayers; l++) {
        cudaFree(m->W[l]);
        cudaFree(m->b[l]);
        cudaFree(m->mW[l]);
        cudaFree(m->vW[l]);
        cudaFree(m->mb[l]);
        cudaFree(m->vb[l]);
        cudaFree(m->gW[l]);
        cudaFree(m->gb[l]);
        cudaFree(m->W16[l]);
        cudaFree(m->Wt16[l]);
        cudaFree(m->Act[l]);
        cudaFree(m->Z[l]);
    }
    cudaFree(m->mean);
    cudaFree(m->stdv);
    cudaFree(m->X);
    cudaFree(m->dZ16);
    cudaFree(m->T);
    cudaFree(m->dA);
    cudaFree(m->dZ);
    cudaFree(m->loss);
    cudaFree(m->fallbacks);
    cudaFree(m->tcErr);
    cudaFree(m->sel);
    if (m->stream)
        cudaStreamDestroy(m->stream);
    delete m;
}

const char *cl_mlp_last_error(const cl_mlp *m) { return m ? m->err.c_str() : ""; }

// Standardisation of the targets (per-component mean and std, host arrays).
int cl_mlp_set_output_scaling(cl_mlp *m, const float *mean, const float *stdv)
{
    if (!m || !mean || !stdv)
        return CL_ERR_ARG;
    m->hmean.assign(mean, mean + m->n);
    m->hstd.assign(stdv, stdv + m->n);
    cudaMemcpy(m->mean, mean, m->n * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(m->stdv, stdv, m->n * 4, cudaMemcpyHostToDevice);
    return CL_OK;
}

// Adam training on pairs (u, alpha) held on the device ([count x n] FP64).
// Minibatches are consecutive slices of a shuffled index order drawn on the
// host; losses[steps] (nullable) receives the batch loss per step.
int cl_mlp_train(cl_mlp *m, const double *d_u, const double *d_alpha, int count, int steps, int batch, float lr,
                 unsigned long long seed, float *losses)
{
    if (!m || !d_u || !d_alpha || count < batch || batch < 1 || steps < 0)
        return CL_ERR_ARG;
    int rc = mlp_reserve(m, batch);
    if (rc)
        return rc;
    const int n = m->n;
    // gather buffers for the minibatch (FP64 on device)
    double *bu = nullptr, *ba = nullptr;
    int *dperm = nullptr;
    if (cudaMalloc(&bu, (size_t)batch * n * 8) != cudaSuccess || cudaMalloc(&ba, (size_t)batch * n * 8) != cudaSuccess ||
        cudaMalloc(&dperm, (size_t)count * sizeof(int)) != cudaSuccess) {
        cudaFree(bu);
        cudaFree(ba);
        m->err = "minibatch allocation failed";
        return CL_ERR_CUDA;
    }
    std::mt19937_64 rng(seed);
    std::vector<int> order(count);
    for (int i = 0; i < count; i++)
        order[i] = i;
    int pos = count;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    cudaError_t e = cudaSuccess;
    for (int s = 0; s < steps && e == cudaSuccess; s++) {
        if (pos + batch > count) {
            // new epoch: a fresh permutation of the training pairs
            std::shuffle(order.begin(), order.end(), rng);
            e = cudaMemcpyAsync(dperm, order.data(), (size_t)count * sizeof(int), cudaMemcpyHostToDevice, m->stream);
            if (e == cudaSuccess)
                e = cudaStreamSynchronize(m->stream);
            pos = 0;
        }
        gather_kernel<<<blocks((size_t)batch * n), 256, 0, m->stream>>>(d_u, d_alpha, dperm + pos, batch, n, bu, ba);
        pos += batch;
        prep_kernel<<<blocks((size_t)batch * n), 256, 0, m->stream>>>(bu, ba, batch, n, m->momentType, m->mean,
                                                                     m->stdv, m->X, m->T);
        if (e == cudaSuccess)
            e = mlp_forward(m, batch);
        float l = 0;
        if (e == cudaSuccess)
            e = mlp_backward(m, batch, losses ? &l : nullptr);
        if (losses)
            losses[s] = l;
        m->adamStep++;
        float c1 = 1.0f - std::pow(b1, (float)m->adamStep), c2 = 1.0f - std::pow(b2, (float)m->adamStep);
        for (int L = 0; L < kLayers && e == cudaSuccess; L++) {
            size_t cnt = (size_t)m->dims[L] * m->dims[L + 1];
            const float lrs = (s >= steps - steps / 5) ? 0.1f * lr : lr;   // step decay for the last fifth
            adam_kernel<<<blocks(cnt), 256, 0, m->stream>>>(m->W[L], m->mW[L], m->vW[L], m->gW[L], cnt, lrs, b1, b2,
                                                           eps, c1, c2);
            adam_kernel<<<blocks(m->dims[L + 1]), 256, 0, m->stream>>>(m->b[L], m->mb[L], m->vb[L], m->gb[L],
                                                                      m->dims[L + 1], lrs, b1, b2, eps, c1, c2);
        }
        if (e == cudaSuccess)
            e = mlp_sync_weights(m);
    }
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(m->stream);
    cudaFree(bu);
    cudaFree(ba);
    cudaFree(dperm);
    if (e != cudaSuccess) {
        m->err = std::string("training: ") + cudaGetErrorString(e);
        return CL_ERR_CUDA;
    }
    return tc_error(m);
}

// Predicted multipliers for count vectors d_u (device, [count x n]) written to
// d_alpha; non-finite predictions keep d_alpha (fallback_kind 0, e.g. the
// previous stage) or take the isotropic multiplier (fallback_kind 1).
// *fallbacks (nullable) receives how many vectors fell back.
int cl_mlp_predict(cl_mlp *m, const double *d_u, double *d_alpha, int count, int fallback_kind, int *fallbacks,
                   void *stream)
{
    if (!m || !d_u || !d_alpha || count < 0)
        return CL_ERR_ARG;
    if (count == 0)
        return CL_OK;
    cudaStream_t st = stream ? (cudaStream_t)stream : m->stream;
    const int chunk = 1 << 18;
    int rc = mlp_reserve(m, count < chunk ? count : chunk);
    if (rc)
        return rc;
    cudaStream_t keep = m->stream;
    m->stream = st;
    cudaError_t e = cudaMemsetAsync(m->fallbacks, 0, sizeof(int), st);
    for (int c0 = 0; c0 < count && e == cudaSuccess; c0 += chunk) {
        int rows = count - c0 < chunk ? count - c0 : chunk;
        prep_kernel<<<blocks((size_t)rows * m->n), 256, 0, st>>>(d_u + (size_t)c0 * m->n, nullptr, rows, m->n,
                                                                m->momentType, m->mean, m->stdv, m->X, nullptr);
        m->keepZ = false;
        e = mlp_forward(m, rows);
        m->keepZ = true;
        predict_out_kernel<<<blocks(rows), 256, 0, st>>>(m->Z[kLayers - 1], d_u + (size_t)c0 * m->n,
                                                         d_alpha + (size_t)c0 * m->n, rows, m->n, m->momentType,
                                                         m->delta, m->mean, m->stdv, fallback_kind, m->fallbacks);
    }
    m->stream = keep;
    if (fallbacks && e == cudaSuccess) {
        e = cudaMemcpyAsync(fallbacks, m->fallbacks, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(st);
    }
    if (e == cudaSuccess)
        e = cudaGetLastError();
    if (e != cudaSuccess) {
        m->err = std::string("predict: ") + cudaGetErrorString(e);
        return CL_ERR_CUDA;
    }
    return CL_OK;
}

// Predicted starts only for the cells whose last optimisation took at least
// min_iters iterations (d_iters, device [count]); the other cells' starts are
// NaN, so the Newton kernel starts them from their previous-stage
// multipliers.  The selection is compacted on the device and the network runs
// over it in chunks whose row counts the GEMMs read from device memory, so
// the call needs no host synchronisation and can be captured in a graph.
int cl_mlp_predict_selected(cl_mlp *m, const double *d_u, const int *d_iters, int min_iters, double *d_alpha,
                            int count, void *stream)
{
    if (!m || !d_u || !d_iters || !d_alpha || count < 0 || min_iters < 1)
        return CL_ERR_ARG;
    if (count == 0)
        return CL_OK;
    cudaStream_t st = stream ? (cudaStream_t)stream : m->stream;
    const int chunk = 1 << 18;
    int rc = mlp_reserve(m, count < chunk ? count : chunk);
    if (rc)
        return rc;
    if (!m->sel || m->selCap < (size_t)count) {
        cudaFree(m->sel);
        m->sel = nullptr;
        if (cudaMalloc(&m->sel, ((size_t)count + 1) * sizeof(int)) != cudaSuccess) {
            m->err = "selection buffer";
            return CL_ERR_CUDA;
        }
        m->selCap = count;
    }
    int *cnt = m->sel + count;
    cudaStream_t keep = m->stream;
    m->stream = st;
    cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(int), st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(m->fallbacks, 0, sizeof(int), st);
    select_kernel<<<blocks(count), 256, 0, st>>>(d_iters, count, min_iters, m->sel, cnt, d_alpha, m->n);
    for (int c0 = 0; c0 < count && e == cudaSuccess; c0 += chunk) {
        const int rows = count - c0 < chunk ? count - c0 : chunk;
        prep_idx_kernel<<<blocks((size_t)rows * m->n), 256, 0, st>>>(d_u, m->sel, cnt, c0, rows, m->n, m->X);
        m->keepZ = false;
        e = mlp_forward(m, rows, cnt, c0);
        m->keepZ = true;
        predict_out_kernel<<<blocks(rows), 256, 0, st>>>(m->Z[kLayers - 1], d_u, d_alpha, rows, m->n, m->momentType,
                                                         m->delta, m->mean, m->stdv, 2, m->fallbacks, m->sel, cnt,
                                                         c0);
    }
    m->stream = keep;
    if (e == cudaSuccess)
        e = cudaGetLastError();
    if (e != cudaSuccess) {
        m->err = std::string("selected predict: ") + cudaGetErrorString(e);
        return CL_ERR_CUDA;
    }
    return CL_OK;
}

// The network's GEMM on its own (device pointers): C [M x N] FP32 = A [M x K]
// . B [N x K]^T with BF16 A, B (row-major, K a multiple of 8).  Waits for the
// result; for the numerics test of the tensor-memory path.
int cl_tc_gemm_bf16(const void *d_A, const void *d_B, int M, int N, int K, float *d_C)
{
    if (!d_A || !d_B || !d_C || M < 1 || N < 1 || K < 8 || K % 8 != 0)
        return CL_ERR_ARG;
    int *err = nullptr;
    if (cudaMalloc(&err, sizeof(int)) != cudaSuccess)
        return CL_ERR_CUDA;
    cudaMemset(err, 0, sizeof(int));
    cudaError_t e = tc_gemm<clb::tc::EPI_STORE>((const __nv_bfloat16 *)d_A, (const __nv_bfloat16 *)d_B, M, N, K, d_C,
                                                 nullptr, nullptr, nullptr, 0, err, nullptr);
    if (e == cudaSuccess)
        e = cudaDeviceSynchronize();
    int h = 0;
    if (e == cudaSuccess)
        e = cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(err);
    if (e != cudaSuccess)
        return CL_ERR_CUDA;
    return h ? CL_ERR_TIMEOUT : CL_OK;
}

// Gradient check support: loss and parameter gradients of one batch (host
// FP64 inputs), copied to host buffers grads[l] = {dW_l [in x out], db_l}.
int cl_mlp_loss_and_grads(cl_mlp *m, const double *u, const double *alpha, int rows, float *loss, float *const *gW,
                          float *const *gb)
{
    if (!m || !u || !alpha || rows < 1)
        return CL_ERR_ARG;
    int rc = mlp_reserve(m, rows);
    if (rc)
        return rc;
    const int n = m->n;
    double *bu = nullptr, *ba = nullptr;
    cudaMalloc(&bu, (size_t)rows * n * 8);
    cudaMalloc(&ba, (size_t)rows * n * 8);
    cudaMemcpy(bu, u, (size_t)rows * n * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(ba, alpha, (size_t)rows * n * 8, cudaMemcpyHostToDevice);
    prep_kernel<<<blocks((size_t)rows * n), 256, 0, m->stream>>>(bu, ba, rows, n, m->momentType, m->mean, m->stdv,
                                                                m->X, m->T);
    cudaError_t e = mlp_forward(m, rows);
    if (e == cudaSuccess)
        e = mlp_backward(m, rows, loss);
    for (int l = 0; l < kLayers && e == cudaSuccess; l++) {
        size_t cnt = (size_t)m->dims[l] * m->dims[l + 1];
        if (gW && gW[l])
            e = cudaMemcpy(gW[l], m->gW[l], cnt * 4, cudaMemcpyDeviceToHost);
        if (gb && gb[l] && e == cudaSuccess)
            e = cudaMemcpy(gb[l], m->gb[l], m->dims[l + 1] * 4, cudaMemcpyDeviceToHost);
    }
    cudaFree(bu);
    cudaFree(ba);
    if (e != cudaSuccess) {
        m->err = std::string("loss/grad: ") + cudaGetErrorString(e);
        return CL_ERR_CUDA;
    }
    return tc_error(m);
}

// Parameters: W_l is [in x out] row-major (y = x W + b).  get/set copy FP32
// masters; set also refreshes the BF16 copies.
int cl_mlp_get_params(cl_mlp *m, float *const *W, float *const *b)
{
    if (!m)
        return CL_ERR_ARG;
    cudaStreamSynchronize(m->stream);
    for (int l = 0; l < kLayers; l++) {
        if (W && W[l])
            cudaMemcpy(W[l], m->W[l], (size_t)m->dims[l] * m->dims[l + 1] * 4, cudaMemcpyDeviceToHost);
        if (b && b[l])
            cudaMemcpy(b[l], m->b[l], m->dims[l + 1] * 4, cudaMemcpyDeviceToHost);
    }
    return CL_OK;
}

int cl_mlp_set_params(cl_mlp *m, float *const *W, float *const *b)
{
    if (!m)
        return CL_ERR_ARG;
    for (int l = 0; l < kLayers; l++) {
        if (W && W[l])
            cudaMemcpy(m->W[l], W[l], (size_t)m->dims[l] * m->dims[l + 1] * 4, cudaMemcpyHostToDevice);
        if (b && b[l])
            cudaMemcpy(m->b[l], b[l], m->dims[l + 1] * 4, cudaMemcpyHostToDevice);
    }
    mlp_sync_weights(m);
    return cudaStreamSynchronize(m->stream) == cudaSuccess ? CL_OK : CL_ERR_CUDA;
}

}  // extern "C"

// Reserves inference buffers ahead of stream capture (used by the grid solver).
int clb_mlp_reserve_for(cl_mlp *m, size_t rows)
{
    const size_t chunk = 1 << 18;
    return mlp_reserve(m, rows < chunk ? rows : chunk);
}
