// common.cuh -- device helpers shared by the closures-2d B200 kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace clb {

constexpr int kThreads = 256;        // 8 warps per CTA
constexpr int kWarps = kThreads / 32;
constexpr int kMaxN = 32;            // moments per cell handled by one warp (order <= 6)
constexpr int kMaxProblems = 8;      // moment orders sharing one persistent launch
constexpr int kNumReg = 5;

// opt/opt.h:39-40
__device__ __constant__ const double kRegularizations[kNumReg] = {0.0, 1e-3, 1e-2, 1e-1, 5e-1};

// FP64 tensor-core MMA, m16n8k8 (A row-major 16x8, B column-major 8x8,
// C/D 16x8).  Fragment ownership (g = lane/4, t = lane%4):
//   a0 A[g][t]   a1 A[g+8][t]   a2 A[g][t+4]   a3 A[g+8][t+4]
//   b0 B[t][g]   b1 B[t+4][g]
//   c0 C[g][2t]  c1 C[g][2t+1]  c2 C[g+8][2t]  c3 C[g+8][2t+1]
__device__ __forceinline__ void dmma16x8x8(double (&c)[4], double a0, double a1, double a2,
                                           double a3, double b0, double b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}

// 16-byte global->shared asynchronous copy (L2 only) and its group fences.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
// Index of the first maximum of v over lanes < n (BLAS idamax semantics).
__device__ __forceinline__ int warp_argmax_first(double v, int lane)
{
    int idx = lane;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double ov = __shfl_xor_sync(0xffffffffu, v, o);
        int oi = __shfl_xor_sync(0xffffffffu, idx, o);
        if (ov > v || (ov == v && oi < idx)) {
            v = ov;
            idx = oi;
        }
    }
    return idx;
}

// Device counters of the optimisation stages; the first kStatU64 fields are
// 64-bit sums, laid out contiguously so a CTA can flush them by index.
struct DevStats {
    unsigned long long hist[kNumReg];   // solves per regularisation level
    unsigned long long totalIter;       // sum of outs.iter
    unsigned long long numSolves;
    unsigned long long trials;          // line-search evaluations
    unsigned long long fallbacks;       // predicted starts abandoned for the fallback start
    int maxIter;
    int pad;
};
constexpr int kStatU64 = kNumReg + 4;

}  // namespace clb
