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
// change-of-basis working state of one Newton slot in global memory: the
// basis T and the rows of L^-1 ([kMaxN][kMaxN] each), then alphaP, the
// line-search alphaM and step, and 1/T_ii ([kMaxN] each)
constexpr int kCbSlotDoubles = 2 * kMaxN * kMaxN + 4 * kMaxN;
// BFGS sub-iterations add the approximations of H and H^-1 in the working
// basis ([kMaxN][kMaxN] each, column j at j * kMaxN, lane i holding row i),
// the previous gradient and the current gradient in that basis
constexpr int kBfgsSlotDoubles = kCbSlotDoubles + 2 * kMaxN * kMaxN + 2 * kMaxN;

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

// TF32 tensor-core MMA m16n8k8 with FP32 accumulation: the same fragment
// ownership as dmma16x8x8, 32-bit registers holding TF32 values.
__device__ __forceinline__ void tmma16x8x8(float (&c)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3,
                                           unsigned b0, unsigned b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// x = hi + lo with hi, lo TF32 (round to nearest): the three products
// hi.hi + hi.lo + lo.hi of two split operands carry about FP32 accuracy.
__device__ __forceinline__ void tf32_split(float x, unsigned &hi, unsigned &lo)
{
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(hi) : "f"(x));
    const float r = x - __uint_as_float(hi);
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(lo) : "f"(r));
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

// Bulk asynchronous copies (global -> shared, completion counted in bytes on
// an mbarrier) and the mbarrier operations they use.  Addresses and sizes of
// a copy are multiples of 16 bytes.
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes)
{
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}
// Waits for the phase with the given parity; gives up after `ns` nanoseconds.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, unsigned parity, unsigned long long ns)
{
    if (mbar_try_wait(bar, parity))
        return true;
    const unsigned long long t0 = global_ns();
    for (;;) {
        if (mbar_try_wait(bar, parity))
            return true;
        if (global_ns() - t0 > ns)
            return false;
    }
}
// Orders this thread's generic-proxy shared-memory accesses before later
// async-proxy (bulk copy) accesses.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

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
    unsigned long long screened;        // solves settled by the screening pass
    unsigned long long screenEvals;     // evaluations of the screening pass
    int maxIter;
    int pad;
    unsigned long long fluxTiles;       // K2+K3 tiles that ran the chunk loop
};
constexpr int kStatU64 = kNumReg + 6;

}  // namespace clb
