// tc_gemm.cuh -- BF16 GEMM on the 5th-generation tensor cores (sm_100a) for
// the learned warm start's network: C = A . B^T with A [M x K] and B [N x K]
// both K-major (row-major with K contiguous), FP32 accumulation in tensor
// memory, and a fused epilogue (bias, GELU, FP32 and/or BF16 stores).
//
// A persistent CTA per SM takes 128 x BN tiles in turn:
//   warp 0, one lane   TMA producer: cp.async.bulk.tensor 2-D loads of the
//                      A and B k-blocks (128 B swizzle, 64 BF16 of K per
//                      row) into a four-stage ring, completion counted in
//                      bytes on the stage's "full" mbarrier; no multicast;
//   warp 1, one lane   MMA issuer: tcgen05.mma.cta_group::1.kind::f16,
//                      M = 128, N = BN, K = 16 per instruction, into one of
//                      two BN-column accumulators in tensor memory;
//                      tcgen05.commit on the stage's "empty" mbarrier hands
//                      the stage back, a commit per tile hands the
//                      accumulator to the epilogue;
//   warps 2-5          epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31
//                      (rows of the tile) with tcgen05.ld.32x32b, 16 columns
//                      at a time, and frees the accumulator, so one tile's
//                      epilogue overlaps the next tile's MMAs.
// Every wait is bounded (2 s of %globaltimer); a wait that gives up records
// an error in *err and the CTA still releases its tensor memory.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "closures_gpu.h"
#include "common.cuh"

namespace clb {
namespace tc {

constexpr int BM = 128;                 // tile rows = TMEM lanes
constexpr int BK = 64;                  // BF16 of K per k-block: one 128 B swizzle row
constexpr unsigned long long kWaitNs = 2000000000ull;

enum Epi { EPI_STORE = 0, EPI_BIAS = 1, EPI_BIAS_GELU = 2 };

__device__ __forceinline__ float gelu_f(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }

// Shared-memory matrix descriptor of a K-major tile in the 128 B swizzle
// layout: rows of 128 B, 8-row groups 1024 B apart (stride byte offset),
// leading byte offset unused (1), descriptor version 1, layout type 2.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;                 // leading byte offset (16 B units)
    d |= (uint64_t)(1024 >> 4) << 32;       // stride byte offset
    d |= (uint64_t)1 << 46;                 // version
    d |= (uint64_t)2 << 61;                 // 128 B swizzle
    return d;
}

// Instruction descriptor of kind::f16: BF16 A and B, FP32 accumulator, both
// K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc_bf16(int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, unsigned long long *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
            smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, int acc)
{
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void umma_commit(unsigned long long *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// Z (nullable) [M x N] FP32 = A B^T (+ bias); Act (nullable) [M x N] BF16 =
// GELU(Z) (EPI_BIAS_GELU) or Z; with Mdev, M = min(M, *Mdev - moff).
// Persistent (one CTA per SM, tiles taken in turn), six warps:
//   warp 0 (one lane)  TMA producer over the tiles' k-blocks, kPStages deep;
//   warp 1 (one lane)  MMA issuer into one of two BN-column accumulators in
//                      tensor memory, alternating per tile;
//   warps 2-5          epilogue of the other accumulator: warp w reads TMEM
//                      lanes 32 (w % 4) .. +31, then frees the buffer.
// So a tile's epilogue runs while the next tile's MMAs accumulate.  Barriers:
// full/empty per stage (TMA / MMA), tfull/tempty per accumulator (MMA /
// epilogue), all waits bounded.
constexpr int kPStages = 4;
constexpr int smem_bytes_persistent(int bn) { return kPStages * (BM * BK * 2 + bn * BK * 2) + 1024; }

template <int BN, int EPI>
__device__ __forceinline__ void epilogue_rows(uint32_t tl, int row, int M, int N, int n0, float *Z,
                                              const float *bias, __nv_bfloat16 *Act)
{
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 16) {
        if (n0 + c0 >= N)
            break;   // uniform over the warp
        uint32_t r[16];
        tmem_ld16(tl + c0, r);
        if (row >= M)
            continue;
        const int col0 = n0 + c0;
        float v[16];
#pragma unroll
        for (int j = 0; j < 16; j++) {
            v[j] = __uint_as_float(r[j]);
            if (EPI != EPI_STORE && col0 + j < N)
                v[j] += bias[col0 + j];
        }
        if (col0 + 16 <= N && (N & 7) == 0) {
            if (Z) {
                float4 *z = reinterpret_cast<float4 *>(Z + (size_t)row * N + col0);
#pragma unroll
                for (int q = 0; q < 4; q++)
                    z[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            }
            if (Act) {
                __align__(16) __nv_bfloat16 b[16];
#pragma unroll
                for (int j = 0; j < 16; j++)
                    b[j] = __float2bfloat16(EPI == EPI_BIAS_GELU ? gelu_f(v[j]) : v[j]);
                uint4 *a = reinterpret_cast<uint4 *>(Act + (size_t)row * N + col0);
                a[0] = reinterpret_cast<const uint4 *>(b)[0];
                a[1] = reinterpret_cast<const uint4 *>(b)[1];
            }
        } else {
#pragma unroll
            for (int j = 0; j < 16; j++) {
                const int col = col0 + j;
                if (col < N) {
                    if (Z)
                        Z[(size_t)row * N + col] = v[j];
                    if (Act)
                        Act[(size_t)row * N + col] = __float2bfloat16(EPI == EPI_BIAS_GELU ? gelu_f(v[j]) : v[j]);
                }
            }
        }
    }
}

template <int BN, int EPI>
__global__ void __launch_bounds__(192, 1)
    tc_gemm_persistent_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                              int M, int N, int K, float *Z, const float *bias, __nv_bfloat16 *Act, const int *Mdev,
                              int moff, int *err)
{
    static_assert(BN == 32 || BN == 64 || BN == 128, "two accumulators of BN columns (power of two)");
    constexpr int A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2, STAGE = A_BYTES + B_BYTES;
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) unsigned long long full[kPStages], empty[kPStages], tfull[2], tempty[2];
    __shared__ uint32_t tmemBase;
    __shared__ int failed;
    unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (Mdev) {
        const int rem = *Mdev - moff;
        M = rem < M ? (rem > 0 ? rem : 0) : M;
    }
    const int tilesN = (N + BN - 1) / BN, tilesM = (M + BM - 1) / BM;
    const int ntiles = tilesM * tilesN;
    if ((int)blockIdx.x >= ntiles)
        return;   // uniform over the CTA, before any allocation
    const int nk = (K + BK - 1) / BK;

    if (tid == 0) {
        for (int s = 0; s < kPStages; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 4);   // one arrival per epilogue warp
        }
        mbar_init_fence();
        failed = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmemBase)),
                     "r"(2 * BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmemBase;

    if (warp == 0) {
        if (lane == 0) {
            int kbAll = 0;   // k-blocks issued so far (ring position)
            for (int t = blockIdx.x; t < ntiles && !failed; t += gridDim.x) {
                const int m0 = (t / tilesN) * BM, n0 = (t % tilesN) * BN;
                for (int kb = 0; kb < nk; kb++, kbAll++) {
                    const int s = kbAll % kPStages;
                    if (kbAll >= kPStages &&
                        !mbar_wait_bounded(&empty[s], ((kbAll / kPStages) - 1) & 1, kWaitNs)) {
                        failed = 1;
                        break;
                    }
                    unsigned char *sa = smem + s * STAGE;
                    mbar_expect_tx(&full[s], STAGE);
                    tma_load_2d(sa, &mapA, kb * BK, m0, &full[s]);
                    tma_load_2d(sa + A_BYTES, &mapB, kb * BK, n0, &full[s]);
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_bf16(BN);
            int kbAll = 0, it = 0;
            for (int t = blockIdx.x; t < ntiles && !failed; t += gridDim.x, it++) {
                const int b = it & 1;
                // the epilogue has freed this accumulator (its previous use)
                if (it >= 2 && !mbar_wait_bounded(&tempty[b], ((it >> 1) - 1) & 1, kWaitNs)) {
                    failed = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint32_t acc = tmem + (uint32_t)(b * BN);
                for (int kb = 0; kb < nk; kb++, kbAll++) {
                    const int s = kbAll % kPStages;
                    if (!mbar_wait_bounded(&full[s], (kbAll / kPStages) & 1, kWaitNs)) {
                        failed = 1;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                    const uint32_t sa = smem_u32(smem + s * STAGE), sb = sa + A_BYTES;
                    const int ksteps = min(BK / 16, (K - kb * BK + 15) / 16);
                    for (int kk = 0; kk < ksteps; kk++)
                        umma_bf16(acc, smem_desc_sw128(sa + kk * 32), smem_desc_sw128(sb + kk * 32), idesc,
                                  (kb > 0 || kk > 0) ? 1 : 0);
                    umma_commit(&empty[s]);
                }
                umma_commit(&tfull[b]);
                if (failed)
                    break;
            }
        }
    } else {
        // epilogue warps 2..5: TMEM lane quarter w % 4
        const int quarter = warp & 3;
        int it = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, it++) {
            const int b = it & 1;
            if (!mbar_wait_bounded(&tfull[b], (it >> 1) & 1, kWaitNs)) {
                if (lane == 0)
                    failed = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const int m0 = (t / tilesN) * BM, n0 = (t % tilesN) * BN;
            const uint32_t tl = tmem + (uint32_t)(b * BN) + ((uint32_t)(quarter * 32) << 16);
            epilogue_rows<BN, EPI>(tl, m0 + quarter * 32 + lane, M, N, n0, Z, bias, Act);
            asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
            __syncwarp();
            if (lane == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(&tempty[b])) : "memory");
        }
    }
    __syncthreads();
    if (failed && tid == 0 && err)
        atomicExch(err, CL_ERR_TIMEOUT);
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(2 * BN) : "memory");
}

}  // namespace tc
}  // namespace clb
