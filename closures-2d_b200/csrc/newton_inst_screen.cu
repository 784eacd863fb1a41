// newton_inst_screen.cu -- the screening pass of K1 (screen_kernel in
// newton_kernel.cuh): layout planning and its instances, one per (gradient
// column tiles, k-steps) of the direction-pair layouts of orders 1-6:
// N = 1..3 -> (2, 2), N = 4 -> (3, 3), N = 5, 6 -> (4, 4).
#include "newton_kernel.cuh"

namespace clb {

bool screen_supported(int nt, int nbk) { return nt == nbk && nt >= 2 && nt <= 4; }

int plan_screen(NewtonArgs &a)
{
    const NewtonProblem &pb = a.prob[0];
    if (a.nprob != 1 || !pb.paired || a.momentType != 0 || a.mixed || a.optType != 0)
        return -1;
    a.nw = kWarps;
    a.T = 32;
    a.kq = 32;
    a.ntq = a.kq / 8;
    a.ldv = pb.nb + 4;
    a.ldE = a.kq + 4;
    a.ldG = pb.K2p + 4;
    a.ldh = (pb.n | 1) + 1;
    const int T = a.T;
    int off = 0;
    auto take = [&](int ndoubles) {
        int o = off;
        off += (ndoubles + 1) & ~1;   // keep 16-byte alignment
        return o;
    };
    a.offAlpha = take(T * a.ldv);
    a.offAold = take(T * a.ldv);
    a.offD = take(T * a.ldv);
    a.offU = take(T * a.ldv);
    a.offScal = take(T * SC_N);
    a.offInt = take((T * SI_N + 1) / 2);
    a.offFpart = take(T * a.ntq);
    a.offStat = take(kStatU64 + 1);
    a.stageEll = 0;
    a.offEllVal = a.offEllIdx = a.offEllPair = a.offEllOff = off;
    a.offExp = take(64);
    a.offBar = take(4);
    a.offEg = take(4 * a.ldv);   // the representative start and results
    a.offE = 0;
    exp_consts_init(a.ex);
    const int unionBase = off;
    const int endG = unionBase + ((T * a.ldG + 1) & ~1);
    const int endA = unionBase + 3 * (a.kq * pb.ldP + a.kq);   // three staged chunks
    a.offP = unionBase;
    a.offG = unionBase;
    a.offH = a.offVec = endG;
    a.doubleBuffer = 1;
    a.ntf = 8;
    a.ntExact = pb.K2p / 8;
    a.nbk = pb.nb / 8;
    a.tpw = 0;
    a.smemBytes = (endA > endG ? endA : endG) * 8;
    if (!screen_supported(a.ntExact, a.nbk) || a.smemBytes > 232448 - 1024)
        return -1;
    return 0;
}

static cudaError_t screen_dispatch(const NewtonArgs &a, int grid, cudaStream_t s, int mode, int *occ)
{
    switch (a.ntExact) {
    case 2:
        return screen_run<2, 2>(a, grid, s, mode, occ);
    case 3:
        return screen_run<3, 3>(a, grid, s, mode, occ);
    case 4:
        return screen_run<4, 4>(a, grid, s, mode, occ);
    default:
        return cudaErrorInvalidValue;
    }
}

cudaError_t prepare_screen(const NewtonArgs &a) { return screen_dispatch(a, 0, nullptr, 1, nullptr); }

cudaError_t launch_screen(const NewtonArgs &a, int grid, cudaStream_t stream)
{
    return screen_dispatch(a, grid, stream, 0, nullptr);
}

cudaError_t launch_screen_gate(const int *iters, int first, int count, int *out, cudaStream_t stream)
{
    int blocks = (count + 255) / 256;
    blocks = blocks < 1 ? 1 : (blocks > 1184 ? 1184 : blocks);
    screen_gate_kernel<<<blocks, 256, 0, stream>>>(iters, first, count, out);
    return cudaGetLastError();
}

namespace {
__global__ void __launch_bounds__(1024) order_cells_kernel(const int *list, const int *listCount, int first, int count,
                                                           const int *gateCount, int gateMin, int wholeMax,
                                                           const int *iters, int *out, int *outCount)
{
    __shared__ int hist[32], start[32];
    const bool useList = list != nullptr && (gateCount == nullptr || *gateCount >= gateMin);
    if (!useList && count > wholeMax) {
        if (threadIdx.x == 0)
            *outCount = -1;   // K1 takes the range in cell order
        return;
    }
    const int cnt = useList ? *listCount : count;
    const unsigned lane = threadIdx.x & 31u;
    if (threadIdx.x < 32)
        hist[threadIdx.x] = 0;
    __syncthreads();
    // one shared atomic per bucket per warp (lanes with equal buckets grouped)
    for (int base = 0; base < cnt; base += blockDim.x) {
        const int i = base + (int)threadIdx.x;
        const int c = (i < cnt) ? (useList ? list[i] : first + i) : 0;
        const int b = (i < cnt) ? 31 - min(iters[c], 31) : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, b);
        if (b >= 0 && lane == (unsigned)(__ffs(peers) - 1))
            atomicAdd(&hist[b], __popc(peers));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int k = 0; k < 32; k++) {
            start[k] = acc;
            acc += hist[k];
        }
        *outCount = cnt;
    }
    __syncthreads();
    for (int base = 0; base < cnt; base += blockDim.x) {
        const int i = base + (int)threadIdx.x;
        const int c = (i < cnt) ? (useList ? list[i] : first + i) : 0;
        const int b = (i < cnt) ? 31 - min(iters[c], 31) : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, b);
        const int leader = __ffs(peers) - 1;
        int pos = 0;
        if (b >= 0 && lane == (unsigned)leader)
            pos = atomicAdd(&start[b], __popc(peers));
        pos = __shfl_sync(0xffffffffu, pos, leader);
        if (b >= 0)
            out[pos + __popc(peers & ((1u << lane) - 1u))] = c;
    }
}
}  // namespace

cudaError_t launch_order_cells(const int *list, const int *listCount, int first, int count, const int *gateCount,
                               int gateMin, int wholeMax, const int *iters, int *out, int *outCount,
                               cudaStream_t stream)
{
    order_cells_kernel<<<1, 1024, 0, stream>>>(list, listCount, first, count, gateCount, gateMin, wholeMax, iters, out,
                                               outCount);
    return cudaGetLastError();
}

int screen_ctas_per_sm(const NewtonArgs &a)
{
    int occ = 1;
    if (screen_dispatch(a, 0, nullptr, 2, &occ) != cudaSuccess)
        return 1;
    return occ;
}

}  // namespace clb
