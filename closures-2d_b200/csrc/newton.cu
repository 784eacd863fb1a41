// newton.cu -- launch planning and instance selection of the persistent
// dual-Newton kernel (device code in newton_kernel.cuh).
#include "newton.cuh"

#include <cfloat>
#include <cmath>

namespace clb {

int plan_newton(NewtonArgs &a)
{
    int nbMax = 8, ldPMax = 0, K2tot = 0, nMax = 1, ellRows = 0, ellChunks = 0;
    for (int p = 0; p < a.nprob; p++) {
        const NewtonProblem &pb = a.prob[p];
        ellRows = pb.ellRows > ellRows ? pb.ellRows : ellRows;
        ellChunks = pb.ellChunks > ellChunks ? pb.ellChunks : ellChunks;
        nbMax = pb.nb > nbMax ? pb.nb : nbMax;
        ldPMax = pb.ldP > ldPMax ? pb.ldP : ldPMax;
        int kt = pb.K2p + (a.momentType == 1 ? pb.nb : 0);
        K2tot = kt > K2tot ? kt : K2tot;
        nMax = pb.n > nMax ? pb.n : nMax;
    }
    if (a.nw == 0)
        a.nw = kWarps;
    if (a.nw != kWarps && a.nw != 4)
        return -1;
    const int nw = a.nw;
    a.T = 4 * nw;   // 16-slot m-tiles x four q-groups of 8 directions = warps
    a.kq = 32;
    a.ntq = a.kq / 8;
    a.ldv = nbMax + 4;
    a.ldE = a.kq + 4;
    a.ldG = K2tot + 4;
    a.ldh = (nMax | 1) + 1;   // even: 16-byte row pairs for the broadcast loads
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
    // the 4-warp shape reads the Gaunt table through L1 so that two CTAs fit
    a.stageEll = (nw == kWarps) ? 1 : 0;   // matches the kernel's compile-time choice
    if (!a.stageEll)
        ellRows = ellChunks = 0;
    a.offEllVal = take(ellRows * 32);
    a.offEllIdx = take((ellRows * 32 + 3) / 4);
    a.offEllPair = take((ellChunks * 32 + 3) / 4);
    a.offEllOff = take((ellChunks + 2) / 2);
    a.offExp = take(64);
    a.offBar = take(4);

    exp_consts_init(a.ex);
    const int unionBase = off;
    const int ntiles2 = (T / 16) * (K2tot / 8);
    a.tpw = (ntiles2 + nw - 1) / nw;
    // fused contractions when every problem's G fits in 16 column tiles
    // (one warp per 16 slots x 8 quadrature rows of a 32-row chunk)
    const int nt2 = K2tot / 8;
    a.ntf = (nt2 <= 16) ? ((nt2 + 7) / 8) * 8 : 0;
    a.ntExact = (a.ntf > 0 && a.nprob == 1) ? nt2 : 0;
    a.nbk = (a.ntf > 0 && a.nprob == 1) ? a.prob[0].nb / 8 : 0;
    if (a.mixed && a.ntExact == 0)
        return -2;
    if (nw != kWarps && (a.ntExact == 0 || a.nprob != 1 || !a.prob[0].paired || a.mixed || a.optType != 0 ||
                         !newton_pair4_supported(a.ntExact, a.nbk)))
        return -1;   // the 4-warp shape: single-order direction-pair Newton only
    // phase-B region
    int offG = unionBase;
    int offH = offG + ((T * a.ldG + 1) & ~1);
    int offVec = offH + ((nw * kMaxN * a.ldh + 1) & ~1);
    int endB = offVec + nw * 64;

    // phase-A region
    const int maxDoubles = (232448 - 1024) / 8;   // opt-in limit minus static shared
    if (a.ntf > 0) {
        const int depth = (nw == kWarps) ? 3 : 2;
        const int endA = unionBase + depth * (a.kq * ldPMax + a.kq);   // staged chunks
        const int end = endA > endB ? endA : endB;
        if (end <= maxDoubles) {
            a.doubleBuffer = 1;
            a.offP = unionBase;
            a.offE = a.offEg = 0;
            a.offG = offG;
            a.offH = offH;
            a.offVec = offVec;
            a.smemBytes = end * 8;
            return 0;
        }
        a.ntf = 0;
        a.ntExact = a.nbk = 0;
        if (a.mixed)
            return -2;
        if (nw != kWarps)
            return -1;
    }
    for (int db = 1; db >= 0; db--) {
        int offP = unionBase;
        int offE = offP + (db ? 2 : 1) * (a.kq * ldPMax + a.kq);
        int offEg = offE + T * a.ldE;
        int endA = offEg + T * a.ldE;
        int end = endA > endB ? endA : endB;
        if (end <= maxDoubles) {
            a.doubleBuffer = db;
            a.offP = offP;
            a.offE = offE;
            a.offEg = offEg;
            a.offG = offG;
            a.offH = offH;
            a.offVec = offVec;
            a.smemBytes = end * 8;
            return 0;
        }
    }
    return -1;
}

// Instance selection: a single-problem launch on the fused path runs the
// kernel specialised to its exact column-tile and k-step counts; mixed
// orders run the fused instance with runtime counts; the rest the general
// contractions.  mode: 0 launch, 1 shared-memory attribute, 2 occupancy.
static cudaError_t run(const NewtonArgs &a, int grid, cudaStream_t stream, int mode, int *occ)
{
    cudaError_t e = cudaErrorInvalidValue;
    if (a.mixed) {
        if (newton_run_mixed_mn(a, grid, stream, mode, occ, &e) || newton_run_mixed_ppn(a, grid, stream, mode, occ, &e))
            return e;
        return cudaErrorInvalidValue;
    }
    if (a.nprob == 1 && a.prob[0].paired) {
        // the direction-pair layout runs only its own fused instances
        if (a.nw == 4)
            return (a.ntf > 0 && a.ntExact > 0 && newton_run_exact_pair4(a, grid, stream, mode, occ, &e))
                       ? e
                       : cudaErrorInvalidValue;
        if (a.ntf > 0 && a.ntExact > 0 && newton_run_exact_pair(a, grid, stream, mode, occ, &e))
            return e;
        return cudaErrorInvalidValue;
    }
    if (a.nw != kWarps)
        return cudaErrorInvalidValue;
    if (a.ntf > 0 && a.ntExact > 0) {
        if (newton_run_exact_mn_a(a, grid, stream, mode, occ, &e) ||
            newton_run_exact_mn_b(a, grid, stream, mode, occ, &e) ||
            newton_run_exact_ppn_a(a, grid, stream, mode, occ, &e) ||
            newton_run_exact_ppn_b(a, grid, stream, mode, occ, &e))
            return e;
    }
    if (newton_run_generic(a, grid, stream, mode, occ, &e))
        return e;
    return cudaErrorInvalidValue;
}

cudaError_t prepare_newton(const NewtonArgs &a) { return run(a, 0, nullptr, 1, nullptr); }

cudaError_t launch_newton(const NewtonArgs &a, int grid, cudaStream_t stream)
{
    return run(a, grid, stream, 0, nullptr);
}

int newton_ctas_per_sm(const NewtonArgs &a)
{
    int occ = 1;
    if (run(a, 0, nullptr, 2, &occ) != cudaSuccess)
        return 1;
    return occ;
}

}  // namespace clb
