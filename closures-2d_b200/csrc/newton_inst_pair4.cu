// newton_inst_pair4.cu -- the direction-pair Mn instances in the 4-warp launch
// shape (16 slots per CTA, two staged chunks, two CTAs per SM), for the
// Gaunt orders 3-6 and the direct order 4: the larger contractions, where
// overlapping one CTA's per-slot Newton logic with the other's contractions
// can pay.  The autotuner chooses between this shape and the 8-warp one.
#include "newton_kernel.cuh"

namespace clb {

namespace {
constexpr int kPair4Shapes[][2] = {{4, 2}, {7, 3}, {9, 4}, {13, 4}, {16, 3}};
}  // namespace

bool newton_pair4_supported(int nt, int nbk)
{
    for (const auto &s : kPair4Shapes)
        if (s[0] == nt && s[1] == nbk)
            return true;
    return false;
}

bool newton_run_exact_pair4(const NewtonArgs &a, int grid, cudaStream_t s, int mode, int *occ, cudaError_t *err)
{
    if (a.momentType != 0 || a.mixed || a.nw != 4)
        return false;
#define CLB_PAIR4(NT_, NBK_)                                                                    \
    if (a.ntExact == NT_ && a.nbk == NBK_) {                                                   \
        *err = newton_run<1, NT_, 0, NT_, NBK_, 0, 1, 4>(a, grid, s, mode, occ);               \
        return true;                                                                           \
    }
    CLB_PAIR4(4, 2)
    CLB_PAIR4(7, 3)
    CLB_PAIR4(9, 4)
    CLB_PAIR4(13, 4)
    CLB_PAIR4(16, 3)
#undef CLB_PAIR4
    return false;
}

}  // namespace clb
