// newton_inst_pair.cu -- Mn instances of the direction-pair layout, one per
// (column tiles, k-steps) of the Gaunt orders 1-6 and the direct orders 1-4.
#include "newton_kernel.cuh"

namespace clb {

namespace {
// (tiles, k-steps) of the paired layouts: Gaunt N = 1..6 -> (2,2) (3,2)
// (4,2) (7,3) (9,4) (13,4); direct N = 3, 4 -> (7,2) (16,3) (N = 1, 2 as Gaunt)
constexpr int kPairShapes[][2] = {{2, 2}, {3, 2}, {4, 2}, {7, 2}, {7, 3}, {9, 4}, {13, 4}, {16, 3}};
}  // namespace

bool newton_pair_supported(int nt, int nbk)
{
    for (const auto &s : kPairShapes)
        if (s[0] == nt && s[1] == nbk)
            return true;
    return false;
}

bool newton_run_exact_pair(const NewtonArgs &a, int grid, cudaStream_t s, int mode, int *occ, cudaError_t *err)
{
    if (a.momentType != 0 || a.mixed)
        return false;
#define CLB_PAIR(NT_, NBK_)                                                                     \
    if (a.ntExact == NT_ && a.nbk == NBK_) {                                                   \
        *err = newton_run<1, NT_, 0, NT_, NBK_, 0, 1>(a, grid, s, mode, occ);                  \
        return true;                                                                           \
    }
    CLB_PAIR(2, 2)
    CLB_PAIR(3, 2)
    CLB_PAIR(4, 2)
    CLB_PAIR(7, 2)
    CLB_PAIR(7, 3)
    CLB_PAIR(9, 4)
    CLB_PAIR(13, 4)
    CLB_PAIR(16, 3)
#undef CLB_PAIR
    return false;
}

}  // namespace clb
