// newton_inst_ppn_b.cu -- PPn instances specialised to the tile counts of Gaunt orders 4-6 and direct order 3.
#include "newton_kernel.cuh"

namespace clb {

bool newton_run_exact_ppn_b(const NewtonArgs &a, int grid, cudaStream_t s, int mode, int *occ, cudaError_t *err)
{
    if (a.momentType != 1)
        return false;
    if (a.ntExact == 8 && a.nbk == 2) {
        *err = newton_run<1, 8, 1, 8, 2>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 9 && a.nbk == 2) {
        *err = newton_run<1, 9, 1, 9, 2>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 12 && a.nbk == 3) {
        *err = newton_run<1, 12, 1, 12, 3>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 16 && a.nbk == 4) {
        *err = newton_run<1, 16, 1, 16, 4>(a, grid, s, mode, occ);
        return true;
    }
    return false;
}

}  // namespace clb
