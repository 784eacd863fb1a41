// newton_inst_ppn_a.cu -- PPn instances specialised to the tile counts of orders 1-2 and Gaunt order 3.
#include "newton_kernel.cuh"

namespace clb {

bool newton_run_exact_ppn_a(const NewtonArgs &a, int grid, cudaStream_t s, int mode, int *occ, cudaError_t *err)
{
    if (a.momentType != 1)
        return false;
    if (a.ntExact == 2 && a.nbk == 1) {
        *err = newton_run<1, 2, 1, 2, 1>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 3 && a.nbk == 1) {
        *err = newton_run<1, 3, 1, 3, 1>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 4 && a.nbk == 1) {
        *err = newton_run<1, 4, 1, 4, 1>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 6 && a.nbk == 2) {
        *err = newton_run<1, 6, 1, 6, 2>(a, grid, s, mode, occ);
        return true;
    }
    return false;
}

}  // namespace clb
