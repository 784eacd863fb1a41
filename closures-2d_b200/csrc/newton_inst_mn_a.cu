// newton_inst_mn_a.cu -- Mn instances specialised to the tile counts of orders 1-2 and Gaunt orders 3-4.
#include "newton_kernel.cuh"

namespace clb {

bool newton_run_exact_mn_a(const NewtonArgs &a, int grid, cudaStream_t s, int mode, int *occ, cudaError_t *err)
{
    if (a.momentType != 0)
        return false;
    if (a.ntExact == 1 && a.nbk == 1) {
        *err = newton_run<1, 1, 0, 1, 1>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 2 && a.nbk == 1) {
        *err = newton_run<1, 2, 0, 2, 1>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 3 && a.nbk == 1) {
        *err = newton_run<1, 3, 0, 3, 1>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 4 && a.nbk == 2) {
        *err = newton_run<1, 4, 0, 4, 2>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 6 && a.nbk == 2) {
        *err = newton_run<1, 6, 0, 6, 2>(a, grid, s, mode, occ);
        return true;
    }
    return false;
}

}  // namespace clb
