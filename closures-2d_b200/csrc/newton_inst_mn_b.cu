// newton_inst_mn_b.cu -- Mn instances specialised to the tile counts of Gaunt orders 5-6 and direct orders 3-4.
#include "newton_kernel.cuh"

namespace clb {

bool newton_run_exact_mn_b(const NewtonArgs &a, int grid, cudaStream_t s, int mode, int *occ, cudaError_t *err)
{
    if (a.momentType != 0)
        return false;
    if (a.ntExact == 7 && a.nbk == 2) {
        *err = newton_run<1, 7, 0, 7, 2>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 9 && a.nbk == 3) {
        *err = newton_run<1, 9, 0, 9, 3>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 12 && a.nbk == 4) {
        *err = newton_run<1, 12, 0, 12, 4>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 15 && a.nbk == 2) {
        *err = newton_run<1, 15, 0, 15, 2>(a, grid, s, mode, occ);
        return true;
    }
    return false;
}

}  // namespace clb
