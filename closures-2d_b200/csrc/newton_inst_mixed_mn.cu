// newton_inst_mixed_mn.cu -- Mn instances with the Hessian-only tiles in split TF32 (CL_MIXED).
#include "newton_kernel.cuh"

namespace clb {

bool newton_run_mixed_mn(const NewtonArgs &a, int grid, cudaStream_t s, int mode, int *occ, cudaError_t *err)
{
    if (a.momentType != 0)
        return false;
    if (a.ntExact == 1 && a.nbk == 1) {   // order 1 with the Gaunt table: no Hessian-only tile
        *err = newton_run<1, 1, 0, 1, 1, 1>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 2 && a.nbk == 1) {
        *err = newton_run<1, 2, 0, 2, 1, 1>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 3 && a.nbk == 1) {
        *err = newton_run<1, 3, 0, 3, 1, 1>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 4 && a.nbk == 2) {
        *err = newton_run<1, 4, 0, 4, 2, 1>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 6 && a.nbk == 2) {
        *err = newton_run<1, 6, 0, 6, 2, 1>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 7 && a.nbk == 2) {
        *err = newton_run<1, 7, 0, 7, 2, 1>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 9 && a.nbk == 3) {
        *err = newton_run<1, 9, 0, 9, 3, 1>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 12 && a.nbk == 4) {
        *err = newton_run<1, 12, 0, 12, 4, 1>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 15 && a.nbk == 2) {
        *err = newton_run<1, 15, 0, 15, 2, 1>(a, grid, s, mode, occ);
        return true;
    }
    return false;
}

}  // namespace clb
