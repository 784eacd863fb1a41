// newton_inst_mixed_ppn.cu -- PPn instances with the Hessian tiles in split TF32 (CL_MIXED).
#include "newton_kernel.cuh"

namespace clb {

bool newton_run_mixed_ppn(const NewtonArgs &a, int grid, cudaStream_t s, int mode, int *occ, cudaError_t *err)
{
    if (a.momentType != 1)
        return false;
    if (a.ntExact == 2 && a.nbk == 1) {
        *err = newton_run<1, 2, 1, 2, 1, 1>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 3 && a.nbk == 1) {
        *err = newton_run<1, 3, 1, 3, 1, 1>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 4 && a.nbk == 1) {
        *err = newton_run<1, 4, 1, 4, 1, 1>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 6 && a.nbk == 2) {
        *err = newton_run<1, 6, 1, 6, 2, 1>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 8 && a.nbk == 2) {
        *err = newton_run<1, 8, 1, 8, 2, 1>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 9 && a.nbk == 2) {
        *err = newton_run<1, 9, 1, 9, 2, 1>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 12 && a.nbk == 3) {
        *err = newton_run<1, 12, 1, 12, 3, 1>(a, grid, s, mode, occ);
        return true;
    }
    if (a.ntExact == 16 && a.nbk == 4) {
        *err = newton_run<1, 16, 1, 16, 4, 1>(a, grid, s, mode, occ);
        return true;
    }
    return false;
}

}  // namespace clb
