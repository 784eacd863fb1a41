// newton_inst_generic.cu -- kernel instances with runtime tile counts: mixed-order launches on the fused path and the general contractions.
#include "newton_kernel.cuh"

namespace clb {

bool newton_run_generic(const NewtonArgs &a, int grid, cudaStream_t s, int mode, int *occ, cudaError_t *err)
{
    if (a.ntf > 0) {
        const bool ppn = a.momentType == 1;
        if (a.ntf <= 8)
            *err = ppn ? newton_run<1, 8, 1, 0, 0>(a, grid, s, mode, occ) : newton_run<1, 8, 0, 0, 0>(a, grid, s, mode, occ);
        else
            *err = ppn ? newton_run<1, 16, 1, 0, 0>(a, grid, s, mode, occ)
                       : newton_run<1, 16, 0, 0, 0>(a, grid, s, mode, occ);
        return true;
    }
    if (a.tpw <= 1)
        *err = newton_run<1, 0, 0, 0, 0>(a, grid, s, mode, occ);
    else if (a.tpw <= 2)
        *err = newton_run<2, 0, 0, 0, 0>(a, grid, s, mode, occ);
    else if (a.tpw <= 4)
        *err = newton_run<4, 0, 0, 0, 0>(a, grid, s, mode, occ);
    else if (a.tpw <= 8)
        *err = newton_run<8, 0, 0, 0, 0>(a, grid, s, mode, occ);
    else if (a.tpw <= 16)
        *err = newton_run<16, 0, 0, 0, 0>(a, grid, s, mode, occ);
    else
        return false;
    return true;
}

}  // namespace clb
