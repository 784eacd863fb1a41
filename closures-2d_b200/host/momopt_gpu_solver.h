// momopt_gpu_solver.h -- MomOptSolver (src/momopt/momopt_solver.h:15-81)
// on the B200: the deck keys, initial state and output files are the
// reference's; update() runs the RK2 step on the device through the C ABI.
#pragma once
#include <string>

#include "closures_gpu.h"
#include "solver.h"

namespace clb {

class MomOptGpuSolver : public Solver {
public:
    ~MomOptGpuSolver() override;

    int tryInit(double dx, double dy, double *maxDt) override;
    int tryUpdate(double dt, double dx, double dy) override;
    int tryOutput(double time) override;
    int tryStage(int stage, double dt, double dx, double dy) override;
    int numMoments() const override { return m_n; }
    int getState(double *moments) override;
    int setState(const double *moments) override;
    int haloCounts(long long counts[4]) override;
    int haloPack(double *const bufs[4]) override;
    int haloUnpack(double *const bufs[4]) override;
    void *stream() override;
    int sync() override;

    cl_ctx *context() { return m_ctx; }

private:
    int ctxError(int rc);
    int m_n = 0;
    double m_maxDt = 0;
    cl_ctx *m_ctx = nullptr;
    cl_options m_opt{};
    bool m_tune = true;   // MOMOPT_GPU_TUNE (default 1): cl_tune once the state is on the device
};

}  // namespace clb
