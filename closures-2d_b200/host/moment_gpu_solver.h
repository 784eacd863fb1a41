// moment_gpu_solver.h -- MomentSolver (src/moment/moment_solver.h:13-51), the
// linear Pn / FPn solver, on the B200: the deck keys, set-up and output file
// are the reference's; the RK2 step runs on the device (cl_pn_*).
#pragma once
#include <string>

#include "closures_gpu.h"
#include "solver.h"

namespace clb {

class MomentGpuSolver : public Solver {
public:
    ~MomentGpuSolver() override;

    int tryInit(double dx, double dy, double *maxDt) override;
    int tryUpdate(double dt, double dx, double dy) override;
    int tryOutput(double time) override;
    int tryStage(int stage, double dt, double dx, double dy) override;
    int numMoments() const override { return m_n; }
    // moment_boundaries.cpp:17-26: the buffer over the interior extent
    int getBoundarySizeX() override { return m_n * 2 * (c_gX[2] - c_gX[1] + 1) * (int)sizeof(double); }
    int getBoundarySizeY() override { return m_n * 2 * (c_gY[2] - c_gY[1] + 1) * (int)sizeof(double); }
    int getState(double *moments) override;
    int setState(const double *moments) override;
    int haloCounts(long long counts[4]) override;
    int haloPack(double *const bufs[4]) override;
    int haloUnpack(double *const bufs[4]) override;
    void *stream() override;
    int sync() override;
    void setExchangedSides(int mask) override;

    cl_pn *context() { return m_pn; }

private:
    int pnError(int rc);
    int m_n = 0;
    cl_pn *m_pn = nullptr;
};

}  // namespace clb
