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
    double init(double dx, double dy) override;
    int getNumGhostCells() override { return 2; }
    void update(double dt, double dx, double dy) override;
    void outputData(double time) override;
    int getBoundarySizeX() override;
    int getBoundarySizeY() override;
    void getInnerBoundaries(char *north, char *south, char *east, char *west) override;
    void setOuterBoundaries(char *north, char *south, char *east, char *west) override;
    void duplicateBoundaries() override;

    // Non-aborting forms used by the C ABI wrappers: return CL_OK or an error.
    int tryInit(double dx, double dy, double *maxDt);
    int tryUpdate(double dt, double dx, double dy);
    int tryOutput(double time);

    cl_ctx *context() { return m_ctx; }
    int numMoments() const { return m_n; }
    std::string lastError;
    std::string outDir = ".";

private:
    int m_n = 0;
    double m_maxDt = 0;
    cl_ctx *m_ctx = nullptr;
    cl_options m_opt{};
};

// The main.cpp driver for SOLVER momopt: reads the deck, builds the solver,
// runs the time loop with outputs.  Returns 0 or an error code (message in err).
int run_deck(const char *deckPath, const char *outDir, int maxSteps, std::string &err);

}  // namespace clb
