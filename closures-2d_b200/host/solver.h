// solver.h -- the Solver interface of closures-2d (src/solver.h:15-61),
// kept so a host driver written against the reference's interface drives the
// B200 path unchanged.  Grid bookkeeping fields keep the reference's names
// and meanings; the state of a solver lives on the device.
//
// Below the reference's virtuals sits the layer the C ABI uses: non-aborting
// forms that return CL_OK or an error code with the message in lastError,
// and the device-side pieces a partitioned run needs (state, halo strips,
// one RK stage, the stream the solver works on).
#pragma once
#include <string>

#include "closures_gpu.h"
#include "deck.h"

namespace clb {

class Solver {
public:
    virtual ~Solver();
    // solver.h:15-61; errors print the message and abort, as utils_abort()
    double init(double dx, double dy);
    int getNumGhostCells() { return 2; }
    void update(double dt, double dx, double dy);
    void outputData(double time);
    virtual int getBoundarySizeX();
    virtual int getBoundarySizeY();
    void getInnerBoundaries(char *north, char *south, char *east, char *west);
    void setOuterBoundaries(char *north, char *south, char *east, char *west);
    void duplicateBoundaries();

    // One node: the periodic copy is the whole exchange (comm.cpp:149-154).
    void communicateBoundaries()
    {
        if (c_initCond == INITCOND_PERIODIC)
            duplicateBoundaries();
    }
    // main.cpp:257-372
    void initializeGrid(int numGhostCells, double dx, double dy, double sigma);

    // The device layer.
    virtual int tryInit(double dx, double dy, double *maxDt) = 0;
    virtual int tryUpdate(double dt, double dx, double dy) = 0;
    virtual int tryOutput(double time) = 0;
    // one RK stage (1 or 2) without the ghost copy; asynchronous
    virtual int tryStage(int stage, double dt, double dx, double dy) = 0;
    virtual int numMoments() const = 0;
    virtual int getState(double *moments) = 0;         // all cells, ghosts included
    virtual int setState(const double *moments) = 0;
    virtual int haloCounts(long long counts[4]) = 0;
    virtual int haloPack(double *const bufs[4]) = 0;
    virtual int haloUnpack(double *const bufs[4]) = 0;
    virtual void *stream() = 0;
    virtual int sync() = 0;
    // sides whose ghost strips a halo exchange fills (bit per CL_NORTH..)
    virtual void setExchangedSides(int mask) { (void)mask; }
    // the .pn file of momopt_output.cpp:21-50 / moment_output.cpp:21-56
    int writePn(double time);

    std::string lastError;
    std::string outDir = ".";

    int c_node = 0, c_numNodes = 1;
    int c_nodeX = 0, c_nodeY = 0, c_numNodesX = 1, c_numNodesY = 1;
    int c_numOmpThreads = 1;
    double *c_initialGrid = nullptr, *c_sigmaT = nullptr, *c_sigmaS = nullptr;
    int c_sizeX = 0, c_sizeY = 0;
    double c_ax = 0, c_ay = 0, c_bx = 0, c_by = 0;
    double c_initX = 0, c_initY = 0;
    int c_gX[4] = {0, 0, 0, 0}, c_gY[4] = {0, 0, 0, 0};
    double c_gaussianSigma = 0, c_floor = 0;
    int c_initCond = 0;
    int c_vectorSize = 0;
    InputDeck c_inputDeckReader;

    enum { INITCOND_LINESOURCE, INITCOND_LATTICE, INITCOND_PERIODIC };
};

// main.cpp:45-251 on one node for the deck's SOLVER (momopt or moment):
// reads the deck, builds the solver, runs the time loop with outputs.
// Returns 0 or an error code (message in err).
int run_deck(const char *deckPath, const char *outDir, int maxSteps, std::string &err);

}  // namespace clb
