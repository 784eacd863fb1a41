// solver.h -- the Solver interface of closures-2d (src/solver.h:15-61),
// kept so a host driver written against the reference's interface drives the
// B200 path unchanged.  Grid bookkeeping fields keep the reference's names
// and meanings; the state of MomOptGpuSolver lives on the device.
#pragma once
#include "deck.h"

namespace clb {

class Solver {
public:
    virtual ~Solver() {}
    virtual double init(double dx, double dy) = 0;
    virtual int getNumGhostCells() = 0;
    virtual void update(double dt, double dx, double dy) = 0;
    virtual void outputData(double time) = 0;

    virtual int getBoundarySizeX() = 0;
    virtual int getBoundarySizeY() = 0;
    virtual void getInnerBoundaries(char *north, char *south, char *east, char *west) = 0;
    virtual void setOuterBoundaries(char *north, char *south, char *east, char *west) = 0;
    virtual void duplicateBoundaries() = 0;

    // One node: the periodic copy is the whole exchange (comm.cpp:149-154).
    void communicateBoundaries()
    {
        if (c_initCond == INITCOND_PERIODIC)
            duplicateBoundaries();
    }
    // main.cpp:257-372
    void initializeGrid(int numGhostCells, double dx, double dy, double sigma);

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

}  // namespace clb
