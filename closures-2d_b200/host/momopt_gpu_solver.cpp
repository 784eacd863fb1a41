// momopt_gpu_solver.cpp -- host side of the B200 momopt solver.
//
//   Solver::initializeGrid      main.cpp:257-372 (IC and sigma fields, ghosts)
//   MomOptGpuSolver::init       momopt_init.cpp:51-160 (deck keys, maxDt,
//                               initial moments and alpha) + device upload
//   update                      momopt_update.cpp:283-382 on the device
//   outputData                  momopt_output.cpp:21-77 (.pn / .opt formats)
//   boundaries                  momopt_boundaries.cpp:18-223
//   run_deck                    main.cpp:45-251 for one node
// Errors in the Solver-interface methods print a message and abort, as the
// reference's utils_abort() does; the try* forms return the code instead.
#include "momopt_gpu_solver.h"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

void clb_set_global_error(const char *msg);

namespace clb {

static const double kPi = 3.14159265358979323846;
static const double kReg[CL_NUM_REG] = {0.0, 1e-3, 1e-2, 1e-1, 5e-1};

static void fail(const std::string &msg)
{
    std::printf("%s\n", msg.c_str());
    std::abort();
}

void Solver::initializeGrid(int numGhostCells, double dx, double dy, double sigma)
{
    c_gX[0] = 0;
    c_gX[1] = numGhostCells;
    c_gX[2] = numGhostCells + c_sizeX - 1;
    c_gX[3] = 2 * numGhostCells + c_sizeX - 1;
    c_gY[0] = 0;
    c_gY[1] = numGhostCells;
    c_gY[2] = numGhostCells + c_sizeY - 1;
    c_gY[3] = 2 * numGhostCells + c_sizeY - 1;
    const int NX = c_gX[3] - c_gX[0] + 1, NY = c_gY[3] - c_gY[0] + 1;
    c_initialGrid = (double *)std::malloc(sizeof(double) * NX * NY);
    c_sigmaT = (double *)std::malloc(sizeof(double) * NX * NY);
    c_sigmaS = (double *)std::malloc(sizeof(double) * NX * NY);
    // absorber blocks of the lattice problem (main.cpp:344-354)
    static const double blocks[11][2] = {{2, 2}, {2, 0}, {2, -2}, {1, 1}, {1, -1}, {0, -2},
                                         {-1, 1}, {-1, -1}, {-2, 2}, {-2, 0}, {-2, -2}};
    for (int i = c_gX[0]; i <= c_gX[3]; i++) {
        for (int j = c_gY[0]; j <= c_gY[3]; j++) {
            const int c = i * NY + j;
            const double x = c_initX + (i - c_gX[1]) * dx + dx / 2.0;
            const double y = c_initY + (j - c_gY[1]) * dy + dy / 2.0;
            const bool ghost = i < c_gX[1] || i > c_gX[2] || j < c_gY[1] || j > c_gY[2];
            if (ghost) {
                c_initialGrid[c] = c_floor;
                c_sigmaT[c] = sigma;
                c_sigmaS[c] = sigma;
            } else if (c_initCond == INITCOND_LINESOURCE && c_gaussianSigma == 0.0) {
                c_initialGrid[c] = c_floor;
                if (c_nodeX == (c_numNodesX - 1) / 2 && c_nodeY == (c_numNodesY - 1) / 2) {
                    bool hitX = (c_numNodesX % 2 != 0 && i == (c_sizeX + numGhostCells) / 2) ||
                                (c_numNodesX % 2 == 0 && i == c_gX[2]);
                    bool hitY = (c_numNodesY % 2 != 0 && j == (c_sizeY + numGhostCells) / 2) ||
                                (c_numNodesY % 2 == 0 && j == c_gY[2]);
                    if (hitX && hitY)
                        c_initialGrid[c] = 1.0 / (dx * dy);
                }
                c_sigmaT[c] = sigma;
                c_sigmaS[c] = sigma;
            } else if (c_initCond == INITCOND_LINESOURCE) {
                const double s2 = c_gaussianSigma * c_gaussianSigma;
                const double gauss = 1.0 / (2.0 * kPi * s2) * std::exp(-(x * x + y * y) / (2.0 * s2));
                c_initialGrid[c] = gauss > c_floor ? gauss : c_floor;
                c_sigmaT[c] = sigma;
                c_sigmaS[c] = sigma;
            } else if (c_initCond == INITCOND_LATTICE) {
                c_initialGrid[c] = c_floor;
                c_sigmaT[c] = 1.0;
                c_sigmaS[c] = 1.0;
                for (const auto &b : blocks) {
                    if (std::fabs(x - b[0]) < 0.5 && std::fabs(y - b[1]) < 0.5) {
                        c_sigmaT[c] = 10.0;
                        c_sigmaS[c] = 0.0;
                        break;
                    }
                }
            } else if (c_initCond == INITCOND_PERIODIC) {
                c_sigmaT[c] = sigma;
                c_sigmaS[c] = sigma;
                c_initialGrid[c] = 1 + std::sin(2 * kPi * x) * std::cos(2 * kPi * y);
            }
        }
    }
}

MomOptGpuSolver::~MomOptGpuSolver()
{
    cl_destroy(m_ctx);
    std::free(c_initialGrid);
    std::free(c_sigmaT);
    std::free(c_sigmaS);
}

int MomOptGpuSolver::tryInit(double dx, double dy, double *maxDtOut)
{
    int momentOrder = 0, quadOrder = 0, useGaunt = 0, maxIterBfgs = 0;
    double cfl = 0, condHMaxBfgs = 0, theta = 0;
    const InputDeck &d = c_inputDeckReader;
    // momopt_init.cpp:56-68: every key is required
    struct IntKey {
        const char *k;
        int *v;
    } ik[] = {{"MOMOPT_MOMENT_ORDER", &momentOrder}, {"MOMOPT_QUAD_ORDER", &quadOrder},
              {"MOMOPT_MAX_ITER", &m_opt.max_iter},   {"MOMOPT_MAX_BFGS_ITER", &maxIterBfgs},
              {"MOMOPT_USE_GAUNT", &useGaunt},        {"MOMOPT_MOMENT_TYPE", &m_opt.moment_type},
              {"MOMOPT_OPTIMIZATION_TYPE", &m_opt.opt_type}};
    struct DblKey {
        const char *k;
        double *v;
    } dk[] = {{"MOMOPT_CFL_FACTOR", &cfl},        {"MOMOPT_TOL", &m_opt.tol},
              {"MOMOPT_COND_H_MAX", &m_opt.cond_h_max}, {"MOMOPT_COND_H_MAX_BFGS", &condHMaxBfgs},
              {"MOMOPT_THETA", &theta},           {"MOMOPT_DELTA_PPN", &m_opt.delta_ppn}};
    for (auto &k : ik)
        if (!d.get(k.k, k.v)) {
            lastError = std::string("momopt input error: missing ") + k.k;
            return CL_ERR_ARG;
        }
    for (auto &k : dk)
        if (!d.get(k.k, k.v)) {
            lastError = std::string("momopt input error: missing ") + k.k;
            return CL_ERR_ARG;
        }
    m_opt.max_bfgs_iter = maxIterBfgs;
    m_opt.cond_h_max_bfgs = condHMaxBfgs;
    // optional extensions (unknown to the reference, ignored by its reader)
    if (!d.get("MOMOPT_TOL_GAMMA", &m_opt.tol_gamma))
        m_opt.tol_gamma = 0.0;
    std::string prec;
    m_opt.precision = CL_FP64;
    if (d.get("MOMOPT_GPU_PRECISION", prec) && prec == "mixed")
        m_opt.precision = CL_MIXED;

    m_maxDt = cfl * (2.0 / (2.0 + theta)) * (dx * dy) / (dx + dy);   // momopt_init.cpp:72
    if (maxDtOut)
        *maxDtOut = m_maxDt;

    cl_angular ang;
    int rc = cl_angular_create(momentOrder, quadOrder, useGaunt, &ang);
    if (rc) {
        lastError = cl_global_error();
        return rc;
    }
    m_n = ang.n;
    c_vectorSize = m_n;
    const int NX = c_gX[3] - c_gX[0] + 1, NY = c_gY[3] - c_gY[0] + 1;
    const size_t C = (size_t)NX * NY;
    std::vector<double> moments(C * m_n, 0.0), alpha(C * m_n, 0.0);
    // momopt_init.cpp:120-143
    for (size_t c = 0; c < C; c++) {
        double u0 = c_initialGrid[c] * 2.0 * std::sqrt(kPi);
        moments[c * m_n] = u0;
        if (m_opt.moment_type == CL_MN)
            alpha[c * m_n] = 2.0 * std::sqrt(kPi) * std::log(u0 / (2.0 * std::sqrt(kPi)));
        else if (m_opt.moment_type == CL_PPN)
            alpha[c * m_n] = u0 - 4.0 * m_opt.delta_ppn * kPi / u0;
    }
    cl_grid g;
    g.nx = c_sizeX;
    g.ny = c_sizeY;
    g.ghost = 2;
    g.init_cond = c_initCond;
    g.init_x = c_initX;
    g.init_y = c_initY;
    g.theta = theta;
    rc = cl_create(&g, &m_opt, &ang, c_sigmaT, c_sigmaS, moments.data(), alpha.data(), &m_ctx);
    cl_angular_free(&ang);
    if (rc) {
        lastError = cl_global_error();
        return rc;
    }
    return CL_OK;
}

double MomOptGpuSolver::init(double dx, double dy)
{
    double maxDt = 0;
    if (tryInit(dx, dy, &maxDt) != CL_OK)
        fail(lastError);
    return maxDt;
}

int MomOptGpuSolver::tryUpdate(double dt, double dx, double dy)
{
    int rc = cl_step(m_ctx, dt, dx, dy);
    if (rc)
        lastError = cl_last_error(m_ctx);
    return rc;
}

void MomOptGpuSolver::update(double dt, double dx, double dy)
{
    if (tryUpdate(dt, dx, dy) != CL_OK)
        fail(lastError);
}

int MomOptGpuSolver::tryOutput(double time)
{
    const int NX = c_gX[3] - c_gX[0] + 1, NY = c_gY[3] - c_gY[0] + 1;
    std::vector<double> moments((size_t)NX * NY * m_n);
    int rc = cl_get_state(m_ctx, moments.data(), nullptr);
    if (rc) {
        lastError = cl_last_error(m_ctx);
        return rc;
    }
    char fn[1024];
    std::snprintf(fn, sizeof(fn), "%s/out_%.3f_%d.pn", outDir.c_str(), time, c_node);
    FILE *f = std::fopen(fn, "wb");
    if (!f) {
        lastError = std::string("cannot open ") + fn;
        return CL_ERR_ARG;
    }
    int64_t v = c_gX[2] - c_gX[1] + 1;
    std::fwrite(&v, sizeof(v), 1, f);
    v = c_gY[2] - c_gY[1] + 1;
    std::fwrite(&v, sizeof(v), 1, f);
    std::fwrite(&c_ax, sizeof(double), 1, f);
    std::fwrite(&c_ay, sizeof(double), 1, f);
    std::fwrite(&c_bx, sizeof(double), 1, f);
    std::fwrite(&c_by, sizeof(double), 1, f);
    v = m_n;
    std::fwrite(&v, sizeof(v), 1, f);
    for (int i = c_gX[1]; i <= c_gX[2]; i++)
        std::fwrite(&moments[((size_t)i * NY + c_gY[1]) * m_n], sizeof(double), (size_t)(c_gY[2] - c_gY[1] + 1) * m_n,
                    f);
    std::fclose(f);

    cl_stats st;
    rc = cl_get_stats(m_ctx, &st);
    if (rc) {
        lastError = cl_last_error(m_ctx);
        return rc;
    }
    std::snprintf(fn, sizeof(fn), "%s/out_%.3f_%d.opt", outDir.c_str(), time, c_node);
    f = std::fopen(fn, "w");
    if (!f) {
        lastError = std::string("cannot open ") + fn;
        return CL_ERR_ARG;
    }
    std::fprintf(f, "Max number of iterations: %d\n", st.max_iter);
    std::fprintf(f, "Mean number of iterations: %f\n", st.iter_mean);
    std::fprintf(f, "Number of optimizations: %d\n", (int)st.num_solves);
    std::fprintf(f, "Regularizations Histogram\n");
    for (int i = 0; i < CL_NUM_REG; i++)
        std::fprintf(f, "r = %.3e   %d\n", kReg[i], (int)st.hist_reg[i]);
    std::fclose(f);
    return CL_OK;
}

void MomOptGpuSolver::outputData(double time)
{
    if (tryOutput(time) != CL_OK)
        fail(lastError);
}

// momopt_boundaries.cpp:18-26
int MomOptGpuSolver::getBoundarySizeX() { return m_n * 2 * (c_gX[3] - c_gX[0] + 1) * (int)sizeof(double); }
int MomOptGpuSolver::getBoundarySizeY() { return m_n * 2 * (c_gY[3] - c_gY[0] + 1) * (int)sizeof(double); }

// momopt_boundaries.cpp:32-107 (host packing from a device snapshot)
void MomOptGpuSolver::getInnerBoundaries(char *north, char *south, char *east, char *west)
{
    const int NY = c_gY[3] - c_gY[0] + 1, NX = c_gX[3] - c_gX[0] + 1;
    std::vector<double> m((size_t)NX * NY * m_n);
    if (cl_get_state(m_ctx, m.data(), nullptr))
        fail(cl_last_error(m_ctx));
    const size_t row = m_n * sizeof(double);
    const int x1 = c_gX[1], x2 = c_gX[2] + 1 - 2, y1 = c_gY[1], y2 = c_gY[2] + 1 - 2;
    const int wx = c_gX[2] - c_gX[1] + 1, wy = c_gY[2] - c_gY[1] + 1;
    for (int i = c_gX[1]; i <= c_gX[2]; i++)
        for (int j = 0; j < 2; j++) {
            int idx = i - c_gX[1] + j * wx;
            if (north)
                std::memcpy(north + idx * row, &m[((size_t)i * NY + y2 + j) * m_n], row);
            if (south)
                std::memcpy(south + idx * row, &m[((size_t)i * NY + y1 + j) * m_n], row);
        }
    for (int i = c_gY[1]; i <= c_gY[2]; i++)
        for (int j = 0; j < 2; j++) {
            int idx = i - c_gY[1] + j * wy;
            if (east)
                std::memcpy(east + idx * row, &m[((size_t)(x2 + j) * NY + i) * m_n], row);
            if (west)
                std::memcpy(west + idx * row, &m[((size_t)(x1 + j) * NY + i) * m_n], row);
        }
}

// momopt_boundaries.cpp:113-188
void MomOptGpuSolver::setOuterBoundaries(char *north, char *south, char *east, char *west)
{
    const int NY = c_gY[3] - c_gY[0] + 1, NX = c_gX[3] - c_gX[0] + 1;
    std::vector<double> m((size_t)NX * NY * m_n);
    if (cl_get_state(m_ctx, m.data(), nullptr))
        fail(cl_last_error(m_ctx));
    const size_t row = m_n * sizeof(double);
    const int x0 = c_gX[0], x3 = c_gX[2] + 1, y0 = c_gY[0], y3 = c_gY[2] + 1;
    const int wx = c_gX[2] - c_gX[1] + 1, wy = c_gY[2] - c_gY[1] + 1;
    for (int i = c_gX[1]; i <= c_gX[2]; i++)
        for (int j = 0; j < 2; j++) {
            int idx = i - c_gX[1] + j * wx;
            if (north)
                std::memcpy(&m[((size_t)i * NY + y3 + j) * m_n], north + idx * row, row);
            if (south)
                std::memcpy(&m[((size_t)i * NY + y0 + j) * m_n], south + idx * row, row);
        }
    for (int i = c_gY[1]; i <= c_gY[2]; i++)
        for (int j = 0; j < 2; j++) {
            int idx = i - c_gY[1] + j * wy;
            if (east)
                std::memcpy(&m[((size_t)(x3 + j) * NY + i) * m_n], east + idx * row, row);
            if (west)
                std::memcpy(&m[((size_t)(x0 + j) * NY + i) * m_n], west + idx * row, row);
        }
    if (cl_set_state(m_ctx, m.data(), nullptr))
        fail(cl_last_error(m_ctx));
}

// momopt_boundaries.cpp:190-223; the RK2 graph performs the same copy on the
// device before each stage, this entry point serves external drivers.
void MomOptGpuSolver::duplicateBoundaries()
{
    const int NY = c_gY[3] - c_gY[0] + 1, NX = c_gX[3] - c_gX[0] + 1;
    std::vector<double> m((size_t)NX * NY * m_n);
    if (cl_get_state(m_ctx, m.data(), nullptr))
        fail(cl_last_error(m_ctx));
    const int x0 = c_gX[0], x1 = c_gX[1], x2 = c_gX[2] + 1 - 2, x3 = c_gX[3] + 1 - 2;
    const int y0 = c_gY[0], y1 = c_gY[1], y2 = c_gY[2] + 1 - 2, y3 = c_gY[3] + 1 - 2;
    auto at = [&](int i, int j) { return &m[((size_t)i * NY + j) * m_n]; };
    for (int i = 0; i < 2; i++)
        for (int j = c_gY[1]; j <= c_gY[2]; j++) {
            std::memcpy(at(x0 + i, j), at(x2 + i, j), m_n * sizeof(double));
            std::memcpy(at(x3 + i, j), at(x1 + i, j), m_n * sizeof(double));
        }
    for (int i = c_gX[1]; i <= c_gX[2]; i++)
        for (int j = 0; j < 2; j++) {
            std::memcpy(at(i, y0 + j), at(i, y2 + j), m_n * sizeof(double));
            std::memcpy(at(i, y3 + j), at(i, y1 + j), m_n * sizeof(double));
        }
    if (cl_set_state(m_ctx, m.data(), nullptr))
        fail(cl_last_error(m_ctx));
}

// main.cpp:157-193: the block of `node` in the nodesX x nodesY partition.
static int partition(int numCellsX, int numCellsY, int nodesX, int nodesY, int numNodes, int node, double ax,
              double ay, double bx, double by, cl_node &out, std::string &err)
{
    if (nodesX < 1 || nodesY < 1 || numCellsX < nodesX || numCellsY < nodesY) {
        err = "Init: Number of partitions larger than number of cells.";
        return CL_ERR_ARG;
    }
    if (nodesX * nodesY != numNodes) {
        err = "Init: Number of Nodes != numPartitionsX * numPartitionsY.";
        return CL_ERR_ARG;
    }
    if (node < 0 || node >= numNodes) {
        err = "Init: node index out of range.";
        return CL_ERR_ARG;
    }
    const double dx = (bx - ax) / numCellsX, dy = (by - ay) / numCellsY;
    out.node = node;
    out.nodes_x = nodesX;
    out.nodes_y = nodesY;
    out.node_x = node / nodesY;
    out.node_y = node % nodesY;
    out.size_x = numCellsX / nodesX;
    if (out.node_x < numCellsX % nodesX) {
        out.size_x++;
        out.init_x = ax + dx * out.size_x * out.node_x;
    } else {
        out.init_x = bx - dx * out.size_x * (nodesX - out.node_x);
    }
    out.size_y = numCellsY / nodesY;
    if (out.node_y < numCellsY % nodesY) {
        out.size_y++;
        out.init_y = ay + dy * out.size_y * out.node_y;
    } else {
        out.init_y = by - dy * out.size_y * (nodesY - out.node_y);
    }
    return CL_OK;
}

// Deck keys of main.cpp:69-83 into a solver: one node (numNodes 1, the
// partition keys are read but unused, as in the build without MPI) or node
// `node` of the deck's NUM_MPI_PARTITIONS_X x _Y partition.
static int setup_from_deck(MomOptGpuSolver &s, const char *deckPath, double &dx, double &dy, double &tFinal,
                           double &outDeltaT, std::string &err, int node = 0, int numNodes = 1)
{
    InputDeck deck;
    if (!deck.read(deckPath)) {
        err = std::string("cannot read ") + deckPath;
        return CL_ERR_ARG;
    }
    std::string solverType;
    int numCellsX = 0, numCellsY = 0, nodesX = 0, nodesY = 0, initCond = 0;
    double ax = 0, ay = 0, bx = 0, by = 0, gaussianSigma = 0, initFloor = 0, sigma = 0;
    bool ok = deck.get("SOLVER", solverType) && deck.get("NUM_CELLS_X", &numCellsX) &&
              deck.get("NUM_CELLS_Y", &numCellsY) && deck.get("NUM_MPI_PARTITIONS_X", &nodesX) &&
              deck.get("NUM_MPI_PARTITIONS_Y", &nodesY) && deck.get("A_X", &ax) && deck.get("B_X", &bx) &&
              deck.get("A_Y", &ay) && deck.get("B_Y", &by) && deck.get("T_FINAL", &tFinal) &&
              deck.get("OUT_DELTA_T", &outDeltaT) && deck.get("GAUSSIAN_SIGMA", &gaussianSigma) &&
              deck.get("FLOOR", &initFloor) && deck.get("INIT_COND", &initCond) && deck.get("SIGMA", &sigma);
    if (!ok) {
        err = "main: input error (missing global deck key)";
        return CL_ERR_ARG;
    }
    if (solverType != "momopt") {
        err = "Solver type does not exist (the B200 build provides SOLVER momopt)";
        return CL_ERR_ARG;
    }
    s.c_gaussianSigma = gaussianSigma;
    s.c_floor = initFloor;
    s.c_initCond = initCond;
    s.c_inputDeckReader = deck;
    dx = (bx - ax) / numCellsX;
    dy = (by - ay) / numCellsY;
    s.c_sizeX = numCellsX;
    s.c_sizeY = numCellsY;
    s.c_ax = ax;
    s.c_ay = ay;
    s.c_bx = bx;
    s.c_by = by;
    s.c_initX = ax;
    s.c_initY = ay;
    if (numNodes > 1 || node != 0) {
        cl_node part;
        int rc = partition(numCellsX, numCellsY, nodesX, nodesY, numNodes, node, ax, ay, bx, by, part, err);
        if (rc)
            return rc;
        s.c_node = node;
        s.c_numNodes = numNodes;
        s.c_nodeX = part.node_x;
        s.c_nodeY = part.node_y;
        s.c_numNodesX = nodesX;
        s.c_numNodesY = nodesY;
        s.c_sizeX = part.size_x;
        s.c_sizeY = part.size_y;
        s.c_initX = part.init_x;
        s.c_initY = part.init_y;
    }
    s.initializeGrid(s.getNumGhostCells(), dx, dy, sigma);
    return CL_OK;
}

int run_deck(const char *deckPath, const char *outDir, int maxSteps, std::string &err)
{
    MomOptGpuSolver s;
    s.outDir = outDir ? outDir : ".";
    double dx, dy, tFinal, outDeltaT;
    int rc = setup_from_deck(s, deckPath, dx, dy, tFinal, outDeltaT, err);
    if (rc)
        return rc;
    double maxDt = 0;
    if ((rc = s.tryInit(dx, dy, &maxDt)) != CL_OK) {
        err = s.lastError;
        return rc;
    }
    // main.cpp:204-230
    double t = 0, dt = maxDt;
    if ((rc = s.tryOutput(t)) != CL_OK) {
        err = s.lastError;
        return rc;
    }
    int steps = 0;
    for (double tOut = std::fmin(t + outDeltaT, tFinal); tOut <= tFinal; tOut = std::fmin(tOut + outDeltaT, tFinal)) {
        dt = maxDt;
        while (t < tOut) {
            t += dt;
            if (t > tOut) {
                dt = tOut - (t - dt);
                t = tOut;
            }
            if ((rc = s.tryUpdate(dt, dx, dy)) != CL_OK) {
                err = s.lastError;
                return rc;
            }
            steps++;
            if (maxSteps >= 0 && steps >= maxSteps)
                return CL_OK;
        }
        if ((rc = s.tryOutput(t)) != CL_OK) {
            err = s.lastError;
            return rc;
        }
        if (tOut > tFinal - 1e-12 * tFinal)
            break;
    }
    return CL_OK;
}

}  // namespace clb

// ------------------------------------------------------------ C ABI wrappers
struct cl_solver {
    clb::MomOptGpuSolver s;
    double dx = 0, dy = 0, tFinal = 0, outDeltaT = 0, maxDt = 0;
    std::string err;
};

extern "C" {

int cl_solver_create(const char *deck_path, const char *out_dir, cl_solver **out, double *max_dt)
{
    if (!deck_path || !out)
        return CL_ERR_ARG;
    *out = nullptr;
    cl_solver *h = new cl_solver();
    h->s.outDir = out_dir ? out_dir : ".";
    std::string err;
    int rc = clb::setup_from_deck(h->s, deck_path, h->dx, h->dy, h->tFinal, h->outDeltaT, err);
    if (rc == CL_OK) {
        rc = h->s.tryInit(h->dx, h->dy, &h->maxDt);
        err = h->s.lastError;
    }
    if (rc != CL_OK) {
        clb_set_global_error(err.c_str());
        delete h;
        return rc;
    }
    if (max_dt)
        *max_dt = h->maxDt;
    *out = h;
    return CL_OK;
}

int cl_partition(int num_cells_x, int num_cells_y, int nodes_x, int nodes_y, int num_nodes, int node, double ax,
                 double ay, double bx, double by, cl_node *out)
{
    if (!out)
        return CL_ERR_ARG;
    std::string err;
    int rc = clb::partition(num_cells_x, num_cells_y, nodes_x, nodes_y, num_nodes, node, ax, ay, bx, by, *out, err);
    if (rc)
        clb_set_global_error(err.c_str());
    return rc;
}

int cl_solver_create_node(const char *deck_path, const char *out_dir, int node, int num_nodes, cl_solver **out,
                          double *max_dt)
{
    if (!deck_path || !out || num_nodes < 1)
        return CL_ERR_ARG;
    *out = nullptr;
    cl_solver *h = new cl_solver();
    h->s.outDir = out_dir ? out_dir : ".";
    std::string err;
    int rc = clb::setup_from_deck(h->s, deck_path, h->dx, h->dy, h->tFinal, h->outDeltaT, err, node, num_nodes);
    if (rc == CL_OK) {
        rc = h->s.tryInit(h->dx, h->dy, &h->maxDt);
        err = h->s.lastError;
    }
    if (rc != CL_OK) {
        clb_set_global_error(err.c_str());
        delete h;
        return rc;
    }
    if (max_dt)
        *max_dt = h->maxDt;
    *out = h;
    return CL_OK;
}

int cl_solver_node(const cl_solver *h, cl_node *out)
{
    if (!h || !out)
        return CL_ERR_ARG;
    out->node = h->s.c_node;
    out->nodes_x = h->s.c_numNodesX;
    out->nodes_y = h->s.c_numNodesY;
    out->node_x = h->s.c_nodeX;
    out->node_y = h->s.c_nodeY;
    out->size_x = h->s.c_sizeX;
    out->size_y = h->s.c_sizeY;
    out->init_x = h->s.c_initX;
    out->init_y = h->s.c_initY;
    return CL_OK;
}

int cl_solver_stage(cl_solver *h, int stage, double dt)
{
    if (!h)
        return CL_ERR_ARG;
    int rc = cl_stage(h->s.context(), stage, dt, h->dx, h->dy);
    if (rc)
        h->err = cl_last_error(h->s.context());
    return rc;
}

int cl_solver_geometry(cl_solver *h, int *nx, int *ny, int *n, double *dx, double *dy, double *t_final,
                       double *out_delta_t)
{
    if (!h)
        return CL_ERR_ARG;
    if (nx)
        *nx = h->s.c_sizeX;
    if (ny)
        *ny = h->s.c_sizeY;
    if (n)
        *n = h->s.numMoments();
    if (dx)
        *dx = h->dx;
    if (dy)
        *dy = h->dy;
    if (t_final)
        *t_final = h->tFinal;
    if (out_delta_t)
        *out_delta_t = h->outDeltaT;
    return CL_OK;
}

int cl_solver_update(cl_solver *h, double dt)
{
    if (!h)
        return CL_ERR_ARG;
    int rc = h->s.tryUpdate(dt, h->dx, h->dy);
    if (rc)
        h->err = h->s.lastError;
    return rc;
}

int cl_solver_output(cl_solver *h, double time)
{
    if (!h)
        return CL_ERR_ARG;
    int rc = h->s.tryOutput(time);
    if (rc)
        h->err = h->s.lastError;
    return rc;
}

cl_ctx *cl_solver_context(cl_solver *h) { return h ? h->s.context() : nullptr; }

const char *cl_solver_last_error(const cl_solver *h) { return h ? h->err.c_str() : cl_global_error(); }

void cl_solver_destroy(cl_solver *h) { delete h; }

int cl_run_deck(const char *deck_path, const char *out_dir, int max_steps)
{
    std::string err;
    int rc = clb::run_deck(deck_path, out_dir, max_steps, err);
    if (rc)
        clb_set_global_error(err.c_str());
    return rc;
}

}  // extern "C"
