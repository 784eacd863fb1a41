// solver.cpp -- the host layer shared by the B200 solvers.
//
//   Solver::initializeGrid      main.cpp:257-372 (IC and sigma fields, ghosts)
//   boundaries                  momopt_boundaries.cpp:18-223 and
//                               moment_boundaries.cpp:17-221 (the same strips)
//   writePn                     momopt_output.cpp:21-50, moment_output.cpp:21-56
//   partition                   main.cpp:157-193
//   setup_from_deck, run_deck   main.cpp:45-251 (SOLVER momopt or moment)
//   cl_solver_* / cl_run_deck   the C ABI over a deck-driven solver
// Errors in the Solver-interface methods print a message and abort, as the
// reference's utils_abort() does; the try* forms return the code instead.
#include "solver.h"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <vector>

#include "moment_gpu_solver.h"
#include "momopt_gpu_solver.h"

void clb_set_global_error(const char *msg);

namespace clb {

static const double kPi = 3.14159265358979323846;

static void fail(const std::string &msg)
{
    std::printf("%s\n", msg.c_str());
    std::abort();
}

Solver::~Solver()
{
    std::free(c_initialGrid);
    std::free(c_sigmaT);
    std::free(c_sigmaS);
}

double Solver::init(double dx, double dy)
{
    double maxDt = 0;
    if (tryInit(dx, dy, &maxDt) != CL_OK)
        fail(lastError);
    return maxDt;
}

void Solver::update(double dt, double dx, double dy)
{
    if (tryUpdate(dt, dx, dy) != CL_OK)
        fail(lastError);
}

void Solver::outputData(double time)
{
    if (tryOutput(time) != CL_OK)
        fail(lastError);
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

// momopt_boundaries.cpp:18-26 (the buffer over the full extent with ghosts)
int Solver::getBoundarySizeX() { return numMoments() * 2 * (c_gX[3] - c_gX[0] + 1) * (int)sizeof(double); }
int Solver::getBoundarySizeY() { return numMoments() * 2 * (c_gY[3] - c_gY[0] + 1) * (int)sizeof(double); }

// momopt_boundaries.cpp:32-107 (host packing from a device snapshot)
void Solver::getInnerBoundaries(char *north, char *south, char *east, char *west)
{
    const int NY = c_gY[3] - c_gY[0] + 1, NX = c_gX[3] - c_gX[0] + 1, n = numMoments();
    std::vector<double> m((size_t)NX * NY * n);
    if (getState(m.data()))
        fail(lastError);
    const size_t row = n * sizeof(double);
    const int x1 = c_gX[1], x2 = c_gX[2] + 1 - 2, y1 = c_gY[1], y2 = c_gY[2] + 1 - 2;
    const int wx = c_gX[2] - c_gX[1] + 1, wy = c_gY[2] - c_gY[1] + 1;
    for (int i = c_gX[1]; i <= c_gX[2]; i++)
        for (int j = 0; j < 2; j++) {
            int idx = i - c_gX[1] + j * wx;
            if (north)
                std::memcpy(north + idx * row, &m[((size_t)i * NY + y2 + j) * n], row);
            if (south)
                std::memcpy(south + idx * row, &m[((size_t)i * NY + y1 + j) * n], row);
        }
    for (int i = c_gY[1]; i <= c_gY[2]; i++)
        for (int j = 0; j < 2; j++) {
            int idx = i - c_gY[1] + j * wy;
            if (east)
                std::memcpy(east + idx * row, &m[((size_t)(x2 + j) * NY + i) * n], row);
            if (west)
                std::memcpy(west + idx * row, &m[((size_t)(x1 + j) * NY + i) * n], row);
        }
}

// momopt_boundaries.cpp:113-188
void Solver::setOuterBoundaries(char *north, char *south, char *east, char *west)
{
    const int NY = c_gY[3] - c_gY[0] + 1, NX = c_gX[3] - c_gX[0] + 1, n = numMoments();
    std::vector<double> m((size_t)NX * NY * n);
    if (getState(m.data()))
        fail(lastError);
    const size_t row = n * sizeof(double);
    const int x0 = c_gX[0], x3 = c_gX[2] + 1, y0 = c_gY[0], y3 = c_gY[2] + 1;
    const int wx = c_gX[2] - c_gX[1] + 1, wy = c_gY[2] - c_gY[1] + 1;
    for (int i = c_gX[1]; i <= c_gX[2]; i++)
        for (int j = 0; j < 2; j++) {
            int idx = i - c_gX[1] + j * wx;
            if (north)
                std::memcpy(&m[((size_t)i * NY + y3 + j) * n], north + idx * row, row);
            if (south)
                std::memcpy(&m[((size_t)i * NY + y0 + j) * n], south + idx * row, row);
        }
    for (int i = c_gY[1]; i <= c_gY[2]; i++)
        for (int j = 0; j < 2; j++) {
            int idx = i - c_gY[1] + j * wy;
            if (east)
                std::memcpy(&m[((size_t)(x3 + j) * NY + i) * n], east + idx * row, row);
            if (west)
                std::memcpy(&m[((size_t)(x0 + j) * NY + i) * n], west + idx * row, row);
        }
    if (setState(m.data()))
        fail(lastError);
}

// momopt_boundaries.cpp:190-223; the device steps perform the same copy
// before each stage, this entry point serves external drivers.
void Solver::duplicateBoundaries()
{
    const int NY = c_gY[3] - c_gY[0] + 1, NX = c_gX[3] - c_gX[0] + 1, n = numMoments();
    std::vector<double> m((size_t)NX * NY * n);
    if (getState(m.data()))
        fail(lastError);
    const int x0 = c_gX[0], x1 = c_gX[1], x2 = c_gX[2] + 1 - 2, x3 = c_gX[3] + 1 - 2;
    const int y0 = c_gY[0], y1 = c_gY[1], y2 = c_gY[2] + 1 - 2, y3 = c_gY[3] + 1 - 2;
    auto at = [&](int i, int j) { return &m[((size_t)i * NY + j) * n]; };
    for (int i = 0; i < 2; i++)
        for (int j = c_gY[1]; j <= c_gY[2]; j++) {
            std::memcpy(at(x0 + i, j), at(x2 + i, j), n * sizeof(double));
            std::memcpy(at(x3 + i, j), at(x1 + i, j), n * sizeof(double));
        }
    for (int i = c_gX[1]; i <= c_gX[2]; i++)
        for (int j = 0; j < 2; j++) {
            std::memcpy(at(i, y0 + j), at(i, y2 + j), n * sizeof(double));
            std::memcpy(at(i, y3 + j), at(i, y1 + j), n * sizeof(double));
        }
    if (setState(m.data()))
        fail(lastError);
}

// momopt_output.cpp:21-50, moment_output.cpp:21-56: "=2q4dq" header (sizes of
// this node, the domain bounds, moments) then the interior [x][y][k]
int Solver::writePn(double time)
{
    const int NX = c_gX[3] - c_gX[0] + 1, NY = c_gY[3] - c_gY[0] + 1, n = numMoments();
    std::vector<double> moments((size_t)NX * NY * n);
    int rc = getState(moments.data());
    if (rc)
        return rc;
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
    v = n;
    std::fwrite(&v, sizeof(v), 1, f);
    for (int i = c_gX[1]; i <= c_gX[2]; i++)
        std::fwrite(&moments[((size_t)i * NY + c_gY[1]) * n], sizeof(double), (size_t)(c_gY[2] - c_gY[1] + 1) * n, f);
    std::fclose(f);
    return CL_OK;
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

// Deck keys of main.cpp:69-83 into a new solver for the deck's SOLVER: one
// node (numNodes 1, the partition keys are read but unused, as in the build
// without MPI) or node `node` of the deck's NUM_MPI_PARTITIONS_X x _Y
// partition.
static int setup_from_deck(std::unique_ptr<Solver> &out, const char *deckPath, double &dx, double &dy,
                           double &tFinal, double &outDeltaT, std::string &err, int node = 0, int numNodes = 1)
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
    // main.cpp:93-106
    if (solverType == "momopt")
        out.reset(new MomOptGpuSolver());
    else if (solverType == "moment")
        out.reset(new MomentGpuSolver());
    else {
        err = "Solver type does not exist (the B200 build provides SOLVER momopt and moment)";
        return CL_ERR_ARG;
    }
    Solver &s = *out;
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
    std::unique_ptr<Solver> sp;
    double dx, dy, tFinal, outDeltaT;
    int rc = setup_from_deck(sp, deckPath, dx, dy, tFinal, outDeltaT, err);
    if (rc)
        return rc;
    Solver &s = *sp;
    s.outDir = outDir ? outDir : ".";
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
    std::unique_ptr<clb::Solver> s;
    double dx = 0, dy = 0, tFinal = 0, outDeltaT = 0, maxDt = 0;
    std::string err;
};

static int solver_create(const char *deck_path, const char *out_dir, int node, int num_nodes, cl_solver **out,
                         double *max_dt)
{
    if (!deck_path || !out || num_nodes < 1)
        return CL_ERR_ARG;
    *out = nullptr;
    cl_solver *h = new cl_solver();
    std::string err;
    int rc = clb::setup_from_deck(h->s, deck_path, h->dx, h->dy, h->tFinal, h->outDeltaT, err, node, num_nodes);
    if (rc == CL_OK) {
        h->s->outDir = out_dir ? out_dir : ".";
        rc = h->s->tryInit(h->dx, h->dy, &h->maxDt);
        err = h->s->lastError;
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

// the solver's own message into h->err
static int note(cl_solver *h, int rc)
{
    if (rc)
        h->err = h->s->lastError;
    return rc;
}

extern "C" {

int cl_solver_create(const char *deck_path, const char *out_dir, cl_solver **out, double *max_dt)
{
    return solver_create(deck_path, out_dir, 0, 1, out, max_dt);
}

int cl_solver_create_node(const char *deck_path, const char *out_dir, int node, int num_nodes, cl_solver **out,
                          double *max_dt)
{
    return solver_create(deck_path, out_dir, node, num_nodes, out, max_dt);
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

int cl_solver_node(const cl_solver *h, cl_node *out)
{
    if (!h || !out)
        return CL_ERR_ARG;
    const clb::Solver &s = *h->s;
    out->node = s.c_node;
    out->nodes_x = s.c_numNodesX;
    out->nodes_y = s.c_numNodesY;
    out->node_x = s.c_nodeX;
    out->node_y = s.c_nodeY;
    out->size_x = s.c_sizeX;
    out->size_y = s.c_sizeY;
    out->init_x = s.c_initX;
    out->init_y = s.c_initY;
    return CL_OK;
}

int cl_solver_stage(cl_solver *h, int stage, double dt)
{
    if (!h)
        return CL_ERR_ARG;
    return note(h, h->s->tryStage(stage, dt, h->dx, h->dy));
}

int cl_solver_geometry(cl_solver *h, int *nx, int *ny, int *n, double *dx, double *dy, double *t_final,
                       double *out_delta_t)
{
    if (!h)
        return CL_ERR_ARG;
    if (nx)
        *nx = h->s->c_sizeX;
    if (ny)
        *ny = h->s->c_sizeY;
    if (n)
        *n = h->s->numMoments();
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
    return note(h, h->s->tryUpdate(dt, h->dx, h->dy));
}

int cl_solver_output(cl_solver *h, double time)
{
    if (!h)
        return CL_ERR_ARG;
    return note(h, h->s->tryOutput(time));
}

int cl_solver_get_state(cl_solver *h, double *moments)
{
    if (!h || !moments)
        return CL_ERR_ARG;
    return note(h, h->s->getState(moments));
}

int cl_solver_set_state(cl_solver *h, const double *moments)
{
    if (!h || !moments)
        return CL_ERR_ARG;
    return note(h, h->s->setState(moments));
}

int cl_solver_halo_counts(cl_solver *h, long long counts[4])
{
    if (!h || !counts)
        return CL_ERR_ARG;
    return note(h, h->s->haloCounts(counts));
}

int cl_solver_halo_pack(cl_solver *h, double *const bufs[4])
{
    if (!h || !bufs)
        return CL_ERR_ARG;
    return note(h, h->s->haloPack(bufs));
}

int cl_solver_halo_unpack(cl_solver *h, double *const bufs[4])
{
    if (!h || !bufs)
        return CL_ERR_ARG;
    return note(h, h->s->haloUnpack(bufs));
}

int cl_solver_set_exchanged_sides(cl_solver *h, int mask)
{
    if (!h || mask < 0 || mask > 0xF)
        return CL_ERR_ARG;
    h->s->setExchangedSides(mask);
    return CL_OK;
}

int cl_solver_stream(cl_solver *h, void **stream)
{
    if (!h || !stream)
        return CL_ERR_ARG;
    *stream = h->s->stream();
    return CL_OK;
}

int cl_solver_sync(cl_solver *h)
{
    if (!h)
        return CL_ERR_ARG;
    return note(h, h->s->sync());
}

int cl_solver_kind(const cl_solver *h)
{
    if (!h)
        return CL_ERR_ARG;
    return dynamic_cast<const clb::MomentGpuSolver *>(h->s.get()) ? CL_SOLVER_MOMENT : CL_SOLVER_MOMOPT;
}

cl_ctx *cl_solver_context(cl_solver *h)
{
    if (!h)
        return nullptr;
    auto *m = dynamic_cast<clb::MomOptGpuSolver *>(h->s.get());
    return m ? m->context() : nullptr;
}

cl_pn *cl_solver_pn(cl_solver *h)
{
    if (!h)
        return nullptr;
    auto *m = dynamic_cast<clb::MomentGpuSolver *>(h->s.get());
    return m ? m->context() : nullptr;
}

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
