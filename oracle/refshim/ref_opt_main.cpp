// ref_opt_main.cpp -- runs the reference's own opt() (opt.cpp, fobj.cpp,
// linesearch.cpp, compiled from its sources) on given moment vectors, with
// the reference's own set-up: MomOptSolver::init from input.deck in the
// working directory (quadrature, basis c_spHarm, Gaunt table g_hStruct,
// initFobj) on the deck's grid.  The options are those solveOptimization
// builds (momopt_update.cpp:216-230).  A regularisation ladder that runs out
// makes opt() call utils_abort() (opt.cpp:256-261); the link wraps that call
// so the vector is reported with status -2 and the next one is solved.
//
//   ref_opt <in> <out>
//   in:  int32 count, int32 n, then u [count*n] and alpha [count*n] float64
//   out: u, alpha [count*n] float64, iters [count] int32, r [count] float64,
//        status [count] int32 (0 or -2)
//
// Test infrastructure (a checker); nothing in the product uses it.  The
// private members of MomOptSolver are read from here, so the class is
// declared with them public in this translation unit only (the layout is
// unchanged).
#include <csetjmp>
#include <cstdio>
#include <cstdlib>
#include <vector>

#define private public
#include "momopt/momopt_solver.h"
#undef private
#include "momopt/opt/opt.h"

static jmp_buf g_jump;
extern "C" void __wrap_utils_abort() { longjmp(g_jump, 1); }

int main(int argc, char **argv)
{
    if (argc != 3) {
        fprintf(stderr, "usage: ref_opt <in> <out>\n");
        return 2;
    }
    MomOptSolver *s = new MomOptSolver();
    InputDeckReader &deck = s->c_inputDeckReader;
    deck.readInputDeck("input.deck");
    int nx = 0, ny = 0, initCond = 0;
    double ax = 0, ay = 0, bx = 0, by = 0, sigma = 0, gs = 0, fl = 0;
    deck.getValue("NUM_CELLS_X", &nx);
    deck.getValue("NUM_CELLS_Y", &ny);
    deck.getValue("A_X", &ax);
    deck.getValue("B_X", &bx);
    deck.getValue("A_Y", &ay);
    deck.getValue("B_Y", &by);
    deck.getValue("SIGMA", &sigma);
    deck.getValue("GAUSSIAN_SIGMA", &gs);
    deck.getValue("FLOOR", &fl);
    deck.getValue("INIT_COND", &initCond);
    // the fields main.cpp sets for a single-node run (main.cpp:97-152)
    s->c_gaussianSigma = gs;
    s->c_floor = fl;
    s->c_initCond = initCond;
    s->c_numOmpThreads = 1;
    const double dx = (bx - ax) / nx, dy = (by - ay) / ny;
    s->c_sizeX = nx;
    s->c_sizeY = ny;
    s->c_node = 0;
    s->c_numNodes = 1;
    s->c_nodeX = s->c_nodeY = 0;
    s->c_numNodesX = s->c_numNodesY = 1;
    s->c_ax = ax;
    s->c_ay = ay;
    s->c_bx = bx;
    s->c_by = by;
    s->c_initX = ax;
    s->c_initY = ay;
    s->initializeGrid(s->getNumGhostCells(), dx, dy, sigma);
    s->init(dx, dy);

    FILE *f = fopen(argv[1], "rb");
    int hdr[2] = {0, 0};
    if (!f || fread(hdr, sizeof(int), 2, f) != 2 || hdr[1] != s->c_numMoments) {
        fprintf(stderr, "ref_opt: bad input (n must be %d)\n", s->c_numMoments);
        return 2;
    }
    const int count = hdr[0], n = hdr[1];
    std::vector<double> u((size_t)count * n), al((size_t)count * n), r(count);
    std::vector<int> it(count), st(count);
    if (fread(u.data(), sizeof(double), u.size(), f) != u.size() ||
        fread(al.data(), sizeof(double), al.size(), f) != al.size()) {
        fprintf(stderr, "ref_opt: short input\n");
        return 2;
    }
    fclose(f);

    OPTIONS o;
    o.momentType = s->c_momentType;
    o.maxIter = s->c_maxIter;
    o.maxBfgsIter = s->c_maxIterBfgs;
    o.tolAbs = s->c_tolerance * s->c_tolerance;
    o.tolRel = s->c_tolerance;
    o.condHMax = s->c_condHMax;
    o.condHMaxBfgs = s->c_condHMaxBfgs;
    o.deltaPPn = s->c_deltaPPn;
    o.useGaunt = s->c_useGaunt == 1;
    for (int v = 0; v < count; v++) {
        OUTS outs = {0.0, 0, 0.0};
        if (setjmp(g_jump) == 0) {
            opt(n, s->c_numManyMoments, s->c_numQuadPoints, &u[(size_t)v * n], &al[(size_t)v * n], o,
                s->c_quadWeights, s->c_spHarm, &outs);
            st[v] = 0;
        } else {
            st[v] = -2;
        }
        it[v] = outs.iter;
        r[v] = outs.r;
    }
    f = fopen(argv[2], "wb");
    fwrite(u.data(), sizeof(double), u.size(), f);
    fwrite(al.data(), sizeof(double), al.size(), f);
    fwrite(it.data(), sizeof(int), it.size(), f);
    fwrite(r.data(), sizeof(double), r.size(), f);
    fwrite(st.data(), sizeof(int), st.size(), f);
    fclose(f);
    return 0;
}
