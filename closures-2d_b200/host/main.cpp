// main.cpp -- drop-in driver for SOLVER momopt and SOLVER moment on one B200.
//
// Mirrors src/main.cpp:45-251 for one node: reads input.deck from the working
// directory (or argv[1]), initialises the grid and the solver, runs the
// fixed-dt time loop with outputs out_<t>_0.{pn,opt}.  Errors print the
// message and abort, as utils_abort() does.
#include <cstdio>
#include <cstdlib>
#include <string>

#include "closures_gpu.h"
#include "solver.h"

int main(int argc, char **argv)
{
    const char *deck = argc > 1 ? argv[1] : "input.deck";
    const char *dir = argc > 2 ? argv[2] : ".";
    int maxSteps = argc > 3 ? std::atoi(argv[3]) : -1;
    std::string err;
    int rc = clb::run_deck(deck, dir, maxSteps, err);
    if (rc != 0) {
        std::printf("%s\n", err.empty() ? cl_error_text(rc) : err.c_str());
        std::fflush(stdout);   // abort() does not flush
        std::abort();
    }
    return 0;
}
