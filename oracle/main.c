/*
 * main.c -- command-line driver of the oracle (TEST INFRASTRUCTURE ONLY).
 *
 * Usage: oracle_momopt [deck-path [out-dir [max-steps]]]
 * Reads input.deck with the reference's key semantics, runs the time loop of
 * main.cpp:204-230 for SOLVER momopt and writes out_<t>_0.{pn,opt} like
 * momopt_output.cpp.  Errors abort like utils_abort() (utils.cpp:25-33).
 */
#include "oracle.h"
#include <stdio.h>
#include <stdlib.h>

int main(int argc, char **argv)
{
    const char *deck = argc > 1 ? argv[1] : "input.deck";
    const char *dir = argc > 2 ? argv[2] : ".";
    int maxSteps = argc > 3 ? atoi(argv[3]) : -1;
    orc_deck d;
    if (orc_deck_read(deck, &d) != ORC_OK) {
        printf("oracle: input error in %s\n", deck);
        abort();
    }
    orc_solver s;
    if (orc_solver_create(&d, &s) != ORC_OK) {
        printf("oracle: unsupported configuration\n");
        abort();
    }
    int st = orc_solver_run(&s, dir, maxSteps);
    if (st == ORC_ERR_U0) {
        printf("u[0] < 0\n");
        abort();
    } else if (st == ORC_ERR_MAXREG) {
        printf("Max regularization achieved.\n");
        abort();
    } else if (st != ORC_OK) {
        printf("oracle: error %d\n", st);
        abort();
    }
    orc_solver_free(&s);
    return 0;
}
