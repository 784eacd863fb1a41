// angular.h -- host FP64 angular set-up (momopt_init.cpp:88-259).
#pragma once
#include <vector>

namespace clb {

struct Angular {
    int order = 0, Q = 0, useGaunt = 0;
    int n = 0, n2 = 0, nq = 0;
    std::vector<double> w, xi, eta;   // [nq]
    std::vector<double> p;            // [nq*n2] row-major
    std::vector<int> goff, gidx;      // Gaunt CSR over (i,j), i*n+j
    std::vector<double> gval;
};

void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w);
double sph_plm(int l, int m, double x);
int build_angular(int order, int Q, int useGaunt, Angular &A);

}  // namespace clb
