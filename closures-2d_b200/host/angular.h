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

namespace clb {

// Gaunt contraction H_ij = sum_k c_ijk G_k (fobj.cpp:130-144) rearranged for
// 32 lanes: the upper pairs (i <= j, CSR row i*n+j) are sorted by entry count
// and grouped 32 to a chunk; chunk c holds rows eoff[c]..eoff[c+1]-1 of
// [row][lane] entries (eidx, eval), zero padded, each pair's entries in CSR
// order so the sum is formed in the reference's order.  pair[c*32+lane] is
// (i << 8) | j, or 0xFFFF for an empty lane.  Fills caller buffers (no
// allocation); returns the number of rows, or -1 if maxRows is too small.
// Buffer sizes: pair and eoff for ceil(n(n+1)/2 / 32) chunks (+1 for eoff).
int build_gaunt_ell(int n, const int *off, const int *idx, const double *val, unsigned short *pair,
                    unsigned short *eidx, double *eval, int *eoff, int maxRows);
inline int gaunt_ell_chunks(int n) { return (n * (n + 1) / 2 + 31) / 32; }

// Column order of the packed Hessian products p_i p_j (j <= i) used without
// the Gaunt table: the n products with p_0 first (they hold the gradient and
// f, which mixed precision keeps in FP64), then j >= 1 row by row.  Fills
// pairs[n(n+1)/2] with (i << 8) | j.
void product_columns(int n, unsigned short *pairs);

}  // namespace clb
