// fexp.cuh -- table-driven FP64 exponential for the evaluation kernels.
//
// Method: P. T. P. Tang, "Table-driven implementation of the exponential
// function in IEEE floating-point arithmetic", ACM TOMS 15(2), 1989, with a
// 32-entry table.  x = (32 m + j) ln2/32 + r with |r| <= ln2/64, so
//   exp(x) = 2^m * 2^(j/32) * exp(r),
// 2^(j/32) held as a head+tail pair (T_hi + T_lo), exp(r) - 1 by its Taylor
// polynomial of degree 6 (truncation below 4e-18 relative on |r| <= ln2/64),
// and the reduction done in two FMA steps with ln2/32 split into a head with
// 24 significant bits (exact products for |N| < 2^29) and a tail.  Inputs
// outside [-700, 700] go to the CUDA library exp.  The constants are built on
// the host from ln 2 and 2^(j/32) (exp_table_init); the table lives in shared
// memory so lanes with different j read it without serialisation.
#pragma once
#include <cuda_runtime.h>

namespace clb {

struct ExpConsts {
    double tab[64];        // tab[2j] = T_hi(j), tab[2j+1] = T_lo(j)
    double invL;           // 32 / ln 2
    double L1, L2;         // ln2/32 = L1 + L2, L1 with 24 significant bits
};

// Host: fills the constants (long double arithmetic for the table tails).
void exp_consts_init(ExpConsts &c);

// Table method for |x| <= 700 (no range check).
__device__ __forceinline__ double fast_exp_core(double x, const double *__restrict__ tab, double invL,
                                                double L1, double L2)
{
    const double shifter = 6755399441055744.0;      // 1.5 * 2^52: rounds to integer in the low bits
    double t = fma(x, invL, shifter);
    long long N = __double_as_longlong(t) - __double_as_longlong(shifter);
    double Nd = t - shifter;
    double r = fma(-Nd, L1, x);
    r = fma(-Nd, L2, r);
    int j = (int)(N & 31);
    long long m = N >> 5;
    // exp(r) - 1 = r (1 + r/2 + r^2/6 + r^3/24 + r^4/120 + r^5/720)
    double q = fma(r, 1.0 / 720.0, 1.0 / 120.0);
    q = fma(r, q, 1.0 / 24.0);
    q = fma(r, q, 1.0 / 6.0);
    q = fma(r, q, 0.5);
    q = fma(r, q, 1.0);
    double p = r * q;
    double hi = tab[2 * j], lo = tab[2 * j + 1];
    double y = hi + fma(hi, p, lo);
    // multiply by 2^m (|m| <= 1011 here, so the scale is a normal number)
    double scale = __longlong_as_double((m + 1023) << 52);
    return y * scale;
}

__device__ __forceinline__ double fast_exp(double x, const double *__restrict__ tab, double invL, double L1,
                                           double L2)
{
    if (!(fabs(x) <= 700.0))
        return exp(x);
    return fast_exp_core(x, tab, invL, L1, L2);
}

// K exponentials as straight-line code (independent evaluations interleave;
// a range branch per value would serialise them), then one branch that
// sends inputs outside [-700, 700] and NaN to the CUDA library exp.
template <int K>
__device__ __forceinline__ void fast_exp_n(double (&y)[K], const double (&x)[K], const double *__restrict__ tab,
                                           double invL, double L1, double L2)
{
    bool out = false;
#pragma unroll
    for (int h = 0; h < K; h++) {
        y[h] = fast_exp_core(fmin(fmax(x[h], -700.0), 700.0), tab, invL, L1, L2);
        out |= !(fabs(x[h]) <= 700.0);
    }
    if (out) {
#pragma unroll
        for (int h = 0; h < K; h++)
            if (!(fabs(x[h]) <= 700.0))
                y[h] = exp(x[h]);
    }
}

}  // namespace clb
