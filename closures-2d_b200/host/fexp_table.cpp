// fexp_table.cpp -- host construction of the fast_exp constants (fexp.cuh):
// 2^(j/32) as head + tail, ln2/32 split for the Cody-Waite reduction, all
// from ln 2 and exp2 in long double.
#include <cmath>

#include "../csrc/fexp.cuh"

namespace clb {

void exp_consts_init(ExpConsts &c)
{
    const long double ln2 = logl(2.0L);
    for (int j = 0; j < 32; j++) {
        long double v = exp2l((long double)j / 32.0L);
        double hi = (double)v;
        c.tab[2 * j] = hi;
        c.tab[2 * j + 1] = (double)(v - (long double)hi);
    }
    const long double L = ln2 / 32.0L;
    c.L1 = (double)(float)L;
    c.L2 = (double)(L - (long double)c.L1);
    c.invL = (double)(32.0L / ln2);
}

}  // namespace clb
