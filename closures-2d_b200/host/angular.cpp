// angular.cpp -- host FP64 angular set-up of the Mn/PPn path.
//
// Replaces MomOptSolver::init's quadrature/basis/Gaunt block
// (src/momopt/momopt_init.cpp:88-259) and utils_getGaussianWeightsAndNodes
// (src/utils.cpp:55-60), which the reference takes from GSL:
//   * Gauss-Legendre nodes on [-1,1] in ascending order (what GSL's
//     glfixed_point reports), by Newton's method on the Legendre recurrence;
//   * mu = first Q/2 nodes, phi_k = (k+1/2) pi / Q for 2Q azimuths, weights
//     2 pi / Q * w_GL (sum 4 pi), q = 2*q1*Q + q2 (momopt_init.cpp:176-190);
//   * z-even real spherical harmonics up to degree N (2N with the Gaunt
//     table), ordered l = 0.., m = -l..l with (l+m) even; sqrt(2) sin(m phi)
//     P_l^|m| for m<0, sqrt(2) cos(m phi) P_l^m for m>0, normalised
//     associated Legendre with the Condon-Shortley phase
//     (momopt_init.cpp:196-215);
//   * Gaunt table: least-squares coefficients of p_i p_j on the extended
//     basis by Householder QR, entries with |beta| > 10e-10 kept
//     (momopt_init.cpp:221-259).
#include "angular.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace clb {

static const double kPi = 3.14159265358979323846;

void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w)
{
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int i = 0; i < (n + 1) / 2; i++) {
        // i-th largest root; Tricomi-style initial guess.
        double z = std::cos(kPi * (4.0 * i + 3.0) / (4.0 * n + 2.0));
        double dp = 1.0;
        for (int it = 0; it < 64; it++) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; k++) {
                double pk = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = pk;
            }
            if (n == 1) {
                p0 = 1.0;
                p1 = z;
            }
            dp = n * (p0 - z * p1) / (1.0 - z * z);
            double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-17 && it > 1)
                break;
        }
        double p0 = 1.0, p1 = z;
        for (int k = 2; k <= n; k++) {
            double pk = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
            p0 = p1;
            p1 = pk;
        }
        dp = n * (p0 - z * p1) / (1.0 - z * z);
        double wi = 2.0 / ((1.0 - z * z) * dp * dp);
        x[n - 1 - i] = z;
        x[i] = -z;
        w[n - 1 - i] = wi;
        w[i] = wi;
    }
    if (n % 2)
        x[n / 2] = 0.0;
}

// Normalised associated Legendre function with Condon-Shortley phase:
// sqrt((2l+1)/(4 pi) (l-m)!/(l+m)!) P_l^m(x), 0 <= m <= l.
double sph_plm(int l, int m, double x)
{
    double somx2 = std::sqrt((1.0 - x) * (1.0 + x));
    double pmm = 1.0 / std::sqrt(4.0 * kPi);
    for (int k = 1; k <= m; k++)
        pmm = -pmm * somx2 * std::sqrt((2.0 * k + 1.0) / (2.0 * k));
    if (l == m)
        return pmm;
    double pmmp1 = std::sqrt(2.0 * m + 3.0) * x * pmm;
    if (l == m + 1)
        return pmmp1;
    double prev = pmm, cur = pmmp1;
    for (int ll = m + 2; ll <= l; ll++) {
        double l2 = (double)ll * ll, m2 = (double)m * m;
        double a = std::sqrt((4.0 * l2 - 1.0) / (l2 - m2));
        double lm1 = ll - 1.0;
        double b = std::sqrt((lm1 * lm1 - m2) / (4.0 * lm1 * lm1 - 1.0));
        double next = a * (x * cur - b * prev);
        prev = cur;
        cur = next;
    }
    return cur;
}

namespace {
// Householder QR least squares on a column-major copy.
struct LeastSquares {
    int rows, cols;
    std::vector<double> a;      // column-major rows x cols (R above, v below)
    std::vector<double> tau;
    LeastSquares(int r, int c, const double *rowmajor, int ld) : rows(r), cols(c), a((size_t)r * c), tau(c)
    {
        for (int i = 0; i < r; i++)
            for (int j = 0; j < c; j++)
                a[(size_t)j * r + i] = rowmajor[(size_t)i * ld + j];
        for (int k = 0; k < c; k++) {
            double *col = &a[(size_t)k * r];
            double nrm = 0.0;
            for (int i = k; i < r; i++)
                nrm += col[i] * col[i];
            nrm = std::sqrt(nrm);
            if (nrm == 0.0) {
                tau[k] = 0.0;
                continue;
            }
            double alpha = col[k];
            double beta = alpha >= 0 ? -nrm : nrm;
            double scale = 1.0 / (alpha - beta);
            for (int i = k + 1; i < r; i++)
                col[i] *= scale;
            tau[k] = (beta - alpha) / beta;
            col[k] = beta;
            for (int j = k + 1; j < c; j++) {
                double *cj = &a[(size_t)j * r];
                double s = cj[k];
                for (int i = k + 1; i < r; i++)
                    s += col[i] * cj[i];
                s *= tau[k];
                cj[k] -= s;
                for (int i = k + 1; i < r; i++)
                    cj[i] -= s * col[i];
            }
        }
    }
    void solve(std::vector<double> &b, std::vector<double> &x) const
    {
        for (int k = 0; k < cols; k++) {
            const double *col = &a[(size_t)k * rows];
            double s = b[k];
            for (int i = k + 1; i < rows; i++)
                s += col[i] * b[i];
            s *= tau[k];
            b[k] -= s;
            for (int i = k + 1; i < rows; i++)
                b[i] -= s * col[i];
        }
        x.assign(cols, 0.0);
        for (int k = cols - 1; k >= 0; k--) {
            double s = b[k];
            for (int j = k + 1; j < cols; j++)
                s -= a[(size_t)j * rows + k] * x[j];
            x[k] = s / a[(size_t)k * rows + k];
        }
    }
};
}  // namespace

int build_angular(int order, int Q, int useGaunt, Angular &A)
{
    // orders above 6 (more than 32 moments) serve the linear moment solver,
    // which has no Gaunt table; the entropy-closure kernels take n <= 32
    if (order < 1 || order > (useGaunt ? 6 : 9) || Q < 2 || Q % 2 != 0)
        return -1;
    A.order = order;
    A.Q = Q;
    A.useGaunt = useGaunt ? 1 : 0;
    A.nq = Q * Q;
    A.n = (order + 1) * (order + 2) / 2;
    A.n2 = A.useGaunt ? (2 * order + 1) * (2 * order + 2) / 2 : A.n;
    const int nq = A.nq, n2 = A.n2;
    A.w.assign(nq, 0.0);
    A.xi.assign(nq, 0.0);
    A.eta.assign(nq, 0.0);
    A.p.assign((size_t)nq * n2, 0.0);
    std::vector<double> glx, glw;
    gauss_legendre(Q, glx, glw);
    const int degMax = A.useGaunt ? 2 * order : order;
    for (int q1 = 0; q1 < Q / 2; q1++) {
        const double mu = glx[q1];
        const double wq = 2.0 * kPi / Q * glw[q1];
        const double st = std::sqrt(1.0 - mu * mu);
        for (int q2 = 0; q2 < 2 * Q; q2++) {
            const double phi = (q2 + 0.5) * kPi / Q;
            const int q = 2 * q1 * Q + q2;
            A.w[q] = wq;
            A.xi[q] = st * std::cos(phi);
            A.eta[q] = st * std::sin(phi);
            double *row = &A.p[(size_t)q * n2];
            int k = 0;
            for (int l = 0; l <= degMax; l++) {
                for (int m = -l; m <= l; m++) {
                    if (((m + l) & 1) != 0)
                        continue;
                    double v;
                    if (m < 0)
                        v = std::sqrt(2.0) * std::sin(m * phi) * sph_plm(l, -m, mu);
                    else if (m > 0)
                        v = std::sqrt(2.0) * std::cos(m * phi) * sph_plm(l, m, mu);
                    else
                        v = sph_plm(l, 0, mu);
                    row[k++] = v;
                }
            }
        }
    }
    A.goff.clear();
    A.gidx.clear();
    A.gval.clear();
    if (A.useGaunt) {
        const int n = A.n;
        LeastSquares ls(nq, n2, A.p.data(), n2);
        std::vector<double> b(nq), beta;
        A.goff.push_back(0);
        for (int i = 0; i < n; i++) {
            for (int j = 0; j < n; j++) {
                for (int q = 0; q < nq; q++)
                    b[q] = A.p[(size_t)q * n2 + i] * A.p[(size_t)q * n2 + j];
                ls.solve(b, beta);
                for (int k = 0; k < n2; k++) {
                    if (std::fabs(beta[k]) > 10e-10) {
                        A.gidx.push_back(k);
                        A.gval.push_back(beta[k]);
                    }
                }
                A.goff.push_back((int)A.gidx.size());
            }
        }
    }
    return 0;
}

}  // namespace clb

namespace clb {

void product_columns(int n, unsigned short *pairs)
{
    int c = 0;
    for (int i = 0; i < n; i++)
        pairs[c++] = (unsigned short)(i << 8);
    for (int i = 1; i < n; i++)
        for (int j = 1; j <= i; j++)
            pairs[c++] = (unsigned short)((i << 8) | j);
}

int build_gaunt_ell(int n, const int *off, const int *idx, const double *val, unsigned short *pair,
                    unsigned short *eidx, double *eval, int *eoff, int maxRows)
{
    const int np = n * (n + 1) / 2;
    int pi[528], pj[528], pc[528];   // n <= 32
    if (np > 528)
        return -1;
    int m = 0;
    for (int i = 0; i < n; i++)
        for (int j = i; j < n; j++) {
            pi[m] = i;
            pj[m] = j;
            pc[m] = off[i * n + j + 1] - off[i * n + j];
            m++;
        }
    // stable insertion sort by descending entry count
    for (int a = 1; a < m; a++) {
        int ti = pi[a], tj = pj[a], tc = pc[a], b = a - 1;
        while (b >= 0 && pc[b] < tc) {
            pi[b + 1] = pi[b];
            pj[b + 1] = pj[b];
            pc[b + 1] = pc[b];
            b--;
        }
        pi[b + 1] = ti;
        pj[b + 1] = tj;
        pc[b + 1] = tc;
    }
    const int chunks = gaunt_ell_chunks(n);
    int rows = 0;
    for (int c = 0; c < chunks; c++) {
        eoff[c] = rows;
        int rc = 0;
        for (int l = 0; l < 32; l++) {
            int p = c * 32 + l;
            if (p < m && pc[p] > rc)
                rc = pc[p];
        }
        if (rows + rc > maxRows)
            return -1;
        for (int l = 0; l < 32; l++) {
            int p = c * 32 + l;
            pair[c * 32 + l] = (p < m) ? (unsigned short)((pi[p] << 8) | pj[p]) : (unsigned short)0xFFFF;
            int r0 = (p < m) ? off[pi[p] * n + pj[p]] : 0;
            for (int e = 0; e < rc; e++) {
                bool live = p < m && e < pc[p];
                eidx[(size_t)(rows + e) * 32 + l] = live ? (unsigned short)idx[r0 + e] : (unsigned short)0;
                eval[(size_t)(rows + e) * 32 + l] = live ? val[r0 + e] : 0.0;
            }
        }
        rows += rc;
    }
    eoff[chunks] = rows;
    return rows;
}

}  // namespace clb
