// moment_gpu_solver.cpp -- host side of the B200 linear Pn / FPn solver.
//
//   MomentGpuSolver::tryInit    moment_init.cpp:53-297 (deck keys, maxDt,
//                               initial moments, basis on the quadrature,
//                               upwind flux operators, filter) + upload
//   tryUpdate / tryStage        moment_update.cpp:169-247 on the device
//   tryOutput                   moment_output.cpp:21-56 (.pn only)
#include "moment_gpu_solver.h"

#include <cmath>
#include <vector>

namespace clb {

static const double kPi = 3.14159265358979323846;

// moment_init.cpp:30-41
static double filterSSpline(double x) { return 1.0 / (1.0 + x * x * x * x); }

static double filterLanczos(double x)
{
    if (x < .0000001)
        return 1.0;
    return std::sin(x) / x;
}

MomentGpuSolver::~MomentGpuSolver() { cl_pn_destroy(m_pn); }

int MomentGpuSolver::pnError(int rc)
{
    if (rc)
        lastError = cl_pn_last_error(m_pn);
    return rc;
}

int MomentGpuSolver::tryInit(double dx, double dy, double *maxDtOut)
{
    int momentOrder = 0, quadOrder = 0, filterType = 0;
    double filterTune = 0, cflFactor = 0;
    const InputDeck &d = c_inputDeckReader;
    // moment_init.cpp:57-61: every key is required
    if (!d.get("MOMENT_MOMENT_ORDER", &momentOrder) || !d.get("MOMENT_QUAD_ORDER", &quadOrder) ||
        !d.get("MOMENT_FILTER_TYPE", &filterType) || !d.get("MOMENT_FILTER_TUNE", &filterTune) ||
        !d.get("MOMENT_CFL_FACTOR", &cflFactor)) {
        lastError = "moment_init.cpp: input error (missing MOMENT_* deck key)";
        return CL_ERR_ARG;
    }
    const double maxDt = cflFactor * 0.5 * std::fmin(dx, dy);   // moment_init.cpp:65
    if (maxDtOut)
        *maxDtOut = maxDt;

    cl_angular ang;
    int rc = cl_angular_create(momentOrder, quadOrder, 0, &ang);
    if (rc) {
        lastError = cl_global_error();
        return rc;
    }
    const int n = ang.n, nq = ang.nq;
    m_n = n;
    c_vectorSize = n;

    // moment_init.cpp:186-222: sums over the quadrature split by the sign of
    // xi (eta), in the reference's order of q
    std::vector<double> ops((size_t)4 * n * n, 0.0);
    double *xp = ops.data(), *xm = xp + n * n, *ep = xm + n * n, *em = ep + n * n;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
            for (int q = 0; q < nq; q++) {
                const double mi = ang.p[(size_t)q * ang.n2 + i], mj = ang.p[(size_t)q * ang.n2 + j];
                const double vx = ang.xi[q] * mi * mj * ang.w[q];
                const double ve = ang.eta[q] * mi * mj * ang.w[q];
                if (ang.xi[q] > 0)
                    xp[i * n + j] += vx;
                else
                    xm[i * n + j] += vx;
                if (ang.eta[q] > 0)
                    ep[i * n + j] += ve;
                else
                    em[i * n + j] += ve;
            }
    cl_angular_free(&ang);

    // moment_init.cpp:225-289
    std::vector<double> filter(n, 1.0);
    const double N = momentOrder;
    int nm = 0;
    for (int l = 0; l <= momentOrder; l++)
        for (int m = -l; m <= l; m++) {
            if ((m + l) % 2 != 0)
                continue;
            if (filterType == 1) {
                const double omega = filterTune, L = 1.0, sigmaT = 1.0;
                const double a = omega / (N * N) / (sigmaT * L + N) / (sigmaT * L + N);
                filter[nm] = 1.0 / (1.0 + a * l * l * (l + 1) * (l + 1));
            } else if (filterType == 2) {
                const double s = -filterTune * maxDt / std::log(filterSSpline(N / (N + 1)));
                filter[nm] = std::pow(filterSSpline(l / (N + 1)), s);
            } else if (filterType == 3) {
                const double s = -filterTune * maxDt / std::log(filterLanczos(N / (N + 1)));
                filter[nm] = std::pow(filterLanczos(l / (N + 1)), s);
            }
            nm++;
        }

    // moment_init.cpp:106-114
    const int NX = c_gX[3] - c_gX[0] + 1, NY = c_gY[3] - c_gY[0] + 1;
    const size_t C = (size_t)NX * NY;
    std::vector<double> moments(C * n, 0.0);
    for (size_t c = 0; c < C; c++)
        moments[c * n] = c_initialGrid[c] * 2.0 * std::sqrt(kPi);

    cl_grid g;
    g.nx = c_sizeX;
    g.ny = c_sizeY;
    g.ghost = 2;
    g.init_cond = c_initCond;
    g.init_x = c_initX;
    g.init_y = c_initY;
    g.theta = 0.0;
    cl_pn_setup setup;
    setup.n = n;
    setup.ops = ops.data();
    setup.filter = (filterType >= 1 && filterType <= 3) ? filter.data() : nullptr;
    rc = cl_pn_create(&g, &setup, c_sigmaT, c_sigmaS, moments.data(), &m_pn);
    if (rc) {
        lastError = cl_global_error();
        return rc;
    }
    return CL_OK;
}

int MomentGpuSolver::tryUpdate(double dt, double dx, double dy) { return pnError(cl_pn_step(m_pn, dt, dx, dy)); }

int MomentGpuSolver::tryStage(int stage, double dt, double dx, double dy)
{
    return pnError(cl_pn_stage(m_pn, stage, dt, dx, dy));
}

int MomentGpuSolver::tryOutput(double time) { return writePn(time); }

int MomentGpuSolver::getState(double *moments) { return pnError(cl_pn_get_state(m_pn, moments)); }

int MomentGpuSolver::setState(const double *moments) { return pnError(cl_pn_set_state(m_pn, moments)); }

int MomentGpuSolver::haloCounts(long long counts[4]) { return pnError(cl_pn_halo_counts(m_pn, counts)); }

int MomentGpuSolver::haloPack(double *const bufs[4]) { return pnError(cl_pn_halo_pack(m_pn, bufs)); }

int MomentGpuSolver::haloUnpack(double *const bufs[4]) { return pnError(cl_pn_halo_unpack(m_pn, bufs)); }

void *MomentGpuSolver::stream()
{
    void *st = nullptr;
    cl_pn_stream(m_pn, &st);
    return st;
}

int MomentGpuSolver::sync() { return pnError(cl_pn_sync(m_pn)); }

void MomentGpuSolver::setExchangedSides(int mask) { cl_pn_set_exchanged_sides(m_pn, mask); }

}  // namespace clb
