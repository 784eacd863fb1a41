// momopt_gpu_solver.cpp -- host side of the B200 momopt solver.
//
//   MomOptGpuSolver::tryInit    momopt_init.cpp:51-160 (deck keys, maxDt,
//                               initial moments and alpha) + device upload
//   tryUpdate / tryStage        momopt_update.cpp:283-382 on the device
//   tryOutput                   momopt_output.cpp:21-77 (.pn / .opt formats)
#include "momopt_gpu_solver.h"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace clb {

static const double kPi = 3.14159265358979323846;
static const double kReg[CL_NUM_REG] = {0.0, 1e-3, 1e-2, 1e-1, 5e-1};

MomOptGpuSolver::~MomOptGpuSolver() { cl_destroy(m_ctx); }

int MomOptGpuSolver::ctxError(int rc)
{
    if (rc)
        lastError = cl_last_error(m_ctx);
    return rc;
}

int MomOptGpuSolver::tryInit(double dx, double dy, double *maxDtOut)
{
    int momentOrder = 0, quadOrder = 0, useGaunt = 0, maxIterBfgs = 0;
    double cfl = 0, condHMaxBfgs = 0, theta = 0;
    const InputDeck &d = c_inputDeckReader;
    // momopt_init.cpp:56-68: every key is required
    struct IntKey {
        const char *k;
        int *v;
    } ik[] = {{"MOMOPT_MOMENT_ORDER", &momentOrder}, {"MOMOPT_QUAD_ORDER", &quadOrder},
              {"MOMOPT_MAX_ITER", &m_opt.max_iter},   {"MOMOPT_MAX_BFGS_ITER", &maxIterBfgs},
              {"MOMOPT_USE_GAUNT", &useGaunt},        {"MOMOPT_MOMENT_TYPE", &m_opt.moment_type},
              {"MOMOPT_OPTIMIZATION_TYPE", &m_opt.opt_type}};
    struct DblKey {
        const char *k;
        double *v;
    } dk[] = {{"MOMOPT_CFL_FACTOR", &cfl},        {"MOMOPT_TOL", &m_opt.tol},
              {"MOMOPT_COND_H_MAX", &m_opt.cond_h_max}, {"MOMOPT_COND_H_MAX_BFGS", &condHMaxBfgs},
              {"MOMOPT_THETA", &theta},           {"MOMOPT_DELTA_PPN", &m_opt.delta_ppn}};
    for (auto &k : ik)
        if (!d.get(k.k, k.v)) {
            lastError = std::string("momopt input error: missing ") + k.k;
            return CL_ERR_ARG;
        }
    for (auto &k : dk)
        if (!d.get(k.k, k.v)) {
            lastError = std::string("momopt input error: missing ") + k.k;
            return CL_ERR_ARG;
        }
    m_opt.max_bfgs_iter = maxIterBfgs;
    m_opt.cond_h_max_bfgs = condHMaxBfgs;
    // optional extensions (unknown to the reference, ignored by its reader)
    if (!d.get("MOMOPT_TOL_GAMMA", &m_opt.tol_gamma))
        m_opt.tol_gamma = 0.0;
    std::string prec;
    m_opt.precision = CL_FP64;
    if (d.get("MOMOPT_GPU_PRECISION", prec) && prec == "mixed")
        m_opt.precision = CL_MIXED;
    std::string contraction;
    m_opt.contraction = CL_CONTRACT_PAIRS;
    int tune = 1;
    if (!d.get("MOMOPT_GPU_TUNE", &tune))
        tune = 1;
    m_tune = tune != 0;
    if (d.get("MOMOPT_GPU_CONTRACTION", contraction) && contraction == "single")
        m_opt.contraction = CL_CONTRACT_SINGLE;

    m_maxDt = cfl * (2.0 / (2.0 + theta)) * (dx * dy) / (dx + dy);   // momopt_init.cpp:72
    if (maxDtOut)
        *maxDtOut = m_maxDt;

    cl_angular ang;
    int rc = cl_angular_create(momentOrder, quadOrder, useGaunt, &ang);
    if (rc) {
        lastError = cl_global_error();
        return rc;
    }
    m_n = ang.n;
    c_vectorSize = m_n;
    const int NX = c_gX[3] - c_gX[0] + 1, NY = c_gY[3] - c_gY[0] + 1;
    const size_t C = (size_t)NX * NY;
    std::vector<double> moments(C * m_n, 0.0), alpha(C * m_n, 0.0);
    // momopt_init.cpp:120-143
    for (size_t c = 0; c < C; c++) {
        double u0 = c_initialGrid[c] * 2.0 * std::sqrt(kPi);
        moments[c * m_n] = u0;
        if (m_opt.moment_type == CL_MN)
            alpha[c * m_n] = 2.0 * std::sqrt(kPi) * std::log(u0 / (2.0 * std::sqrt(kPi)));
        else if (m_opt.moment_type == CL_PPN)
            alpha[c * m_n] = u0 - 4.0 * m_opt.delta_ppn * kPi / u0;
    }
    cl_grid g;
    g.nx = c_sizeX;
    g.ny = c_sizeY;
    g.ghost = 2;
    g.init_cond = c_initCond;
    g.init_x = c_initX;
    g.init_y = c_initY;
    g.theta = theta;
    rc = cl_create(&g, &m_opt, &ang, c_sigmaT, c_sigmaS, moments.data(), alpha.data(), &m_ctx);
    cl_angular_free(&ang);
    if (rc) {
        lastError = cl_global_error();
        return rc;
    }
    // launch shapes chosen by the autotuner on the initial state (or taken
    // from its cache); grids too small to time keep the defaults
    if (m_tune)
        return ctxError(cl_tune(m_ctx, 1, nullptr));
    return CL_OK;
}

int MomOptGpuSolver::tryOutput(double time)
{
    int rc = writePn(time);
    if (rc)
        return rc;
    char fn[1024];
    FILE *f;
    cl_stats st;
    rc = cl_get_stats(m_ctx, &st);
    if (rc) {
        lastError = cl_last_error(m_ctx);
        return rc;
    }
    std::snprintf(fn, sizeof(fn), "%s/out_%.3f_%d.opt", outDir.c_str(), time, c_node);
    f = std::fopen(fn, "w");
    if (!f) {
        lastError = std::string("cannot open ") + fn;
        return CL_ERR_ARG;
    }
    std::fprintf(f, "Max number of iterations: %d\n", st.max_iter);
    std::fprintf(f, "Mean number of iterations: %f\n", st.iter_mean);
    std::fprintf(f, "Number of optimizations: %d\n", (int)st.num_solves);
    std::fprintf(f, "Regularizations Histogram\n");
    for (int i = 0; i < CL_NUM_REG; i++)
        std::fprintf(f, "r = %.3e   %d\n", kReg[i], (int)st.hist_reg[i]);
    std::fclose(f);
    return CL_OK;
}

int MomOptGpuSolver::tryUpdate(double dt, double dx, double dy) { return ctxError(cl_step(m_ctx, dt, dx, dy)); }

int MomOptGpuSolver::tryStage(int stage, double dt, double dx, double dy)
{
    return ctxError(cl_stage(m_ctx, stage, dt, dx, dy));
}

int MomOptGpuSolver::getState(double *moments) { return ctxError(cl_get_state(m_ctx, moments, nullptr)); }

int MomOptGpuSolver::setState(const double *moments) { return ctxError(cl_set_state(m_ctx, moments, nullptr)); }

int MomOptGpuSolver::haloCounts(long long counts[4]) { return ctxError(cl_halo_counts(m_ctx, counts)); }

int MomOptGpuSolver::haloPack(double *const bufs[4]) { return ctxError(cl_halo_pack(m_ctx, bufs)); }

int MomOptGpuSolver::haloUnpack(double *const bufs[4]) { return ctxError(cl_halo_unpack(m_ctx, bufs)); }

void *MomOptGpuSolver::stream()
{
    void *st = nullptr;
    cl_stream(m_ctx, &st);
    return st;
}

int MomOptGpuSolver::sync() { return ctxError(cl_sync(m_ctx)); }

}  // namespace clb
