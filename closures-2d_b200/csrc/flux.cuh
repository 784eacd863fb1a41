// flux.cuh -- host interface of the kinetic-flux + RK-stage kernel (K2+K3)
// and the periodic ghost fill (K4).
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"
#include "fexp.cuh"

namespace clb {

struct FluxArgs {
    const double *alpha;        // [C][n]
    double *moments;            // [C][n], updated in place on interior cells
    const double *momentsOld;   // Heun average partner (stage 2) or null (stage 1)
    const double *sigmaT, *sigmaS;  // [C]
    const double *P;            // [nqp][ldPf] basis rows, padding columns zero
    const double *xi, *eta;     // 16 per chunk, zero on padded directions
    const double *cxw, *cyw;    // xi*w, eta*w per direction
    int n, nb, ldPf, nqp;
    // direction pairs: a chunk's 8 rows of P serve directions q (0..7) and
    // q + Q (8..15); columns are grouped by degree parity (nbe even ones
    // first) and binv[c] is the moment of column c (-1 padding)
    int paired, nbe;
    const short *binv;
    int NX, NY;                 // grid with ghosts
    int momentType, initCond;
    double theta, deltaPPn;
    double dt, dx, dy, initX, initY;
    // layout (doubles), filled by plan_flux()
    int kq, ldAl, ldA, ldF;
    int offAl, offA, offF, offP, offQ, offExp;
    ExpConsts ex;
    int smemBytes;
    int tilesX, tilesY;
    int tileBase;               // first tile of the launch (row-major over tilesX x tilesY)
    unsigned long long *tilesRun;   // nullable: tiles that ran the chunk loop (non-uniform)
    int skipUniform;                // 1: uniform tiles apply zero flux without the chunk loop
};

int plan_flux(FluxArgs &f);
cudaError_t prepare_flux(const FluxArgs &f);
cudaError_t launch_flux(const FluxArgs &f, cudaStream_t stream);
// The tiles first .. first + count - 1 only (one launch of a split stage).
cudaError_t launch_flux_tiles(const FluxArgs &f, int first, int count, cudaStream_t stream);
int flux_tile_rows(const FluxArgs &f);   // interior cells per tile along x
// duplicateBoundaries (momopt_boundaries.cpp:190-223) on device moments.
cudaError_t launch_ghost_periodic(double *moments, int n, int NX, int NY, cudaStream_t stream);
// Halo strips of a node's block: pack (1) the inner strips into p[side] or
// unpack (0) p[side] into the ghost strips; null sides are skipped.
struct HaloBuffers {
    double *p[4];
};
cudaError_t launch_halo(double *moments, int n, int NX, int NY, const HaloBuffers &b, int pack,
                        cudaStream_t stream);

}  // namespace clb
