// Point-implicit species update (src/lib/solvesp.f), FP64.
//
// Lane = cell; every warp walks 32-cell tiles. The per-cell update program
// is generated (generated/update_program.cuh) from the reference's statement
// sequence with its A-terms resolved into products of RC, the pass-start Y
// (YO) and the freshly updated Y (YN), so only those live per cell. RC
// comes from the plane written by the rate kernel ([544][npad], coalesced
// per warp). The relaxation passes run inside one cooperative launch: the
// residual sum|dY| is reduced per block, the blocks meet at a grid barrier,
// and every block sums the partials in the same order, so all of them take
// the same convergence decision (src/lib/solvesp.f:2833).
#pragma once
#include <cooperative_groups.h>

#include "uc_device.cuh"
#include "generated/update_program.cuh"

namespace uc {

struct UpdArgs {
    const DevParams *P;
    const double *rc, *sour, *rho, *y0, *soot0;  // y0 [52][npad]: old time level; soot0 [2][npad]
    const double *face_sum, *face_nbr;           // [51][npad] or null
    double *y, *soot;                            // updated in place
    double *partial;                             // [2][gridDim.x]
    int *passes;                                 // out: pass count as ISOR1 reports it
    double dt, sor1, tol, spnorm;
    int isor, n, npad, ntile;
};

constexpr int UPD_THREADS = 128;

__global__ void __launch_bounds__(UPD_THREADS) update_fp64_kernel(const UpdArgs a)
{
    namespace cg = cooperative_groups;
    cg::grid_group grid = cg::this_grid();
    __shared__ double s_part[UPD_THREADS / 32];
    const DevParams &P = *a.P;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int gwarp = (blockIdx.x * UPD_THREADS + threadIdx.x) >> 5;
    const int nwarp = (gridDim.x * UPD_THREADS) >> 5;
    const double sor1 = a.sor1, sor2 = 1.0 - a.sor1, dt = a.dt;
    const size_t np = a.npad;
    int pass;
    for (pass = 1; pass <= a.isor; ++pass) {
        double rsd = 0.0;
        for (int tile = gwarp; tile < a.ntile; tile += nwarp) {
            const size_t cell = (size_t)tile * TILE + lane;
            const bool live = cell < (size_t)a.n;
            double yo[LSP], yn[LSP];
#pragma unroll
            for (int k = 0; k < LSP - 1; ++k) { yo[k] = a.y[k * np + cell]; yn[k] = 0.0; }
            const double rho = a.rho[cell];
            double crsd = 0.0;
            {
                double &rsd = crsd;
#define RC(r) __ldg(a.rc + (size_t)(r) * np + cell)
#define YO(k) yo[k]
#define YN(k) yn[k]
#define Y0(k) __ldg(a.y0 + (size_t)(k) * np + cell)
#define SOUR(m) __ldg(a.sour + (size_t)(m) * np + cell)
#define WM(k) P.WM[k]
#define FACE_SUM(k) (a.face_sum ? a.face_sum[(size_t)(k) * np + cell] : 0.0)
#define FACE_NBR(k) (a.face_nbr ? a.face_nbr[(size_t)(k) * np + cell] : 0.0)
#define UC_UPDATE_TAIL(k) do { if (fnew < 0.0) fnew = 0.0; yn[k] = fnew; } while (0)
                UC_UPDATE_PROGRAM();
#undef RC
#undef YO
#undef YN
#undef Y0
#undef SOUR
#undef WM
#undef FACE_SUM
#undef FACE_NBR
#undef UC_UPDATE_TAIL
                // soot mass fraction and number density (solvesp.f:2807-2832)
                const double s1 = a.soot[cell], s2 = a.soot[np + cell];
                const double so0 = a.sour[cell], so1 = a.sour[np + cell], so2 = a.sour[2 * np + cell],
                             so3 = a.sour[3 * np + cell], so4 = a.sour[4 * np + cell], so5 = a.sour[5 * np + cell];
                double rhs1 = rho * a.soot0[cell] + dt * ((double)0.012011f / P.WMSTR) *
                                                        (2.0 * so0 * yn[21] - so2 * yn[1] - so3 * yn[4] - so4 * yn[3]);
                double fnew = sor2 * s1 + rhs1 * sor1 / ((rho - 0.0) - 0.0);
                crsd += fabs(s1 - fnew);
                if (fnew < 0.0) fnew = 0.0;
                const double n1 = fnew;
                rhs1 = rho * a.soot0[np + cell] + dt * so1 * yn[21];
                const double rhs2 = -(dt * so5);
                fnew = sor2 * s2 + rhs1 * sor1 / ((rho - 0.0) - rhs2);
                if (fnew < 0.0) fnew = 0.0;
                if (live) {
#pragma unroll
                    for (int k = 0; k < LSP - 1; ++k) a.y[k * np + cell] = yn[k];
                    a.soot[cell] = n1;
                    a.soot[np + cell] = fnew;
                }
            }
            if (live) rsd += crsd;
        }
        // deterministic block reduction of the residual
        for (int o = 16; o > 0; o >>= 1) rsd += __shfl_xor_sync(0xffffffffu, rsd, o);
        if (lane == 0) s_part[wib] = rsd;
        __syncthreads();
        if (threadIdx.x == 0) {
            double b = 0.0;
            for (int w = 0; w < UPD_THREADS / 32; ++w) b += s_part[w];
            a.partial[(pass & 1) * gridDim.x + blockIdx.x] = b;
        }
        grid.sync();
        double tot = 0.0;
        for (int b = 0; b < (int)gridDim.x; ++b) tot += a.partial[(pass & 1) * gridDim.x + b];
        if (tot / a.spnorm <= a.tol) break;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *a.passes = pass;   // ISOR1+1 if not converged
    // N2 closure and renormalisation (solvesp.f:2839-2915)
    for (size_t cell = (size_t)blockIdx.x * UPD_THREADS + threadIdx.x; cell < (size_t)a.n;
         cell += (size_t)gridDim.x * UPD_THREADS) {
        double ft = a.y[cell];
        for (int k = 1; k < LSP - 1; ++k) ft = ft + a.y[k * np + cell];
        ft = ft + a.soot[cell];
        double n2 = 1.0 - ft;
        if (ft > 1.0) {
            for (int k = 0; k < LSP - 1; ++k) a.y[k * np + cell] = a.y[k * np + cell] / ft;
            a.soot[cell] = a.soot[cell] / ft;
            n2 = 0.0;
        }
        a.y[(LSP - 1) * np + cell] = n2;
    }
}

}  // namespace uc
