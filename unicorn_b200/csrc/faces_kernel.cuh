// Species-equation face coefficients on the device (src/lib/spgsolv.f:233-1290).
//
// For an lj x li grid (J fastest, cell c = (I-1) lj + (J-1)) every interior
// cell gets, per species k, the coefficients of its east, west, north and
// south neighbours: the hybrid convection-diffusion form of the reference,
//   E = DT/XXC(I) * (rho u_e - max(|rho u_e|, D_e)) / 2, and likewise W, N, S,
// with the face conductances D (spgsolv.f:233-348: the mean of EMU VDF_k of
// the two cells plus the eddy part REI (TMU + TMU)/SIGSP, over the spacing)
// and, on the N and S faces, the axisymmetric terms of spgsolv.f:354-406.
// The update takes them as face_sum = E+W+N+S and face_nbr = N Y(J+1) +
// S Y(J-1) + E Y(I+1) + W Y(I-1), with the neighbour values of the start of
// the update (Jacobi over cells: the reference's lexicographic Gauss-Seidel
// has no parallel form); the grid's boundary cells are held.
#pragma once
#include "uc_device.cuh"

namespace uc {

struct FaceArgs {
    const DevParams *P;
    int lj, li, npad, isym;
    const double *rho, *vdf, *u, *v, *tmu, *yr;      // [npad], vdf [52][npad]
    const double *xxs, *xxc, *yys, *yyc;             // [li], [li], [lj], [lj]
    double dt, sigsp;
    double *e, *w, *n, *s;                           // [51][npad]
};

__global__ void faces_kernel(const FaceArgs a)
{
    const DevParams &P = *a.P;
    const int lj = a.lj, li = a.li;
    const size_t np = a.npad;
    const double SYM = (double)a.isym, REI = P.REI, BETA3 = P.BETA3;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < lj * li; idx += gridDim.x * blockDim.x) {
        const int j = idx % lj, i = idx / lj;
        if (j == 0 || j == lj - 1 || i == 0 || i == li - 1) continue;
        const size_t c = idx, cE = c + lj, cW = c - lj, cN = c + 1, cS = c - 1;
        const double *rho = a.rho, *tmu = a.tmu;
        const double DTBRX = a.dt / a.xxc[i], DTBRY = a.dt / a.yyc[j];
        const double RHOUE = 0.5 * (rho[cE] + rho[c]) * a.u[cE];
        const double RHOUW = 0.5 * (rho[c] + rho[cW]) * a.u[c];
        const double RHOVN = 0.5 * (rho[cN] + rho[c]) * a.v[cN];
        const double RHOVS = 0.5 * (rho[c] + rho[cS]) * a.v[c];
        const double EMUc = REI * BETA3 * rho[c], EMUe = REI * BETA3 * rho[cE], EMUw = REI * BETA3 * rho[cW];
        const double EMUn = REI * BETA3 * rho[cN], EMUs = REI * BETA3 * rho[cS];
        const double SYM1 = SYM * a.dt * 0.5 * EMUc / a.yr[c];
        const double SYM2 = SYM * a.dt * 0.5 * REI * tmu[c] / a.sigsp / a.yr[c];
        const double TURE = REI * (tmu[cE] + tmu[c]) / a.sigsp, TURW = REI * (tmu[c] + tmu[cW]) / a.sigsp;
        const double TURN = REI * (tmu[cN] + tmu[c]) / a.sigsp, TURS = REI * (tmu[c] + tmu[cS]) / a.sigsp;
        const double xe = a.xxs[i + 1], xw = a.xxs[i], yn = a.yys[j + 1], ys = a.yys[j];
        for (int k = 0; k < LSP - 1; ++k) {
            const double *d = a.vdf + (size_t)k * np;
            const double dc = d[c];
            const double DE = (EMUe * d[cE] + EMUc * dc + TURE) / xe;
            const double DW = (EMUc * dc + EMUw * d[cW] + TURW) / xw;
            const double DN = (EMUn * d[cN] + EMUc * dc + TURN) / yn;
            const double DS = (EMUc * dc + EMUs * d[cS] + TURS) / ys;
            const double SYMA = SYM1 * dc + SYM2;
            double cv;
            cv = fabs(RHOUE); if (DE >= cv) cv = DE;
            a.e[(size_t)k * np + c] = DTBRX * 0.5 * (RHOUE - cv);
            cv = fabs(RHOUW); if (DW >= cv) cv = DW;
            a.w[(size_t)k * np + c] = DTBRX * 0.5 * (-RHOUW - cv);
            cv = fabs(RHOVN); if (DN >= cv) cv = DN;
            a.n[(size_t)k * np + c] = DTBRY * 0.5 * (RHOVN - cv) - SYMA / yn;
            cv = fabs(RHOVS); if (DS >= cv) cv = DS;
            a.s[(size_t)k * np + c] = DTBRY * 0.5 * (-RHOVS - cv) + SYMA / ys;
        }
    }
}

// face_sum / face_nbr of the update from the coefficients and the current Y;
// boundary cells get zeros (they are held)
__global__ void faces_apply_kernel(int lj, int li, int npad, const double *e, const double *w, const double *n,
                                   const double *s, const double *y, double *fsum, double *fnbr)
{
    const size_t np = npad;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < lj * li; idx += gridDim.x * blockDim.x) {
        const int j = idx % lj, i = idx / lj;
        const bool inner = !(j == 0 || j == lj - 1 || i == 0 || i == li - 1);
        for (int k = 0; k < LSP - 1; ++k) {
            const size_t o = (size_t)k * np + idx;
            if (!inner) { fsum[o] = 0.0; fnbr[o] = 0.0; continue; }
            const double *yk = y + (size_t)k * np;
            fsum[o] = e[o] + w[o] + n[o] + s[o];
            fnbr[o] = n[o] * yk[idx + 1] + s[o] * yk[idx - 1] + e[o] * yk[idx + lj] + w[o] * yk[idx - lj];
        }
    }
}

// 1 for the grid's boundary cells (and padding), 0 inside
__global__ void hold_mask_kernel(int lj, int li, int npad, uint8_t *hold)
{
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < npad; idx += gridDim.x * blockDim.x) {
        const int j = idx % lj, i = idx / lj;
        hold[idx] = (idx >= lj * li || j == 0 || j == lj - 1 || i == 0 || i == li - 1) ? 1 : 0;
    }
}

}  // namespace uc
