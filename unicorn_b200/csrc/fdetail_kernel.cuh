// Regular-grid detail output (src/lib/stdata.f:24-119, the FDETAIL dump).
//
// The staggered fields of an lj x li grid are averaged onto the cell corners
// (four-point means; velocities from their two faces), the last row and
// column copied from their neighbours, and dimensional values formed with the
// reference scales; the mixture cp and the species enthalpies h_k are then
// evaluated at the corner temperature. The 218 output rows per point, in the
// order of the reference's record (stdata.f:127-133): z, r, RHO, v (axial),
// u (radial), T, QDOT, VMU, VTC, CP, then for each species Y_k, D_k,
// QDSP_k, h_k. One thread per point, J fastest (coalesced).
#pragma once
#include "uc_device.cuh"

namespace uc {

constexpr int FD_ROWS = 10 + 4 * LSP;

struct FdArgs {
    const DevParams *P;
    int lj, li, npad;
    const double *x, *y, *u, *v;                   // [npad] grid coordinates and velocities
    const double *rho, *tk, *qdot, *vmu, *vtc;     // [npad]
    const double *fsp, *vdf, *qdsp;                // [52][npad]
    double ALSTR, RSTR, TSTR, AMSTR, ACSTR, VSTR, DSTR;
    double *out;                                   // [FD_ROWS][npad]
};

__global__ void fdetail_kernel(const FdArgs a)
{
    const DevParams &P = *a.P;
    const int lj = a.lj, li = a.li;
    const size_t np = a.npad;
    const double XSHIFT = 0.5 * (a.x[0] + a.x[lj]), YSHIFT = 0.5 * (a.y[0] + a.y[1]);
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < lj * li; idx += gridDim.x * blockDim.x) {
        const int j = idx % lj, i = idx / lj;
        // the interior corner whose values this point takes (stdata.f:1322-1325 copies)
        const int jj = j == lj - 1 ? lj - 2 : j, ii = i == li - 1 ? li - 2 : i;
        const size_t c = (size_t)ii * lj + jj, cE = c + lj, cN = c + 1, cNE = c + lj + 1;
        auto avg4 = [&](const double *f) { return 0.25 * (f[c] + f[cN] + f[cE] + f[cNE]); };
        double *o = a.out + idx;
        double XRG = (0.5 * (a.x[c] + a.x[cE]) - XSHIFT) * a.ALSTR;
        double YRG = (0.5 * (a.y[c] + a.y[cN]) - YSHIFT) * a.ALSTR;
        if (j == lj - 1) YRG = a.y[(size_t)ii * lj + j] * a.ALSTR;   // last row (stdata.f:1322); the corner
        if (i == li - 1) XRG = a.x[idx] * a.ALSTR;                      // takes row LJ's LI-1 value (:1324)
        o[0 * np] = XRG;
        o[1 * np] = YRG;
        o[2 * np] = avg4(a.rho) * a.RSTR;
        o[3 * np] = 0.5 * (a.u[cE] + a.u[cNE]) * a.VSTR;
        o[4 * np] = 0.5 * (a.v[cN] + a.v[cNE]) * a.VSTR;
        const double TKD = avg4(a.tk) * a.TSTR;
        o[5 * np] = TKD;
        o[6 * np] = avg4(a.qdot);
        o[7 * np] = avg4(a.vmu) * a.AMSTR;
        o[8 * np] = avg4(a.vtc) * a.ACSTR;
        const double TKD2 = TKD * TKD, TKD3 = TKD * TKD2, TKD4 = TKD * TKD3, TKD5 = TKD * TKD4;
        const int ip = TKD > UC_TPOL1 ? 7 : 0;
        double FTOT = 0.0, TCP = 0.0;
        for (int k = 0; k < LSP; ++k) {
            const size_t kk = (size_t)k * np;
            double Y;
            if (k < LSP - 1) {
                Y = 0.25 * (a.fsp[kk + c] + a.fsp[kk + cN] + a.fsp[kk + cE] + a.fsp[kk + cNE]);
                FTOT = FTOT + Y;
            } else {
                Y = 1.0 - FTOT;
            }
            const double *p = P.poly + k * 14 + ip;
            TCP = TCP + (p[0] + p[1] * TKD + p[2] * TKD2 + p[3] * TKD3 + p[4] * TKD4) * Y * P.GASC / P.WM[k] / P.WMSTR;
            double *ok = o + (size_t)(10 + 4 * k) * np;
            ok[0] = Y;
            ok[np] = 0.25 * (a.vdf[kk + c] + a.vdf[kk + cN] + a.vdf[kk + cE] + a.vdf[kk + cNE]) * a.DSTR;
            ok[2 * np] = 0.25 * (a.qdsp[kk + c] + a.qdsp[kk + cN] + a.qdsp[kk + cE] + a.qdsp[kk + cNE]);
            ok[3 * np] = (p[0] * TKD + p[1] * TKD2 / 2.0 + p[2] * TKD3 / 3.0 + p[3] * TKD4 / 4.0 + p[4] * TKD5 / 5.0 + p[5]) *
                         P.GASC / P.WM[k] / P.WMSTR;
        }
        o[9 * np] = TCP;
    }
}

}  // namespace uc
