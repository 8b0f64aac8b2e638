// Property kernels, FP64: Y clip + mixture-averaged transport, cp/h, and
// temperature from enthalpy. Thread = cell.
#pragma once
#include "uc_device.cuh"

namespace uc {

struct PropArgs {
    const DevParams *P;
    const double *tk;
    double *y;                       // [52][npad], clipped in place (main:821-828)
    double *vmu, *vtc, *vdf;         // outputs (vdf [52][npad])
    int n, npad;
};

__device__ __forceinline__ int ci_range(double TKDS)
{
    int K = 0;
    if (TKDS >= 2.0) K = 1;
    if (TKDS > 5.0) K = 2;
    if (TKDS > 70.0) K = 3;
    return K;
}

// Omega(1,1) quartic fit CI11 in T* (main:944-952), for the pair (i, j)
__device__ __forceinline__ double ci11t(const DevParams &P, int i, int j, double TKD1, double TKD2, double TKD3,
                                        double TKD4)
{
    const int ij = i * LSP + j;
    const double TKDS = TKD1 / P.ETLJ1[ij];
    const double *c = P.ci11 + ci_range(TKDS) * 5;
    return c[0] + c[1] * TKDS + c[2] * TKD2 / P.ETLJ2[ij] + c[3] * TKD3 / P.ETLJ3[ij] + c[4] * TKD4 / P.ETLJ4[ij];
}

// src/unicornd-mild-sd-5.f:821-1006 for one cell per thread.
__global__ void __launch_bounds__(128) props_fp64_kernel(const PropArgs a)
{
    const DevParams &P = *a.P;
    const size_t np = a.npad;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < (size_t)a.n; c += (size_t)gridDim.x * blockDim.x) {
        // Y clip and N2 closure (main:821-828)
        double TMASS = 0.0;
        for (int k = 0; k < LSP - 1; ++k) {
            double yk = a.y[k * np + c];
            if (yk < 0.0) { yk = 0.0; a.y[k * np + c] = 0.0; }
            TMASS = TMASS + yk;
        }
        a.y[(LSP - 1) * np + c] = 1.0 - TMASS;
        // sub-mixture: species with Y >= 1e-3 plus N2 last (main:842-915)
        int8_t sub[LSP];
        double X[LSP];
        int IA = 0;
        TMASS = 0.0;
        double TMOLE = 0.0;
        for (int k = 0; k < LSP - 1; ++k) {
            const double yk = a.y[k * np + c];
            if (yk < 1.0e-03) continue;
            sub[IA] = (int8_t)k;
            TMASS = TMASS + yk;
            X[IA] = yk / P.WM[k];
            TMOLE = TMOLE + X[IA];
            ++IA;
        }
        int LSPT = IA + 1;
        if (LSPT >= LSP) LSPT = LSP;
        sub[LSPT - 1] = LSP - 1;
        X[LSPT - 1] = (1.0 - TMASS) / P.WM[LSP - 1];
        TMOLE = TMOLE + X[LSPT - 1];
        const double tk = a.tk[c];
        const double TKRT = sqrt(tk);
        const double TKD1 = tk * P.TSTR;
        const double TKD2 = TKD1 * TKD1, TKD3 = TKD2 * TKD1, TKD4 = TKD3 * TKD1, TKD5 = TKD4 * TKD1;
        const int IPL1 = TKD1 >= UC_TPOL1 ? 7 : 0, IPL2 = TKD1 >= UC_TPOL1 ? 6 : 0;
        const double TKBP = tk * TKRT / P.PBACK;
        double ATC[LSP], AMU[LSP];
        for (int i = 0; i < LSPT; ++i) {
            const int k = sub[i];
            const double *p = P.poly + k * 14 + IPL1;
            const double *q = P.om22 + k * 12 + IPL2;
            const double EUKEN = (double)0.115f + (double)0.354f * (p[0] + p[1] * TKD1 + p[2] * TKD2 + p[3] * TKD3 + p[4] * TKD4);
            const double SIOME = P.cdia[k] * P.cdia[k] * (q[0] + q[1] * TKD1 + q[2] * TKD2 + q[3] * TKD3 + q[4] * TKD4 + q[5] * TKD5);
            ATC[i] = P.CONVRC * EUKEN * TKRT / P.WMIK[k * LSP + k] / SIOME;
            AMU[i] = P.CONVRM * TKRT * P.WMIK[k * LSP + k] / SIOME;
        }
        double VTC = 0.0, VMU = 0.0;
        double VDFQ[LSP];
        for (int i = 0; i < LSPT; ++i) {
            const int k = sub[i];
            double PHIK = 0.0, PHDIK = 0.0, EFDIK = 0.0;
            for (int j = 0; j < LSPT; ++j) {
                if (j == i) continue;
                const int kb = sub[j];
                const int ij = k * LSP + kb;
                const double t1 = 1.0 + sqrt(ATC[i] / ATC[j]) * P.WMIK[ij];
                const double t2 = 1.0 + sqrt(AMU[i] / AMU[j]) * P.WMIK[ij];
                PHIK = PHIK + X[j] * (t1 * t1) / P.DWMIK[ij];
                PHDIK = PHDIK + X[j] * (t2 * t2) / P.DWMIK[ij];
                // binary diffusion D_ij (main:940-953); the fit value is symmetric in (i, j)
                const double CI = ci11t(P, i < j ? k : kb, i < j ? kb : k, TKD1, TKD2, TKD3, TKD4);
                EFDIK = EFDIK + X[j] / (P.WMCD[ij] * TKBP / CI);
            }
            VTC = VTC + ATC[i] * X[i] / (X[i] + (double)1.065f * PHIK);
            VMU = VMU + AMU[i] * X[i] / (X[i] + PHDIK);
            const double AA = TMOLE - X[i];
            if (AA <= 1.0e-10) {
                // DIFSP(i, LSPT): assigned above the diagonal only; the diagonal stays zero
                double d = 0.0;
                if (i != LSPT - 1) {
                    const int kl = sub[LSPT - 1];
                    d = P.WMCD[k * LSP + kl] * TKBP / ci11t(P, k, kl, TKD1, TKD2, TKD3, TKD4);
                }
                VDFQ[i] = P.CONVRD * d;
            } else {
                VDFQ[i] = P.CONVRD * (TMOLE - X[i]) / EFDIK;
            }
        }
        a.vtc[c] = VTC;
        a.vmu[c] = VMU;
        // D_k of every species (main:981-1003); N2 (never flagged in ISPQ) takes this path too
        int pos = 0;
        for (int k = 0; k < LSP; ++k) {
            double v;
            if (k < LSP - 1 && pos < LSPT - 1 && sub[pos] == k) {
                v = VDFQ[pos];
                ++pos;
            } else {
                double EFD = 0.0;
                for (int b = 0; b < LSPT; ++b) {
                    const int nb = sub[b];
                    const double CI = ci11t(P, k, nb, TKD1, TKD2, TKD3, TKD4);
                    EFD = EFD + X[b] / (P.WMCD[k * LSP + nb] * TKBP / CI);
                }
                v = P.CONVRD * TMOLE / EFD;
            }
            a.vdf[k * np + c] = v;
        }
    }
}

// Mixture cp (spgsolv.f:102-173) and h = sum_k Y_k h_k (h_k: solveh.f:39-57).
struct CpHArgs {
    const DevParams *P;
    const double *tk, *y;
    double *cp, *h;
    int n, npad;
};

__global__ void __launch_bounds__(256) cp_h_fp64_kernel(const CpHArgs a)
{
    const DevParams &P = *a.P;
    const size_t np = a.npad;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < (size_t)a.n; c += (size_t)gridDim.x * blockDim.x) {
        const double TKD = a.tk[c] * P.TSTR;
        const double TKD2 = TKD * TKD, TKD3 = TKD * TKD2, TKD4 = TKD * TKD3, TKD5 = TKD * TKD4;
        const int ip = TKD > UC_TPOL1 ? 7 : 0;
        double TCP = 0.0, hs = 0.0;
        for (int k = 0; k < LSP; ++k) {
            const double *p = P.poly + k * 14 + ip;
            const double yk = a.y[k * np + c];
            const double t = (p[0] + p[1] * TKD + p[2] * TKD2 + p[3] * TKD3 + p[4] * TKD4) / P.WM[k];
            TCP = TCP + t * yk;
            const double HSSP = (p[0] * TKD + p[1] * TKD2 / 2.0 + p[2] * TKD3 / 3.0 + p[3] * TKD4 / 4.0 + p[4] * TKD5 / 5.0) /
                                P.WM[k] * P.HCONVR;
            const double H = HSSP * P.WMSTR * P.HSTR + p[5] / P.WM[k] * P.GASC;
            hs = hs + yk * H;
        }
        if (a.cp) a.cp[c] = TCP / P.WMSTR * P.GASC * P.TSTR / P.HSTR;
        if (a.h) a.h[c] = hs;
    }
}

// Temperature from the sensible enthalpy by Newton (solveh.f:1170-1234).
struct TempArgs {
    const DevParams *P;
    const double *y, *ht;
    double *tk;
    int *status;
    int n, npad;
};

__global__ void __launch_bounds__(128) temperature_fp64_kernel(const TempArgs a)
{
    const DevParams &P = *a.P;
    const size_t np = a.npad;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < (size_t)a.n; c += (size_t)gridDim.x * blockDim.x) {
        double ENTH = (a.ht[c] - (double)0.5f * 0.0) * P.HSTR;
        for (int k = 0; k < LSP; ++k) ENTH = ENTH + a.y[k * np + c] * P.HFO[k] * P.HSTR;
        int IPL = 0;
        double TPOLY = UC_TPOL1;
        double TKD = a.tk[c] * P.TSTR;
        double A1, A2, A3, A4, A5, A6;
        for (int guard = 0; guard < 3; ++guard) {
            if (TKD > TPOLY) TKD = TPOLY / 2.0;
            A1 = A2 = A3 = A4 = A5 = A6 = 0.0;
            for (int k = 0; k < LSP; ++k) {
                const double *p = P.poly + k * 14 + IPL;
                const double yk = a.y[k * np + c];
                A1 = A1 + p[0] * yk / P.WM[k];
                A2 = A2 + p[1] * yk / P.WM[k] / 2.0;
                A3 = A3 + p[2] * yk / P.WM[k] / 3.0;
                A4 = A4 + p[3] * yk / P.WM[k] / 4.0;
                A5 = A5 + p[4] * yk / P.WM[k] / 5.0;
                A6 = A6 + p[5] * yk / P.WM[k];
            }
            const double FUNT = ((A1 + (A2 + (A3 + (A4 + A5 * TPOLY) * TPOLY) * TPOLY) * TPOLY) * TPOLY + A6) * P.GASC / P.WMSTR - ENTH;
            if (FUNT >= 1.0e-07) break;
            if (IPL >= 7) break;
            IPL = 7;
            if (TKD <= TPOLY) TKD = UC_TPOL2 / 2.0;
            TPOLY = UC_TPOL2;
        }
        bool conv = false;
        for (int it = 1; it <= 100; ++it) {
            const double DTKD = ((A1 + (A2 + (A3 + (A4 + A5 * TKD) * TKD) * TKD) * TKD) * TKD + A6 - ENTH * P.WMSTR / P.GASC) /
                                (A1 + (2.0 * A2 + (3.0 * A3 + (4.0 * A4 + 5.0 * A5 * TKD) * TKD) * TKD) * TKD);
            if (fabs(DTKD) <= (double)0.001f) { conv = true; break; }
            TKD = TKD - DTKD;
        }
        if (!conv && a.status) atomicCAS(a.status, ST_OK, ST_NEWTON_NOCONV);
        if (TKD > UC_TPOL2) TKD = UC_TPOL2;
        if (TKD < P.TKDMIN) TKD = P.TKDMIN;
        a.tk[c] = TKD / P.TSTR;
    }
}

}  // namespace uc
