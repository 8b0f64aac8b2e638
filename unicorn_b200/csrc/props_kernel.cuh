// Property kernels: Y clip + mixture-averaged transport, cp/h (FP64, or with the
// property arithmetic in FP32 for the mixed form), and temperature from
// enthalpy (FP64). Thread = cell.
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

// Omega(1,1) quartic fit CI11 in T* (main:944-952), for the pair (i, j); R is the
// arithmetic type (double: the drop-in form; float: the mixed form)
template <typename R>
__device__ __forceinline__ R ci11t(const DevParams &P, int i, int j, R TKD1, R TKD2, R TKD3, R TKD4)
{
    const int ij = i * LSP + j;
    const R TKDS = TKD1 / (R)P.ETLJ1[ij];
    const double *c = P.ci11 + ci_range((double)TKDS) * 5;
    return (R)c[0] + (R)c[1] * TKDS + (R)c[2] * TKD2 / (R)P.ETLJ2[ij] + (R)c[3] * TKD3 / (R)P.ETLJ3[ij] +
           (R)c[4] * TKD4 / (R)P.ETLJ4[ij];
}

// src/unicornd-mild-sd-5.f:821-1006 for one cell per thread. R = double is the
// drop-in form; R = float runs the polynomials, square roots and property sums
// in FP32 (the mixed form), with the clip/closure of the state in FP64.
template <typename R>
__global__ void __launch_bounds__(128) props_kernel(const PropArgs a)
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
        R X[LSP];
        int IA = 0;
        double TMASSD = 0.0;
        R TMOLE = 0;
        for (int k = 0; k < LSP - 1; ++k) {
            const double yk = a.y[k * np + c];
            if (yk < 1.0e-03) continue;
            sub[IA] = (int8_t)k;
            TMASSD = TMASSD + yk;
            X[IA] = (R)(yk / P.WM[k]);
            TMOLE = TMOLE + X[IA];
            ++IA;
        }
        int LSPT = IA + 1;
        if (LSPT >= LSP) LSPT = LSP;
        sub[LSPT - 1] = LSP - 1;
        X[LSPT - 1] = (R)((1.0 - TMASSD) / P.WM[LSP - 1]);
        TMOLE = TMOLE + X[LSPT - 1];
        const double tkd = a.tk[c];
        const R tk = (R)tkd;
        const R TKRT = sqrt(tk);
        const R TKD1 = (R)(tkd * P.TSTR);
        const R TKD2 = TKD1 * TKD1, TKD3 = TKD2 * TKD1, TKD4 = TKD3 * TKD1, TKD5 = TKD4 * TKD1;
        const int IPL1 = (double)TKD1 >= UC_TPOL1 ? 7 : 0, IPL2 = (double)TKD1 >= UC_TPOL1 ? 6 : 0;
        const R TKBP = tk * TKRT / (R)P.PBACK;
        R ATC[LSP], AMU[LSP];
        for (int i = 0; i < LSPT; ++i) {
            const int k = sub[i];
            const double *p = P.poly + k * 14 + IPL1;
            const double *q = P.om22 + k * 12 + IPL2;
            const R EUKEN = (R)(double)0.115f + (R)(double)0.354f * ((R)p[0] + (R)p[1] * TKD1 + (R)p[2] * TKD2 + (R)p[3] * TKD3 + (R)p[4] * TKD4);
            const R SIOME = (R)P.cdia[k] * (R)P.cdia[k] *
                            ((R)q[0] + (R)q[1] * TKD1 + (R)q[2] * TKD2 + (R)q[3] * TKD3 + (R)q[4] * TKD4 + (R)q[5] * TKD5);
            ATC[i] = (R)P.CONVRC * EUKEN * TKRT / (R)P.WMIK[k * LSP + k] / SIOME;
            AMU[i] = (R)P.CONVRM * TKRT * (R)P.WMIK[k * LSP + k] / SIOME;
        }
        R VTC = 0, VMU = 0;
        R VDFQ[LSP];
        for (int i = 0; i < LSPT; ++i) {
            const int k = sub[i];
            R PHIK = 0, PHDIK = 0, EFDIK = 0;
            for (int j = 0; j < LSPT; ++j) {
                if (j == i) continue;
                const int kb = sub[j];
                const int ij = k * LSP + kb;
                const R t1 = (R)1 + sqrt(ATC[i] / ATC[j]) * (R)P.WMIK[ij];
                const R t2 = (R)1 + sqrt(AMU[i] / AMU[j]) * (R)P.WMIK[ij];
                PHIK = PHIK + X[j] * (t1 * t1) / (R)P.DWMIK[ij];
                PHDIK = PHDIK + X[j] * (t2 * t2) / (R)P.DWMIK[ij];
                // binary diffusion D_ij (main:940-953); the fit value is symmetric in (i, j)
                const R CI = ci11t<R>(P, i < j ? k : kb, i < j ? kb : k, TKD1, TKD2, TKD3, TKD4);
                EFDIK = EFDIK + X[j] / ((R)P.WMCD[ij] * TKBP / CI);
            }
            VTC = VTC + ATC[i] * X[i] / (X[i] + (R)(double)1.065f * PHIK);
            VMU = VMU + AMU[i] * X[i] / (X[i] + PHDIK);
            const R AA = TMOLE - X[i];
            if ((double)AA <= 1.0e-10) {
                // DIFSP(i, LSPT): assigned above the diagonal only; the diagonal stays zero
                R d = 0;
                if (i != LSPT - 1) {
                    const int kl = sub[LSPT - 1];
                    d = (R)P.WMCD[k * LSP + kl] * TKBP / ci11t<R>(P, k, kl, TKD1, TKD2, TKD3, TKD4);
                }
                VDFQ[i] = (R)P.CONVRD * d;
            } else {
                VDFQ[i] = (R)P.CONVRD * (TMOLE - X[i]) / EFDIK;
            }
        }
        a.vtc[c] = (double)VTC;
        a.vmu[c] = (double)VMU;
        // D_k of every species (main:981-1003); N2 (never flagged in ISPQ) takes this path too
        int pos = 0;
        for (int k = 0; k < LSP; ++k) {
            R v;
            if (k < LSP - 1 && pos < LSPT - 1 && sub[pos] == k) {
                v = VDFQ[pos];
                ++pos;
            } else {
                R EFD = 0;
                for (int b = 0; b < LSPT; ++b) {
                    const int nb = sub[b];
                    const R CI = ci11t<R>(P, k, nb, TKD1, TKD2, TKD3, TKD4);
                    EFD = EFD + X[b] / ((R)P.WMCD[k * LSP + nb] * TKBP / CI);
                }
                v = (R)P.CONVRD * TMOLE / EFD;
            }
            a.vdf[k * np + c] = (double)v;
        }
    }
}

// The collision integral CI11 of the pair (i, j) in Horner form with the
// argument t = T / ETLJ1 from the reciprocal table: FP64, no division
// (the quartic in T* has alternating-sign coefficients and cancels).
__device__ __forceinline__ double ci11_horner(const DevParams &P, int ij, double TKD1)
{
    const double t = TKD1 * P.RETLJ1[ij];
    const double *c = P.ci11 + ci_range(t) * 5;
    return fma(fma(fma(fma(c[4], t, c[3]), t, c[2]), t, c[1]), t, c[0]);
}

// The mixed form of src/unicornd-mild-sd-5.f:821-1006: the per-pair work of
// the Wilke sums and of the binary diffusion sums (square roots, divisions,
// the products of each term) runs in FP32; what cancels or accumulates stays
// FP64 -- the polynomials in T (cp/R of the Eucken factor, the Omega(2,2) fit
// to T^5, the CI11 quartic, all in Horner form), the sums over species, the
// mole numbers and TMOLE - X_i, and the per-species values ATC, AMU. Every
// pair term then carries a few FP32 roundings and nothing adds them up, so
// mu, lambda and D_k stay within a few 1e-7 of the FP64 form.
__global__ void __launch_bounds__(128) props_mixed_kernel(const PropArgs a)
{
    const DevParams &P = *a.P;
    const size_t np = a.npad;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < (size_t)a.n; c += (size_t)gridDim.x * blockDim.x) {
        double TMASS = 0.0;
        for (int k = 0; k < LSP - 1; ++k) {
            double yk = a.y[k * np + c];
            if (yk < 0.0) { yk = 0.0; a.y[k * np + c] = 0.0; }
            TMASS = TMASS + yk;
        }
        a.y[(LSP - 1) * np + c] = 1.0 - TMASS;
        int8_t sub[LSP];
        double X[LSP];
        int IA = 0;
        double TMASSD = 0.0, TMOLE = 0.0;
        for (int k = 0; k < LSP - 1; ++k) {
            const double yk = a.y[k * np + c];
            if (yk < 1.0e-03) continue;
            sub[IA] = (int8_t)k;
            TMASSD = TMASSD + yk;
            X[IA] = yk / P.WM[k];
            TMOLE = TMOLE + X[IA];
            ++IA;
        }
        int LSPT = IA + 1;
        if (LSPT >= LSP) LSPT = LSP;
        sub[LSPT - 1] = LSP - 1;
        X[LSPT - 1] = (1.0 - TMASSD) / P.WM[LSP - 1];
        TMOLE = TMOLE + X[LSPT - 1];
        const double tk = a.tk[c];
        const double TKRT = sqrt(tk);
        const double TKD1 = tk * P.TSTR;
        const int IPL1 = TKD1 >= UC_TPOL1 ? 7 : 0, IPL2 = TKD1 >= UC_TPOL1 ? 6 : 0;
        const float TKBP = (float)(tk * TKRT / P.PBACK);
        double ATC[LSP], AMU[LSP];
        float ATCf[LSP], AMUf[LSP], Xf[LSP];
        for (int i = 0; i < LSPT; ++i) {
            const int k = sub[i];
            const double *p = P.poly + k * 14 + IPL1;
            const double *q = P.om22 + k * 12 + IPL2;
            const double cpr = fma(fma(fma(fma(p[4], TKD1, p[3]), TKD1, p[2]), TKD1, p[1]), TKD1, p[0]);
            const double EUKEN = (double)0.115f + (double)0.354f * cpr;
            const double om = fma(fma(fma(fma(fma(q[5], TKD1, q[4]), TKD1, q[3]), TKD1, q[2]), TKD1, q[1]), TKD1, q[0]);
            const double SIOME = P.cdia[k] * P.cdia[k] * om;
            ATC[i] = P.CONVRC * EUKEN * TKRT / P.WMIK[k * LSP + k] / SIOME;
            AMU[i] = P.CONVRM * TKRT * P.WMIK[k * LSP + k] / SIOME;
            ATCf[i] = (float)ATC[i];
            AMUf[i] = (float)AMU[i];
            Xf[i] = (float)X[i];
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
                const float w = (float)P.WMIK[ij], dw = (float)P.DWMIK[ij];
                const float t1 = 1.0f + sqrtf(ATCf[i] / ATCf[j]) * w;
                const float t2 = 1.0f + sqrtf(AMUf[i] / AMUf[j]) * w;
                PHIK += (double)(Xf[j] * (t1 * t1) / dw);
                PHDIK += (double)(Xf[j] * (t2 * t2) / dw);
                const float CI = (float)ci11_horner(P, i < j ? k * LSP + kb : kb * LSP + k, TKD1);
                EFDIK += (double)(Xf[j] * CI / ((float)P.WMCD[ij] * TKBP));
            }
            VTC = VTC + ATC[i] * X[i] / (X[i] + (double)1.065f * PHIK);
            VMU = VMU + AMU[i] * X[i] / (X[i] + PHDIK);
            const double AA = TMOLE - X[i];
            if (AA <= 1.0e-10) {
                double d = 0.0;
                if (i != LSPT - 1) {
                    const int kl = sub[LSPT - 1];
                    d = P.WMCD[k * LSP + kl] * (double)TKBP / ci11_horner(P, k * LSP + kl, TKD1);
                }
                VDFQ[i] = P.CONVRD * d;
            } else {
                VDFQ[i] = P.CONVRD * AA / EFDIK;
            }
        }
        a.vtc[c] = VTC;
        a.vmu[c] = VMU;
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
                    const float CI = (float)ci11_horner(P, k * LSP + nb, TKD1);
                    EFD += (double)(Xf[b] * CI / ((float)P.WMCD[k * LSP + nb] * TKBP));
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

// cp and h of each cell from the coefficient tables of DevParams (the polynomials of
// spgsolv.f:102-173 and solveh.f:39-57 with the divisions by W_k, by the powers' orders and
// the scale factors folded in at set-up), in Horner form: a few fused multiply-adds per
// species, so the kernel is bound by reading the 52 Y rows (the table form rounds differently
// from the reference's expression by a few units in the last place). The sums over species
// keep the reference's order.
template <typename R>
__global__ void __launch_bounds__(256) cp_h_kernel(const CpHArgs a)
{
    const DevParams &P = *a.P;
    const size_t np = a.npad;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < (size_t)a.n; c += (size_t)gridDim.x * blockDim.x) {
        const double T = a.tk[c] * P.TSTR;
        const int r = T > UC_TPOL1 ? 1 : 0;
        double TCP = 0.0, hs = 0.0;
#pragma unroll 4
        for (int k = 0; k < LSP; ++k) {
            const double yk = a.y[k * np + c];
            const double *q = P.cpc + (k * 2 + r) * 5;
            const double *e = P.hc + (k * 2 + r) * 6;
            const double cpk = fma(fma(fma(fma(q[4], T, q[3]), T, q[2]), T, q[1]), T, q[0]);
            const double hk = fma(T * fma(fma(fma(fma(e[4], T, e[3]), T, e[2]), T, e[1]), T, e[0]), 1.0, e[5]);
            TCP = TCP + cpk * yk;
            hs = hs + yk * hk;
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
    const int8_t *skip;              // optional ISKIP class: skipped cells keep T (solveh.f:1173)
};

__global__ void __launch_bounds__(128) temperature_fp64_kernel(const TempArgs a)
{
    const DevParams &P = *a.P;
    const size_t np = a.npad;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < (size_t)a.n; c += (size_t)gridDim.x * blockDim.x) {
        if (a.skip && a.skip[c]) continue;
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
