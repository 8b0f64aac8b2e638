// Rate coefficients and species source terms, mixed precision.
//
// Same tile structure as chem_fp64_kernel (16 warps, 32 cells per tile, the
// whole RC plane of a tile on chip), with the arithmetic split as follows:
//   FP64  the Gibbs exponents G0_k and ln Kc = sum of +-G0 over the
//         reaction's species (the equilibrium constant of the reverse rate),
//         and the assembly of each exponent (ln A + beta ln T - E/T + ln of the
//         constant factors), so that no large-argument cancellation happens
//         in single precision;
//   FP32  every exponential (range-reduced in FP64, polynomial in FP32), the
//         fall-off blend (log10, pow), the RC plane, RA = RC*prod(Y), the
//         species sums (Neumaier-compensated) and d(omega)/dY.
// The RC plane is written as FP32 ([544][npad] floats): the point-implicit
// update reads it and computes in FP64.
#pragma once
#include "uc_device.cuh"

namespace uc {

// Reaction-pair table of the mixed kernel, built at set-up from the same
// mechanism tables: logarithms of the constant factors folded per slot.
struct __align__(16) PairTabM {
    double lnakf, alf, exaf;    // forward slot: ln AKF, beta, Ea/R
    double lnc0, lnc1;          // ln(C_order / prod W) of the forward / reverse slot
    double lnaklow, allow, ealow;   // fall-off low-pressure limit (falloff != 0)
    float troe[4];
    int8_t has_rev, rut, qlen, dmole, order0, order1, tb0, tb1;
    int8_t ny0, ny1, falloff, pad0[5];
    int8_t qsp[8], qsgn[8];     // ln q = sum qsgn[t] * G0[qsp[t]]
    int8_t yk0[4], yk1[4];      // post factors Y[yk] of the two slots
};
static_assert(sizeof(PairTabM) == 128, "PairTabM layout");
constexpr int PAIRTABM_BYTES = NPAIR * (int)sizeof(PairTabM);

struct ChemMArgs {
    const DevParams *P;
    const PairTabM *tab;
    const double *tk, *rho, *y, *stmf, *stnd;
    float *rc32;                 // [544][npad] or null
    double *rc64;                // [544][npad] or null: the same values stored as doubles
    int *tile_flag;              // [ntile]: 1 if a rate of the tile leaves the FP32 range
    double *sour;                // [6][npad] or null
    double *qdsp, *qdot, *dwdy;  // outputs (any may be null)
    int n, npad, ntile;
    int *status;
    const int8_t *skip;          // optional ISKIP class per cell (see ChemArgs): tiles with one go to FP64
};

enum { SM_TKD = 0, SM_LNT, SM_INVT, SM_LNRHO, SM_LNRUT, SM_RHO, SM_LNDMOLEA, SM_TB0, SM_STMF = SM_TB0 + 11,
       SM_STND, SM_N };

constexpr size_t CHEMM_SMEM = PAIRTABM_BYTES + sizeof(float) * (size_t)(LRX * TILE + 3 * LSP * TILE) +
                              sizeof(double) * (size_t)(2 * LSP * TILE + SM_N * TILE) + 64;

// Error control of the FP32 species sums. Every term of a net rate carries at
// most UC_MIXED_TERM_ERR relative error (a few FP32 roundings of the rate
// coefficient, the fall-off factor and the Y products), so the net of species k
// is off by at most UC_MIXED_TERM_ERR * gross_k. A tile in which that bound
// exceeds UC_MIXED_OMEGA_TOL * max(|omega_k|, 1e-6 * max_j |omega_j|) for a
// species above 1e-8 mass fraction is recomputed in FP64, as are tiles with a
// rate beyond the FP32 range.
#ifndef UC_MIXED_TERM_ERR
#define UC_MIXED_TERM_ERR 2.0e-6
#endif
#ifndef UC_MIXED_OMEGA_TOL
#define UC_MIXED_OMEGA_TOL 1.0e-3
#endif

// e^x for a double argument: n = round(x/ln2) and the remainder in FP64,
// the exponential of the remainder in FP32, scaled by 2^n.
__device__ __forceinline__ float exp_split(double x)
{
    if (!(x > -110.0)) return 0.0f;                       // below the FP32 range (and NaN -> 0 handled by caller)
    if (x > 88.7) return 3.4028234663852886e38f;            // clamp at FLT_MAX
    const double n = rint(x * 1.4426950408889634);
    const double r = fma(-n, 6.93147180369123816490e-01, x) - n * 1.90821492927058770002e-10;
    return scalbnf(expf((float)r), (int)n);
}

__device__ __forceinline__ void neumaier_add(float &s, float &c, float t)
{
    const float u = s + t;
    const float a = (s - u) + t, b = (t - u) + s;
    c += fabsf(s) >= fabsf(t) ? a : b;
    s = u;
}

__global__ void __launch_bounds__(CHEM_THREADS, 1) chem_mixed_kernel(const ChemMArgs a)
{
    extern __shared__ __align__(128) unsigned char smem[];
    PairTabM *sTab = reinterpret_cast<PairTabM *>(smem);
    float *sRC = reinterpret_cast<float *>(smem + PAIRTABM_BYTES);   // [544][32]
    float *sYf = sRC + LRX * TILE;                                   // [52][32]
    float *sNet = sYf + LSP * TILE;                                  // [52][32] |W_k net_k|
    float *sGross = sNet + LSP * TILE;                               // [52][32] W_k sum |terms|
    double *sY = reinterpret_cast<double *>(sGross + LSP * TILE);    // [52][32]
    double *sG = sY + LSP * TILE;                                    // [52][32] Gibbs exponents, then HRR terms
    double *sC = sG + LSP * TILE;                                    // [SM_N][32]
    uint64_t *bar = reinterpret_cast<uint64_t *>(sC + SM_N * TILE);
    __shared__ int s_flag;
    const DevParams &P = *a.P;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    if (tid == 0) { mbar_init(bar, 1); s_flag = 0; }
    __syncthreads();
    if (tid == 0) {
        mbar_expect_tx(bar, PAIRTABM_BYTES);
        constexpr int CH = 8192;
        for (int off = 0; off < PAIRTABM_BYTES; off += CH) {
            const int bytes = PAIRTABM_BYTES - off < CH ? PAIRTABM_BYTES - off : CH;
            bulk_g2s(reinterpret_cast<unsigned char *>(sTab) + off,
                     reinterpret_cast<const unsigned char *>(a.tab) + off, bytes, bar);
        }
    }
    if (!mbar_wait_bounded(bar, 0, 1 << 20)) {
        if (tid == 0) atomicExch(a.status, ST_TMA_TIMEOUT);
        mbar_wait_bounded(bar, 0, 1 << 20);
        return;
    }
    const float RCONVf = (float)P.RCONV;

    for (int tile = blockIdx.x; tile < a.ntile; tile += gridDim.x) {
        const size_t cell = (size_t)tile * TILE + lane;
        const bool skipped = a.skip && a.skip[cell] != 0;   // the FP64 kernel redoes this tile
        // ---------------- phase 0: load
        for (int k = warp; k < LSP; k += CHEM_WARPS) {
            const double yk = a.y[(size_t)k * a.npad + cell];
            sY[k * TILE + lane] = yk;
            sYf[k * TILE + lane] = (float)yk;
        }
        if (warp == CHEM_WARPS - 1) {
            const double TKD = a.tk[cell] * P.TSTR;
            const double rho = a.rho[cell];
            sC[SM_TKD * TILE + lane] = TKD;
            sC[SM_LNT * TILE + lane] = log(TKD);
            sC[SM_INVT * TILE + lane] = 1.0 / TKD;
            sC[SM_LNRHO * TILE + lane] = log(rho);
            sC[SM_LNRUT * TILE + lane] = log((double)82.06f * TKD);
            sC[SM_RHO * TILE + lane] = rho;
            sC[SM_LNDMOLEA * TILE + lane] = log(rho * P.RSTR_WMSTR * 1.0e-06);
            sC[SM_STMF * TILE + lane] = a.stmf ? a.stmf[cell] : 0.0;
            sC[SM_STND * TILE + lane] = a.stnd ? a.stnd[cell] : 0.0;
        }
        __syncthreads();
        // ---------------- phase 1a: Gibbs exponents (FP64); Y/W rows (scratch in sRC as floats)
        {
            const double TKD = sC[SM_TKD * TILE + lane], ELOGT = sC[SM_LNT * TILE + lane];
            const double IT = sC[SM_INVT * TILE + lane];
            const int ip = TKD > UC_TPOL1 ? 7 : 0;
            const double T1 = TKD * 0.5, T2 = TKD * TKD * (1.0 / 6.0), T3 = T1 * T2, T4 = 1.2 * T1 * T3;
            for (int k = warp; k < LSP; k += CHEM_WARPS) {
                const double *c = P.poly + k * 14 + ip;
                sG[k * TILE + lane] = c[0] * (ELOGT - 1.0) + c[1] * T1 + c[2] * T2 + c[3] * T3 + c[4] * T4 - c[5] * IT + c[6];
            }
        }
        __syncthreads();
        // ---------------- phase 1b: third bodies (FP32 sums of Y/W)
        if (warp == 0) {
            float tb = 0.0f, cmp = 0.0f;
            for (int k = 0; k < LSP; ++k) neumaier_add(tb, cmp, sYf[k * TILE + lane] * (float)(1.0 / P.WM[k]));
            sC[SM_TB0 * TILE + lane] = (double)(tb + cmp);
        }
        __syncthreads();
        if (warp >= 1 && warp <= 10) {
            const int g = warp;
            double acc = sC[SM_TB0 * TILE + lane];
            const int o = P.tb_off[g];
            for (int t = 0; t < P.tb_len[g]; ++t) {
                const int k = P.tb_sp[o + t];
                const double term = (P.tb_hascoef[o + t] ? P.tb_coef[o + t] : 1.0) * sY[k * TILE + lane] / P.WM[k];
                acc = P.tb_sign[o + t] > 0 ? acc + term : acc - term;
            }
            sC[(SM_TB0 + g) * TILE + lane] = acc;
        } else if (warp == 11 && a.sour && !skipped) {
            // soot sources (ckrates.f:1337-1352); FP64, a handful of terms per cell
            const double PI = 3.1415927e+00, RSOOT = 1.9000e+03, SIGB = 1.38e-23, AVNO = 6.0232e+23;
            const double TKD = sC[SM_TKD * TILE + lane], rho = sC[SM_RHO * TILE + lane];
            const double stmf = sC[SM_STMF * TILE + lane], stnd = sC[SM_STND * TILE + lane];
            const double TBODY = sC[SM_TB0 * TILE + lane];
            const double C1ST = P.C1ST;
            double DPST = 0.0;
            if (stnd >= 1.0) DPST = pow(6.0 * stmf / (PI * RSOOT * stnd), (double)0.333333f);
            const double ASST = PI * DPST * DPST * P.RSTR * rho * stnd;
            const double SOURNU = C1ST * rho * 1.000e+04 * exp(-(2.0632e+04 / TKD)) / P.WM[21];
            const size_t np = a.npad;
            a.sour[cell] = SOURNU + C1ST * rho * ASST * 3.468e+03 * exp(-(1.2077e+04 / TKD)) / P.WM[21];
            a.sour[np + cell] = 2.0 * SOURNU * AVNO / (double)100.0f / P.WMSTR;
            a.sour[2 * np + cell] = C1ST * rho * ASST * 1.000e+04 * sqrt(TKD) * exp(-(1.9626e+04 / TKD)) / P.WM[1];
            a.sour[3 * np + cell] = (double)0.13f * C1ST * ASST * 1.060e+02 / sqrt(TKD) / P.WM[4] / TBODY;
            a.sour[4 * np + cell] = 0.5 * C1ST * ASST * 5.54e+00 / sqrt(TKD) / P.WM[3] / TBODY;
            a.sour[5 * np + cell] = 2.0 * C1ST * P.RSTR * (double)9.0f * sqrt(DPST * 6.0 * SIGB * TKD / RSOOT) * rho * rho * stnd;
        }
        __syncthreads();
        // ---------------- phase 2: reaction pairs -> RC plane (FP32)
        {
            const double ELOGT = sC[SM_LNT * TILE + lane], IT = sC[SM_INVT * TILE + lane];
            const double LNRHO = sC[SM_LNRHO * TILE + lane], LNRUT = sC[SM_LNRUT * TILE + lane];
            const float TKDf = (float)sC[SM_TKD * TILE + lane];
            const int np = P.npair_of_warp[warp];
            for (int i = 0; i < np; ++i) {
                const int p = P.pair_of_warp[warp][i];
                const PairTabM &T = sTab[p];
                const double lnkf = T.lnakf + T.alf * ELOGT - T.exaf * IT;
                double lnkr = -1.0e300;
                if (T.has_rev) {
                    double lnq = 0.0;
                    for (int t = 0; t < T.qlen; ++t) lnq += T.qsgn[t] * sG[T.qsp[t] * TILE + lane];
                    lnkr = lnkf + T.rut * LNRUT - lnq;          // AKF of a reverse slot is 1
                }
                double lafp = 0.0;                                 // ln of the fall-off blend factor
                if (T.falloff) {
                    // ckrates.f:740-794: Pr = k0 [M] / (k_inf + 1e-20), exactly as ckrates.f:770 has
                    // it (at low T the 1e-20 dominates k_inf for several reactions and keeps Pr small)
                    const double l20 = -46.051701859880914;      // ln 1e-20
                    const double lden = lnkf > l20 ? lnkf + log1p(exp(l20 - lnkf)) : l20 + log1p(exp(lnkf - l20));
                    const double lnk0m = T.lnaklow + T.allow * ELOGT - T.ealow * IT +
                                         log(sC[(SM_TB0 + T.dmole) * TILE + lane]) + sC[SM_LNDMOLEA * TILE + lane] - lden;
                    float RFACT;                                   // Troe / SRI / Lindemann factor in FP32
                    if (T.troe[0] > 0.0f) {
                        float FCLOG;
                        if (T.troe[1] == 0.0f) FCLOG = log10f(T.troe[0]);
                        else FCLOG = log10f((1.0f - T.troe[0]) * expf(-(TKDf / T.troe[1])) +
                                            T.troe[0] * expf(-(TKDf / T.troe[2])) + expf(-(T.troe[3] / TKDf)));
                        const float CPLOG = (float)(lnk0m * 0.43429448190325176) - (0.4f + 0.67f * FCLOG);
                        const float z = CPLOG / (0.75f - 1.27f * FCLOG - 0.14f * CPLOG);
                        RFACT = exp10f(FCLOG / (1.0f + z * z));
                    } else if (T.troe[0] == 0.0f) {
                        RFACT = 1.0f;
                    } else {
                        const float l = (float)(lnk0m * 0.43429448190325176);
                        const float XFACT = 1.0f / (1.0f + l * l);
                        RFACT = powf(-(T.troe[0] * expf(-(T.troe[1] / TKDf))) + expf(-(TKDf / T.troe[2])), XFACT);
                    }
                    // ln(Pr/(1+Pr) * RFACT); Pr itself can leave every floating range at low T
                    lafp = (double)logf(RFACT) - (lnk0m > 0.0 ? log1p(exp(-lnk0m)) : log1p(exp(lnk0m)) - lnk0m);
                }
                float rc0 = 0.0f, rc1 = 0.0f;
                const double e0 = lnkf + lafp + T.lnc0 + T.order0 * LNRHO;
                const double e1 = lnkr + lafp + T.lnc1 + T.order1 * LNRHO;
                // a rate beyond the FP32 range (cold cells: reverse rates up to 1e78) sends the
                // tile to the FP64 kernel
                if ((T.order0 && e0 > 85.0) || (T.order1 && T.has_rev && e1 > 85.0)) s_flag = 1;
                if (T.order0) {
                    float v = exp_split(e0);
                    if (T.tb0 >= 0) v *= (float)sC[(SM_TB0 + T.tb0) * TILE + lane];
                    for (int t = 0; t < T.ny0; ++t) v *= sYf[T.yk0[t] * TILE + lane];
                    rc0 = v;
                }
                if (T.order1 && T.has_rev) {
                    float v = exp_split(e1);
                    if (T.tb1 >= 0) v *= (float)sC[(SM_TB0 + T.tb1) * TILE + lane];
                    for (int t = 0; t < T.ny1; ++t) v *= sYf[T.yk1[t] * TILE + lane];
                    rc1 = v;
                }
                sRC[(2 * p) * TILE + lane] = rc0;
                sRC[(2 * p + 1) * TILE + lane] = rc1;
            }
        }
        __syncthreads();
        // ---------------- phase 3: RC out (FP32), species sums
        if (skipped) s_flag = 1;
        if (a.rc32 && !skipped)
            for (int r = warp; r < LRX; r += CHEM_WARPS) a.rc32[(size_t)r * a.npad + cell] = sRC[r * TILE + lane];
        if (a.rc64 && !skipped)
            for (int r = warp; r < LRX; r += CHEM_WARPS) a.rc64[(size_t)r * a.npad + cell] = (double)sRC[r * TILE + lane];
        {
            const float TKD = (float)sC[SM_TKD * TILE + lane];
            const float TKD2 = TKD * TKD, TKD3 = TKD * TKD2, TKD4 = TKD * TKD3, TKD5 = TKD * TKD4;
            const int ip = TKD > (float)UC_TPOL1 ? 7 : 0;
            const int ns = P.nspec_of_warp[warp];
            for (int s = 0; s < ns; ++s) {
                const int k = P.spec_of_warp[warp][s];
                float sum = 0.0f, cmp = 0.0f, gross = 0.0f;
                const int len = P.prd_len[k], off = P.prd_off[k];
                for (int t = 0; t < len; ++t) {
                    const unsigned code = P.prd_term[off + t];
                    if (code & 0x2000) continue;                 // SRA terms are zero
                    const int r = code & 0x1FFF;
                    float v = sRC[r * TILE + lane];
                    for (int q = 0; q < P.ra_len[r]; ++q) v *= sYf[P.ra_sp[r * 3 + q] * TILE + lane];
                    if (code & 0x4000) v *= (float)P.prd_coef[off + t];
                    neumaier_add(sum, cmp, (code & 0x8000) ? -v : v);
                    gross += fabsf(v);
                }
                const float net = sum + cmp;                      // sum over the PRD list of species k
                const float wnet = (float)P.WM[k] * net;
                sNet[k * TILE + lane] = fabsf(wnet);
                sGross[k * TILE + lane] = (float)P.WM[k] * gross;
                if (a.qdsp && !skipped) a.qdsp[(size_t)k * a.npad + cell] = -(double)(RCONVf * wnet);
                const double *pa = P.poly + k * 14 + ip;
                const float HS = ((float)pa[0] * TKD + (float)pa[1] * TKD2 * 0.5f + (float)pa[2] * TKD3 * (1.0f / 3.0f) +
                                  (float)pa[3] * TKD4 * 0.25f + (float)pa[4] * TKD5 * 0.2f + (float)pa[5]) *
                                 (float)(P.GASC / P.WM[k]);
                sG[k * TILE + lane] = (double)(wnet * HS);         // PRD*HENTH/HFO
                if (a.dwdy && !skipped) {
                    float L = 0.0f;
                    const int lo = P.loss_off[k], ll = P.loss_len[k];
                    for (int t = 0; t < ll; ++t) {
                        const int r = P.loss_term[lo + t];
                        float v = sRC[r * TILE + lane];
                        bool skipped = false;
                        for (int q = 0; q < P.ra_len[r]; ++q) {
                            const int sp = P.ra_sp[r * 3 + q];
                            if (sp == k && !skipped) { skipped = true; continue; }
                            v *= sYf[sp * TILE + lane];
                        }
                        L += v;
                    }
                    a.dwdy[(size_t)k * a.npad + cell] = -(double)(RCONVf * (float)P.WM[k] * L);
                }
            }
        }
        __syncthreads();
        // ---------------- phase 4: QDOT (compensated); tile flag
        if (warp == 0 && a.qdot && !skipped) {
            float s = 0.0f, c = 0.0f;
            for (int k = 0; k < LSP; ++k) neumaier_add(s, c, (float)sG[k * TILE + lane]);
            a.qdot[cell] = -(double)((s + c) * RCONVf);
        }
        if (warp == 1) {
            // error bound of the FP32 nets against the stated accuracy (see UC_MIXED_TERM_ERR)
            float wmax = 0.0f;
            for (int k = 0; k < LSP; ++k) wmax = fmaxf(wmax, sNet[k * TILE + lane]);
            bool bad = false;
            for (int k = 0; k < LSP; ++k) {
                const float ref = fmaxf(sNet[k * TILE + lane], 1.0e-6f * wmax);
                if (sY[k * TILE + lane] > 1.0e-8 &&
                    (double)UC_MIXED_TERM_ERR * sGross[k * TILE + lane] > (double)UC_MIXED_OMEGA_TOL * ref)
                    bad = true;
            }
            if (__any_sync(0xffffffffu, bad) && lane == 0) s_flag = 1;
        }
        __syncthreads();
        if (tid == 0) {
            a.tile_flag[tile] = s_flag;
            s_flag = 0;                 // read again only after the next tile's first barrier
        }
    }
}

}  // namespace uc
