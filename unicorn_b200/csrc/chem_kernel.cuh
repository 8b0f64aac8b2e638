// Rate coefficients and species source terms, FP64 (the drop-in form).
//
// One CTA of 16 warps works on tiles of 32 cells (lane = cell), looping over
// tiles persistently. For each tile it keeps the whole rate-coefficient
// plane RC[544][32] on chip, so the 544 coefficients of a cell are never
// written to HBM unless the species update asks for them:
//   phase 0  load Y[52][32], T, rho, soot of the tile (coalesced rows)
//   phase 1  Gibbs functions exp(G_k) and Y_k/W_k rows; third-body sums;
//            soot sources                 (src/lib/ckrates.f:103-115, 643-731, 1337-1352)
//   phase 2  per reaction pair: k_f, k_r = k_f/Kc, fall-off blend, RC
//            (warp-uniform pair -> no divergence)  (ckrates.f:95-101, 116-642, 740-1333)
//   phase 3  per species: RA = RC*prod(Y), PRD sums in the reference's order,
//            QDSP, the heat-release terms, and d(omega)/dY   (solveh.f:116-1140)
//   phase 4  QDOT (ordered sum over species)                 (solveh.f:1134-1142)
// The reaction-pair table (Arrhenius, fall-off, Troe, Kc formula, RC assembly)
// is staged into shared memory once per CTA by a bulk (TMA) copy.
#pragma once
#include "uc_device.cuh"

namespace uc {

// per-cell scalar rows of the tile (shared memory)
enum { SC_TK = 0, SC_TKD, SC_LNT, SC_RHO, SC_RUT, SC_DMOLEA, SC_TB0, SC_STMF = SC_TB0 + 11, SC_STND,
       SC_N };

struct ChemArgs {
    const DevParams *P;
    const PairTab *tab;          // [NPAIR] in global memory
    const double *tk, *rho, *y, *stmf, *stnd;   // y: [52][npad]
    double *rc;                  // [544][npad] or null
    double *sour;                // [6][npad] or null
    double *qdsp, *qdot, *dwdy;  // outputs (any may be null)
    int n, npad, ntile;
    int *status;
    const int *tile_list;        // optional: only these tiles ([*tile_count] entries)
    const int *tile_count;
    // optional ISKIP class per cell (0: computed; 1: 3 <= ISKIP < 10; 2: ISKIP >= 10). Classes 1 and 2
    // keep their RC and SOUR (ckrates.f:94); class 2 keeps its omega, QDOT and d(omega)/dY too
    // (solveh.f:119), class 1 takes them from its kept RC (rc_stale, zero when null).
    const int8_t *skip;
    const double *rc_stale;
};

constexpr size_t CHEM_SMEM = PAIRTAB_BYTES + sizeof(double) * (size_t)(LRX * TILE + 2 * LSP * TILE + SC_N * TILE) + 64;

__device__ __forceinline__ double gibbs_exp(const double *a, double ELOGT, double TKD)
{
    // ckrates.f:103-115: exp(a1(lnT-1) + a2 T/2 + a3 T^2/6 + a4 T^3/12 + a5 T^4/20 - a6/T + a7)
    double TKD1 = TKD / 2.0;
    double TKD2 = TKD * TKD / 6.0;
    double TKD3 = TKD1 * TKD2;
    double TKD4 = (double)1.2f * TKD1 * TKD3;
    double g0 = a[0] * (ELOGT - 1.0) + a[1] * TKD1 + a[2] * TKD2 + a[3] * TKD3 + a[4] * TKD4 - a[5] / TKD + a[6];
    return exp(g0);
}

// Phases 1b-1c of a tile: TBODY from the Y/W rows left in sRC by phase 1a, the
// third-body groups TB001..TB010 and the soot sources (ckrates.f:643-731,
// 1337-1352). Ends with the barrier that publishes them.
template <int NW>
__device__ __forceinline__ void tile_tb_soot(const DevParams &P, const double *sRC, const double *sY, double *sC,
                                             double *sour, size_t sstride, size_t soff, int lane, int warp,
                                             bool keep_sour)
{
    const double C1ST = P.C1ST;
    // ---------------- phase 1b: TBODY (ordered sum)
    if (warp == 0) {
        double tb = sRC[lane];
        for (int k = 1; k < LSP; ++k) tb = tb + sRC[k * TILE + lane];
        sC[SC_TB0 * TILE + lane] = tb;
    }
    __syncthreads();
    // ---------------- phase 1c: third-body groups TB001..TB010; soot sources
    for (int j = (warp == 0 ? NW : warp); j <= 11; j += NW) {
        if (j <= 10) {
            const int g = j;
            double acc = sC[SC_TB0 * TILE + lane];
            const int o = P.tb_off[g];
            for (int t = 0; t < P.tb_len[g]; ++t) {
                const int k = P.tb_sp[o + t];
                const double yk = sY[k * TILE + lane];
                const double term = P.tb_hascoef[o + t] ? (P.tb_coef[o + t] * yk) / P.WM[k] : yk / P.WM[k];
                acc = P.tb_sign[o + t] > 0 ? acc + term : acc - term;
            }
            sC[(SC_TB0 + g) * TILE + lane] = acc;
        } else if (sour && !keep_sour) {
            // ckrates.f:1337-1352 (skipped cells, ISKIP >= 3, keep theirs: ckrates.f:94)
            const double PI = 3.1415927e+00, RSOOT = 1.9000e+03, SIGB = 1.38e-23, AVNO = 6.0232e+23;
            const double CMIN = (double)100.0f, CAGL = (double)9.0f;
            const double TKD = sC[SC_TKD * TILE + lane], rho = sC[SC_RHO * TILE + lane];
            const double stmf = sC[SC_STMF * TILE + lane], stnd = sC[SC_STND * TILE + lane];
            const double TBODY = sC[SC_TB0 * TILE + lane];
            double DPST = 0.0;
            if (stnd >= 1.0) DPST = pow(6.0 * stmf / (PI * RSOOT * stnd), (double)0.333333f);
            const double ASST = PI * DPST * DPST * P.RSTR * rho * stnd;
            const double SOURNU = C1ST * rho * 1.000e+04 * exp(-(2.0632e+04 / TKD)) / P.WM[21];
            sour[soff] = SOURNU + C1ST * rho * ASST * 3.468e+03 * exp(-(1.2077e+04 / TKD)) / P.WM[21];
            sour[sstride + soff] = 2.0 * SOURNU * AVNO / CMIN / P.WMSTR;
            sour[2 * sstride + soff] = C1ST * rho * ASST * 1.000e+04 * pow(TKD, (double)0.5f) * exp(-(1.9626e+04 / TKD)) / P.WM[1];
            sour[3 * sstride + soff] = (double)0.13f * C1ST * ASST * 1.060e+02 * pow(TKD, (double)-0.5f) * exp(-(0.0 / TKD)) / P.WM[4] / TBODY;
            sour[4 * sstride + soff] = (double)0.5f * C1ST * ASST * 5.54e+00 * pow(TKD, (double)-0.5f) * exp(-(0.0 / TKD)) / P.WM[3] / TBODY;
            sour[5 * sstride + soff] = 2.0 * C1ST * P.RSTR * CAGL * sqrt(DPST * 6.0 * SIGB * TKD / RSOOT) * rho * rho * stnd;
        }
    }
    __syncthreads();
}

// Phases 1a-2 of a tile: Gibbs functions, third bodies, soot sources and
// the RC plane of the tile in shared memory, with NW warps (NW divides 16:
// a warp takes the pair lists of the virtual warps w, w+NW, ...). Expects the
// tile's Y rows in sY and the scalar rows of sC; writes sRC and sG, and the
// six soot sources to sour[m*sstride + soff] when sour is not null. Ends
// before the barrier that publishes sRC.
template <int NW>
__device__ __forceinline__ void tile_rates_fp64(const DevParams &P, const PairTab *sTab, double *sRC,
                                                const double *sY, double *sG, double *sC, double *sour,
                                                size_t sstride, size_t soff, int lane, int warp,
                                                bool keep_sour = false)
{
    const double C1ST = P.C1ST, C2ND = P.C2ND, C3RD = P.C3RD;
    // ---------------- phase 1a: Gibbs functions; Y/W rows (scratch in sRC)
    {
        const double TKD = sC[SC_TKD * TILE + lane];
        const double ELOGT = sC[SC_LNT * TILE + lane];
        const int ip = TKD > UC_TPOL1 ? 7 : 0;
        for (int k = warp; k < LSP; k += NW) {
            sG[k * TILE + lane] = gibbs_exp(P.poly + k * 14 + ip, ELOGT, TKD);
            sRC[k * TILE + lane] = sY[k * TILE + lane] / P.WM[k];
        }
    }
    __syncthreads();
    tile_tb_soot<NW>(P, sRC, sY, sC, sour, sstride, soff, lane, warp, keep_sour);
    // ---------------- phase 2: reaction pairs -> RC plane
    {
        const double TKD = sC[SC_TKD * TILE + lane];
        const double ELOGT = sC[SC_LNT * TILE + lane];
        const double RUT = sC[SC_RUT * TILE + lane];
        const double rho = sC[SC_RHO * TILE + lane];
        const double CR[4] = {0.0, C1ST * rho, C2ND * (rho * rho), C3RD * (rho * rho * rho)};
        for (int vw = warp; vw < CHEM_WARPS; vw += NW)
        for (int i = 0; i < P.npair_of_warp[vw]; ++i) {
            const int p = P.pair_of_warp[vw][i];
            const PairTab &T = sTab[p];
            double kf = T.akf * exp(T.alf * ELOGT - T.exaf / TKD);
            double kr = 0.0;
            if (T.has_rev) {
                double q = sG[T.qsp[0] * TILE + lane];
                for (int t = 1; t < T.qlen; ++t) {
                    const double g = sG[T.qsp[t] * TILE + lane];
                    q = T.qdiv[t] ? q / g : q * g;
                }
                double v = T.akf_r * kf;
                if (T.rut < 0) v = v / RUT;
                else if (T.rut > 0) v = v * RUT;
                kr = v / q;
            }
            if (T.aklow != 0.0) {
                // ckrates.f:740-794 (AKLOW < 0, the Tseng form, is not used by this data)
                const double DMOLE = sC[(SC_TB0 + T.dmole) * TILE + lane] * sC[SC_DMOLEA * TILE + lane];
                const double ACTV = T.allow * ELOGT - T.ealow / TKD;
                const double AK0M = T.aklow * exp(ACTV) * DMOLE / (kf + 1.0e-20);
                double RFACT;
                if (T.troe[0] > 0.0) {
                    double FCLOG;
                    if (T.troe[1] == 0.0) FCLOG = log10(T.troe[0]);
                    else FCLOG = log10((1.0 - T.troe[0]) * exp(-(TKD / T.troe[1])) +
                                       T.troe[0] * exp(-(TKD / T.troe[2])) + exp(-(T.troe[3] / TKD)));
                    const double CPLOG = log10(AK0M) - ((double)0.4f + (double)0.67f * FCLOG);
                    const double z = CPLOG / ((double)0.75f - (double)1.27f * FCLOG - (double)0.14f * CPLOG);
                    RFACT = pow(10.0, FCLOG / (1.0 + z * z));
                } else if (T.troe[0] == 0.0) {
                    RFACT = 1.0;
                } else {
                    const double l = log10(AK0M);
                    const double XFACT = 1.0 / (1.0 + l * l);
                    RFACT = pow(-(T.troe[0] * exp(-(T.troe[1] / TKD))) + exp(-(TKD / T.troe[2])), XFACT);
                }
                const double AFP = (AK0M / (1.0 + AK0M)) * RFACT;
                kf = AFP * kf;
                kr = AFP * kr;
            }
            // RC assembly, ckrates.f:796-1333
            double rc0 = 0.0, rc1 = 0.0;
            if (T.rc_order0) {
                double v = CR[T.rc_order0];
                if (T.rc_tb0 >= 0) v = v * sC[(SC_TB0 + T.rc_tb0) * TILE + lane];
                v = v * kf;
                for (int t = 0; t < T.rc_len0; ++t)
                    v = T.rc_kind0[t] ? v * sY[T.rc_idx0[t] * TILE + lane] : v / P.WM[T.rc_idx0[t]];
                rc0 = v;
            }
            if (T.rc_order1) {
                double v = CR[T.rc_order1];
                if (T.rc_tb1 >= 0) v = v * sC[(SC_TB0 + T.rc_tb1) * TILE + lane];
                v = v * kr;
                for (int t = 0; t < T.rc_len1; ++t)
                    v = T.rc_kind1[t] ? v * sY[T.rc_idx1[t] * TILE + lane] : v / P.WM[T.rc_idx1[t]];
                rc1 = v;
            }
            sRC[(2 * p) * TILE + lane] = rc0;
            sRC[(2 * p + 1) * TILE + lane] = rc1;
        }
    }
}

__global__ void __launch_bounds__(CHEM_THREADS, 1) chem_fp64_kernel(const ChemArgs a)
{
    extern __shared__ __align__(128) unsigned char smem[];
    PairTab *sTab = reinterpret_cast<PairTab *>(smem);
    double *sRC = reinterpret_cast<double *>(smem + PAIRTAB_BYTES);   // [544][32]
    double *sY = sRC + LRX * TILE;                                    // [52][32]
    double *sG = sY + LSP * TILE;                                     // [52][32]
    double *sC = sG + LSP * TILE;                                     // [SC_N][32]
    uint64_t *bar = reinterpret_cast<uint64_t *>(sC + SC_N * TILE);
    const DevParams &P = *a.P;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    // ---- stage the reaction-pair table (bulk copy, bounded wait)
    if (tid == 0) mbar_init(bar, 1);
    __syncthreads();
    if (tid == 0) {
        mbar_expect_tx(bar, PAIRTAB_BYTES);
        constexpr int CH = 8192;
        for (int off = 0; off < PAIRTAB_BYTES; off += CH) {
            int bytes = PAIRTAB_BYTES - off < CH ? PAIRTAB_BYTES - off : CH;
            bulk_g2s(reinterpret_cast<unsigned char *>(sTab) + off,
                     reinterpret_cast<const unsigned char *>(a.tab) + off, bytes, bar);
        }
    }
    if (!mbar_wait_bounded(bar, 0, 1 << 20)) {
        if (tid == 0) atomicExch(a.status, ST_TMA_TIMEOUT);
        mbar_wait_bounded(bar, 0, 1 << 20);   // let the copy in flight land before exiting
        return;
    }

    const double RCONV = P.RCONV;

    const int nwork = a.tile_list ? *a.tile_count : a.ntile;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int tile = a.tile_list ? a.tile_list[w] : w;
        const size_t c0 = (size_t)tile * TILE;
        const size_t cell = c0 + lane;
        const int cls = a.skip ? a.skip[cell] : 0;
        const bool tile_skips = a.skip && __syncthreads_or(cls != 0);
        // ---------------- phase 0: load
        for (int k = warp; k < LSP; k += CHEM_WARPS) sY[k * TILE + lane] = a.y[(size_t)k * a.npad + cell];
        if (warp == CHEM_WARPS - 1) {
            double tk = a.tk[cell];
            double TKD = tk * P.TSTR;
            sC[SC_TK * TILE + lane] = tk;
            sC[SC_TKD * TILE + lane] = TKD;
            sC[SC_LNT * TILE + lane] = log(TKD);
            sC[SC_RUT * TILE + lane] = (double)82.06f * TKD;
            double rho = a.rho[cell];
            sC[SC_RHO * TILE + lane] = rho;
            sC[SC_DMOLEA * TILE + lane] = rho * P.RSTR / P.WMSTR * 1.0e-06;
            sC[SC_STMF * TILE + lane] = a.stmf ? a.stmf[cell] : 0.0;
            sC[SC_STND * TILE + lane] = a.stnd ? a.stnd[cell] : 0.0;
        }
        __syncthreads();
        tile_rates_fp64<CHEM_WARPS>(P, sTab, sRC, sY, sG, sC, a.sour, a.npad, cell, lane, warp, cls != 0);
        __syncthreads();
        // ---------------- phase 3: RC out (optional), species sums
        if (a.rc && cls == 0)
            for (int r = warp; r < LRX; r += CHEM_WARPS) a.rc[(size_t)r * a.npad + cell] = sRC[r * TILE + lane];
        if (tile_skips) {
            // a skipped cell's omega comes from the RC it kept (solveh.f:116-1145 reads RC as it is)
            if (cls == 1)
                for (int r = warp; r < LRX; r += CHEM_WARPS)
                    sRC[r * TILE + lane] = a.rc_stale ? a.rc_stale[(size_t)r * a.npad + cell] : 0.0;
            __syncthreads();
        }
        if (!a.qdsp && !a.qdot && !a.dwdy) continue;      // RC and SOUR only: no species sums (uniform branch)
        const bool put = cls < 2;
        {
            const double TKD = sC[SC_TKD * TILE + lane];
            const double TKD2 = TKD * TKD, TKD3 = TKD * TKD2, TKD4 = TKD * TKD3, TKD5 = TKD * TKD4;
            const int ip = TKD > UC_TPOL1 ? 7 : 0;
            const int ns = P.nspec_of_warp[warp];
            for (int s = 0; s < ns; ++s) {
                const int k = P.spec_of_warp[warp][s];
                double prd = 0.0;
                const int len = P.prd_len[k];
                if (len > 0) {
                    const int off = P.prd_off[k];
                    double acc = 0.0;
                    for (int t = 0; t < len; ++t) {
                        const unsigned code = P.prd_term[off + t];
                        const int r = code & 0x1FFF;
                        double v = 0.0;
                        if (!(code & 0x2000)) {           // SRA terms are zero
                            v = sRC[r * TILE + lane];
                            for (int q = 0; q < P.ra_len[r]; ++q) v = v * sY[P.ra_sp[r * 3 + q] * TILE + lane];
                            if (code & 0x4000) v = P.prd_coef[off + t] * v;
                        }
                        const bool neg = code & 0x8000;
                        acc = (t == 0) ? (neg ? -v : v) : (neg ? acc - v : acc + v);
                    }
                    prd = P.WM[k] * P.HFO[k] * acc;
                }
                if (a.qdsp && put) a.qdsp[(size_t)k * a.npad + cell] = -(RCONV * prd / P.HFO[k]);
                // species enthalpy (solveh.f:39-57) for the heat-release sum
                const double *pa = P.poly + k * 14 + ip;
                const double HSSP = (pa[0] * TKD + pa[1] * TKD2 / 2.0 + pa[2] * TKD3 / 3.0 + pa[3] * TKD4 / 4.0 +
                                     pa[4] * TKD5 / 5.0) / P.WM[k] * P.HCONVR;
                const double H = HSSP * P.WMSTR * P.HSTR + pa[5] / P.WM[k] * P.GASC;
                sG[k * TILE + lane] = prd * H / P.HFO[k];
                if (a.dwdy && put) {
                    double L = 0.0;
                    const int lo = P.loss_off[k], ll = P.loss_len[k];
                    for (int t = 0; t < ll; ++t) {
                        const int r = P.loss_term[lo + t];
                        double v = sRC[r * TILE + lane];
                        bool skipped = false;
                        for (int q = 0; q < P.ra_len[r]; ++q) {
                            const int sp = P.ra_sp[r * 3 + q];
                            if (sp == k && !skipped) { skipped = true; continue; }
                            v = v * sY[sp * TILE + lane];
                        }
                        L = L + v;
                    }
                    a.dwdy[(size_t)k * a.npad + cell] = -(RCONV * P.WM[k] * L);
                }
            }
        }
        __syncthreads();
        // ---------------- phase 4: QDOT
        if (warp == 0 && a.qdot && put) {
            double hrr = 0.0;
            for (int k = 0; k < LSP; ++k) hrr = hrr + sG[k * TILE + lane];
            a.qdot[cell] = -(hrr * RCONV);
        }
        // the next tile's phase-0 barrier orders these reads before sG is rewritten
    }
}

}  // namespace uc

namespace uc {
// List of the tiles whose flag is set (one CTA; order of the tile index).
__global__ void compact_tiles_kernel(const int *flag, int ntile, int *list, int *count)
{
    __shared__ int s_base;
    if (threadIdx.x == 0) s_base = 0;
    __syncthreads();
    for (int t0 = 0; t0 < ntile; t0 += blockDim.x) {
        const int t = t0 + threadIdx.x;
        const int f = (t < ntile) ? flag[t] : 0;
        const unsigned m = __ballot_sync(0xffffffffu, f);
        __shared__ int s_warp[32];
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        if (lane == 0) s_warp[w] = __popc(m);
        __syncthreads();
        if (threadIdx.x == 0) {
            int acc = s_base;
            for (int i = 0; i < (int)(blockDim.x >> 5); ++i) { const int c = s_warp[i]; s_warp[i] = acc; acc += c; }
            s_base = acc;
        }
        __syncthreads();
        if (f) list[s_warp[w] + __popc(m & ((1u << lane) - 1))] = t;
        __syncthreads();
    }
    if (threadIdx.x == 0) *count = s_base;
}
}  // namespace uc
