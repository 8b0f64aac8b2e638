// Enthalpy equation on the device (src/lib/solveh.f with the coefficients of
// src/lib/spgsolv.f:174,233-1290).
//
// For an lj x li grid (J fastest, cell c = (I-1) lj + (J-1)):
//   enth_source_kernel  heat release of the start-state rate coefficients and
//                       the updated mass fractions: RA = RC * prod(Y), PRD,
//                       PROD = sum PRD, QDSP, QDOT          (solveh.f:116-1145)
//                       (two 16-warp CTAs per SM, RC read through L1)
//   enth_coef_kernel    EKT, EMU and the species-enthalpy diffusion factors
//                       RDHSP_k of every cell      (spgsolv.f:174, solveh.f:39-57)
//   enth_rhs_kernel     interior cells: coefficients ZE, ZW, ZN, ZS (hybrid
//                       convection-diffusion of EKT), RHSZ = diffusion of
//                       species enthalpy - radiation + RHO HT - DT PROD
//                       (solveh.f:58-114, 1143), PPP; written in the skewed
//                       layout of the relaxation
//   enth_relax_kernel   the point relaxation of FPZ (solveh.f:1146-1167) as the
//                       reference orders it: lexicographic Gauss-Seidel, J outer
//                       and I inner, so every pass gives the reference's iterate
//   enth_temp_kernel    T from FPZ less the kinetic energy (solveh.f:1170-1234),
//                       HT := FPZ and the residual of spgsolv.f:1304
//
// Relaxation. Cell (J, I) of a pass needs (J-1, I) and (J, I-1) of the same
// pass and (J+1, I), (J, I+1) of the previous one. One CTA runs a pass with a
// thread per interior row jj = J-2; at step s thread jj updates column
// ii = s - jj (a wavefront over the anti-diagonals), its west value in a
// register and its south value from the row below through shared memory.
// Pass p at step s reads what pass p-1 wrote at steps s and s+1, so the passes
// run as a pipeline, two steps apart: CTA p waits for the published step count
// of pass p-1. Pass values are stored skewed, index s*nj + jj, so the loads of
// a step are contiguous across the rows; a ring of R pass buffers holds them.
// A pass starts only when pass p-R+1 (the last reader of the slot it
// overwrites) has finished. Each pass sums |dFPZ| per row in I order and then
// over rows in J order (the reference keeps one running sum; the two agree to
// rounding, so the pass count can differ only when the residual lies within
// rounding of the tolerance). Passes finish in order; a pass whose residual
// meets the tolerance records itself as the stop pass, and every later pass
// drops out at its next wait. All waits are bounded (wall clock) and end on
// the error word or the stop pass.
#pragma once
#include "uc_device.cuh"

namespace uc {

// ------------------------------------------------------------------ heat release

struct EnthSrcArgs {
    const DevParams *P;
    const double *rc;          // [544][npad] start-state rate coefficients (FP64 plane)
    const float *rc32;         // [544][npad] FP32 plane of the mixed form (RCT = float)
    const int *tile_flag;      // mixed form: tiles whose RC is in the FP64 plane
    const double *tk, *y;      // start temperature; Y after the species update
    const uint8_t *hold;       // cells whose QDSP/QDOT are not written (grid boundary)
    double *qdsp, *qdot, *prod;
    int npad, ntile;
};

constexpr size_t ENTH_SRC_SMEM = (size_t)(3 * LSP + 1) * TILE * sizeof(double);

// RC is read straight from the plane (through L1: a row of the tile is read by
// the PRD lists of several species), so that shared memory holds only the
// tile's Y and the species sums and two CTAs share an SM: the loads of one
// overlap the arithmetic of the other. (Staging the tile's RC block [544][32]
// in shared memory allowed one CTA per SM: 2.98 ms for the C2 field, 3.7 % of
// DRAM bandwidth, stalled on the barriers between its load and species phases.)
template <typename RCT>
__global__ void __launch_bounds__(CHEM_THREADS, 2) enth_source_kernel(const EnthSrcArgs a)
{
    extern __shared__ __align__(16) double esm[];
    double *sY = esm;                  // [52][32]
    double *sP = sY + LSP * TILE;      // [52][32] PRD
    double *sH = sP + LSP * TILE;      // [52][32] PRD * HENTH / HFO
    double *sT = sH + LSP * TILE;      // [32] TKD
    const DevParams &P = *a.P;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const size_t np = a.npad;
    for (int tile = blockIdx.x; tile < a.ntile; tile += gridDim.x) {
        const size_t cell = (size_t)tile * TILE + lane;
        const bool f64 = sizeof(RCT) == 8 || (a.tile_flag && a.tile_flag[tile]);
        for (int k = warp; k < LSP; k += CHEM_WARPS) sY[k * TILE + lane] = a.y[(size_t)k * np + cell];
        if (warp == 0) sT[lane] = a.tk[cell] * P.TSTR;
        __syncthreads();
        {
            const double TKD = sT[lane];
            const double TKD2 = TKD * TKD, TKD3 = TKD * TKD2, TKD4 = TKD * TKD3, TKD5 = TKD * TKD4;
            const int ip = TKD > UC_TPOL1 ? 7 : 0;
            const bool out = !(a.hold && a.hold[cell]);
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
                        if (!(code & 0x2000)) {           // SRA terms are zero (solveh.f:671-676)
                            v = f64 ? __ldg(a.rc + (size_t)r * np + cell) : (double)__ldg(a.rc32 + (size_t)r * np + cell);
                            for (int q = 0; q < P.ra_len[r]; ++q) v = v * sY[P.ra_sp[r * 3 + q] * TILE + lane];
                            if (code & 0x4000) v = P.prd_coef[off + t] * v;
                        }
                        const bool neg = code & 0x8000;
                        acc = (t == 0) ? (neg ? -v : v) : (neg ? acc - v : acc + v);
                    }
                    prd = P.WM[k] * P.HFO[k] * acc;
                }
                if (out) a.qdsp[(size_t)k * np + cell] = -(P.RCONV * prd / P.HFO[k]);
                const double *pa = P.poly + k * 14 + ip;
                const double HSSP = (pa[0] * TKD + pa[1] * TKD2 / 2.0 + pa[2] * TKD3 / 3.0 + pa[3] * TKD4 / 4.0 +
                                     pa[4] * TKD5 / 5.0) / P.WM[k] * P.HCONVR;
                const double H = HSSP * P.WMSTR * P.HSTR + pa[5] / P.WM[k] * P.GASC;
                sP[k * TILE + lane] = prd;
                sH[k * TILE + lane] = prd * H / P.HFO[k];
            }
        }
        __syncthreads();
        if (warp == 0) {                      // ordered sums over the species (solveh.f:1134-1144)
            double prod = 0.0, hrr = 0.0;
            for (int k = 0; k < LSP; ++k) {
                prod = prod + sP[k * TILE + lane];
                hrr = hrr + sH[k * TILE + lane];
            }
            a.prod[cell] = prod;
            if (!(a.hold && a.hold[cell])) a.qdot[cell] = -(hrr * P.RCONV);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ EKT, RDHSP

struct EnthCoefArgs {
    const DevParams *P;
    const double *tk, *rho, *cp, *vtc, *vdf, *tmu;   // start state; cp = TCP of spgsolv.f:102-173
    double sigsp, sigh, beta2;
    double *ekt, *rdhsp;                             // [npad], [52][npad]
    int n, npad;
};

__global__ void enth_coef_kernel(const EnthCoefArgs a)
{
    const DevParams &P = *a.P;
    const size_t np = a.npad;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < (size_t)a.n; c += (size_t)gridDim.x * blockDim.x) {
        const double EKT = P.REI * (a.beta2 * a.vtc[c] / a.cp[c] + a.tmu[c] / a.sigh);   // spgsolv.f:174
        const double EMU = P.REI * P.BETA3 * a.rho[c];                                   // spgsolv.f:175
        const double TURB = P.REI * a.tmu[c] / a.sigsp;
        a.ekt[c] = EKT;
        const double TKD = a.tk[c] * P.TSTR;
        const double TKD2 = TKD * TKD, TKD3 = TKD * TKD2, TKD4 = TKD * TKD3, TKD5 = TKD * TKD4;
        const int ip = TKD > UC_TPOL1 ? 7 : 0;
        for (int k = 0; k < LSP; ++k) {                                                  // solveh.f:39-57
            const double *pa = P.poly + k * 14 + ip;
            const double HSSP = (pa[0] * TKD + pa[1] * TKD2 / 2.0 + pa[2] * TKD3 / 3.0 + pa[3] * TKD4 / 4.0 +
                                 pa[4] * TKD5 / 5.0) / P.WM[k] * P.HCONVR;
            a.rdhsp[(size_t)k * np + c] = (EMU * a.vdf[(size_t)k * np + c] + TURB - EKT) * HSSP;
        }
    }
}

// ------------------------------------------------------------------ RHSZ, Z

// coefficient rows of the skewed layout
enum { CF_RHSZ = 0, CF_PPP = 1, CF_ZN = 2, CF_ZS = 3, CF_ZE = 4, CF_ZW = 5, CF_N = 6 };

struct EnthRhsArgs {
    const DevParams *P;
    int lj, li, npad, isym;
    const double *tk, *rho, *y, *ht, *stmf, *u, *v;    // y after the species update; stmf at the start
    const double *ekt, *rdhsp, *prod;
    const double *yr, *xxs, *xxc, *yys, *yyc;
    double dt, crad, rsoot;
    double *ze, *zw, *zn, *zs, *rhsz;                 // natural layout [npad], interior cells
    double *cf, *f0s;                                 // skewed: [CF_N][plane], [plane]
};

__device__ __forceinline__ size_t skew_index(int jj, int ii, int nj) { return (size_t)(ii + jj) * nj + jj; }

__global__ void enth_rhs_kernel(const EnthRhsArgs a)
{
    const DevParams &P = *a.P;
    const int lj = a.lj, li = a.li, nj = lj - 2, ni = li - 2;
    const size_t np = a.npad, plane = (size_t)(ni + nj - 1) * nj;
    const double SYM = (double)a.isym, dt = a.dt;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < lj * li; idx += gridDim.x * blockDim.x) {
        const int j = idx % lj, i = idx / lj;
        if (j == 0 || j == lj - 1 || i == 0 || i == li - 1) continue;
        const size_t c = idx, cE = c + lj, cW = c - lj, cN = c + 1, cS = c - 1;
        const double *rho = a.rho, *ekt = a.ekt;
        // ---- enthalpy coefficients (spgsolv.f:240, 294, 350-1290: the Z lines)
        const double DTBRX = dt / a.xxc[i], DTBRY = dt / a.yyc[j];
        const double RHOUE = 0.5 * (rho[cE] + rho[c]) * a.u[cE];
        const double RHOUW = 0.5 * (rho[c] + rho[cW]) * a.u[c];
        const double RHOVN = 0.5 * (rho[cN] + rho[c]) * a.v[cN];
        const double RHOVS = 0.5 * (rho[c] + rho[cS]) * a.v[c];
        const double SYMZ = SYM * dt * 0.5 * ekt[c] / a.yr[c];
        const double DE = (ekt[cE] + ekt[c]) / a.xxs[i + 1];
        const double DW = (ekt[c] + ekt[cW]) / a.xxs[i];
        const double DN = (ekt[cN] + ekt[c]) / a.yys[j + 1];
        const double DS = (ekt[c] + ekt[cS]) / a.yys[j];
        double cv;
        cv = fabs(RHOUE); if (DE >= cv) cv = DE;
        const double ZE = DTBRX * 0.5 * (RHOUE - cv);
        cv = fabs(RHOUW); if (DW >= cv) cv = DW;
        const double ZW = DTBRX * 0.5 * (-RHOUW - cv);
        cv = fabs(RHOVN); if (DN >= cv) cv = DN;
        const double ZN = DTBRY * 0.5 * (RHOVN - cv) - SYMZ / a.yys[j + 1];
        cv = fabs(RHOVS); if (DS >= cv) cv = DS;
        const double ZS = DTBRY * 0.5 * (-RHOVS - cv) + SYMZ / a.yys[j];
        // ---- diffusion of species enthalpy (solveh.f:59-80)
        double RDHE = 0.0, RDHW = 0.0, RDHN = 0.0, RDHS = 0.0, RDHP = 0.0, TMOLE = 0.0;
        for (int k = 0; k < LSP; ++k) {
            const double *rd = a.rdhsp + (size_t)k * np;
            const double *ys = a.y + (size_t)k * np;
            const double rc = rd[c], yc = ys[c], yn = ys[cN], ysv = ys[cS];
            TMOLE = TMOLE + yc / P.WM[k];
            RDHE = RDHE + (rd[cE] + rc) * (ys[cE] - yc);
            RDHW = RDHW + (rc + rd[cW]) * (yc - ys[cW]);
            RDHN = RDHN + (rd[cN] + rc) * (yn - yc);
            RDHS = RDHS + (rc + rd[cS]) * (yc - ysv);
            RDHP = RDHP + rc * (yn - ysv);
        }
        // ---- radiation of CH4, CO2, CO, H2O and soot, 40% included (solveh.f:81-108)
        const double TKD = a.tk[c] * P.TSTR;
        const double TKDI = 1000.0 / TKD, TKDIS = TKDI * TKDI;
        const double PLANK1 = (double)6.6334f +
                              TKD * (-3.5686e-03 + TKD * (1.6682e-08 + TKD * (2.5611e-10 - 2.6558e-14 * TKD)));
        const double PLANK2 = 1.8741e+01 - TKDI * (1.2131e+02 - 2.7350e+02 * TKDI + 1.9405e+02 * TKDIS -
                                                   5.6310e+01 * TKDIS * TKDI + (double)5.81690f * TKDIS * TKDIS);
        double PLANK3;
        if (TKD <= 750.0)
            PLANK3 = (double)4.7869f +
                     TKD * (-6.953e-02 + TKD * (2.95775e-04 + TKD * (-4.25732e-07 + 2.02894e-10 * TKD)));
        else
            PLANK3 = 1.009e+01 + TKD * (-1.183e-02 + TKD * (4.7753e-06 + TKD * (-5.87209e-10 - 2.5334e-14 * TKD)));
        const double PLANK4 = -(double)0.23093f -
                              TKDI * ((double)1.12390f - (double)9.41530f * TKDI + (double)2.99880f * TKDIS -
                                      (double)0.51382f * TKDIS * TKDI + 1.86840e-05 * TKDIS * TKDIS);
        const double PLANKC = (PLANK1 * a.y[12 * np + c] / P.WM[12] + PLANK2 * a.y[9 * np + c] / P.WM[9] +
                               PLANK3 * a.y[8 * np + c] / P.WM[8] + PLANK4 * a.y[5 * np + c] / P.WM[5]) / TMOLE;
        const double T2 = TKD * TKD, T5 = T2 * TKD * T2;
        const double QRAD = a.crad * (double)0.4f *
                            (4.0 * 5.669e-08 * PLANKC * (pow(TKD, 4.0) - 8.1e+09) +
                             3.334e-04 * a.stmf[c] * (rho[c] / a.rsoot) * T5);
        double RHSZ = dt * 0.5 * ((RDHE / a.xxs[i + 1] - RDHW / a.xxs[i]) / a.xxc[i] +
                                  (RDHN / a.yys[j + 1] - RDHS / a.yys[j]) / a.yyc[j] + SYM * RDHP / a.yr[c] / a.yyc[j]) -
                      QRAD * dt;
        RHSZ = RHSZ + rho[c] * a.ht[c] - dt * a.prod[c];                    // solveh.f:1143
        const double PPP = rho[c] - (ZE + ZW + ZN + ZS);                    // solveh.f:1155
        a.ze[c] = ZE; a.zw[c] = ZW; a.zn[c] = ZN; a.zs[c] = ZS; a.rhsz[c] = RHSZ;
        const size_t k = skew_index(j - 1, i - 1, nj);
        a.cf[CF_RHSZ * plane + k] = RHSZ;
        a.cf[CF_PPP * plane + k] = PPP;
        a.cf[CF_ZN * plane + k] = ZN;
        a.cf[CF_ZS * plane + k] = ZS;
        a.cf[CF_ZE * plane + k] = ZE;
        a.cf[CF_ZW * plane + k] = ZW;
        a.f0s[k] = a.ht[c];
    }
}

// ------------------------------------------------------------------ relaxation

constexpr int RELAX_MAX_ROWS = 1024;

struct RelaxArgs {
    int lj, li, nj, ni, nstep;       // nj = lj-2 rows, ni = li-2 columns, nstep = ni + nj - 1
    const double *cf;                // [CF_N][nstep*nj] skewed coefficients
    const double *f0;                // [lj*li] FPZ on entry (natural layout; boundary values)
    const double *f0s;               // [nstep*nj] skewed interior copy of f0 (the input of pass 0)
    double *ring;                    // [R][nstep*nj] pass results
    double *rsdz;                    // [isor] residual of each pass
    int *progress, *done;            // [isor] steps published by a pass; pass finished
    int *stop_at;                    // first pass whose residual met the tolerance (isor: none)
    int *status;
    int isor, R;
    double sor1, sor2, tol, hnorm;
    long long timeout_ns;
};

__device__ __forceinline__ long long gtimer()
{
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ int ld_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(int *p, int v)
{
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Wait until *flag >= need. Returns the value seen, or -1 when the pass must
// drop out: the error word is set, a pass before p met the tolerance, or the
// wall-clock limit passed (then the error word is set here).
__device__ __noinline__ int relax_wait(const int *flag, int need, int p, int *status, const int *stop_at,
                                       long long timeout_ns)
{
    const long long t0 = gtimer();
    for (int it = 0;; ++it) {
        const int v = ld_acquire(flag);
        if (v >= need) {
            __threadfence();
            return v;
        }
        if (timeout_ns <= 0) {                  // a limit of zero: no waiting at all
            atomicCAS(status, ST_OK, ST_RELAX_TIMEOUT);
            return -1;
        }
        if ((it & 15) == 15) {
            if (ld_acquire(status) != ST_OK || ld_acquire(stop_at) < p) return -1;
            if (gtimer() - t0 > timeout_ns) {
                atomicCAS(status, ST_OK, ST_RELAX_TIMEOUT);
                return -1;
            }
            __nanosleep(32);
        }
    }
}

__global__ void __launch_bounds__(RELAX_MAX_ROWS) enth_relax_kernel(const RelaxArgs a)
{
    extern __shared__ __align__(16) double rsm[];
    double *sF = rsm;                  // [2][nj] value of the previous step, by step parity
    double *sRow = rsm + 2 * a.nj;     // [nj] row residuals
    __shared__ int s_drop[2];
    const int jj = threadIdx.x, nj = a.nj, ni = a.ni;
    const bool rowthr = jj < nj;
    const size_t plane = (size_t)a.nstep * nj;
    const double *cRH = a.cf + CF_RHSZ * plane, *cPP = a.cf + CF_PPP * plane, *cZN = a.cf + CF_ZN * plane;
    const double *cZS = a.cf + CF_ZS * plane, *cZE = a.cf + CF_ZE * plane, *cZW = a.cf + CF_ZW * plane;
    const double sor1 = a.sor1, sor2 = a.sor2;
    for (int p = blockIdx.x; p < a.isor; p += gridDim.x) {
        // ---- slot of this pass free (pass p-R+1 read it last) and no earlier stop
        if (threadIdx.x == 0) {
            int drop = 0;
            if (p - a.R + 1 >= 1 && relax_wait(a.done + (p - a.R + 1), 1, p, a.status, a.stop_at, a.timeout_ns) < 0) drop = 1;
            if (!drop && (ld_acquire(a.stop_at) < p || ld_acquire(a.status) != ST_OK)) drop = 1;
            s_drop[0] = drop;
        }
        __syncthreads();
        const int dropped_early = s_drop[0];
        __syncthreads();
        if (dropped_early) return;
        const double *prev = p == 0 ? a.f0s : a.ring + (size_t)((p - 1) % a.R) * plane;
        double *cur = a.ring + (size_t)(p % a.R) * plane;
        double fw = 0.0, res = 0.0;
        int seen = 0;                  // thread 0: steps of pass p-1 known to be published
        bool dropped = false;
        for (int s = 0; s < a.nstep; ++s) {
            if (threadIdx.x == 0) {
                int drop = 0;
                const int need = min(s + 2, a.nstep);
                if (p > 0 && seen < need) {
                    seen = relax_wait(a.progress + (p - 1), need, p, a.status, a.stop_at, a.timeout_ns);
                    if (seen < 0) drop = 1;
                }
                s_drop[s & 1] = drop;
            }
            __syncthreads();
            // steps < s of this pass are complete in every thread
            if (threadIdx.x == 0 && s > 0) {
                __threadfence();
                st_release(a.progress + p, s);
            }
            if (s_drop[s & 1]) { dropped = true; break; }
            const int ii = s - jj;
            if (rowthr && ii >= 0 && ii < ni) {
                const int j = jj + 1, i = ii + 1;
                const size_t k = (size_t)s * nj + jj;
                const double fold = __ldcg(prev + k);
                const double fn = jj == nj - 1 ? a.f0[(size_t)i * a.lj + (a.lj - 1)] : __ldcg(prev + k + nj + 1);
                const double fe = ii == ni - 1 ? a.f0[(size_t)(a.li - 1) * a.lj + j] : __ldcg(prev + k + nj);
                const double fs = jj == 0 ? a.f0[(size_t)i * a.lj] : sF[((s - 1) & 1) * nj + jj - 1];
                const double fwv = ii == 0 ? a.f0[j] : fw;
                // FNEW = SOR2 FPZ + (RHSZ - ZN FN - ZS FS - ZE FE - ZW FW) SOR1 / PPP, rounded as written
                double t = __dsub_rn(cRH[k], __dmul_rn(cZN[k], fn));
                t = __dsub_rn(t, __dmul_rn(cZS[k], fs));
                t = __dsub_rn(t, __dmul_rn(cZE[k], fe));
                t = __dsub_rn(t, __dmul_rn(cZW[k], fwv));
                const double fnew = __dadd_rn(__dmul_rn(sor2, fold), __ddiv_rn(__dmul_rn(t, sor1), cPP[k]));
                res = __dadd_rn(res, fabs(__dsub_rn(fold, fnew)));
                cur[k] = fnew;
                sF[(s & 1) * nj + jj] = fnew;
                fw = fnew;
            }
        }
        if (dropped) return;
        if (rowthr) sRow[jj] = res;
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            st_release(a.progress + p, a.nstep);
            double r = 0.0;
            for (int q = 0; q < nj; ++q) r = __dadd_rn(r, sRow[q]);
            a.rsdz[p] = r;
            // passes finish in order, so the first pass that meets the tolerance is the stop pass
            bool ok = p == 0 || relax_wait(a.done + (p - 1), 1, p, a.status, a.stop_at, a.timeout_ns) >= 0;
            if (ok) {
                if (r / a.hnorm <= a.tol) atomicMin(a.stop_at, p);
                __threadfence();
                st_release(a.done + p, 1);
            }
            s_drop[0] = ok ? 0 : 1;
        }
        __syncthreads();
        if (s_drop[0]) return;
        __syncthreads();
    }
}

// FPZ of the result pass in the natural layout; pass count as ISOR2 reports it
// (the converging pass, or isor + 1: solveh.f:1163-1167).
__global__ void enth_relax_final_kernel(const RelaxArgs a, double *fpz, int *passes)
{
    if (ld_acquire(a.status) != ST_OK) return;
    const int stop = *a.stop_at;
    const int q = stop < a.isor ? stop : a.isor - 1;
    if (blockIdx.x == 0 && threadIdx.x == 0) *passes = stop < a.isor ? stop + 1 : a.isor + 1;
    const double *src = a.ring + (size_t)(q % a.R) * ((size_t)a.nstep * a.nj);
    const int lj = a.lj, li = a.li;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < lj * li; idx += gridDim.x * blockDim.x) {
        const int j = idx % lj, i = idx / lj;
        const bool inner = !(j == 0 || j == lj - 1 || i == 0 || i == li - 1);
        fpz[idx] = inner ? src[skew_index(j - 1, i - 1, a.nj)] : a.f0[idx];
    }
}

// ------------------------------------------------------------------ temperature

struct EnthTempArgs {
    const DevParams *P;
    int lj, li, npad;
    const double *y, *fpz, *u, *v, *w;   // w may be null (no swirl)
    double *tk, *ht;                     // tk: guess in, T out; ht := fpz on the interior
    double *partial;                     // [gridDim.x] partial sums of |FPZ - HT|
    int *status;
    const int *relax_status;             // error word of the relaxation: when set, nothing is changed
};

__global__ void __launch_bounds__(256) enth_temp_kernel(const EnthTempArgs a)
{
    const DevParams &P = *a.P;
    const int lj = a.lj, li = a.li;
    __shared__ double s_part[256];
    double res = 0.0;
    const bool skip = a.relax_status && *a.relax_status != ST_OK;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; !skip && idx < lj * li; idx += gridDim.x * blockDim.x) {
        const int j = idx % lj, i = idx / lj;
        if (j == 0 || j == lj - 1 || i == 0 || i == li - 1) continue;
        const size_t c = idx;
        const double f = a.fpz[c], wc = a.w ? a.w[c] : 0.0;
        double ENTH = (f - (double)0.5f * (a.u[c] * a.u[c] + a.v[c] * a.v[c] + wc * wc)) * P.HSTR;
        for (int k = 0; k < LSP; ++k) ENTH = ENTH + a.y[(size_t)k * a.npad + c] * P.HFO[k] * P.HSTR;
        bool conv;
        a.tk[c] = temperature_at(P, a.tk[c], a.y + c, a.npad, ENTH, &conv);
        if (!conv && a.status) atomicCAS(a.status, ST_OK, ST_NEWTON_NOCONV);
        res += fabs(f - a.ht[c]);                                     // spgsolv.f:1304
        a.ht[c] = f;                                                  // spgsolv.f:1358
    }
    s_part[threadIdx.x] = res;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int t = 0; t < (int)blockDim.x; ++t) b += s_part[t];
        a.partial[blockIdx.x] = b;
    }
}

// ------------------------------------------------------------------ density

// RHONP = PBACK / (BETA1 TK RBAR), RBAR = sum Y_k / W_k (src/unicornd-mild-sd-5.f:1056-1062)
__global__ void density_kernel(const DevParams *Pp, double pback, int n, int npad, const double *tk, const double *y,
                               double *rho)
{
    const DevParams &P = *Pp;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        double rbar = 0.0;
        for (int k = 0; k < LSP; ++k) rbar = rbar + y[(size_t)k * npad + c] / P.WM[k];
        rho[c] = pback / (P.BETA1 * tk[c] * rbar);
    }
}

// edge rules of src/unicornd-mild-sd-5.f:1063-1068 (one CTA): the last column
// extrapolated linearly, then the first row copied from the second
__global__ void density_edges_kernel(int lj, int li, double *rho)
{
    const size_t last = (size_t)(li - 1) * lj;
    for (int j = threadIdx.x; j < lj; j += blockDim.x)
        rho[last + j] = 2.0 * rho[last + j - lj] - rho[last + j - 2 * (size_t)lj];
    __syncthreads();
    for (int i = threadIdx.x; i < li; i += blockDim.x) rho[(size_t)i * lj] = rho[(size_t)i * lj + 1];
}

}  // namespace uc
