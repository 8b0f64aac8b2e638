// Batched stiff point-implicit integration of independent cells (FP64, or FP32 rates with the FP64 update).
//
// Each cell is advanced over dt by n_sub sub-steps of dt/n_sub; every
// sub-step is the reference's own chain for a one-cell field: the rate
// coefficients (src/lib/ckrates.f), the point-implicit species update with
// its closure (src/lib/solvesp.f; the cell converges on its own residual,
// SPNORM = LSP-1, no face terms), T from the cell's constant total enthalpy
// (src/lib/solveh.f:1186-1234) and rho from the ideal gas at the cell's
// pressure (src/unicornd-mild-sd-5.f:1056-1062).
//
// n_sub comes from the cell's chemical time scale (nsub_kernel) and spans
// 1..~200, so the cost per cell is very uneven. The cells are ordered by
// n_sub (a stable counting sort, longest first) and a persistent kernel, one
// CTA per SM, takes 32-cell tiles from an atomic work queue: tiles hold cells
// of equal or neighbouring n_sub, and the longest tiles start first.
//
// Per tile the CTA keeps everything on chip: the reaction-pair table (one
// bulk copy per CTA), the tile's RC plane [544][32], Y, Y at the sub-step
// start and the update's scratch. The rates of a sub-step run on all NW
// warps (the phases of chem_fp64_kernel); the update program, the closure
// and the Newton for T run on warp 0 (lane = cell) with RC read from shared
// memory.
#pragma once
#include "chem_kernel.cuh"
#include "chem_mixed_kernel.cuh"
#include "generated/update_program.cuh"

namespace uc {

// The rate coefficients of a tile in the mixed form of chem_mixed_kernel (FP64
// Gibbs exponents, ln Kc and exponent assembly; FP32 exponentials, fall-off
// blend and RC products), stored as doubles in sRC so that the FP64 update reads
// them unchanged; third bodies and soot sources as in the FP64 form. Reads the
// scalar rows of sC (SC_*), uses sG as scratch for the Gibbs exponents and the
// mixed pair table in global memory. Returns, uniformly over the block, whether
// a rate of the tile left the FP32 range (the caller then recomputes the tile
// in FP64).
template <int NW>
__device__ bool tile_rates_mixed(const DevParams &P, const PairTabM *tabm, double *sRC, const double *sY, double *sG,
                                 double *sC, double *sour, size_t sstride, size_t soff, int lane, int warp)
{
    {   // phase 1a: Gibbs exponents (FP64) and the Y/W rows
        const double TKD = sC[SC_TKD * TILE + lane], ELOGT = sC[SC_LNT * TILE + lane];
        const double IT = 1.0 / TKD;
        const int ip = TKD > UC_TPOL1 ? 7 : 0;
        const double T1 = TKD * 0.5, T2 = TKD * TKD * (1.0 / 6.0), T3 = T1 * T2, T4 = 1.2 * T1 * T3;
        for (int k = warp; k < LSP; k += NW) {
            const double *c = P.poly + k * 14 + ip;
            sG[k * TILE + lane] = c[0] * (ELOGT - 1.0) + c[1] * T1 + c[2] * T2 + c[3] * T3 + c[4] * T4 - c[5] * IT + c[6];
            sRC[k * TILE + lane] = sY[k * TILE + lane] / P.WM[k];
        }
    }
    __syncthreads();
    tile_tb_soot<NW>(P, sRC, sY, sC, sour, sstride, soff, lane, warp, false);
    bool out = false;
    {   // phase 2: reaction pairs -> RC (FP32 arithmetic, stored as doubles)
        const double TKD = sC[SC_TKD * TILE + lane], ELOGT = sC[SC_LNT * TILE + lane], IT = 1.0 / TKD;
        const double LNRHO = log(sC[SC_RHO * TILE + lane]), LNRUT = log(sC[SC_RUT * TILE + lane]);
        const double LNDMOLEA = log(sC[SC_DMOLEA * TILE + lane]);
        const float TKDf = (float)TKD;
        for (int vw = warp; vw < CHEM_WARPS; vw += NW)
        for (int i = 0; i < P.npair_of_warp[vw]; ++i) {
            const int p = P.pair_of_warp[vw][i];
            const PairTabM &T = tabm[p];
            const double lnkf = T.lnakf + T.alf * ELOGT - T.exaf * IT;
            double lnkr = -1.0e300;
            if (T.has_rev) {
                double lnq = 0.0;
                for (int t = 0; t < T.qlen; ++t) lnq += T.qsgn[t] * sG[T.qsp[t] * TILE + lane];
                lnkr = lnkf + T.rut * LNRUT - lnq;
            }
            double lafp = 0.0;
            if (T.falloff) {
                const double l20 = -46.051701859880914;      // ln 1e-20 (ckrates.f:770)
                const double lden = lnkf > l20 ? lnkf + log1p(exp(l20 - lnkf)) : l20 + log1p(exp(lnkf - l20));
                const double lnk0m = T.lnaklow + T.allow * ELOGT - T.ealow * IT +
                                     log(sC[(SC_TB0 + T.dmole) * TILE + lane]) + LNDMOLEA - lden;
                float RFACT;
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
                lafp = (double)logf(RFACT) - (lnk0m > 0.0 ? log1p(exp(-lnk0m)) : log1p(exp(lnk0m)) - lnk0m);
            }
            float rc0 = 0.0f, rc1 = 0.0f;
            const double e0 = lnkf + lafp + T.lnc0 + T.order0 * LNRHO;
            const double e1 = lnkr + lafp + T.lnc1 + T.order1 * LNRHO;
            if ((T.order0 && e0 > 85.0) || (T.order1 && T.has_rev && e1 > 85.0)) out = true;
            if (T.order0) {
                float v = exp_split(e0);
                if (T.tb0 >= 0) v *= (float)sC[(SC_TB0 + T.tb0) * TILE + lane];
                for (int t = 0; t < T.ny0; ++t) v *= (float)sY[T.yk0[t] * TILE + lane];
                rc0 = v;
            }
            if (T.order1 && T.has_rev) {
                float v = exp_split(e1);
                if (T.tb1 >= 0) v *= (float)sC[(SC_TB0 + T.tb1) * TILE + lane];
                for (int t = 0; t < T.ny1; ++t) v *= (float)sY[T.yk1[t] * TILE + lane];
                rc1 = v;
            }
            sRC[(2 * p) * TILE + lane] = (double)rc0;
            sRC[(2 * p + 1) * TILE + lane] = (double)rc1;
        }
    }
    return __syncthreads_or(out) != 0;
}

struct IntArgs {
    const DevParams *P;
    const PairTab *tab;
    const PairTabM *tabm;            // the mixed form's pair table (global memory)
    double *tk, *rho, *y, *soot;     // state, updated in place: [npad], [npad], [52][npad], [2][npad]
    const double *pnd;               // p / PSTR per cell [npad]
    const int *nsub;                 // sub-steps per cell [npad]
    const int *order;                // [npad]: position -> cell (sorted by n_sub), or null (identity)
    int *next_tile;                  // work-queue counter, zero at launch
    int *passes;                     // [npad] out: update passes summed over the sub-steps
    int *status;
    double dt, sor1, tol;
    int isor, n, npad, ntile;
};

constexpr size_t INT_SMEM =
    PAIRTAB_BYTES + sizeof(double) * (size_t)(LRX * TILE + 3 * LSP * TILE + SC_N * TILE + 6 * TILE) + 64;
static_assert(INT_SMEM <= 232448, "integrator tile does not fit in shared memory");

// Total enthalpy of a cell at its own temperature, in the units of ENTH in
// solveh.f:1186-1205; y has stride ys between species.
__device__ __forceinline__ double enthalpy_total(const DevParams &P, double tk, const double *y, int ys)
{
    const double TKD = tk * P.TSTR;
    const int ip = TKD > UC_TPOL1 ? 7 : 0;
    double A1 = 0.0, A2 = 0.0, A3 = 0.0, A4 = 0.0, A5 = 0.0, A6 = 0.0;
    for (int k = 0; k < LSP; ++k) {
        const double *a = P.poly + k * 14 + ip;
        const double yk = y[k * ys];
        A1 = A1 + a[0] * yk / P.WM[k];
        A2 = A2 + a[1] * yk / P.WM[k] / 2.0;
        A3 = A3 + a[2] * yk / P.WM[k] / 3.0;
        A4 = A4 + a[3] * yk / P.WM[k] / 4.0;
        A5 = A5 + a[4] * yk / P.WM[k] / 5.0;
        A6 = A6 + a[5] * yk / P.WM[k];
    }
    return ((A1 + (A2 + (A3 + (A4 + A5 * TKD) * TKD) * TKD) * TKD) * TKD + A6) * P.GASC / P.WMSTR;
}

// Newton for T at total enthalpy ENTH (solveh.f:1186-1234). Returns tk;
// sets *conv to false if 100 iterations did not meet the step tolerance.
__device__ __forceinline__ double temperature_at(const DevParams &P, double tk, const double *y, int ys, double ENTH,
                                                 bool *conv)
{
    int IPL = 0;
    double TPOLY = UC_TPOL1;
    double TKD = tk * P.TSTR;
    double A1, A2, A3, A4, A5, A6;
    for (int guard = 0; guard < 3; ++guard) {
        if (TKD > TPOLY) TKD = TPOLY / 2.0;
        A1 = A2 = A3 = A4 = A5 = A6 = 0.0;
        for (int k = 0; k < LSP; ++k) {
            const double *p = P.poly + k * 14 + IPL;
            const double yk = y[k * ys];
            A1 = A1 + p[0] * yk / P.WM[k];
            A2 = A2 + p[1] * yk / P.WM[k] / 2.0;
            A3 = A3 + p[2] * yk / P.WM[k] / 3.0;
            A4 = A4 + p[3] * yk / P.WM[k] / 4.0;
            A5 = A5 + p[4] * yk / P.WM[k] / 5.0;
            A6 = A6 + p[5] * yk / P.WM[k];
        }
        const double FUNT =
            ((A1 + (A2 + (A3 + (A4 + A5 * TPOLY) * TPOLY) * TPOLY) * TPOLY) * TPOLY + A6) * P.GASC / P.WMSTR - ENTH;
        if (FUNT >= 1.0e-07) break;
        if (IPL >= 7) break;
        IPL = 7;
        if (TKD <= TPOLY) TKD = UC_TPOL2 / 2.0;
        TPOLY = UC_TPOL2;
    }
    *conv = false;
    for (int it = 1; it <= 100; ++it) {
        const double DTKD = ((A1 + (A2 + (A3 + (A4 + A5 * TKD) * TKD) * TKD) * TKD) * TKD + A6 - ENTH * P.WMSTR / P.GASC) /
                            (A1 + (2.0 * A2 + (3.0 * A3 + (4.0 * A4 + 5.0 * A5 * TKD) * TKD) * TKD) * TKD);
        if (fabs(DTKD) <= (double)0.001f) { *conv = true; break; }
        TKD = TKD - DTKD;
    }
    if (TKD > UC_TPOL2) TKD = UC_TPOL2;
    if (TKD < P.TKDMIN) TKD = P.TKDMIN;
    return TKD / P.TSTR;
}

// Sub-step count per cell from the omega of the start state (QDSP rows):
// x = max over Y_k > y_tau of dt*|QDSP_k|/(RCONV*rho*Y_k), n_sub = clamp(ceil(x/c_tau), 1, nsub_max).
__global__ void nsub_kernel(const DevParams *Pp, const double *rho, const double *y, const double *qdsp, int n, int npad,
                            double dt, double c_tau, double y_tau, int nsub_max, int *nsub)
{
    const DevParams &P = *Pp;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < npad; c += gridDim.x * blockDim.x) {
        double x = 0.0;
        for (int k = 0; k < LSP; ++k) {
            const double yk = y[(size_t)k * npad + c];
            if (yk > y_tau) {
                const double v = dt * fabs(qdsp[(size_t)k * npad + c]) / (P.RCONV * rho[c] * yk);
                if (!(v <= x)) x = v;
            }
        }
        const double m = ceil(x / c_tau);
        nsub[c] = (m != m || m >= (double)nsub_max) ? nsub_max : (m < 1.0 ? 1 : (int)m);
    }
}

// Total enthalpy of each cell of a field (held while the composition changes)
__global__ void hold_enthalpy_kernel(const DevParams *Pp, const double *tk, const double *y, int npad, double *enth)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < npad; c += gridDim.x * blockDim.x)
        enth[c] = enthalpy_total(*Pp, tk[c], y + c, npad);
}

// T from the held total enthalpy and the current Y (solveh.f:1186-1234), then rho
// from the ideal gas at the cell pressure (main:1056-1062); the first *nlive cells when nlive is given,
// else all npad
__global__ void temperature_held_kernel(const DevParams *Pp, const double *enth, const double *y, const double *pnd,
                                        int npad, double *tk, double *rho, int *status, const int *nlive = nullptr)
{
    const DevParams &P = *Pp;
    const int nc = nlive ? *nlive : npad;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        bool conv;
        const double t = temperature_at(P, tk[c], y + c, npad, enth[c], &conv);
        if (!conv && status) atomicCAS(status, ST_OK, ST_NEWTON_NOCONV);
        double rbar = 0.0;
        for (int k = 0; k < LSP; ++k) rbar = rbar + y[(size_t)k * npad + c] / P.WM[k];
        tk[c] = t;
        rho[c] = pnd[c] / (P.BETA1 * t * rbar);
    }
}

// ---- stable counting sort of positions by n_sub, largest first.
// Chunk j of SORT_CHUNK cells is owned by CTA j; key = nsub_max - n_sub.
constexpr int SORT_CHUNK = 4096;
constexpr int SORT_MAXBIN = 1024;

__global__ void sort_count_kernel(const int *nsub, int n, int nsub_max, int nchunk, int *hist)
{
    __shared__ int h[SORT_MAXBIN + 1];
    const int j = blockIdx.x;
    for (int b = threadIdx.x; b <= nsub_max; b += blockDim.x) h[b] = 0;
    __syncthreads();
    const int c0 = j * SORT_CHUNK, c1 = min(n, c0 + SORT_CHUNK);
    for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) atomicAdd(&h[nsub_max - nsub[c]], 1);
    __syncthreads();
    for (int b = threadIdx.x; b <= nsub_max; b += blockDim.x) hist[(size_t)b * nchunk + j] = h[b];
}

// Exclusive scan of hist in (bin, chunk) order, in place; one CTA.
__global__ void sort_scan_kernel(int *hist, int total)
{
    __shared__ int s_carry;
    __shared__ int s_warp[32];
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int base = 0; base < total; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int v = i < total ? hist[i] : 0;
        int incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) s_warp[w] = incl;
        __syncthreads();
        if (threadIdx.x == 0) {
            int acc = 0;
            for (int q = 0; q < nw; ++q) { const int t = s_warp[q]; s_warp[q] = acc; acc += t; }
        }
        __syncthreads();
        const int excl = s_carry + s_warp[w] + incl - v;
        if (i < total) hist[i] = excl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) s_carry = excl + v;
        __syncthreads();
    }
}

// Scatter: one warp per chunk walks its cells in index order (stable).
__global__ void sort_scatter_kernel(const int *nsub, int n, int npad, int nsub_max, int nchunk, const int *offs,
                                    int *order)
{
    __shared__ int off[SORT_MAXBIN + 1];
    const int j = blockIdx.x, lane = threadIdx.x;
    for (int b = lane; b <= nsub_max; b += 32) off[b] = offs[(size_t)b * nchunk + j];
    __syncwarp();
    const int c0 = j * SORT_CHUNK, c1 = min(n, c0 + SORT_CHUNK);
    for (int base = c0; base < c1; base += 32) {
        const int c = base + lane;
        const bool v = c < c1;
        const int key = v ? nsub_max - nsub[c] : -1;
        const unsigned act = __ballot_sync(0xffffffffu, v);
        const unsigned peers = __match_any_sync(0xffffffffu, key) & act;
        const int rank = __popc(peers & ((1u << lane) - 1));
        int pos = 0;
        if (v) pos = off[key] + rank;
        __syncwarp();
        if (v && rank == 0) off[key] += __popc(peers);
        __syncwarp();
        if (v) order[pos] = c;
    }
    // positions n..npad-1 keep the padding cells
    if (j == 0)
        for (int c = n + lane; c < npad; c += 32) order[c] = c;
}

// ---- rounds form: the cells in n_sub order (longest first) advance one sub-step per round; round r
// (0-based) advances the cells with n_sub > r, a prefix of that order. After the sort's scan, hist[b * nchunk]
// counts the cells whose key nsub_max - n_sub is below b, so round r has hist[(nsub_max - r) * nchunk] cells.
__global__ void round_counts_kernel(const int *hist, int nchunk, int nsub_max, int *cells, int *tiles)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nsub_max; r += gridDim.x * blockDim.x) {
        const int c = hist[(size_t)(nsub_max - r) * nchunk];
        cells[r] = c;
        tiles[r] = (c + TILE - 1) / TILE;
    }
}

__global__ void iota_kernel(int *v, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

// The state of the rounds form, position by position: y [52][npad], tk, rho, pnd, soot [2][npad], enth in
// doubles; nsub, passes (summed over the sub-steps), last (passes of the last sub-step) and ord (the cell at
// the position) in ints. Two such buffers alternate: between rounds the live cells are re-ordered.
struct RoundState {
    double *y, *tk, *rho, *pnd, *soot, *enth;
    int *nsub, *passes, *last, *ord;
};

// The state in n_sub order: position pos holds cell order[pos] (pos < n; the padding cells keep their place)
__global__ void gather_state_kernel(const int *order, int n, int npad, const double *y, const double *tk,
                                    const double *rho, const double *pnd, const double *soot, const int *nsub,
                                    RoundState d)
{
    for (int pos = blockIdx.x * blockDim.x + threadIdx.x; pos < npad; pos += gridDim.x * blockDim.x) {
        const int c = pos < n ? order[pos] : pos;
        for (int k = 0; k < LSP; ++k) d.y[(size_t)k * npad + pos] = y[(size_t)k * npad + c];
        d.tk[pos] = tk[c];
        d.rho[pos] = rho[c];
        d.pnd[pos] = pnd[c];
        d.soot[pos] = soot[c];
        d.soot[npad + pos] = soot[(size_t)npad + c];
        d.nsub[pos] = nsub[c];
        d.passes[pos] = 0;
        d.last[pos] = 0;
        d.ord[pos] = c;
    }
}

// Sort key of the positions of round r for round r + 1: the cells that go on (n_sub > r + 1) by the passes
// their last sub-step took, most first (a cell's pass count changes little from one sub-step to the next,
// so warps then hold cells that stop together), the others after them.
constexpr int ROUND_KEYS = 102;            // 0..99: 100 - min(passes, 100) of a live cell; 101: done
__global__ void round_key_kernel(const int *nsub, const int *last, const int *nlive, int r, int *key)
{
    const int n = *nlive;
    for (int pos = blockIdx.x * blockDim.x + threadIdx.x; pos < n; pos += gridDim.x * blockDim.x)
        key[pos] = nsub[pos] > r + 1 ? 100 - min(max(last[pos], 1), 100) : ROUND_KEYS - 1;
}

// Stable counting sort of the first *nlive keys (chunks of SORT_CHUNK; hist [nbins][nchunk], scanned by
// sort_scan_kernel in between): perm[new position] = old position.
__global__ void key_count_kernel(const int *key, const int *nlive, int nbins, int nchunk, int *hist)
{
    __shared__ int h[SORT_MAXBIN];
    const int j = blockIdx.x, n = *nlive;
    for (int b = threadIdx.x; b < nbins; b += blockDim.x) h[b] = 0;
    __syncthreads();
    const int c0 = j * SORT_CHUNK, c1 = min(n, c0 + SORT_CHUNK);
    for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) atomicAdd(&h[key[c]], 1);
    __syncthreads();
    for (int b = threadIdx.x; b < nbins; b += blockDim.x) hist[(size_t)b * nchunk + j] = h[b];
}

__global__ void key_scatter_kernel(const int *key, const int *nlive, int nbins, int nchunk, const int *offs,
                                   int *perm)
{
    __shared__ int off[SORT_MAXBIN];
    const int j = blockIdx.x, lane = threadIdx.x, n = *nlive;
    for (int b = lane; b < nbins; b += 32) off[b] = offs[(size_t)b * nchunk + j];
    __syncwarp();
    const int c0 = j * SORT_CHUNK, c1 = min(n, c0 + SORT_CHUNK);
    for (int base = c0; base < c1; base += 32) {
        const int c = base + lane;
        const bool v = c < c1;
        const int k = v ? key[c] : -1;
        const unsigned act = __ballot_sync(0xffffffffu, v);
        const unsigned peers = __match_any_sync(0xffffffffu, k) & act;
        const int rank = __popc(peers & ((1u << lane) - 1));
        int pos = 0;
        if (v) pos = off[k] + rank;
        __syncwarp();
        if (v && rank == 0) off[k] += __popc(peers);
        __syncwarp();
        if (v) perm[pos] = c;
    }
}

// d[pos] = s[perm[pos]] for the first *nlive positions, d[pos] = s[pos] beyond
__global__ void permute_state_kernel(const int *perm, const int *nlive, int npad, RoundState s, RoundState d)
{
    const int n = *nlive;
    for (int pos = blockIdx.x * blockDim.x + threadIdx.x; pos < npad; pos += gridDim.x * blockDim.x) {
        const int q = pos < n ? perm[pos] : pos;
        for (int k = 0; k < LSP; ++k) d.y[(size_t)k * npad + pos] = s.y[(size_t)k * npad + q];
        d.tk[pos] = s.tk[q];
        d.rho[pos] = s.rho[q];
        d.pnd[pos] = s.pnd[q];
        d.soot[pos] = s.soot[q];
        d.soot[npad + pos] = s.soot[npad + q];
        d.enth[pos] = s.enth[q];
        d.nsub[pos] = s.nsub[q];
        d.passes[pos] = s.passes[q];
        d.last[pos] = s.last[q];
        d.ord[pos] = s.ord[q];
    }
}

// back to cell order (the first n positions)
__global__ void scatter_state_kernel(int n, int npad, RoundState s, double *y, double *tk, double *rho,
                                     double *soot, int *passes)
{
    for (int pos = blockIdx.x * blockDim.x + threadIdx.x; pos < n; pos += gridDim.x * blockDim.x) {
        const int c = s.ord[pos];
        for (int k = 0; k < LSP; ++k) y[(size_t)k * npad + c] = s.y[(size_t)k * npad + pos];
        tk[c] = s.tk[pos];
        rho[c] = s.rho[pos];
        soot[c] = s.soot[pos];
        soot[(size_t)npad + c] = s.soot[npad + pos];
        passes[c] = s.passes[pos];
    }
}

// MIXED: the rates of every sub-step in the mixed form (tile_rates_mixed; a tile with a rate beyond the
// FP32 range is recomputed in FP64), the update, closure and Newton in FP64 as in the FP64 form.
template <int NW, bool MIXED>
__global__ void __launch_bounds__(NW * 32, 1) integrate_fp64_kernel(const IntArgs a)
{
    extern __shared__ __align__(128) unsigned char smem[];
    PairTab *sTab = reinterpret_cast<PairTab *>(smem);
    double *sRC = reinterpret_cast<double *>(smem + PAIRTAB_BYTES);   // [544][32]
    double *sY = sRC + LRX * TILE;                                    // [52][32] current Y (YO)
    double *sYN = sY + LSP * TILE;                                    // [52][32] Gibbs scratch / YN
    double *sY0 = sYN + LSP * TILE;                                   // [52][32] Y at the sub-step start
    double *sC = sY0 + LSP * TILE;                                    // [SC_N][32]
    double *sS = sC + SC_N * TILE;                                    // [6][32] soot sources
    uint64_t *bar = reinterpret_cast<uint64_t *>(sS + 6 * TILE);
    __shared__ int s_tile, s_smax;
    const DevParams &P = *a.P;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    if (tid == 0) mbar_init(bar, 1);
    __syncthreads();
    if (tid == 0) {
        mbar_expect_tx(bar, PAIRTAB_BYTES);
        constexpr int CH = 8192;
        for (int off = 0; off < PAIRTAB_BYTES; off += CH) {
            const int bytes = PAIRTAB_BYTES - off < CH ? PAIRTAB_BYTES - off : CH;
            bulk_g2s(reinterpret_cast<unsigned char *>(sTab) + off, reinterpret_cast<const unsigned char *>(a.tab) + off,
                     bytes, bar);
        }
    }
    if (!mbar_wait_bounded(bar, 0, 1 << 20)) {
        if (tid == 0) atomicExch(a.status, ST_TMA_TIMEOUT);
        mbar_wait_bounded(bar, 0, 1 << 20);
        return;
    }
    const size_t np = a.npad;
    const double sor1 = a.sor1, sor2 = 1.0 - a.sor1;

    for (;;) {
        if (tid == 0) s_tile = atomicAdd(a.next_tile, 1);
        __syncthreads();
        const int tile = s_tile;
        if (tile >= a.ntile) break;
        const int pos = tile * TILE + lane;
        size_t cell = a.order ? (size_t)a.order[pos] : (size_t)pos;
        if (cell >= (size_t)a.npad) {          // a broken order: keep the access in bounds and report it
            cell = pos;
            atomicExch(a.status, ST_BAD_ORDER);
        }
        // ---- load the tile's state (gathered through the order)
        for (int k = warp; k < LSP; k += NW) sY[k * TILE + lane] = a.y[k * np + cell];
        double tk = 0.0, rho = 0.0, pnd = 0.0, s1 = 0.0, s2 = 0.0, ENTH0 = 0.0;
        int ns = 0, npass = 0;
        bool tconv = true;
        if (warp == 0) {
            tk = a.tk[cell];
            rho = a.rho[cell];
            pnd = a.pnd[cell];
            s1 = a.soot[cell];
            s2 = a.soot[np + cell];
            ns = a.nsub[cell];
        }
        __syncthreads();
        if (warp == 0) {
            ENTH0 = enthalpy_total(P, tk, sY + lane, TILE);
            int m = ns;
            for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (lane == 0) s_smax = m;
        }
        __syncthreads();
        const int smax = s_smax;
        for (int st = 0; st < smax; ++st) {
            if (warp == 0) {
                const double TKD = tk * P.TSTR;
                sC[SC_TK * TILE + lane] = tk;
                sC[SC_TKD * TILE + lane] = TKD;
                sC[SC_LNT * TILE + lane] = log(TKD);
                sC[SC_RUT * TILE + lane] = (double)82.06f * TKD;
                sC[SC_RHO * TILE + lane] = rho;
                sC[SC_DMOLEA * TILE + lane] = rho * P.RSTR / P.WMSTR * 1.0e-06;
                sC[SC_STMF * TILE + lane] = s1;
                sC[SC_STND * TILE + lane] = s2;
            }
            __syncthreads();
            if (!MIXED || tile_rates_mixed<NW>(P, a.tabm, sRC, sY, sYN, sC, sS, TILE, lane, lane, warp))
                tile_rates_fp64<NW>(P, sTab, sRC, sY, sYN, sC, sS, TILE, lane, lane, warp);
            __syncthreads();
            if (warp == 0 && st < ns) {
                const double dt = a.dt / (double)ns;
                double so[6];
#pragma unroll
                for (int m = 0; m < 6; ++m) so[m] = sS[m * TILE + lane];
                for (int k = 0; k < LSP; ++k) sY0[k * TILE + lane] = sY[k * TILE + lane];
                const double s10 = s1, s20 = s2;
                for (int pass = 1; pass <= a.isor; ++pass) {
                    double rsd = 0.0;
                    // Shared-memory operands; the empty asm with a memory clobber before each
                    // species block keeps the compiler from hoisting loads across blocks (it
                    // runs out of registers otherwise), while loads within a block still overlap.
#define YO(k) sY[(k) * TILE + lane]
#define YN(k) sYN[(k) * TILE + lane]
#define Y0(k) sY0[(k) * TILE + lane]
#define RC(r) sRC[(r) * TILE + lane]
#define RC_LAST(r) sRC[(r) * TILE + lane]
#define SOUR(m) so[m]
#define WM(k) P.WM[k]
#define FACE_SUM(k) 0.0
#define FACE_NBR(k) 0.0
#define UC_UPDATE_TAIL(k) do { if (fnew < 0.0) fnew = 0.0; sYN[(k) * TILE + lane] = fnew; } while (0)
#define UC_UPDATE_SYNC() do { } while (0)
#define UC_UPDATE_BLOCK_BEGIN(b) asm volatile("" ::: "memory")
                    UC_UPDATE_PROGRAM();
#undef YO
#undef YN
#undef Y0
#undef RC
#undef RC_LAST
#undef SOUR
#undef WM
#undef FACE_SUM
#undef FACE_NBR
#undef UC_UPDATE_TAIL
#undef UC_UPDATE_SYNC
#undef UC_UPDATE_BLOCK_BEGIN
                    // soot mass fraction and number density (solvesp.f:2807-2832)
                    const double y2 = sYN[1 * TILE + lane], y4 = sYN[3 * TILE + lane], y5 = sYN[4 * TILE + lane];
                    const double y22 = sYN[21 * TILE + lane];
                    double rhs1 = rho * s10 + dt * ((double)0.012011f / P.WMSTR) *
                                                  (2.0 * so[0] * y22 - so[2] * y2 - so[3] * y5 - so[4] * y4);
                    double fnew = sor2 * s1 + rhs1 * sor1 / ((rho - 0.0) - 0.0);
                    rsd += fabs(s1 - fnew);
                    if (fnew < 0.0) fnew = 0.0;
                    const double n1 = fnew;
                    rhs1 = rho * s20 + dt * so[1] * y22;
                    const double rhs2 = -(dt * so[5]);
                    fnew = sor2 * s2 + rhs1 * sor1 / ((rho - 0.0) - rhs2);
                    if (fnew < 0.0) fnew = 0.0;
                    for (int k = 0; k < LSP - 1; ++k) sY[k * TILE + lane] = sYN[k * TILE + lane];
                    s1 = n1;
                    s2 = fnew;
                    ++npass;
                    if (rsd / (double)(LSP - 1) <= a.tol) break;
                }
                // N2 closure and renormalisation (solvesp.f:2839-2915)
                double ft = sY[lane];
                for (int k = 1; k < LSP - 1; ++k) ft = ft + sY[k * TILE + lane];
                ft = ft + s1;
                double n2 = 1.0 - ft;
                if (ft > 1.0) {
                    for (int k = 0; k < LSP - 1; ++k) sY[k * TILE + lane] = sY[k * TILE + lane] / ft;
                    s1 = s1 / ft;
                    n2 = 0.0;
                }
                sY[(LSP - 1) * TILE + lane] = n2;
                bool conv;
                tk = temperature_at(P, tk, sY + lane, TILE, ENTH0, &conv);
                tconv = tconv && conv;
                double rbar = 0.0;
                for (int k = 0; k < LSP; ++k) rbar = rbar + sY[k * TILE + lane] / P.WM[k];
                rho = pnd / (P.BETA1 * tk * rbar);
            }
            __syncthreads();
        }
        // ---- store
        for (int k = warp; k < LSP; k += NW) a.y[k * np + cell] = sY[k * TILE + lane];
        if (warp == 0) {
            a.tk[cell] = tk;
            a.rho[cell] = rho;
            a.soot[cell] = s1;
            a.soot[np + cell] = s2;
            a.passes[cell] = npass;
            if (!tconv && a.status) atomicCAS(a.status, ST_OK, ST_NEWTON_NOCONV);
        }
        __syncthreads();
    }
}

}  // namespace uc
