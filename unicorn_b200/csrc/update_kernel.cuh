// Point-implicit species update (src/lib/solvesp.f), FP64.
//
// Lane = cell; each warp of a CTA walks its own 32-cell tiles. The per-cell
// update program is generated (generated/update_program.cuh) from the
// reference's statement sequence with its A-terms resolved into products of
// RC, the pass-start Y (YO) and the freshly updated Y (YN). Both Y sets live
// in shared memory ([52][32] per warp each), so registers go to keeping RC
// loads in flight. The in-place form (IP, the FP64 default) keeps one set
// ([51][32] per warp: each species is overwritten by its own update), so 14
// warps fit per SM instead of 8; the eight species whose start-of-pass value
// the program still reads after their update (through A-terms built before
// it) are read from the tile's Y rows in global memory, which hold the
// start-of-pass values until the tile's program has ended. The warps of a CTA can run the program in lockstep (a
// barrier after every species) so that the instruction cache holds only the code of
// the current species (optional, see UC_LOCKSTEP); RC (the plane written by
// the rate kernel, [544][npad]) is read with loads that do not allocate in L1
// and tell L2 whether the line is read again in the pass.
//
// The relaxation passes run inside one cooperative launch: the residual
// sum|dY| is reduced per CTA, the CTAs meet at a grid barrier, and every CTA
// sums the partials in the same order, so all take the same convergence
// decision (src/lib/solvesp.f:2833).
#pragma once
#include <cooperative_groups.h>

#include "uc_device.cuh"
#include "generated/update_program.cuh"

namespace uc {

struct UpdArgs {
    const DevParams *P;
    const double *rc;                            // [544][npad] FP64 plane (update_kernel<double>)
    const float *rc32;                           // [544][npad] FP32 plane (update_kernel<float>)
    const double *sour, *rho, *y0, *soot0;       // y0 [52][npad]: old time level; soot0 [2][npad]
    const double *face_sum, *face_nbr;           // [51][npad] or null
    double *y, *soot;                            // updated in place
    const int *tile_flag;                        // update_kernel<float>: tiles whose RC is in the FP64 plane
    const uint8_t *hold;                         // optional [npad]: cells that keep their state (grid boundary)
    double *partial;                             // [2][gridDim.x]
    int *passes;                                 // out: pass count as ISOR1 reports it
    double dt, sor1, tol, spnorm;
    int isor, n, npad, ntile;
};

#ifndef UC_UPD_WARPS
#define UC_UPD_WARPS 8
#endif
#ifndef UC_L2_HINTS
#define UC_L2_HINTS 1
#endif
// Measured on B200 (C2 field, 20 passes): an L2 prefetch of the next
// species' RC rows (UC_PF = 1, 2, 4) costs 0.82-0.84 ms/pass against 0.65
// without, and a barrier after every species (UC_LOCKSTEP) changes nothing,
// so both are off; the options stay for re-measurement on other parts.
#ifndef UC_PF
#define UC_PF 0          // species blocks of look-ahead for an L2 prefetch of RC rows (0: none)
#endif
#ifndef UC_LOCKSTEP
#define UC_LOCKSTEP 0    // barrier after every species block
#endif
constexpr int UPD_WARPS = UC_UPD_WARPS;
constexpr int UPD_THREADS = UPD_WARPS * 32;
constexpr size_t UPD_SMEM = (size_t)UPD_WARPS * 2 * LSP * TILE * sizeof(double);

// Read-only loads that skip L1 and carry an L2 eviction priority: lines that
// are read again later in the pass are kept (evict_last), the last read of a
// line in the pass lets it go first (evict_first). The asm is not volatile:
// the data is read-only during the kernel, and the compiler must be free to
// issue these loads early (a volatile form pins each load to its use and
// leaves only a few loads in flight per warp).
// Measured on the C2 sweep with the in-place kernel (update time of 3 sweeps):
// evict_last 161.5 ms, evict_normal 161.4, evict_first everywhere 171.3, no
// hints 171.6 -- the last-use evict_first is what helps.
#ifndef UC_L2_KEEP
#define UC_L2_KEEP 0     // policy of RC reads that are read again in the pass: 0 evict_last, 1 evict_normal, 2 evict_first
#endif
__device__ __forceinline__ uint64_t l2_policy_keep()
{
    uint64_t p;
#if UC_L2_KEEP == 1
    asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
#elif UC_L2_KEEP == 2
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
#else
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
#endif
    return p;
}
__device__ __forceinline__ uint64_t l2_policy_drop()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ double ld_hint(const double *p, uint64_t pol)
{
    double v;
#if UC_L2_HINTS
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
#else
    asm("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
#endif
    return v;
}
__device__ __forceinline__ double ld_hint(const float *p, uint64_t pol)
{
    float v;
#if UC_L2_HINTS
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
#else
    asm("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
#endif
    return (double)v;
}


// Prefetch into L2 the RC rows (256 B per 32-cell tile row) that species
// block b of the program reads; each lane pair takes one row, 16 rows per step.
template <typename RCT>
__device__ __forceinline__ void prefetch_block_rows(int b, const RCT *tile_base, size_t np, int lane)
{
    const int o = uc_upd_row_off[b], e = uc_upd_row_off[b + 1];
    for (int i = o + (lane >> 1); i < e; i += 16) {
        const RCT *p = tile_base + (size_t)uc_upd_rows[i] * np + (lane & 1) * (128 / sizeof(RCT));
        asm volatile("prefetch.global.L2::evict_last [%0];" ::"l"(p));
    }
}

// Shared memory of a CTA of NW warps: two Y sets [52][32] per warp, or with
// IP (in place) one set of the 51 updated species. In place, the few species
// the program reads at their start-of-pass value after their own update are
// read from the Y rows in global memory, which keep the start-of-pass values
// until the tile's program ends.
template <int NW, bool IP>
constexpr size_t upd_smem()
{
    return (size_t)NW * (IP ? (LSP - 1) : 2 * LSP) * TILE * sizeof(double);
}

// RCT: storage type of the RC plane (double for the FP64 form, float for the
// mixed form); the update itself is FP64 in both. NW warps per CTA; IP: Y in
// place (one array per warp), so that more warps fit per SM.
template <typename RCT, int NW = UPD_WARPS, bool IP = false>
__global__ void __launch_bounds__(NW * 32, 1) update_kernel(const UpdArgs a)
{
    // the plane is addressed through the kernel parameter itself (not a local
    // pointer copy): ptxas then rebuilds addresses from the parameter bank and
    // the generated program fits in registers (a local copy spilled 5 KB/thread)
    namespace cg = cooperative_groups;
    cg::grid_group grid = cg::this_grid();
    extern __shared__ __align__(128) double s_upd[];
    __shared__ double s_part[NW];
    __shared__ double s_wm[LSP];
    const DevParams &P = *a.P;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double *syo = s_upd + (size_t)wib * (IP ? LSP - 1 : 2 * LSP) * TILE + lane;   // YO(k) = syo[k*32]
    double *syn = IP ? syo : syo + LSP * TILE;                   // YN(k) = syn[k*32]
    const int nwarp = gridDim.x * NW;
    const int gwarp = blockIdx.x * NW + wib;
    const int rounds = (a.ntile + nwarp - 1) / nwarp;            // same trip count for every warp of the grid
    const double sor1 = a.sor1, sor2 = 1.0 - a.sor1, dt = a.dt;
    const size_t np = a.npad;
    const uint64_t keep = l2_policy_keep(), drop = l2_policy_drop();
    for (int k = threadIdx.x; k < LSP; k += blockDim.x) s_wm[k] = P.WM[k];
    __syncthreads();
    int pass;
    for (pass = 1; pass <= a.isor; ++pass) {
        double rsd = 0.0;
        for (int round = 0; round < rounds; ++round) {
            int tile = gwarp + round * nwarp;
            const bool own = tile < a.ntile;            // warps without a tile repeat the last one, unstored
            if (!own) tile = a.ntile - 1;
            const size_t cell = (size_t)tile * TILE + lane;
            const bool live = own && cell < (size_t)a.n && !(a.hold && a.hold[cell]);
            for (int k = 0; k < LSP - 1; ++k) syo[k * TILE] = a.y[k * np + cell];
            const double rho = a.rho[cell];
            double so[6];
#pragma unroll
            for (int m = 0; m < 6; ++m) so[m] = a.sour[m * np + cell];
            double crsd = 0.0;
            {
                double &rsd = crsd;
#define YO(k) syo[(k) * TILE]
#define YN(k) syn[(k) * TILE]
#define Y0(k) ld_hint(a.y0 + (size_t)(k) * np + cell, drop)
#define SOUR(m) so[m]
#define WM(k) s_wm[k]
#define FACE_SUM(k) (a.face_sum ? __ldg(a.face_sum + (size_t)(k) * np + cell) : 0.0)
#define FACE_NBR(k) (a.face_nbr ? __ldg(a.face_nbr + (size_t)(k) * np + cell) : 0.0)
#define UC_UPDATE_TAIL(k) do { if (fnew < 0.0) fnew = 0.0; syn[(k) * TILE] = fnew; } while (0)
#if UC_LOCKSTEP
#define UC_UPDATE_SYNC() __syncthreads()
#else
#define UC_UPDATE_SYNC() do { } while (0)
#endif
#define UC_UPDATE_BLOCK_BEGIN(b) do { } while (0)
#define YOS(m) __ldcg(a.y + (size_t)uc_ip_shadow[m] * np + cell)
                if constexpr (IP) {
                    if (sizeof(RCT) == 4 && a.tile_flag && a.tile_flag[tile]) {
#define RC(r) ld_hint(a.rc + (size_t)(r) * np + cell, keep)
#define RC_LAST(r) ld_hint(a.rc + (size_t)(r) * np + cell, drop)
                        UC_UPDATE_PROGRAM_IP();
#undef RC
#undef RC_LAST
                    } else {
#define UC_RCP (sizeof(RCT) == 4 ? reinterpret_cast<const RCT *>(a.rc32) : reinterpret_cast<const RCT *>(a.rc))
#define RC(r) ld_hint(UC_RCP + (size_t)(r) * np + cell, keep)
#define RC_LAST(r) ld_hint(UC_RCP + (size_t)(r) * np + cell, drop)
                        UC_UPDATE_PROGRAM_IP();
#undef RC
#undef RC_LAST
#undef UC_RCP
                    }
                } else if (sizeof(RCT) == 4 && a.tile_flag && a.tile_flag[tile]) {
                    // a tile the mixed rate kernel sent to FP64: its RC is in the FP64 plane
#define RC(r) ld_hint(a.rc + (size_t)(r) * np + cell, keep)
#define RC_LAST(r) ld_hint(a.rc + (size_t)(r) * np + cell, drop)
                    UC_UPDATE_PROGRAM();
#undef RC
#undef RC_LAST
                } else {
#define UC_RCP (sizeof(RCT) == 4 ? reinterpret_cast<const RCT *>(a.rc32) : reinterpret_cast<const RCT *>(a.rc))
#define RC(r) ld_hint(UC_RCP + (size_t)(r) * np + cell, keep)
#define RC_LAST(r) ld_hint(UC_RCP + (size_t)(r) * np + cell, drop)
                    UC_UPDATE_PROGRAM();
                }
#undef RC
#undef RC_LAST
#undef UC_RCP
#undef YO
#undef YN
#undef Y0
#undef SOUR
#undef WM
#undef FACE_SUM
#undef FACE_NBR
#undef UC_UPDATE_TAIL
#undef UC_UPDATE_SYNC
#undef UC_UPDATE_BLOCK_BEGIN
#undef YOS
                // soot mass fraction and number density (solvesp.f:2807-2832)
                const double s1 = a.soot[cell], s2 = a.soot[np + cell];
                const double so0 = so[0], so1 = so[1], so2 = so[2], so3 = so[3], so4 = so[4], so5 = so[5];
                const double y2 = syn[1 * TILE], y4 = syn[3 * TILE], y5 = syn[4 * TILE], y22 = syn[21 * TILE];
                double rhs1 = rho * a.soot0[cell] + dt * ((double)0.012011f / P.WMSTR) *
                                                        (2.0 * so0 * y22 - so2 * y2 - so3 * y5 - so4 * y4);
                double fnew = sor2 * s1 + rhs1 * sor1 / ((rho - 0.0) - 0.0);
                crsd += fabs(s1 - fnew);
                if (fnew < 0.0) fnew = 0.0;
                const double n1 = fnew;
                rhs1 = rho * a.soot0[np + cell] + dt * so1 * y22;
                const double rhs2 = -(dt * so5);
                fnew = sor2 * s2 + rhs1 * sor1 / ((rho - 0.0) - rhs2);
                if (fnew < 0.0) fnew = 0.0;
                if (live) {
                    for (int k = 0; k < LSP - 1; ++k) a.y[k * np + cell] = syn[k * TILE];
                    a.soot[cell] = n1;
                    a.soot[np + cell] = fnew;
                }
            }
            if (live) rsd += crsd;
        }
        // deterministic CTA reduction of the residual
        for (int o = 16; o > 0; o >>= 1) rsd += __shfl_xor_sync(0xffffffffu, rsd, o);
        if (lane == 0) s_part[wib] = rsd;
        __syncthreads();
        if (threadIdx.x == 0) {
            double b = 0.0;
            for (int w = 0; w < NW; ++w) b += s_part[w];
            a.partial[(pass & 1) * gridDim.x + blockIdx.x] = b;
        }
        grid.sync();
        double tot = 0.0;
        for (int b = 0; b < (int)gridDim.x; ++b) tot += a.partial[(pass & 1) * gridDim.x + b];
        if (tot / a.spnorm <= a.tol) break;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *a.passes = pass;   // ISOR1+1 if not converged
    // N2 closure and renormalisation (solvesp.f:2839-2915)
    for (size_t cell = (size_t)blockIdx.x * (NW * 32) + threadIdx.x; cell < (size_t)a.n;
         cell += (size_t)gridDim.x * (NW * 32)) {
        if (a.hold && a.hold[cell]) continue;
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
