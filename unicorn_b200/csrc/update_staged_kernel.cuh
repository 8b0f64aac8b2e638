// Point-implicit species update (src/lib/solvesp.f), FP64, with the rate
// coefficients staged through shared memory.
//
// The same per-cell program as update_kernel (lane = cell, 32-cell tiles, the
// reference's species order), but every RC operand is read from a ring of
// rows in shared memory that the warp fills ahead of use with asynchronous
// copies (cp.async, 16 bytes per lane; completion on an mbarrier per chunk of
// UC_STG_C rows, every lane arriving when its own copies have landed). The row stream of a pass (uc_stg_rows) lists the
// RC rows in use order, a row reused while still resident is read again from
// the ring. The warp waits for chunk c before its first use and, after its
// last use, hands the slot to chunk c + UC_STG_NR: bytes in flight no longer
// cost registers, and the stream runs on across tiles and passes (the RC plane
// does not change during the update). Y lives in shared memory in place; the
// eight species whose start-of-pass value the program reads after their own
// update keep a shadow copy (uc_stg_shadow). All
// mbarrier waits are bounded; a wait that gives up sets ST_TMA_TIMEOUT and
// the update runs on to its end so that every block reaches the grid
// barriers, after which the host reports the error.
#pragma once
#include <cooperative_groups.h>

#include "uc_device.cuh"
#include "update_kernel.cuh"
#include "generated/update_program.cuh"

namespace uc {

#ifndef UC_STG_WARPS
#define UC_STG_WARPS 6
#endif
constexpr int STG_WARPS = UC_STG_WARPS;
constexpr int STG_THREADS = STG_WARPS * 32;
constexpr int STG_RING = UC_STG_C * UC_STG_NR;                    // rows per warp ring
constexpr size_t STG_WARP_DOUBLES = (size_t)(LSP + UC_STG_NSHADOW) * TILE + (size_t)STG_RING * TILE;
constexpr size_t STG_SMEM = STG_WARPS * STG_WARP_DOUBLES * sizeof(double) + STG_WARPS * UC_STG_NR * sizeof(uint64_t);
static_assert(UC_STG_NCHUNK % UC_STG_NR == 0, "chunks per pass must fill whole rings");
constexpr long long STG_WAIT_NS = 2000000000LL;   // a chunk that has not landed in 2 s is an error

// The warp's row stream: position seq (chunk) -> pass, round, chunk of the tile-pass.
struct StgStream {
    const double *rc;
    double *ring;              // this warp's ring (lane 0 view)
    uint64_t *bars;            // UC_STG_NR mbarriers
    size_t np;
    int gwarp, nwarp, rounds, ntile, isor;
};

__device__ __forceinline__ void cp_async16_cg(void *dst, const void *src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

// Arrive on the mbarrier when all earlier cp.async copies of this thread have landed.
__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t *bar)
{
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Issue chunk c of tile `tile` into its ring slot: its rows (256 B of the tile
// each) in 16-byte asynchronous copies spread over the warp's lanes, then every
// lane arrives on the chunk's mbarrier (initialised for 32 arrivals) once its
// own copies have landed. tile < 0: nothing to issue (past the last pass).
__device__ __forceinline__ void stg_issue(const StgStream &s, int tile, int c, int lane)
{
    if (tile < 0) return;
    const int slot = c % UC_STG_NR;
    const int piece = lane & 15;                       // 16-byte piece of a 256-byte row
    const double *src = s.rc + (size_t)tile * TILE + 2 * piece;
    double *dst = s.ring + (size_t)slot * UC_STG_C * TILE + 2 * piece;
#pragma unroll
    for (int j = 0; j < UC_STG_C / 2; ++j) {
        const int q = 2 * j + (lane >> 4);             // row of the chunk
        const int r = uc_stg_rows[c * UC_STG_C + q];
        if (r >= 0) cp_async16_cg(dst + (size_t)q * TILE, src + (size_t)r * s.np);
    }
    cp_async_arrive_noinc(s.bars + slot);
}

// Tile of round `round` of `pass` for this warp, or -1 past the last pass.
__device__ __forceinline__ int stg_tile(const StgStream &s, int pass, int round)
{
    if (round >= s.rounds) { ++pass; round = 0; }
    if (pass > s.isor) return -1;
    const int t = s.gwarp + round * s.nwarp;
    return t < s.ntile ? t : s.ntile - 1;
}

__global__ void __launch_bounds__(STG_THREADS, 1) update_staged_kernel(const UpdArgs a)
{
    namespace cg = cooperative_groups;
    cg::grid_group grid = cg::this_grid();
    extern __shared__ __align__(128) double s_stg[];
    __shared__ double s_part[STG_WARPS];
    __shared__ double s_wm[LSP];
    const DevParams &P = *a.P;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double *sy = s_stg + (size_t)wib * STG_WARP_DOUBLES + lane;          // Y(k) = sy[k*32]
    double *ysh = sy + (size_t)LSP * TILE;                               // YOS(m) = ysh[m*32]
    double *ring = s_stg + (size_t)wib * STG_WARP_DOUBLES + (size_t)(LSP + UC_STG_NSHADOW) * TILE;
    const double *rl = ring + lane;                                      // RCS(i) = rl[(i % ring)*32]
    uint64_t *bars = reinterpret_cast<uint64_t *>(s_stg + STG_WARPS * STG_WARP_DOUBLES) + wib * UC_STG_NR;
    StgStream S;
    S.rc = a.rc; S.ring = ring; S.bars = bars; S.np = a.npad;
    S.nwarp = gridDim.x * STG_WARPS;
    S.gwarp = blockIdx.x * STG_WARPS + wib;
    S.rounds = (a.ntile + S.nwarp - 1) / S.nwarp;
    S.ntile = a.ntile; S.isor = a.isor;
    const double sor1 = a.sor1, sor2 = 1.0 - a.sor1, dt = a.dt;
    const size_t np = a.npad;
    const uint64_t drop = l2_policy_drop();
    for (int k = threadIdx.x; k < LSP; k += blockDim.x) s_wm[k] = P.WM[k];
    if (lane == 0)
        for (int j = 0; j < UC_STG_NR; ++j) mbar_init(bars + j, 32);
    __syncthreads();
    bool timed_out = false;
    long long base = 0;                 // stream position of chunk 0 of the current tile-pass
    for (int j = 0; j < UC_STG_NR; ++j) stg_issue(S, stg_tile(S, 1, 0), j, lane);
    int pass;
    for (pass = 1; pass <= a.isor; ++pass) {
        double rsd = 0.0;
        for (int round = 0; round < S.rounds; ++round, base += UC_STG_NCHUNK) {
            int tile = S.gwarp + round * S.nwarp;
            const bool own = tile < a.ntile;
            if (!own) tile = a.ntile - 1;
            const int tile_next = stg_tile(S, pass, round + 1);   // where chunks c + NR >= NCHUNK go
            const size_t cell = (size_t)tile * TILE + lane;
            const bool live = own && cell < (size_t)a.n && !(a.hold && a.hold[cell]);
            for (int k = 0; k < LSP - 1; ++k) sy[k * TILE] = a.y[k * np + cell];
#pragma unroll
            for (int m = 0; m < UC_STG_NSHADOW; ++m) ysh[m * TILE] = sy[uc_stg_shadow[m] * TILE];
            const double rho = a.rho[cell];
            double so[6];
#pragma unroll
            for (int m = 0; m < 6; ++m) so[m] = a.sour[m * np + cell];
            __syncwarp();
            double crsd = 0.0;
            {
                double &rsd = crsd;
#define YO(k) sy[(k) * TILE]
#define YN(k) sy[(k) * TILE]
#define YOS(m) ysh[(m) * TILE]
#define Y0(k) ld_hint(a.y0 + (size_t)(k) * np + cell, drop)
#define SOUR(m) so[m]
#define WM(k) s_wm[k]
#define FACE_SUM(k) (a.face_sum ? __ldg(a.face_sum + (size_t)(k) * np + cell) : 0.0)
#define FACE_NBR(k) (a.face_nbr ? __ldg(a.face_nbr + (size_t)(k) * np + cell) : 0.0)
#define UC_UPDATE_TAIL(k) do { if (fnew < 0.0) fnew = 0.0; sy[(k) * TILE] = fnew; } while (0)
#define RCS(i) rl[((i) % STG_RING) * TILE]
#define UC_RC_WAIT(c)                                                                                   \
    do {                                                                                                \
        const long long q_ = base + (c);                                                                \
        if (!timed_out && !mbar_wait_ns(bars + (c) % UC_STG_NR, (uint32_t)((q_ / UC_STG_NR) & 1), STG_WAIT_NS)) \
            timed_out = true;                                                                           \
    } while (0)
#define UC_RC_RELEASE(c)                                                                                \
    do {                                                                                                \
        __syncwarp();                                                                                   \
        if ((c) + UC_STG_NR < UC_STG_NCHUNK) stg_issue(S, tile, (c) + UC_STG_NR, lane);                 \
        else stg_issue(S, tile_next, (c) + UC_STG_NR - UC_STG_NCHUNK, lane);                            \
    } while (0)
                UC_UPDATE_PROGRAM_STAGED();
#undef YO
#undef YN
#undef YOS
#undef Y0
#undef SOUR
#undef WM
#undef FACE_SUM
#undef FACE_NBR
#undef UC_UPDATE_TAIL
#undef RCS
#undef UC_RC_WAIT
#undef UC_RC_RELEASE
                // soot mass fraction and number density (solvesp.f:2807-2832)
                const double s1 = a.soot[cell], s2 = a.soot[np + cell];
                const double so0 = so[0], so1 = so[1], so2 = so[2], so3 = so[3], so4 = so[4], so5 = so[5];
                const double y2 = sy[1 * TILE], y4 = sy[3 * TILE], y5 = sy[4 * TILE], y22 = sy[21 * TILE];
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
                    for (int k = 0; k < LSP - 1; ++k) a.y[k * np + cell] = sy[k * TILE];
                    a.soot[cell] = n1;
                    a.soot[np + cell] = fnew;
                }
            }
            if (live) rsd += crsd;
            __syncwarp();
        }
        // deterministic CTA reduction of the residual
        for (int o = 16; o > 0; o >>= 1) rsd += __shfl_xor_sync(0xffffffffu, rsd, o);
        if (lane == 0) s_part[wib] = rsd;
        __syncthreads();
        if (threadIdx.x == 0) {
            double b = 0.0;
            for (int w = 0; w < STG_WARPS; ++w) b += s_part[w];
            a.partial[(pass & 1) * gridDim.x + blockIdx.x] = b;
        }
        grid.sync();
        double tot = 0.0;
        for (int b = 0; b < (int)gridDim.x; ++b) tot += a.partial[(pass & 1) * gridDim.x + b];
        if (tot / a.spnorm <= a.tol) break;
    }
    // let the copies issued ahead land before the block exits
    for (int j = 0; j < UC_STG_NR; ++j) {
        const long long q = base + j;
        if (q / ((long long)S.rounds * UC_STG_NCHUNK) + 1 > a.isor) break;
        if (!mbar_wait_ns(bars + j, (uint32_t)((q / UC_STG_NR) & 1), timed_out ? STG_WAIT_NS / 16 : STG_WAIT_NS))
            timed_out = true;
    }
    if (__any_sync(0xffffffffu, timed_out) && lane == 0 && a.status) atomicExch(a.status, ST_TMA_TIMEOUT);
    if (blockIdx.x == 0 && threadIdx.x == 0) *a.passes = pass;   // ISOR1+1 if not converged
    // N2 closure and renormalisation (solvesp.f:2839-2915)
    for (size_t cell = (size_t)blockIdx.x * STG_THREADS + threadIdx.x; cell < (size_t)a.n;
         cell += (size_t)gridDim.x * STG_THREADS) {
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
