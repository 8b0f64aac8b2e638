// Point-implicit species update (src/lib/solvesp.f:85-2915) with each tile's
// rate coefficients held on chip across passes: the FP64 default.
//
// Within one update call the cells are independent (the transport terms are
// frozen at the start), and only the stopping test couples them: the pass
// loop ends at the first pass whose residual sum|dY| over all cells meets the
// tolerance (solvesp.f:2833). The kernel therefore runs the passes in chunks
// of C: a warp stages one 32-cell tile's RC block [544][32] on chip once,
// runs C passes of that tile back to back, records the tile's residual of
// each pass and, for all but the last pass of the chunk, a snapshot of the
// tile's Y; then the next tile. After a grid barrier every block sums the
// residual partials of each pass of the chunk in the same order and finds the
// first pass that met the tolerance; if it lies inside the chunk, its snapshot
// becomes the result. The RC plane is read from HBM once per chunk instead of
// once per pass.
//
// On chip: the 537 RC rows the program reads are split between tensor memory
// (256 rows, two 32-bit columns each, in the warp's lane quarter of the
// 512-column allocation) and shared memory (281 rows per warp); three warps,
// each owning one tile, so a block holds 96 cells' RC blocks (417 KB). Y of
// the cell lives in registers (lane = cell). The generated program
// (generated/update_program_tr.cuh) loads tensor-memory operands into two
// register banks ahead of use; shared-memory rows are read where used.
// Slots 0..255 live in tensor memory and slots 256..543 in shared memory, so
// each part is one contiguous range of the plane's rows. A tile is staged by
// three tiled bulk copies through tensor maps of the plane ([32 cells] x [rows]
// boxes, completion on the warp's mbarrier with a bounded wait): first the
// tensor-memory rows into the warp's shared-memory slot, from where tcgen05.st
// moves them on, then the shared-memory rows (loads of the rows into
// registers, or one 256-byte bulk copy per row, were bound by latency or by
// the copy count: 4-5 and 3-4 ms per chunk on 1M cells).
//
// Every cell goes through the same operations in the same order as in the
// in-place kernel, so Y is bit for bit that kernel's; the residual is summed
// per tile, then per warp in tile order, per block in warp order and over the
// blocks in block order.
#pragma once
#include <cooperative_groups.h>
#include <cuda.h>                       // CUtensorMap (the type only; encoded through the runtime's entry point)

#include "uc_device.cuh"
#include "update_kernel.cuh"
#include "generated/update_program_tr.cuh"

namespace uc {

constexpr int TR_WARPS = 3;
constexpr int TR_CHUNK_MAX = 32;
constexpr int TR_SNAP_ROWS = LSP - 1 + 2;          // Y of species 1..51 and the two soot scalars
constexpr size_t TR_SLOT_DOUBLES = (size_t)UC_TR_NS * TILE;
constexpr size_t TR_SMEM = TR_WARPS * TR_SLOT_DOUBLES * sizeof(double);
static_assert(TR_SMEM + 8192 <= 232448, "shared memory of the tile-resident update");
static_assert(UC_TR_NT * 2 <= 512 && UC_TR_NT % 16 == 0, "tensor-memory rows of the tile-resident update");
static_assert(UC_TR_NT <= 256 && UC_TR_NS % 2 == 0 && UC_TR_NS / 2 <= 256 && UC_TR_NT <= UC_TR_NS,
              "boxes of the tiled bulk copies (at most 256 rows each; the tensor-memory rows pass through the slot)");
constexpr uint32_t TR_BOX_T = UC_TR_NT, TR_BOX_S = UC_TR_NS / 2;   // rows per box

struct TrArgs {
    double *snap;          // [chunk - 1][TR_SNAP_ROWS][npad]
    double *partial;       // [2][TR_CHUNK_MAX][gridDim.x]
    int chunk;             // passes per chunk, 1..TR_CHUNK_MAX
    int *status;
    int adapt;             // longer chunks (up to TR_CHUNK_MAX) while the previous call's count says that
                           // many passes are still to come
};

#ifndef UC_TR_WAIT_TRIES
#define UC_TR_WAIT_TRIES (1 << 22)
#endif

__device__ __forceinline__ void tr_tmem_st16(uint32_t taddr, const uint32_t (&v)[32])
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
        "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]),
        "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15]), "r"(v[16]),
        "r"(v[17]), "r"(v[18]), "r"(v[19]), "r"(v[20]), "r"(v[21]), "r"(v[22]), "r"(v[23]), "r"(v[24]),
        "r"(v[25]), "r"(v[26]), "r"(v[27]), "r"(v[28]), "r"(v[29]), "r"(v[30]), "r"(v[31])
        : "memory");
}

// The loads of a bank complete at tcgen05.wait::ld; its registers are operands
// of the wait, so no use of them can be scheduled before it.
#define UC_TR_WAIT_BANK(b)                                                                                     \
    asm volatile("tcgen05.wait::ld.sync.aligned;"                                                             \
                 : "+r"(b[0]), "+r"(b[1]), "+r"(b[2]), "+r"(b[3]), "+r"(b[4]), "+r"(b[5]), "+r"(b[6]),       \
                   "+r"(b[7]), "+r"(b[8]), "+r"(b[9]), "+r"(b[10]), "+r"(b[11]), "+r"(b[12]), "+r"(b[13]),    \
                   "+r"(b[14]), "+r"(b[15]), "+r"(b[16]), "+r"(b[17]), "+r"(b[18]), "+r"(b[19]), "+r"(b[20]), \
                   "+r"(b[21]), "+r"(b[22]), "+r"(b[23])                                                      \
                 :                                                                                            \
                 : "memory")
static_assert(UC_TR_SEG == 12, "UC_TR_WAIT_BANK names 2 x 12 registers");

// FACES: the frozen transport terms are given (else they are zero, as in SOLVESP without faces);
// LOCK: the warps of a block run each species of the program together (a barrier after each), so
// that they fetch the program's instructions once instead of three times.
// rows [y, y + box) of the RC plane for the 32 cells from x, into shared memory as [box][32]: one tiled bulk
// copy through the plane's tensor map (no multicast), completion on the mbarrier
__device__ __forceinline__ void tr_box_load(double *dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// Stage one 32-cell tile's RC block on chip, all rows by bulk copies (bandwidth-bound, not latency-bound):
// first the tensor-memory rows (slots 0..NT-1) into the warp's shared-memory slot, moved on into the warp's
// lane quarter of tensor memory by tcgen05.st, then the shared-memory rows (slots NT..543) into the slot.
// The second copy is still in flight on return: tr_stage_wait completes it (the caller loads the cells'
// state meanwhile). Bounded waits: on a timeout the status is set and the copies in flight are waited for.
__device__ __forceinline__ void tr_stage_begin(double *slot, uint32_t tbase, const CUtensorMap *map_t,
                                               const CUtensorMap *map_s, int tile, uint64_t *bar, uint32_t &phase,
                                               int lane, int *status)
{
    __syncwarp();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncwarp();
    if (lane == 0) {
        mbar_expect_tx(bar, (uint32_t)(UC_TR_NT * TILE * sizeof(double)));
        tr_box_load(slot, map_t, tile * TILE, 0, bar);            // slots 0 .. NT-1
    }
    __syncwarp();
    if (!mbar_wait_bounded(bar, phase, UC_TR_WAIT_TRIES)) {
        if (lane == 0) atomicExch(status, ST_TMA_TIMEOUT);
        mbar_wait_bounded(bar, phase, UC_TR_WAIT_TRIES);   // let copies in flight land
    }
    phase ^= 1u;
    for (int i0 = 0; i0 < UC_TR_NT; i0 += 16) {
        uint32_t v[32];
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const double d = slot[(size_t)(i0 + q) * TILE + lane];
            v[2 * q] = (uint32_t)__double2loint(d);
            v[2 * q + 1] = (uint32_t)__double2hiint(d);
        }
        tr_tmem_st16(tbase + (uint32_t)(2 * i0), v);
    }
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    __syncwarp();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncwarp();
    if (lane == 0) {
        mbar_expect_tx(bar, (uint32_t)(UC_TR_NS * TILE * sizeof(double)));
        tr_box_load(slot, map_s, tile * TILE, UC_TR_NT, bar);     // slots NT .. NT+NS/2-1
        tr_box_load(slot + (size_t)TR_BOX_S * TILE, map_s, tile * TILE, UC_TR_NT + TR_BOX_S, bar);
    }
    __syncwarp();
}

__device__ __forceinline__ void tr_stage_wait(uint64_t *bar, uint32_t &phase, int lane, int *status)
{
    if (!mbar_wait_bounded(bar, phase, UC_TR_WAIT_TRIES)) {
        if (lane == 0) atomicExch(status, ST_TMA_TIMEOUT);
        mbar_wait_bounded(bar, phase, UC_TR_WAIT_TRIES);   // let copies in flight land
    }
    phase ^= 1u;
}

template <bool FACES, bool LOCK>
__global__ void __launch_bounds__(TR_WARPS * 32, 1)
update_tr_kernel(const UpdArgs a, const TrArgs t, const __grid_constant__ CUtensorMap map_t,
                 const __grid_constant__ CUtensorMap map_s)
{
    namespace cg = cooperative_groups;
    cg::grid_group grid = cg::this_grid();
    extern __shared__ __align__(128) double s_rc[];          // [TR_WARPS][UC_TR_NS][32]
    __shared__ double s_wm[LSP];
    __shared__ double s_part[TR_WARPS][TR_CHUNK_MAX];
    __shared__ double s_cell[TR_WARPS][8][TILE];            // SOUR 1..6 and the two soot values of the old level
    __shared__ __align__(8) uint64_t s_bar[TR_WARPS];
    __shared__ uint32_t s_tmem;
    __shared__ int s_stop, s_pred;
    const DevParams &P = *a.P;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const size_t np = a.npad;
    const double sor1 = a.sor1, sor2 = 1.0 - a.sor1, dt = a.dt;

    if (w == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x < TR_WARPS) mbar_init(&s_bar[threadIdx.x], 1);
    for (int k = threadIdx.x; k < LSP; k += blockDim.x) s_wm[k] = P.WM[k];
    // the pass count of the previous call (*a.passes, written by block 0 at the end: every block reads it
    // before the first grid barrier). Only the chunk schedule depends on it, not the result: a chunk runs
    // passes beyond the stopping pass at most, whose Y is dropped for the snapshot of the stopping pass.
    if (threadIdx.x == 0) s_pred = t.adapt ? __ldcg(a.passes) : 0;
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tbase = s_tmem + ((uint32_t)(32 * w) << 16);   // this warp's lane quarter
    double *slot = s_rc + (size_t)w * TR_SLOT_DOUBLES;
    uint32_t phase = 0;
    const int nwarp = gridDim.x * TR_WARPS, gwarp = blockIdx.x * TR_WARPS + w;
    const int rounds = (a.ntile + nwarp - 1) / nwarp;
    uint32_t bank0[2 * UC_TR_SEG], bank1[2 * UC_TR_SEG];
#pragma unroll
    for (int i = 0; i < 2 * UC_TR_SEG; ++i) bank0[i] = bank1[i] = 0u;

    int p0 = 0, passes = 0, cpar = 0;
    for (;;) {
        int want = t.chunk;
        if (s_pred > 0) want = max(want, min(TR_CHUNK_MAX, s_pred - p0 - 4));
        const int C = min(want, a.isor - p0);
        if (lane < TR_CHUNK_MAX) s_part[w][lane] = 0.0;
        __syncwarp();
        for (int round = 0; round < rounds; ++round) {
            int tile = gwarp + round * nwarp;
            const bool own = tile < a.ntile;          // without a tile of its own a warp repeats the last
            if (!own) tile = a.ntile - 1;             // one (nothing stored) to keep the barriers matched
            const size_t cell = (size_t)tile * TILE + lane;
            const bool live = own && cell < (size_t)a.n && !(a.hold && a.hold[cell]);
            tr_stage_begin(slot, tbase, &map_t, &map_s, tile, &s_bar[w], phase, lane, t.status);
            // ---- the cell's state (Y in registers)
            double yv[LSP], ysh[UC_IP_NSHADOW];
#pragma unroll
            for (int k = 0; k < LSP; ++k) yv[k] = a.y[k * np + cell];
            const double rho = a.rho[cell];
            double *sc = &s_cell[w][0][lane];        // sc[m * TILE]: SOUR(m), m < 6; old soot at 6, 7
#pragma unroll
            for (int m = 0; m < 6; ++m) sc[m * TILE] = a.sour[m * np + cell];
            sc[6 * TILE] = a.soot0[cell];
            sc[7 * TILE] = a.soot0[np + cell];
            double st1 = a.soot[cell], st2 = a.soot[np + cell];
            double y0s0, y0s1, fss0 = 0.0, fss1 = 0.0, fns0 = 0.0, fns1 = 0.0;
            tr_stage_wait(&s_bar[w], phase, lane, t.status);
            for (int j = 0; j < C; ++j) {
                double crsd = 0.0;
                {
                    double &rsd = crsd;
#define YO(k) yv[k]
#define YN(k) yv[k]
#define YOS(m) ysh[m]
#define SOUR(m) sc[(m) * TILE]
#define WM(k) s_wm[k]
#define UC_TR_PF(s, k)                                                                  \
    do {                                                                                \
        y0s##s = __ldg(a.y0 + (size_t)(k) * np + cell);                                \
        if (FACES) {                                                                    \
            fss##s = a.face_sum ? __ldg(a.face_sum + (size_t)(k) * np + cell) : 0.0;   \
            fns##s = a.face_nbr ? __ldg(a.face_nbr + (size_t)(k) * np + cell) : 0.0;   \
        }                                                                               \
    } while (0)
#define Y0S(s) y0s##s
#define FSS(s) fss##s
#define FNS(s) fns##s
#define UC_TR_SYNC() do { if (LOCK) __syncthreads(); } while (0)
#define UC_UPDATE_TAIL(k) do { if (fnew < 0.0) fnew = 0.0; yv[k] = fnew; } while (0)
#define RCS(i) slot[(i) * TILE + lane]
#define TM_LD(b, q, col)                                                                              \
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];"                             \
                 : "=r"(bank##b[2 * (q)]), "=r"(bank##b[2 * (q) + 1])                                \
                 : "r"(tbase + (uint32_t)(col)))
#define TM_WAIT(b) UC_TR_WAIT_BANK(bank##b)
#define RCT(b, q) __hiloint2double((int)bank##b[2 * (q) + 1], (int)bank##b[2 * (q)])
                    UC_TR_SHADOW_SAVE();
                    UC_UPDATE_PROGRAM_TR();
#undef YO
#undef YN
#undef YOS
#undef SOUR
#undef WM
#undef UC_TR_PF
#undef Y0S
#undef FSS
#undef FNS
#undef UC_TR_SYNC
#undef UC_UPDATE_TAIL
#undef RCS
#undef TM_LD
#undef TM_WAIT
#undef RCT
                }
                // soot mass fraction and number density (solvesp.f:2807-2832)
                {
                    const double y2 = yv[1], y4 = yv[3], y5 = yv[4], y22 = yv[21];
                    const double so0 = sc[0], so1 = sc[TILE], so2 = sc[2 * TILE], so3 = sc[3 * TILE],
                                 so4 = sc[4 * TILE], so5 = sc[5 * TILE];
                    double rhs1 = rho * sc[6 * TILE] + dt * ((double)0.012011f / P.WMSTR) *
                                                       (2.0 * so0 * y22 - so2 * y2 - so3 * y5 - so4 * y4);
                    double fnew = sor2 * st1 + rhs1 * sor1 / ((rho - 0.0) - 0.0);
                    crsd += fabs(st1 - fnew);
                    if (fnew < 0.0) fnew = 0.0;
                    const double n1 = fnew;
                    rhs1 = rho * sc[7 * TILE] + dt * so1 * y22;
                    const double rhs2 = -(dt * so5);
                    fnew = sor2 * st2 + rhs1 * sor1 / ((rho - 0.0) - rhs2);
                    if (fnew < 0.0) fnew = 0.0;
                    st1 = n1;
                    st2 = fnew;
                }
                double r = live ? crsd : 0.0;
                for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
                if (lane == 0) s_part[w][j] += r;
                if (j < C - 1 && live) {
                    double *sn = t.snap + (size_t)j * TR_SNAP_ROWS * np + cell;
#pragma unroll
                    for (int k = 0; k < LSP - 1; ++k) sn[k * np] = yv[k];
                    sn[(LSP - 1) * np] = st1;
                    sn[LSP * np] = st2;
                }
            }
            if (live) {
#pragma unroll
                for (int k = 0; k < LSP - 1; ++k) a.y[k * np + cell] = yv[k];
                a.soot[cell] = st1;
                a.soot[np + cell] = st2;
            }
        }
        // ---- residual of each pass of the chunk, and the stopping test (solvesp.f:2833-2838)
        __syncthreads();
        if (threadIdx.x < C) {
            double b = 0.0;
            for (int v = 0; v < TR_WARPS; ++v) b += s_part[v][threadIdx.x];
            t.partial[((size_t)cpar * TR_CHUNK_MAX + threadIdx.x) * gridDim.x + blockIdx.x] = b;
        }
        grid.sync();
        if (threadIdx.x == 0) {
            int stop = -1;
            for (int j = 0; j < C && stop < 0; ++j) {
                double tot = 0.0;
                const double *pp = t.partial + ((size_t)cpar * TR_CHUNK_MAX + j) * gridDim.x;
                for (int b = 0; b < (int)gridDim.x; ++b) tot += __ldcg(pp + b);
                if (tot / a.spnorm <= a.tol) stop = j;
            }
            s_stop = stop;
        }
        __syncthreads();
        const int stop = s_stop;
        cpar ^= 1;
        if (stop >= 0) {
            passes = p0 + stop + 1;
            if (stop < C - 1) {
                // the pass that met the tolerance lies inside the chunk: its snapshot is the result
                // (written by other blocks before the grid barrier: read through L2)
                const double *sn = t.snap + (size_t)stop * TR_SNAP_ROWS * np;
                for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < (size_t)a.n;
                     c += (size_t)gridDim.x * blockDim.x) {
                    if (a.hold && a.hold[c]) continue;
                    for (int k = 0; k < LSP - 1; ++k) a.y[k * np + c] = __ldcg(sn + k * np + c);
                    a.soot[c] = __ldcg(sn + (LSP - 1) * np + c);
                    a.soot[np + c] = __ldcg(sn + LSP * np + c);
                }
            }
            break;
        }
        p0 += C;
        if (p0 >= a.isor) {
            passes = a.isor + 1;          // ISOR1 + 1 when the tolerance was not met
            break;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *a.passes = passes;
    // N2 closure and renormalisation (solvesp.f:2839-2915); the cells this thread copied above
    for (size_t cell = (size_t)blockIdx.x * blockDim.x + threadIdx.x; cell < (size_t)a.n;
         cell += (size_t)gridDim.x * blockDim.x) {
        if (a.hold && a.hold[cell]) continue;
        double ft = __ldcg(a.y + cell);
        for (int k = 1; k < LSP - 1; ++k) ft = ft + __ldcg(a.y + k * np + cell);
        ft = ft + __ldcg(a.soot + cell);
        double n2 = 1.0 - ft;
        if (ft > 1.0) {
            for (int k = 0; k < LSP - 1; ++k) a.y[k * np + cell] = __ldcg(a.y + k * np + cell) / ft;
            a.soot[cell] = __ldcg(a.soot + cell) / ft;
            n2 = 0.0;
        }
        a.y[(LSP - 1) * np + cell] = n2;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (w == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s_tmem), "r"(512));
}

// Per-cell form of the tile-resident update, for the batched integration (uc_integrate, rounds form):
// every cell runs its own pass loop with its own step a.dt / nsub[cell] and stops on its own residual
// (SPNORM = LSP - 1: solvesp.f:2833-2838 for a one-cell field), then the N2 closure and renormalisation
// (solvesp.f:2839-2915), all in registers. Only the first *nlive cells of the arrays are live (the caller
// orders the cells so that the ones still integrating come first); tiles beyond them are not touched.
// The old time level (a.y0, a.soot0) is the state at the sub-step start, and the caller may pass the
// state arrays themselves: each warp reads its tile's rows before it writes them. passes[cell] is
// incremented by the passes the cell ran, last[cell] set to them. No grid barrier: warps take tiles gwarp,
// gwarp + nwarp, ...
// The arithmetic of a pass is that of update_tr_kernel; a lane that has converged keeps its Y while the
// others of its warp run on (its values are computed and dropped).
__global__ void __launch_bounds__(TR_WARPS * 32, 1)
update_cells_kernel(const UpdArgs a, const int *nlive, const int *nsub, int *passes, int *last, int *status,
                    const __grid_constant__ CUtensorMap map_t, const __grid_constant__ CUtensorMap map_s)
{
    extern __shared__ __align__(128) double s_rc[];          // [TR_WARPS][UC_TR_NS][32]
    __shared__ double s_wm[LSP];
    __shared__ double s_cell[TR_WARPS][8][TILE];            // SOUR 1..6 and the two soot values of the old level
    __shared__ __align__(8) uint64_t s_bar[TR_WARPS];
    __shared__ uint32_t s_tmem;
    const int n = *nlive;
    if (n <= 0) return;                                     // uniform over the grid
    const DevParams &P = *a.P;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const size_t np = a.npad;
    const double sor1 = a.sor1, sor2 = 1.0 - a.sor1;
    const int ntile = (n + TILE - 1) / TILE;

    if (w == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x < TR_WARPS) mbar_init(&s_bar[threadIdx.x], 1);
    for (int k = threadIdx.x; k < LSP; k += blockDim.x) s_wm[k] = P.WM[k];
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tbase = s_tmem + ((uint32_t)(32 * w) << 16);   // this warp's lane quarter
    double *slot = s_rc + (size_t)w * TR_SLOT_DOUBLES;
    uint32_t phase = 0;
    const int nwarp = gridDim.x * TR_WARPS;
    uint32_t bank0[2 * UC_TR_SEG], bank1[2 * UC_TR_SEG];
#pragma unroll
    for (int i = 0; i < 2 * UC_TR_SEG; ++i) bank0[i] = bank1[i] = 0u;

    for (int tile = blockIdx.x * TR_WARPS + w; tile < ntile; tile += nwarp) {
        const size_t cell = (size_t)tile * TILE + lane;
        const bool live = cell < (size_t)n;
        tr_stage_begin(slot, tbase, &map_t, &map_s, tile, &s_bar[w], phase, lane, status);
        double yv[LSP], ysh[UC_IP_NSHADOW];
#pragma unroll
        for (int k = 0; k < LSP; ++k) yv[k] = a.y[k * np + cell];
        const double rho = a.rho[cell];
        const double dt = a.dt / (double)max(1, nsub[cell]);
        double *sc = &s_cell[w][0][lane];        // sc[m * TILE]: SOUR(m), m < 6; old soot at 6, 7
#pragma unroll
        for (int m = 0; m < 6; ++m) sc[m * TILE] = a.sour[m * np + cell];
        sc[6 * TILE] = a.soot0[cell];
        sc[7 * TILE] = a.soot0[np + cell];
        double st1 = a.soot[cell], st2 = a.soot[np + cell];
        double y0s0, y0s1;
        tr_stage_wait(&s_bar[w], phase, lane, status);
        bool done = !live;
        int npass = 0;
        for (int pass = 1; pass <= a.isor; ++pass) {
            if (__all_sync(0xffffffffu, done)) break;
            double crsd = 0.0;
            {
                double &rsd = crsd;
#define YO(k) yv[k]
#define YN(k) yv[k]
#define YOS(m) ysh[m]
#define SOUR(m) sc[(m) * TILE]
#define WM(k) s_wm[k]
#define UC_TR_PF(s, k) do { y0s##s = __ldg(a.y0 + (size_t)(k) * np + cell); } while (0)
#define Y0S(s) y0s##s
#define FSS(s) 0.0
#define FNS(s) 0.0
#define UC_TR_SYNC() do { } while (0)
#define UC_UPDATE_TAIL(k) do { if (fnew < 0.0) fnew = 0.0; if (!done) yv[k] = fnew; } while (0)
#define RCS(i) slot[(i) * TILE + lane]
#define TM_LD(b, q, col)                                                                              \
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];"                             \
                 : "=r"(bank##b[2 * (q)]), "=r"(bank##b[2 * (q) + 1])                                \
                 : "r"(tbase + (uint32_t)(col)))
#define TM_WAIT(b) UC_TR_WAIT_BANK(bank##b)
#define RCT(b, q) __hiloint2double((int)bank##b[2 * (q) + 1], (int)bank##b[2 * (q)])
                UC_TR_SHADOW_SAVE();
                UC_UPDATE_PROGRAM_TR();
#undef YO
#undef YN
#undef YOS
#undef SOUR
#undef WM
#undef UC_TR_PF
#undef Y0S
#undef FSS
#undef FNS
#undef UC_TR_SYNC
#undef UC_UPDATE_TAIL
#undef RCS
#undef TM_LD
#undef TM_WAIT
#undef RCT
            }
            // soot mass fraction and number density (solvesp.f:2807-2832)
            const double y2 = yv[1], y4 = yv[3], y5 = yv[4], y22 = yv[21];
            const double so0 = sc[0], so1 = sc[TILE], so2 = sc[2 * TILE], so3 = sc[3 * TILE], so4 = sc[4 * TILE],
                         so5 = sc[5 * TILE];
            double rhs1 = rho * sc[6 * TILE] + dt * ((double)0.012011f / P.WMSTR) *
                                               (2.0 * so0 * y22 - so2 * y2 - so3 * y5 - so4 * y4);
            double fnew = sor2 * st1 + rhs1 * sor1 / ((rho - 0.0) - 0.0);
            crsd += fabs(st1 - fnew);
            if (fnew < 0.0) fnew = 0.0;
            const double n1 = fnew;
            rhs1 = rho * sc[7 * TILE] + dt * so1 * y22;
            const double rhs2 = -(dt * so5);
            fnew = sor2 * st2 + rhs1 * sor1 / ((rho - 0.0) - rhs2);
            if (fnew < 0.0) fnew = 0.0;
            if (!done) {
                st1 = n1;
                st2 = fnew;
                ++npass;
                if (crsd / (double)(LSP - 1) <= a.tol) done = true;
            }
        }
        if (live) {
            // N2 closure and renormalisation (solvesp.f:2839-2915)
            double ft = yv[0];
#pragma unroll
            for (int k = 1; k < LSP - 1; ++k) ft = ft + yv[k];
            ft = ft + st1;
            double n2 = 1.0 - ft;
            if (ft > 1.0) {
#pragma unroll
                for (int k = 0; k < LSP - 1; ++k) yv[k] = yv[k] / ft;
                st1 = st1 / ft;
                n2 = 0.0;
            }
            yv[LSP - 1] = n2;
#pragma unroll
            for (int k = 0; k < LSP; ++k) a.y[k * np + cell] = yv[k];
            a.soot[cell] = st1;
            a.soot[np + cell] = st2;
            passes[cell] += npass;
            last[cell] = npass;
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (w == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s_tmem), "r"(512));
}

}  // namespace uc
