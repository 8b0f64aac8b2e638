// Device-side data structures shared by the unichem kernels (sm_100a).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "generated/mech_tables.h"

namespace uc {

constexpr int LSP = UC_LSP;
constexpr int LRX = UC_LRX;
constexpr int NPAIR = UC_NPAIR;
constexpr int TILE = 32;                 // cells per tile = lanes of a warp
constexpr int CHEM_WARPS = 16;           // warps of the rate/omega kernel
constexpr int CHEM_THREADS = CHEM_WARPS * 32;
constexpr int MAX_SPEC_PER_WARP = 8;

// status words written by kernels (device side; the host maps them to UC_E*)
constexpr int ST_OK = 0;
constexpr int ST_TMA_TIMEOUT = 1;
constexpr int ST_NEWTON_NOCONV = 2;
constexpr int ST_BAD_ORDER = 3;
constexpr int ST_MMA_TIMEOUT = 4;
constexpr int ST_RELAX_TIMEOUT = 5;

// One reaction pair of the mechanism: forward slot 2p and reverse slot 2p+1
// (0-based). Staged into shared memory by a bulk (TMA) copy at kernel start.
struct __align__(16) PairTab {
    double akf, alf, exaf, akf_r;          // Arrhenius of the forward slot; AKF of the reverse slot
    double aklow, allow, ealow, pad0;      // fall-off low-pressure limit (aklow = 0: none)
    double troe[4];                        // TROE(IR,1..4)
    int8_t has_rev, rut, qlen, dmole;      // reverse formula present; RUT power; q length; TB group of DMOLE
    int8_t rc_order0, rc_order1, rc_tb0, rc_tb1;   // RC assembly (order 0 = slot never written)
    int8_t rc_len0, rc_len1, pad1[6];
    int8_t qsp[8], qdiv[8];                // q = G[qsp0] (*|/) G[qsp1] ...
    int8_t rc_kind0[4], rc_idx0[4];        // post factors: kind 1 = *Y[idx], 0 = /WM[idx]
    int8_t rc_kind1[4], rc_idx1[4];
};
static_assert(sizeof(PairTab) == 144, "PairTab layout");
constexpr int PAIRTAB_BYTES = NPAIR * (int)sizeof(PairTab);
static_assert(PAIRTAB_BYTES % 16 == 0, "bulk copy size must be a multiple of 16 bytes");

// Constants of one context: scales, tables prepared at set-up, and the
// static work split of the species phase.
struct DevParams {
    double TSTR, RSTR, WMSTR, ALSTR, VSTR, HSTR, GASC, PBACK, CONVRC, CONVRM, CONVRD;
    double C1ST, C2ND, C3RD, RCONV, HCONVR, TKDMIN, RSTR_WMSTR, BETA1, BETA3, REI;
    double WM[LSP], HFO[LSP];
    int8_t elem[LSP * 3];                 // atoms of C, H, O per species
    double poly[LSP * 14];
    double om22[LSP * 12];
    double cdia[LSP];
    double ci11[20];
    double WMIK[LSP * LSP], DWMIK[LSP * LSP], WMCD[LSP * LSP];
    double ETLJ1[LSP * LSP], ETLJ2[LSP * LSP], ETLJ3[LSP * LSP], ETLJ4[LSP * LSP];
    double RETLJ1[LSP * LSP];             // 1 / ETLJ1 (the mixed form's collision-integral argument)
    // cp/R / W and h of every species as polynomials in T for Horner evaluation, per temperature range
    // (0: T <= TPOL1, 1: above): cp_k / W_k = sum_i cpc[i] T^i, h_k = T (sum_i hc[i] T^i) + hc[5]
    double cpc[LSP * 2 * 5], hc[LSP * 2 * 6];
    // third-body groups 1..10 (TBODY + sum sign*coef*Y/W)
    int16_t tb_off[11], tb_len[11];
    int8_t tb_sp[64], tb_sign[64], tb_hascoef[64];
    double tb_coef[64];
    // omega phase
    int16_t prd_off[LSP], prd_len[LSP], loss_off[LSP], loss_len[LSP];
    uint16_t prd_term[UC_NPRD_TERMS];
    double prd_coef[UC_NPRD_TERMS];
    uint16_t loss_term[UC_NLOSS_TERMS];
    int8_t ra_len[LRX], ra_sp[LRX * 3];
    // species assigned to each warp of the rate/omega kernel (balanced by terms)
    int8_t spec_of_warp[CHEM_WARPS][MAX_SPEC_PER_WARP];
    int8_t nspec_of_warp[CHEM_WARPS];
    // reaction pairs assigned to each warp (balanced by cost)
    int16_t pair_of_warp[CHEM_WARPS][24];
    int8_t npair_of_warp[CHEM_WARPS];
};

// ------------------------------------------------------------------ TMA / mbarrier

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// 1-D bulk copy global -> shared (no multicast), completion on the mbarrier.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// Bounded wait on phase `parity` of the mbarrier: returns false if it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int max_tries)
{
    for (int i = 0; i < max_tries; ++i) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

}  // namespace uc
