// unichem: host side of the C ABI (include/unichem.h) and kernel launches.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/unichem.h"
#include "chem_kernel.cuh"
#include "chem_mixed_kernel.cuh"
#include "props_kernel.cuh"
#include "update_kernel.cuh"
#include "update_tr_kernel.cuh"
#include "integrate_kernel.cuh"
#include "faces_kernel.cuh"
#include "fdetail_kernel.cuh"
#include "enthalpy_kernel.cuh"
#include "mlp_gemm.cuh"
#include "mlp.cuh"

using namespace uc;

// Device buffers of the enthalpy relaxation, grown on demand: the ring of pass
// results, the residual of each pass and the flags (progress [isor],
// done [isor], stop pass, pass count, error word).
struct RelaxBuffers {
    double *ring = nullptr, *rsdz = nullptr;
    int *flags = nullptr;
    size_t ring_cap = 0, isor_cap = 0;
    void release()
    {
        if (ring) cudaFree(ring);
        if (rsdz) cudaFree(rsdz);
        if (flags) cudaFree(flags);
        ring = rsdz = nullptr;
        flags = nullptr;
        ring_cap = isor_cap = 0;
    }
};

#define F32(x) ((double)(float)(x))

struct uc_ctx {
    int device = 0, n = 0, npad = 0, ntile = 0, nsm = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t io_stream = nullptr;  // uc_sweep_host: copies of the outputs while the update runs
    cudaEvent_t io_event = nullptr;
    uc_scales sc{};
    uc_inputs inputs{};               // the input-card values of uc_init
    DevParams *hP = nullptr;          // host copy
    DevParams *dP = nullptr;
    PairTab *dTab = nullptr;
    PairTabM *dTabM = nullptr;
    float *rc32 = nullptr;
    int rc_prec = UC_FP64;            // precision of the RC plane of the last uc_rates/uc_sweep
    int *tile_flag = nullptr, *tile_list = nullptr, *tile_count = nullptr;   // mixed form: tiles sent to FP64
    double *tk = nullptr, *rho = nullptr, *y = nullptr, *y0 = nullptr, *soot = nullptr, *soot0 = nullptr;
    double *rc = nullptr, *sour = nullptr;
    double *qdsp = nullptr, *qdot = nullptr, *dwdy = nullptr;
    double *vmu = nullptr, *vtc = nullptr, *vdf = nullptr, *cp = nullptr, *h = nullptr;
    double *face_sum = nullptr, *face_nbr = nullptr, *ht = nullptr, *partial = nullptr;
    int *status = nullptr, *passes = nullptr;
    bool have_fields = false, have_rc = false;
    int upd_grid = 0;
    int upd_ip = 0, ip_grid = 0;       // FP64 update with Y in place: warps per CTA (0: two Y sets, 8 warps)
    int upd_kind = 0;                  // 0: tile-resident (default), 1: Y in place per pass, 2: two Y sets per pass
    int tr_chunk = 16;                 // tile-resident update: passes per chunk (1M cells, 100 passes:
                                       // chunks of 4, 8, 16 took 234, 202, 182 ms)
    bool tr_adapt = true;              // ... longer while the last call's pass count says more are to come
                                       // (off when UNICHEM_TR_CHUNK fixes the chunk, or when the snapshots
    bool tr_adapt_nomem = false;       // of the longer chunks did not fit in device memory)
    bool tr_lock = false;              // ... with the warps of a block in step species by species
                                       // (measured on 1M cells, 100 passes: 227 ms in step, 221 ms free)
    double *tr_snap = nullptr, *tr_partial = nullptr;
    CUtensorMap tr_map[2];             // the RC plane as a 2-D tensor [544][npad], boxes of 256 and 144 rows
    const double *tr_map_base = nullptr;
    size_t tr_snap_cap = 0;
    // species-equation faces assembled on the device (grid, flow, coefficients)
    int lj = 0, li = 0, isym = 0;
    double sigsp = 0.0;
    double *g_xxs = nullptr, *g_xxc = nullptr, *g_yys = nullptr, *g_yyc = nullptr, *g_yr = nullptr;
    double *f_u = nullptr, *f_v = nullptr, *f_tmu = nullptr;
    double *fe = nullptr, *fw = nullptr, *fn = nullptr, *fs = nullptr;
    uint8_t *hold = nullptr;
    // ISKIP of the reference (src/lib/skipdf.f): class per cell 0 (computed), 1 (3 <= ISKIP < 10),
    // 2 (ISKIP >= 10); skip_hold = class >= 1; hold_comb = that or the grid boundary
    int8_t *skip = nullptr;
    uint8_t *skip_hold = nullptr, *hold_comb = nullptr;
    bool have_skip = false;
    bool have_grid = false, have_flow = false, faces_ready = false;
    double *fd_x = nullptr, *fd_y = nullptr, *fd_u = nullptr, *fd_v = nullptr, *fd_out = nullptr;
    // enthalpy equation (SOLVEH)
    bool rc_start = false;            // the RC plane belongs to the start state of the last species update
    bool have_ht = false;
    double *e_w = nullptr, *e_ekt = nullptr, *e_rdhsp = nullptr, *e_prod = nullptr, *e_fpz = nullptr;
    double *e_ze = nullptr, *e_zw = nullptr, *e_zn = nullptr, *e_zs = nullptr, *e_rhsz = nullptr;
    double *e_cf = nullptr, *e_f0s = nullptr, *e_part = nullptr;
    RelaxBuffers e_rb;
    // batched integration
    double *pnd = nullptr, *enth = nullptr;
    int *nsub = nullptr, *order = nullptr, *hist = nullptr, *next_tile = nullptr, *cpasses = nullptr;
    cudaGraph_t int_graph = nullptr;
    cudaGraphExec_t int_exec = nullptr;
    uc_integrate_opts int_opts{};
    int int_prec = -1, int_gwarps = 0, int_gsorted = -1;   // what the captured graph was built for
    int int_warps = 16, int_sorted = 1;                     // kernel shape in use (tuned); 3 warps: rounds form
    double *rnd_state = nullptr;       // rounds form: y [52], tk, rho, pnd, soot [2], enth rows in n_sub order
    int *rnd_int = nullptr;            // ... nsub and passes in that order, cells and tiles per round, tiles 0..ntile-1
    double tune_best = 0.0, tune_worst = 0.0;
    // tracing: CUDA event pairs around launches
    bool prof = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<int, int>> ev_used;   // (kind, index of the start event)
    char err[512] = {0};
};

static void prof_begin(uc_ctx *c, int kind, int &slot)
{
    slot = -1;
    if (!c->prof) return;
    const int i = (int)c->ev_used.size() * 2;
    while ((int)c->ev_pool.size() < i + 2) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return;
        c->ev_pool.push_back(e);
    }
    cudaEventRecord(c->ev_pool[i], c->stream);
    c->ev_used.push_back({kind, i});
    slot = i;
}

static void prof_end(uc_ctx *c, int slot)
{
    if (slot >= 0) cudaEventRecord(c->ev_pool[slot + 1], c->stream);
}

static int set_err(uc_ctx *c, int code, const char *fmt, ...)
{
    if (c) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(c->err, sizeof(c->err), fmt, ap);
        va_end(ap);
    }
    return code;
}

#define CK(call)                                                                                 \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            return set_err(ctx, UC_E_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                           __FILE__, __LINE__);                                                  \
    } while (0)

// ------------------------------------------------------------------ set-up

// Tables and scales of src/unicornd-mild-sd-5.f:327-483 (all reactions on,
// IRSW=1), written for the device parameter block. Literal constants keep
// the reference's single-precision kind where it has one.
static void build_params(const uc_inputs &in, DevParams &P, std::vector<PairTab> &tab, std::vector<PairTabM> &tabm,
                         uc_scales &sc)
{
    const double RUCAL = F32(1.9872), GASC = F32(8.3144);
    double AKF[LRX], ALF[LRX], EXAF[LRX], AKLOW[LRX], ALLOW[LRX], EALOW[LRX], TROE[LRX][4];
    for (int r = 0; r < LRX; ++r) {
        AKF[r] = uc_raw_akf[r]; ALF[r] = uc_raw_alf[r]; EXAF[r] = uc_raw_exaf[r];
        AKLOW[r] = uc_raw_aklow[r]; ALLOW[r] = uc_raw_allow[r]; EALOW[r] = uc_raw_ealow[r];
        for (int c = 0; c < 4; ++c) TROE[r][c] = uc_raw_troe[r * 4 + c];
    }
    for (int i = 0; i < LRX; i += 2) {   // main:364-413
        EXAF[i] = EXAF[i] / RUCAL;
        if (AKF[i] < 0) {
            AKF[i] = -AKF[i];
            EALOW[i] = EALOW[i] / RUCAL;
        } else {
            EALOW[i] = AKLOW[i] = ALLOW[i] = 0.0;
            for (int c = 0; c < 4; ++c) TROE[i][c] = 0.0;
        }
        AKF[i + 1] = 1.0;
        EXAF[i + 1] = ALF[i + 1] = EALOW[i + 1] = AKLOW[i + 1] = ALLOW[i + 1] = 0.0;
        for (int c = 0; c < 4; ++c) TROE[i + 1][c] = 0.0;
    }
    // main:421-459
    const double WMREF = 1.0 / (in.fo2in / uc_wsp[1] + (1.0 - in.fo2in) / uc_wsp[LSP - 1]) / 1000.0;
    const double AMREF = 5.69428e-07 * pow(in.tref, F32(0.62245));
    const double ACREF = 2.78763e-04 * pow(in.tref, F32(0.796783));
    const double DREF = 1.2e-04;
    const double RREF = in.pref / (GASC / WMREF) / in.tref;
    sc.gasc = GASC;
    sc.alstr = in.rtot - in.rtin;
    sc.vstr = in.vref;
    sc.rstr = RREF;
    sc.pstr = RREF * in.vref * in.vref;
    sc.pback = in.pref / sc.pstr;
    sc.tstr = in.tref;
    sc.hstr = in.vref * in.vref;
    sc.akstr = in.vref * in.vref;
    sc.epstr = in.vref * in.vref * in.vref / sc.alstr;
    sc.cpstr = in.vref * in.vref / in.tref;
    sc.acstr = ACREF;
    sc.tmstr = sc.alstr / in.vref;
    sc.amstr = AMREF;
    sc.dstr = DREF;
    sc.wmstr = WMREF;
    sc.rei = AMREF / RREF / in.vref / sc.alstr;
    sc.beta1 = GASC * sc.rstr * sc.tstr / sc.pstr / sc.wmstr;
    sc.beta2 = sc.tstr * sc.acstr / sc.amstr / sc.vstr / sc.vstr;
    sc.beta3 = sc.rstr * sc.dstr / sc.amstr;
    sc.beta4 = 0.0;
    sc.hconv = GASC / sc.wmstr / sc.hstr;
    sc.convrc = F32(418.68) * 1.9891e-04 * sqrt(sc.tstr / 1000.0 / sc.wmstr) / sc.acstr;
    sc.convrm = F32(0.1) * 2.6693e-05 * sqrt(1000.0 * sc.wmstr * sc.tstr) / sc.amstr;
    sc.convrd = F32(0.02628) * sc.tstr * sqrt(sc.tstr) / sc.pstr / sqrt(sc.wmstr * 1000.0) / sc.dstr;

    memset(&P, 0, sizeof(P));
    P.TSTR = sc.tstr; P.RSTR = sc.rstr; P.WMSTR = sc.wmstr; P.ALSTR = sc.alstr; P.VSTR = sc.vstr;
    P.HSTR = sc.hstr; P.GASC = GASC; P.PBACK = sc.pback;
    P.CONVRC = sc.convrc; P.CONVRM = sc.convrm; P.CONVRD = sc.convrd;
    // ckrates.f:87-89, solveh.f:35-38
    P.C1ST = sc.alstr / sc.vstr;
    P.C2ND = sc.alstr / sc.vstr * (sc.rstr / sc.wmstr * 1.0e-06);
    P.C3RD = sc.alstr / sc.vstr * (sc.rstr * sc.rstr / sc.wmstr / sc.wmstr * 1.0e-12);
    P.RCONV = sc.vstr / sc.wmstr / sc.alstr * 1.0e-06;
    P.HCONVR = GASC / sc.wmstr / sc.hstr;
    P.TKDMIN = sc.tstr - 1.0;
    P.RSTR_WMSTR = sc.rstr / sc.wmstr;
    P.BETA1 = sc.beta1;
    P.BETA3 = sc.beta3;
    P.REI = sc.rei;
    for (int k = 0; k < LSP; ++k) {   // main:461-464
        P.WM[k] = uc_wsp[k] / 1000.0 / sc.wmstr;
        P.HFO[k] = sc.hconv * uc_poly[k * 14 + 5] / P.WM[k];
        P.cdia[k] = uc_cdia[k];
    }
    memcpy(P.poly, uc_poly, sizeof(P.poly));
    memcpy(P.elem, uc_elem_cho, sizeof(P.elem));
    for (int k = 0; k < LSP; ++k)      // spgsolv.f:102-173 and solveh.f:39-57 as coefficient tables
        for (int r = 0; r < 2; ++r) {
            const double *p = uc_poly + k * 14 + 7 * r;
            const double hs = P.HCONVR * P.WMSTR * P.HSTR / P.WM[k];
            for (int i = 0; i < 5; ++i) {
                P.cpc[(k * 2 + r) * 5 + i] = p[i] / P.WM[k];
                P.hc[(k * 2 + r) * 6 + i] = p[i] / (double)(i + 1) * hs;
            }
            P.hc[(k * 2 + r) * 6 + 5] = p[5] / P.WM[k] * P.GASC;
        }
    memcpy(P.om22, uc_om22, sizeof(P.om22));
    memcpy(P.ci11, uc_ci11, sizeof(P.ci11));
    for (int i = 0; i < LSP; ++i)       // main:471-483
        for (int j = 0; j < LSP; ++j) {
            const int ij = i * LSP + j;
            P.WMIK[ij] = (i == j) ? sqrt(P.WM[i]) : pow(P.WM[i] / P.WM[j], F32(0.25));
            P.DWMIK[ij] = F32(2.828427125) * sqrt(1.0 + P.WM[i] / P.WM[j]);
            const double ECDIA = F32(0.5) * (uc_cdia[i] + uc_cdia[j]);
            P.WMCD[ij] = sqrt((P.WM[i] + P.WM[j]) / 2.0 / P.WM[i] / P.WM[j]) / ECDIA / ECDIA;
            P.ETLJ1[ij] = sqrt(uc_tlj[i] * uc_tlj[j]);
            P.ETLJ2[ij] = P.ETLJ1[ij] * P.ETLJ1[ij];
            P.ETLJ3[ij] = P.ETLJ2[ij] * P.ETLJ1[ij];
            P.ETLJ4[ij] = P.ETLJ3[ij] * P.ETLJ1[ij];
            P.RETLJ1[ij] = 1.0 / P.ETLJ1[ij];
        }
    for (int g = 0; g < 11; ++g) { P.tb_off[g] = uc_tb_off[g]; P.tb_len[g] = uc_tb_len[g]; }
    const int ntb = (int)(sizeof(uc_tb_sp) / sizeof(uc_tb_sp[0]));
    for (int t = 0; t < ntb; ++t) {
        P.tb_sp[t] = uc_tb_sp[t]; P.tb_sign[t] = uc_tb_sign[t];
        P.tb_hascoef[t] = uc_tb_hascoef[t]; P.tb_coef[t] = uc_tb_coef[t];
    }
    for (int k = 0; k < LSP; ++k) {
        P.prd_off[k] = uc_prd_off[k]; P.prd_len[k] = uc_prd_len[k];
        P.loss_off[k] = uc_loss_off[k]; P.loss_len[k] = uc_loss_len[k];
    }
    memcpy(P.prd_term, uc_prd_term, sizeof(P.prd_term));
    memcpy(P.prd_coef, uc_prd_coef, sizeof(P.prd_coef));
    memcpy(P.loss_term, uc_loss_term, sizeof(P.loss_term));
    memcpy(P.ra_len, uc_ra_len, sizeof(P.ra_len));
    memcpy(P.ra_sp, uc_ra_sp, sizeof(P.ra_sp));

    // reaction-pair table
    tab.assign(NPAIR, PairTab{});
    std::vector<double> pcost(NPAIR);
    for (int p = 0; p < NPAIR; ++p) {
        PairTab &T = tab[p];
        memset(&T, 0, sizeof(T));
        const int r0 = 2 * p, r1 = 2 * p + 1;
        T.akf = AKF[r0]; T.alf = ALF[r0]; T.exaf = EXAF[r0]; T.akf_r = AKF[r1];
        T.aklow = AKLOW[r0]; T.allow = ALLOW[r0]; T.ealow = EALOW[r0];
        for (int c = 0; c < 4; ++c) T.troe[c] = TROE[r0][c];
        T.has_rev = uc_rev_has[r1];
        T.rut = uc_rev_rut[r1];
        T.qlen = uc_rev_len[r1];
        for (int t = 0; t < T.qlen; ++t) { T.qsp[t] = uc_rev_sp[r1 * UC_QMAX + t]; T.qdiv[t] = uc_rev_div[r1 * UC_QMAX + t]; }
        T.dmole = uc_dmole_grp[r0];
        T.rc_order0 = uc_rc_order[r0]; T.rc_order1 = uc_rc_order[r1];
        T.rc_tb0 = uc_rc_tb[r0]; T.rc_tb1 = uc_rc_tb[r1];
        T.rc_len0 = uc_rc_len[r0]; T.rc_len1 = uc_rc_len[r1];
        for (int t = 0; t < 4; ++t) {
            if (t < T.rc_len0) { T.rc_kind0[t] = uc_rc_kind[r0 * UC_PMAX + t]; T.rc_idx0[t] = uc_rc_idx[r0 * UC_PMAX + t]; }
            if (t < T.rc_len1) { T.rc_kind1[t] = uc_rc_kind[r1 * UC_PMAX + t]; T.rc_idx1[t] = uc_rc_idx[r1 * UC_PMAX + t]; }
        }
        pcost[p] = 3.0 + (T.has_rev ? 1.0 + 0.5 * T.qlen : 0.0) + (T.aklow != 0.0 ? 6.0 : 0.0);
    }
    // balance pairs and species over the warps (longest first onto the least loaded warp)
    auto balance = [](const std::vector<double> &cost, int nw, int cap, std::vector<std::vector<int>> &out) {
        std::vector<int> idx(cost.size());
        for (size_t i = 0; i < idx.size(); ++i) idx[i] = (int)i;
        std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return cost[a] > cost[b]; });
        std::vector<double> load(nw, 0.0);
        out.assign(nw, {});
        for (int i : idx) {
            int best = -1;
            for (int w = 0; w < nw; ++w)
                if ((int)out[w].size() < cap && (best < 0 || load[w] < load[best])) best = w;
            out[best].push_back(i);
            load[best] += cost[i];
        }
        for (auto &v : out) std::sort(v.begin(), v.end());
    };
    // pair table of the mixed kernel: logarithms of the constant factors
    tabm.assign(NPAIR, PairTabM{});
    const double CO[4] = {0.0, P.C1ST, P.C2ND, P.C3RD};
    for (int p = 0; p < NPAIR; ++p) {
        const PairTab &T = tab[p];
        PairTabM &M = tabm[p];
        memset(&M, 0, sizeof(M));
        M.lnakf = T.akf > 0.0 ? log(T.akf) : -1.0e300;
        M.alf = T.alf;
        M.exaf = T.exaf;
        M.falloff = T.aklow != 0.0;
        M.lnaklow = M.falloff ? log(T.aklow) : 0.0;
        M.allow = T.allow;
        M.ealow = T.ealow;
        for (int c = 0; c < 4; ++c) M.troe[c] = (float)T.troe[c];
        M.has_rev = T.has_rev; M.rut = T.rut; M.qlen = T.qlen; M.dmole = T.dmole;
        for (int t = 0; t < T.qlen; ++t) { M.qsp[t] = T.qsp[t]; M.qsgn[t] = (t > 0 && T.qdiv[t]) ? -1 : 1; }
        M.order0 = T.rc_order0; M.order1 = T.rc_order1; M.tb0 = T.rc_tb0; M.tb1 = T.rc_tb1;
        double l0 = T.rc_order0 ? log(CO[T.rc_order0]) : 0.0, l1 = T.rc_order1 ? log(CO[T.rc_order1]) : 0.0;
        for (int t = 0; t < T.rc_len0; ++t) {
            if (T.rc_kind0[t]) M.yk0[M.ny0++] = T.rc_idx0[t];
            else l0 -= log(P.WM[T.rc_idx0[t]]);
        }
        for (int t = 0; t < T.rc_len1; ++t) {
            if (T.rc_kind1[t]) M.yk1[M.ny1++] = T.rc_idx1[t];
            else l1 -= log(P.WM[T.rc_idx1[t]]);
        }
        M.lnc0 = l0;
        M.lnc1 = l1 + (T.akf_r > 0.0 ? log(T.akf_r) : 0.0);
    }
    std::vector<std::vector<int>> pw, sw;
    balance(pcost, CHEM_WARPS, 24, pw);
    for (int w = 0; w < CHEM_WARPS; ++w) {
        P.npair_of_warp[w] = (int8_t)pw[w].size();
        for (size_t i = 0; i < pw[w].size(); ++i) P.pair_of_warp[w][i] = (int16_t)pw[w][i];
    }
    std::vector<double> scost(LSP);
    for (int k = 0; k < LSP; ++k) scost[k] = 8.0 + 2.0 * uc_prd_len[k] + 2.5 * uc_loss_len[k];
    balance(scost, CHEM_WARPS, MAX_SPEC_PER_WARP, sw);
    for (int w = 0; w < CHEM_WARPS; ++w) {
        P.nspec_of_warp[w] = (int8_t)sw[w].size();
        for (size_t i = 0; i < sw[w].size(); ++i) P.spec_of_warp[w][i] = (int8_t)sw[w][i];
    }
}

// ------------------------------------------------------------------ helpers

static void free_ctx(uc_ctx *c)
{
    if (!c) return;
    double **bufs[] = {&c->tk, &c->rho, &c->y, &c->y0, &c->soot, &c->soot0, &c->rc, &c->sour, &c->qdsp,
                       &c->qdot, &c->dwdy, &c->vmu, &c->vtc, &c->vdf, &c->cp, &c->h, &c->face_sum,
                       &c->face_nbr, &c->ht, &c->partial, &c->tr_snap, &c->tr_partial};
    for (auto b : bufs)
        if (*b) { cudaFree(*b); *b = nullptr; }
    if (c->dP) cudaFree(c->dP);
    if (c->dTab) cudaFree(c->dTab);
    if (c->dTabM) cudaFree(c->dTabM);
    if (c->rc32) cudaFree(c->rc32);
    if (c->tile_flag) cudaFree(c->tile_flag);
    if (c->tile_list) cudaFree(c->tile_list);
    if (c->tile_count) cudaFree(c->tile_count);
    if (c->status) cudaFree(c->status);
    if (c->passes) cudaFree(c->passes);
    {
        int **ibufs[] = {&c->nsub, &c->order, &c->hist, &c->next_tile, &c->cpasses};
        for (auto b : ibufs)
            if (*b) { cudaFree(*b); *b = nullptr; }
        if (c->pnd) cudaFree(c->pnd);
        if (c->enth) cudaFree(c->enth);
        if (c->rnd_state) cudaFree(c->rnd_state);
        if (c->rnd_int) cudaFree(c->rnd_int);
        void *fb[] = {c->g_xxs, c->g_xxc, c->g_yys, c->g_yyc, c->g_yr, c->f_u, c->f_v, c->f_tmu,
                      c->fe, c->fw, c->fn, c->fs, c->hold, c->skip, c->skip_hold, c->hold_comb, c->fd_x, c->fd_y, c->fd_u, c->fd_v, c->fd_out,
                      c->e_w, c->e_ekt, c->e_rdhsp, c->e_prod, c->e_fpz, c->e_ze, c->e_zw, c->e_zn, c->e_zs,
                      c->e_rhsz, c->e_cf, c->e_f0s, c->e_part};
        for (void *b : fb)
            if (b) cudaFree(b);
        c->e_rb.release();
        if (c->int_exec) cudaGraphExecDestroy(c->int_exec);
        if (c->int_graph) cudaGraphDestroy(c->int_graph);
    }
    for (auto e : c->ev_pool) cudaEventDestroy(e);
    c->ev_pool.clear();
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->io_stream) cudaStreamDestroy(c->io_stream);
    if (c->io_event) cudaEventDestroy(c->io_event);
    delete c->hP;
}

static int dalloc(uc_ctx *ctx, double **p, size_t count)
{
    if (*p) return UC_OK;
    cudaError_t e = cudaMalloc((void **)p, count * sizeof(double));
    if (e != cudaSuccess) {
        *p = nullptr;
        return set_err(ctx, UC_E_NOMEM, "cudaMalloc of %zu doubles failed: %s", count, cudaGetErrorString(e));
    }
    return UC_OK;
}

// copies of the last real cell into the padding cells of a [rows][npad] array
__global__ void pad_rows_kernel(double *a, int rows, int n, int npad)
{
    const int pad = npad - n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows * pad; i += gridDim.x * blockDim.x) {
        const int r = i / pad, c = n + i % pad;
        a[(size_t)r * npad + c] = a[(size_t)r * npad + n - 1];
    }
}

static int upload_rows(uc_ctx *ctx, double *dst, const double *src, int rows)
{
    if (src) {
        CK(cudaMemcpy2DAsync(dst, (size_t)ctx->npad * sizeof(double), src, (size_t)ctx->n * sizeof(double),
                             (size_t)ctx->n * sizeof(double), rows, cudaMemcpyHostToDevice, ctx->stream));
    } else {
        CK(cudaMemsetAsync(dst, 0, (size_t)rows * ctx->npad * sizeof(double), ctx->stream));
    }
    if (ctx->npad > ctx->n) {
        pad_rows_kernel<<<64, 256, 0, ctx->stream>>>(dst, rows, ctx->n, ctx->npad);
        CK(cudaGetLastError());
    }
    return UC_OK;
}

static int download_rows(uc_ctx *ctx, double *dst, const double *src, int rows)
{
    if (!dst) return UC_OK;
    CK(cudaMemcpy2DAsync(dst, (size_t)ctx->n * sizeof(double), src, (size_t)ctx->npad * sizeof(double),
                         (size_t)ctx->n * sizeof(double), rows, cudaMemcpyDeviceToHost, ctx->stream));
    return UC_OK;
}

static int check_status(uc_ctx *ctx)
{
    int st = 0;
    CK(cudaMemcpyAsync(&st, ctx->status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (st == ST_TMA_TIMEOUT) {
        CK(cudaMemsetAsync(ctx->status, 0, sizeof(int), ctx->stream));
        return set_err(ctx, UC_E_TIMEOUT, "table staging (bulk copy) timed out on the device");
    }
    if (st == ST_BAD_ORDER) {
        CK(cudaMemsetAsync(ctx->status, 0, sizeof(int), ctx->stream));
        return set_err(ctx, UC_E_CUDA, "integration work order out of range (internal error)");
    }
    if (st == ST_NEWTON_NOCONV) {
        CK(cudaMemsetAsync(ctx->status, 0, sizeof(int), ctx->stream));
        return set_err(ctx, UC_E_NOCONV, "temperature Newton iteration did not converge in 100 steps for some cell");
    }
    return UC_OK;
}

// Species update with Y in place: 14 warps per CTA (one CTA per SM). Measured on
// the C2 sweep against the two-Y-set kernel at 8 warps: 0.56 against 0.65 ms
// per pass; 12, 16 and 17 warps gave 0.62, 0.57 and 0.66 (fewer registers per
// thread as the warps grow: 168, 128, 96); over 5 sweeps 13, 14 and 15 warps
// took 257.3, 257.2 and 250.8 ms of update time. 14 warps stay at 128 registers: each
// of the SM's four schedulers holds four of them in its 16K-register share, so
// a 144-register build has no resident CTA and cannot be launched.
#ifndef UC_UPD_IP_WARPS
#define UC_UPD_IP_WARPS 14
#endif
constexpr int UPD_IP_WARPS = UC_UPD_IP_WARPS;
static void ip_kernel(bool mixed, const void **fn, size_t *sm)
{
    *fn = mixed ? (const void *)update_kernel<float, UPD_IP_WARPS, true>
                : (const void *)update_kernel<double, UPD_IP_WARPS, true>;
    *sm = upd_smem<UPD_IP_WARPS, true>();
}

// The RC plane [544][npad] (FP64) as a tiled tensor map: boxes of 32 cells x `rows` rows, no swizzle,
// no interleave (a box lands in shared memory as [rows][32], the slot layout). cuTensorMapEncodeTiled
// is reached through the runtime's driver entry point, so the library links no driver library.
typedef CUresult (*uc_encode_tiled_fn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                       const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                       CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static uc_encode_tiled_fn tensor_map_encoder()
{
    static uc_encode_tiled_fn encode = nullptr;
    if (!encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        if (e == cudaSuccess && q == cudaDriverEntryPointSuccess && fn) encode = (uc_encode_tiled_fn)fn;
    }
    return encode;
}

static int encode_rc_map(uc_ctx *ctx)
{
    if (ctx->tr_map_base == ctx->rc) return UC_OK;
    uc_encode_tiled_fn encode = tensor_map_encoder();
    if (!encode) return set_err(ctx, UC_E_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const cuuint64_t dims[2] = {(cuuint64_t)ctx->npad, (cuuint64_t)LRX};
    const cuuint64_t strides[1] = {(cuuint64_t)ctx->npad * sizeof(double)};
    const cuuint32_t estr[2] = {1, 1};
    const cuuint32_t rows[2] = {TR_BOX_T, TR_BOX_S};      // the tensor-memory box and the shared-memory boxes
    for (int m = 0; m < 2; ++m) {
        const cuuint32_t box[2] = {(cuuint32_t)TILE, rows[m]};
        CUresult r = encode(&ctx->tr_map[m], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, (void *)ctx->rc, dims, strides, box,
                            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return set_err(ctx, UC_E_CUDA, "tensor map of the RC plane: error %d", (int)r);
    }
    ctx->tr_map_base = ctx->rc;
    return UC_OK;
}

// the tile-resident update kernel for the face terms given or not, warps in step or not
static const void *tr_kernel(bool faces, bool lock)
{
    if (faces) return lock ? (const void *)update_tr_kernel<true, true> : (const void *)update_tr_kernel<true, false>;
    return lock ? (const void *)update_tr_kernel<false, true> : (const void *)update_tr_kernel<false, false>;
}

#define RET_IF(x)                 \
    do {                          \
        int r_ = (x);             \
        if (r_ != UC_OK) return r_; \
    } while (0)

// ------------------------------------------------------------------ C ABI

extern "C" int uc_init(const uc_inputs *in, int ncell, int device, uc_ctx **out)
{
    if (!out) return UC_E_ARG;
    *out = nullptr;
    if (!in || ncell <= 0) return UC_E_ARG;
    if (!(in->rtot > in->rtin) || !(in->vref > 0) || !(in->tref > 0) || !(in->pref > 0) ||
        !(in->fo2in >= 0 && in->fo2in <= 1))
        return UC_E_ARG;
    uc_ctx *ctx = new (std::nothrow) uc_ctx();
    if (!ctx) return UC_E_NOMEM;
    int rc = UC_OK;
    do {
        cudaError_t e = cudaSetDevice(device);
        if (e != cudaSuccess) { rc = set_err(ctx, UC_E_CUDA, "cudaSetDevice(%d): %s", device, cudaGetErrorString(e)); break; }
        ctx->device = device;
        cudaDeviceProp prop;
        cudaGetDeviceProperties(&prop, device);
        ctx->nsm = prop.multiProcessorCount;
        e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) { rc = set_err(ctx, UC_E_CUDA, "stream: %s", cudaGetErrorString(e)); break; }
        ctx->n = ncell;
        ctx->inputs = *in;
        ctx->ntile = (ncell + TILE - 1) / TILE;
        ctx->npad = ctx->ntile * TILE;
        ctx->hP = new (std::nothrow) DevParams();
        if (!ctx->hP) { rc = UC_E_NOMEM; break; }
        std::vector<PairTab> tab;
        std::vector<PairTabM> tabm;
        build_params(*in, *ctx->hP, tab, tabm, ctx->sc);
        if (cudaMalloc((void **)&ctx->dP, sizeof(DevParams)) != cudaSuccess ||
            cudaMalloc((void **)&ctx->dTab, PAIRTAB_BYTES) != cudaSuccess ||
            cudaMalloc((void **)&ctx->dTabM, PAIRTABM_BYTES) != cudaSuccess ||
            cudaMalloc((void **)&ctx->status, sizeof(int)) != cudaSuccess ||
            cudaMalloc((void **)&ctx->passes, sizeof(int)) != cudaSuccess) {
            rc = set_err(ctx, UC_E_NOMEM, "device allocation of the parameter block failed");
            break;
        }
        cudaMemcpy(ctx->dP, ctx->hP, sizeof(DevParams), cudaMemcpyHostToDevice);
        cudaMemset(ctx->passes, 0, sizeof(int));        // no previous update: fixed chunks on the first call
        cudaMemcpy(ctx->dTab, tab.data(), PAIRTAB_BYTES, cudaMemcpyHostToDevice);
        cudaMemcpy(ctx->dTabM, tabm.data(), PAIRTABM_BYTES, cudaMemcpyHostToDevice);
        cudaMemset(ctx->status, 0, sizeof(int));
        const size_t np = ctx->npad;
        if ((rc = dalloc(ctx, &ctx->tk, np)) || (rc = dalloc(ctx, &ctx->rho, np)) ||
            (rc = dalloc(ctx, &ctx->y, LSP * np)) || (rc = dalloc(ctx, &ctx->y0, LSP * np)) ||
            (rc = dalloc(ctx, &ctx->soot, 2 * np)) || (rc = dalloc(ctx, &ctx->soot0, 2 * np)) ||
            (rc = dalloc(ctx, &ctx->sour, 6 * np)))
            break;
        cudaMemset(ctx->sour, 0, 6 * np * sizeof(double));
        e = cudaFuncSetAttribute(chem_fp64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CHEM_SMEM);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(chem_mixed_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CHEMM_SMEM);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(update_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)UPD_SMEM);
        if (e != cudaSuccess) { rc = set_err(ctx, UC_E_CUDA, "smem attribute: %s", cudaGetErrorString(e)); break; }
        e = cudaFuncSetAttribute(update_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)UPD_SMEM);
        if (e != cudaSuccess) { rc = set_err(ctx, UC_E_CUDA, "smem attribute: %s", cudaGetErrorString(e)); break; }
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, update_kernel<double>, UPD_THREADS, UPD_SMEM);
        if (const char *cap = getenv("UNICHEM_UPD_CTAS_PER_SM")) per_sm = std::min(per_sm, std::max(1, atoi(cap)));
        if (per_sm < 1) per_sm = 1;
        ctx->upd_grid = std::min(per_sm * ctx->nsm, std::max(1, (ctx->ntile + UPD_THREADS / 32 - 1) / (UPD_THREADS / 32)));
        if ((rc = dalloc(ctx, &ctx->partial, 2 * (size_t)per_sm * ctx->nsm))) break;
        // the update kernel: the tile-resident form unless UNICHEM_UPDATE names a per-pass one
        ctx->upd_ip = UPD_IP_WARPS;
        ctx->upd_kind = 0;
        if (const char *k = getenv("UNICHEM_UPDATE")) {
            if (!strcmp(k, "twoset")) { ctx->upd_ip = 0; ctx->upd_kind = 2; }
            else if (!strcmp(k, "inplace")) ctx->upd_kind = 1;
        }
        if (const char *k = getenv("UNICHEM_TR_CHUNK")) {
            ctx->tr_chunk = std::max(1, std::min(TR_CHUNK_MAX, atoi(k)));
            ctx->tr_adapt = false;
        }
        // shape of the batched integration until uc_integrate_tune picks one: 16 or 8 (persistent kernel), 3 (rounds).
        // By default the rounds form once every SM has four tiles or more (1M cells: 4.1 s per step against 7.4 s
        // for the persistent kernel; 333 cells: the persistent kernel is faster)
        if (ctx->ntile >= 4 * ctx->nsm) ctx->int_warps = 3;
        if (const char *k = getenv("UNICHEM_INT_WARPS")) {
            const int v = atoi(k);
            if (v == 3 || v == 8 || v == 16) ctx->int_warps = v;
        }
        if (ctx->upd_kind == 0) {
            if (const char *k = getenv("UNICHEM_TR_LOCKSTEP")) ctx->tr_lock = atoi(k) != 0;
            for (int f = 0; f < 2 && e == cudaSuccess; ++f) {
                const void *fn = tr_kernel(f != 0, ctx->tr_lock);
                e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TR_SMEM);
                int tr_per_sm = 0;
                if (e == cudaSuccess) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&tr_per_sm, fn, TR_WARPS * 32, TR_SMEM);
                if (e == cudaSuccess && tr_per_sm < 1) e = cudaErrorInvalidConfiguration;
            }
            if (e != cudaSuccess) { rc = set_err(ctx, UC_E_CUDA, "tile-resident update set-up: %s", cudaGetErrorString(e)); break; }
        }
        if (ctx->upd_ip) {
            const void *fn, *fnm; size_t sm;
            ip_kernel(true, &fnm, &sm);
            e = cudaFuncSetAttribute(fnm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            if (e != cudaSuccess) { rc = set_err(ctx, UC_E_CUDA, "smem attribute: %s", cudaGetErrorString(e)); break; }
            ip_kernel(false, &fn, &sm);
            e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            if (e != cudaSuccess) { rc = set_err(ctx, UC_E_CUDA, "smem attribute: %s", cudaGetErrorString(e)); break; }
            int ip_per_sm = 0, ipm_per_sm = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ip_per_sm, fn, ctx->upd_ip * 32, sm);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ipm_per_sm, fnm, ctx->upd_ip * 32, sm);
            ip_per_sm = std::max(1, std::min(std::min(ip_per_sm, ipm_per_sm), per_sm));
            ctx->ip_grid = std::min(ip_per_sm * ctx->nsm, std::max(1, (ctx->ntile + ctx->upd_ip - 1) / ctx->upd_ip));
        }
        e = cudaDeviceSynchronize();
        if (e != cudaSuccess) { rc = set_err(ctx, UC_E_CUDA, "init: %s", cudaGetErrorString(e)); break; }
    } while (0);
    if (rc != UC_OK) {
        fprintf(stderr, "uc_init: %s\n", ctx->err);
        free_ctx(ctx);
        delete ctx;
        return rc;
    }
    *out = ctx;
    return UC_OK;
}

extern "C" int uc_get_scales(const uc_ctx *ctx, uc_scales *sc, double *wm, double *hfo)
{
    if (!ctx) return UC_E_ARG;
    if (sc) *sc = ctx->sc;
    if (wm) memcpy(wm, ctx->hP->WM, sizeof(double) * LSP);
    if (hfo) memcpy(hfo, ctx->hP->HFO, sizeof(double) * LSP);
    return UC_OK;
}

extern "C" int uc_upload_fields(uc_ctx *ctx, const double *tk, const double *rho, const double *fsp,
                                const double *stmf, const double *stnd)
{
    if (!ctx || !tk || !rho || !fsp) return set_err(ctx, UC_E_ARG, "uc_upload_fields: tk, rho and fsp are required");
    CK(cudaSetDevice(ctx->device));
    RET_IF(upload_rows(ctx, ctx->tk, tk, 1));
    RET_IF(upload_rows(ctx, ctx->rho, rho, 1));
    RET_IF(upload_rows(ctx, ctx->y, fsp, LSP));
    RET_IF(upload_rows(ctx, ctx->soot, stmf, 1));
    RET_IF(upload_rows(ctx, ctx->soot + ctx->npad, stnd, 1));
    CK(cudaMemcpyAsync(ctx->y0, ctx->y, (size_t)LSP * ctx->npad * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->soot0, ctx->soot, 2 * (size_t)ctx->npad * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->have_fields = true;
    ctx->have_rc = false;
    ctx->rc_start = false;
    return UC_OK;
}

static int ensure_u8(uc_ctx *ctx, uint8_t **p, size_t count)
{
    if (*p) return UC_OK;
    if (cudaMalloc((void **)p, count) != cudaSuccess) {
        *p = nullptr;
        return set_err(ctx, UC_E_NOMEM, "device allocation of a %zu-byte mask failed", count);
    }
    return UC_OK;
}

// ISKIP (int per cell) -> class 0 (computed), 1 (3 <= ISKIP < 10), 2 (ISKIP >= 10) and the mask of
// cells that keep their state in the update; padding cells are class 0
__global__ void skip_class_kernel(const int *iskip, int n, int npad, int8_t *cls, uint8_t *keep)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < npad; c += gridDim.x * blockDim.x) {
        const int v = c < n ? iskip[c] : 0;
        const int8_t k = v >= 10 ? 2 : (v >= 3 ? 1 : 0);
        cls[c] = k;
        keep[c] = k != 0;
    }
}

__global__ void or_mask_kernel(const uint8_t *a, const uint8_t *b, int npad, uint8_t *out)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < npad; c += gridDim.x * blockDim.x)
        out[c] = (uint8_t)(a[c] | b[c]);
}

extern "C" int uc_set_iskip(uc_ctx *ctx, const int *iskip)
{
    if (!ctx) return UC_E_ARG;
    CK(cudaSetDevice(ctx->device));
    if (!iskip) {
        ctx->have_skip = false;
        return UC_OK;
    }
    if (!ctx->skip && cudaMalloc((void **)&ctx->skip, ctx->npad) != cudaSuccess) {
        ctx->skip = nullptr;
        return set_err(ctx, UC_E_NOMEM, "ISKIP class array");
    }
    RET_IF(ensure_u8(ctx, &ctx->skip_hold, ctx->npad));
    int *tmp = nullptr;
    CK(cudaMalloc((void **)&tmp, (size_t)ctx->n * sizeof(int)));
    cudaError_t e = cudaMemcpyAsync(tmp, iskip, (size_t)ctx->n * sizeof(int), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) {
        skip_class_kernel<<<ctx->nsm * 4, 256, 0, ctx->stream>>>(tmp, ctx->n, ctx->npad, ctx->skip, ctx->skip_hold);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(tmp);
    if (e != cudaSuccess) return set_err(ctx, UC_E_CUDA, "uc_set_iskip: %s", cudaGetErrorString(e));
    ctx->have_skip = true;
    return UC_OK;
}

// rows of a device array with row stride ld (elements) into a context array [rows][npad]
static int copy_rows_device(uc_ctx *ctx, double *dst, const double *src, int rows, int ld)
{
    if (src) {
        CK(cudaMemcpy2DAsync(dst, (size_t)ctx->npad * sizeof(double), src, (size_t)ld * sizeof(double),
                             (size_t)ctx->n * sizeof(double), rows, cudaMemcpyDeviceToDevice, ctx->stream));
    } else {
        CK(cudaMemsetAsync(dst, 0, (size_t)rows * ctx->npad * sizeof(double), ctx->stream));
    }
    if (ctx->npad > ctx->n) {
        pad_rows_kernel<<<64, 256, 0, ctx->stream>>>(dst, rows, ctx->n, ctx->npad);
        CK(cudaGetLastError());
    }
    return UC_OK;
}

extern "C" int uc_upload_fields_device(uc_ctx *ctx, const double *tk, const double *rho, const double *fsp,
                                       const double *stmf, const double *stnd, int ld)
{
    if (!ctx || !tk || !rho || !fsp)
        return set_err(ctx, UC_E_ARG, "uc_upload_fields_device: tk, rho and fsp are required");
    if (ld < ctx->n) return set_err(ctx, UC_E_ARG, "uc_upload_fields_device: row stride %d below n = %d", ld, ctx->n);
    CK(cudaSetDevice(ctx->device));
    RET_IF(copy_rows_device(ctx, ctx->tk, tk, 1, ld));
    RET_IF(copy_rows_device(ctx, ctx->rho, rho, 1, ld));
    RET_IF(copy_rows_device(ctx, ctx->y, fsp, LSP, ld));
    RET_IF(copy_rows_device(ctx, ctx->soot, stmf, 1, ld));
    RET_IF(copy_rows_device(ctx, ctx->soot + ctx->npad, stnd, 1, ld));
    CK(cudaMemcpyAsync(ctx->y0, ctx->y, (size_t)LSP * ctx->npad * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->soot0, ctx->soot, 2 * (size_t)ctx->npad * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    ctx->have_fields = true;
    ctx->have_rc = false;
    ctx->rc_start = false;
    return UC_OK;
}

extern "C" int uc_download_fields(uc_ctx *ctx, double *tk, double *rho, double *fsp, double *stmf, double *stnd)
{
    if (!ctx) return UC_E_ARG;
    if (!ctx->have_fields) return set_err(ctx, UC_E_STATE, "no fields uploaded");
    CK(cudaSetDevice(ctx->device));
    RET_IF(download_rows(ctx, tk, ctx->tk, 1));
    RET_IF(download_rows(ctx, rho, ctx->rho, 1));
    RET_IF(download_rows(ctx, fsp, ctx->y, LSP));
    RET_IF(download_rows(ctx, stmf, ctx->soot, 1));
    RET_IF(download_rows(ctx, stnd, ctx->soot + ctx->npad, 1));
    CK(cudaStreamSynchronize(ctx->stream));
    return UC_OK;
}

static int launch_chem(uc_ctx *ctx, int precision, bool want_rc, bool want_omega)
{
    if (precision != UC_FP64 && precision != UC_MIXED) return set_err(ctx, UC_E_ARG, "unknown precision %d", precision);
    if (precision == UC_MIXED && want_rc && ctx->upd_kind != 0 && !ctx->rc32) {
        cudaError_t e = cudaMalloc((void **)&ctx->rc32, (size_t)LRX * ctx->npad * sizeof(float));
        if (e != cudaSuccess) { ctx->rc32 = nullptr; return set_err(ctx, UC_E_NOMEM, "FP32 RC plane: %s", cudaGetErrorString(e)); }
    }
    if (want_rc && !ctx->rc) {         // mixed: FP64 plane of fallback tiles
        RET_IF(dalloc(ctx, &ctx->rc, (size_t)LRX * ctx->npad));
        // zero like the reference's COMMON: cells skipped by ISKIP keep what the plane holds
        CK(cudaMemsetAsync(ctx->rc, 0, (size_t)LRX * ctx->npad * sizeof(double), ctx->stream));
    }
    if (precision == UC_MIXED && !ctx->tile_flag) {
        if (cudaMalloc((void **)&ctx->tile_flag, ctx->ntile * sizeof(int)) != cudaSuccess ||
            cudaMalloc((void **)&ctx->tile_list, ctx->ntile * sizeof(int)) != cudaSuccess ||
            cudaMalloc((void **)&ctx->tile_count, sizeof(int)) != cudaSuccess)
            return set_err(ctx, UC_E_NOMEM, "tile flag buffers");
    }
    if (want_omega && !ctx->qdsp) {
        RET_IF(dalloc(ctx, &ctx->qdsp, (size_t)LSP * ctx->npad));
        CK(cudaMemsetAsync(ctx->qdsp, 0, (size_t)LSP * ctx->npad * sizeof(double), ctx->stream));
    }
    if (want_omega && !ctx->qdot) {
        RET_IF(dalloc(ctx, &ctx->qdot, ctx->npad));
        CK(cudaMemsetAsync(ctx->qdot, 0, (size_t)ctx->npad * sizeof(double), ctx->stream));
    }
    if (want_omega && !ctx->dwdy) {
        RET_IF(dalloc(ctx, &ctx->dwdy, (size_t)LSP * ctx->npad));
        CK(cudaMemsetAsync(ctx->dwdy, 0, (size_t)LSP * ctx->npad * sizeof(double), ctx->stream));
    }
    const int8_t *skip = ctx->have_skip ? ctx->skip : nullptr;
    if (precision == UC_MIXED) {
        ChemMArgs m{};
        m.P = ctx->dP; m.tab = ctx->dTabM;
        m.tk = ctx->tk; m.rho = ctx->rho; m.y = ctx->y; m.stmf = ctx->soot; m.stnd = ctx->soot + ctx->npad;
        // the tile-resident update reads an FP64 plane: the FP32 rates are stored as doubles
        m.rc32 = want_rc && ctx->upd_kind != 0 ? ctx->rc32 : nullptr;
        m.rc64 = want_rc && ctx->upd_kind == 0 ? ctx->rc : nullptr;
        m.sour = ctx->sour;
        m.qdsp = want_omega ? ctx->qdsp : nullptr;
        m.qdot = want_omega ? ctx->qdot : nullptr;
        m.dwdy = want_omega ? ctx->dwdy : nullptr;
        m.n = ctx->n; m.npad = ctx->npad; m.ntile = ctx->ntile; m.status = ctx->status;
        m.tile_flag = ctx->tile_flag;
        m.skip = skip;
        const int grid = std::min(ctx->ntile, ctx->nsm);
        int slot;
        prof_begin(ctx, UC_K_CHEM, slot);
        chem_mixed_kernel<<<grid, CHEM_THREADS, CHEMM_SMEM, ctx->stream>>>(m);
        prof_end(ctx, slot);
        CK(cudaGetLastError());
        // tiles with a rate beyond the FP32 range: recompute them in FP64
        compact_tiles_kernel<<<1, 1024, 0, ctx->stream>>>(ctx->tile_flag, ctx->ntile, ctx->tile_list, ctx->tile_count);
        CK(cudaGetLastError());
        ChemArgs f{};
        f.P = ctx->dP; f.tab = ctx->dTab;
        f.tk = ctx->tk; f.rho = ctx->rho; f.y = ctx->y; f.stmf = ctx->soot; f.stnd = ctx->soot + ctx->npad;
        f.rc = want_rc ? ctx->rc : nullptr;
        f.sour = ctx->sour;
        f.qdsp = m.qdsp; f.qdot = m.qdot; f.dwdy = m.dwdy;
        f.n = ctx->n; f.npad = ctx->npad; f.ntile = ctx->ntile; f.status = ctx->status;
        f.tile_list = ctx->tile_list; f.tile_count = ctx->tile_count;
        f.skip = skip; f.rc_stale = ctx->rc;
        prof_begin(ctx, UC_K_CHEM, slot);
        chem_fp64_kernel<<<std::min(ctx->ntile, ctx->nsm), CHEM_THREADS, CHEM_SMEM, ctx->stream>>>(f);
        prof_end(ctx, slot);
        CK(cudaGetLastError());
        if (want_rc) ctx->rc_prec = ctx->upd_kind == 0 ? UC_FP64 : UC_MIXED;   // the type of the plane
        return UC_OK;
    }
    ChemArgs a{};
    a.P = ctx->dP;
    a.tab = ctx->dTab;
    a.tk = ctx->tk; a.rho = ctx->rho; a.y = ctx->y; a.stmf = ctx->soot; a.stnd = ctx->soot + ctx->npad;
    a.rc = want_rc ? ctx->rc : nullptr;
    a.sour = ctx->sour;
    a.qdsp = want_omega ? ctx->qdsp : nullptr;
    a.qdot = want_omega ? ctx->qdot : nullptr;
    a.dwdy = want_omega ? ctx->dwdy : nullptr;
    a.n = ctx->n; a.npad = ctx->npad; a.ntile = ctx->ntile;
    a.status = ctx->status;
    a.skip = skip; a.rc_stale = ctx->rc;
    const int grid = std::min(ctx->ntile, ctx->nsm);
    int slot;
    prof_begin(ctx, UC_K_CHEM, slot);
    chem_fp64_kernel<<<grid, CHEM_THREADS, CHEM_SMEM, ctx->stream>>>(a);
    prof_end(ctx, slot);
    CK(cudaGetLastError());
    if (want_rc) ctx->rc_prec = UC_FP64;
    return UC_OK;
}

extern "C" int uc_rates(uc_ctx *ctx, int precision, double *rc)
{
    if (!ctx) return UC_E_ARG;
    if (!ctx->have_fields) return set_err(ctx, UC_E_STATE, "uc_rates before uc_upload_fields");
    CK(cudaSetDevice(ctx->device));
    RET_IF(launch_chem(ctx, precision, true, false));
    ctx->have_rc = true;
    ctx->rc_start = false;
    if (rc && ctx->rc_prec == UC_FP64) {
        RET_IF(download_rows(ctx, rc, ctx->rc, LRX));
        CK(cudaStreamSynchronize(ctx->stream));
        RET_IF(check_status(ctx));
    } else if (rc) {
        // FP32 plane, with the FP64 values of the tiles that fell back to FP64
        std::vector<float> tmp((size_t)LRX * ctx->n);
        std::vector<int> flag(ctx->ntile);
        CK(cudaMemcpy2DAsync(tmp.data(), (size_t)ctx->n * sizeof(float), ctx->rc32, (size_t)ctx->npad * sizeof(float),
                             (size_t)ctx->n * sizeof(float), LRX, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(flag.data(), ctx->tile_flag, ctx->ntile * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        RET_IF(download_rows(ctx, rc, ctx->rc, LRX));
        CK(cudaStreamSynchronize(ctx->stream));
        for (int r = 0; r < LRX; ++r)
            for (int c = 0; c < ctx->n; ++c)
                if (!flag[c / TILE]) rc[(size_t)r * ctx->n + c] = tmp[(size_t)r * ctx->n + c];
        RET_IF(check_status(ctx));
    }
    return UC_OK;
}

extern "C" int uc_omega(uc_ctx *ctx, int precision, double *qdsp, double *qdot, double *domega_dy)
{
    if (!ctx) return UC_E_ARG;
    if (!ctx->have_fields) return set_err(ctx, UC_E_STATE, "uc_omega before uc_upload_fields");
    CK(cudaSetDevice(ctx->device));
    RET_IF(launch_chem(ctx, precision, false, true));
    if (qdsp || qdot || domega_dy) {
        RET_IF(download_rows(ctx, qdsp, ctx->qdsp, LSP));
        RET_IF(download_rows(ctx, qdot, ctx->qdot, 1));
        RET_IF(download_rows(ctx, domega_dy, ctx->dwdy, LSP));
        RET_IF(check_status(ctx));
    }
    return UC_OK;
}

static int props_impl(uc_ctx *ctx, int precision, double *vmu, double *vtc, double *vdf)
{
    if (!ctx) return UC_E_ARG;
    if (!ctx->have_fields) return set_err(ctx, UC_E_STATE, "uc_props before uc_upload_fields");
    CK(cudaSetDevice(ctx->device));
    RET_IF(dalloc(ctx, &ctx->vmu, ctx->npad));
    RET_IF(dalloc(ctx, &ctx->vtc, ctx->npad));
    RET_IF(dalloc(ctx, &ctx->vdf, (size_t)LSP * ctx->npad));
    PropArgs a{ctx->dP, ctx->tk, ctx->y, ctx->vmu, ctx->vtc, ctx->vdf, ctx->n, ctx->npad};
    const int grid = std::min((ctx->n + 127) / 128, ctx->nsm * 16);
    int slot;
    prof_begin(ctx, UC_K_PROPS, slot);
    if (precision == UC_MIXED)
        props_mixed_kernel<<<grid, 128, 0, ctx->stream>>>(a);
    else
        props_kernel<double><<<grid, 128, 0, ctx->stream>>>(a);
    prof_end(ctx, slot);
    CK(cudaGetLastError());
    if (vmu || vtc || vdf) {
        RET_IF(download_rows(ctx, vmu, ctx->vmu, 1));
        RET_IF(download_rows(ctx, vtc, ctx->vtc, 1));
        RET_IF(download_rows(ctx, vdf, ctx->vdf, LSP));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return UC_OK;
}

extern "C" int uc_props(uc_ctx *ctx, double *vmu, double *vtc, double *vdf)
{
    return props_impl(ctx, UC_FP64, vmu, vtc, vdf);
}

static int cp_h_impl(uc_ctx *ctx, int precision, double *cp, double *h)
{
    if (!ctx) return UC_E_ARG;
    if (!ctx->have_fields) return set_err(ctx, UC_E_STATE, "uc_cp_h before uc_upload_fields");
    CK(cudaSetDevice(ctx->device));
    RET_IF(dalloc(ctx, &ctx->cp, ctx->npad));
    RET_IF(dalloc(ctx, &ctx->h, ctx->npad));
    CpHArgs a{ctx->dP, ctx->tk, ctx->y, ctx->cp, ctx->h, ctx->n, ctx->npad};
    const int grid = std::min((ctx->n + 255) / 256, ctx->nsm * 8);
    int slot;
    prof_begin(ctx, UC_K_CPH, slot);
    // cp and h stay FP64 in the mixed form too: the kernel is bound by reading the 52 Y rows, and h is
    // a signed sum (formation enthalpies) that FP32 cannot hold to 1e-6 of itself
    (void)precision;
    cp_h_kernel<double><<<grid, 256, 0, ctx->stream>>>(a);
    prof_end(ctx, slot);
    CK(cudaGetLastError());
    if (cp || h) {
        RET_IF(download_rows(ctx, cp, ctx->cp, 1));
        RET_IF(download_rows(ctx, h, ctx->h, 1));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return UC_OK;
}

extern "C" int uc_cp_h(uc_ctx *ctx, double *cp, double *h)
{
    return cp_h_impl(ctx, UC_FP64, cp, h);
}

extern "C" int uc_chem_props(uc_ctx *ctx, int precision)
{
    if (!ctx) return UC_E_ARG;
    if (!ctx->have_fields) return set_err(ctx, UC_E_STATE, "uc_chem_props before uc_upload_fields");
    if (precision != UC_FP64 && precision != UC_MIXED) return set_err(ctx, UC_E_ARG, "unknown precision %d", precision);
    RET_IF(props_impl(ctx, precision, nullptr, nullptr, nullptr));
    RET_IF(cp_h_impl(ctx, precision, nullptr, nullptr));
    CK(cudaSetDevice(ctx->device));
    return launch_chem(ctx, precision, false, true);
}

extern "C" int uc_species_update(uc_ctx *ctx, double dt, int isor, double relx, double tol, double spnorm,
                                 const double *face_sum, const double *face_nbr, int *passes)
{
    if (!ctx) return UC_E_ARG;
    if (!ctx->have_rc) return set_err(ctx, UC_E_STATE, "uc_species_update needs the RC plane of uc_rates");
    if (isor < 1 || !(relx > 0.0) || !(dt >= 0.0)) return set_err(ctx, UC_E_ARG, "invalid isor/relx/dt");
    CK(cudaSetDevice(ctx->device));
    // old time level = state at the start of the update (SPGSOLV copies FSP -> SA, src/lib/spgsolv.f:177-231)
    CK(cudaMemcpyAsync(ctx->y0, ctx->y, (size_t)LSP * ctx->npad * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->soot0, ctx->soot, 2 * (size_t)ctx->npad * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    const double *fs = nullptr, *fn = nullptr;
    const uint8_t *hold = nullptr;
    if (!face_sum && !face_nbr && ctx->faces_ready) {
        // assembled coefficients with the neighbours' Y of this moment
        RET_IF(dalloc(ctx, &ctx->face_sum, (size_t)(LSP - 1) * ctx->npad));
        RET_IF(dalloc(ctx, &ctx->face_nbr, (size_t)(LSP - 1) * ctx->npad));
        CK(cudaMemsetAsync(ctx->face_sum, 0, (size_t)(LSP - 1) * ctx->npad * sizeof(double), ctx->stream));
        CK(cudaMemsetAsync(ctx->face_nbr, 0, (size_t)(LSP - 1) * ctx->npad * sizeof(double), ctx->stream));
        faces_apply_kernel<<<ctx->nsm * 4, 256, 0, ctx->stream>>>(ctx->lj, ctx->li, ctx->npad, ctx->fe, ctx->fw, ctx->fn,
                                                                ctx->fs, ctx->y, ctx->face_sum, ctx->face_nbr);
        CK(cudaGetLastError());
        fs = ctx->face_sum;
        fn = ctx->face_nbr;
        hold = ctx->hold;
    }
    if (face_sum) {
        RET_IF(dalloc(ctx, &ctx->face_sum, (size_t)(LSP - 1) * ctx->npad));
        RET_IF(upload_rows(ctx, ctx->face_sum, face_sum, LSP - 1));
        fs = ctx->face_sum;
    }
    if (face_nbr) {
        RET_IF(dalloc(ctx, &ctx->face_nbr, (size_t)(LSP - 1) * ctx->npad));
        RET_IF(upload_rows(ctx, ctx->face_nbr, face_nbr, LSP - 1));
        fn = ctx->face_nbr;
    }
    if (ctx->have_skip) {
        // cells skipped by ISKIP keep their state and leave the residual (solvesp.f:89,2842)
        if (hold) {
            RET_IF(ensure_u8(ctx, &ctx->hold_comb, ctx->npad));
            or_mask_kernel<<<ctx->nsm * 4, 256, 0, ctx->stream>>>(hold, ctx->skip_hold, ctx->npad, ctx->hold_comb);
            CK(cudaGetLastError());
            hold = ctx->hold_comb;
        } else {
            hold = ctx->skip_hold;
        }
    }
    UpdArgs a{};
    a.P = ctx->dP; a.rc = ctx->rc; a.rc32 = ctx->rc32; a.sour = ctx->sour;
    a.tile_flag = ctx->rc_prec == UC_MIXED ? ctx->tile_flag : nullptr; a.rho = ctx->rho; a.y0 = ctx->y0; a.soot0 = ctx->soot0;
    a.face_sum = fs; a.face_nbr = fn; a.y = ctx->y; a.soot = ctx->soot; a.partial = ctx->partial;
    a.hold = hold;
    a.passes = ctx->passes;
    a.dt = dt; a.sor1 = relx; a.tol = tol; a.spnorm = spnorm > 0.0 ? spnorm : (double)ctx->n * (LSP - 1);
    a.isor = isor; a.n = ctx->n; a.npad = ctx->npad; a.ntile = ctx->ntile;
    void *args[] = {&a};
    int slot;
    if (ctx->upd_kind == 0 && ctx->rc_prec == UC_FP64) {
        const int C = std::min(ctx->tr_chunk, isor);
        // Y snapshots for the longest chunk of the call: TR_CHUNK_MAX passes where the chunk schedule may
        // lengthen chunks, else C. Where those do not fit in device memory, fixed chunks of C from then on.
        auto snaps = [&](int c) { return (size_t)std::max(1, std::min(c, isor) - 1) * TR_SNAP_ROWS * ctx->npad; };
        bool adapt = ctx->tr_adapt && !ctx->tr_adapt_nomem;
        size_t need = snaps(adapt ? TR_CHUNK_MAX : C);
        if (ctx->tr_snap_cap < need) {
            if (ctx->tr_snap) cudaFree(ctx->tr_snap);
            ctx->tr_snap = nullptr;
            ctx->tr_snap_cap = 0;
            if (dalloc(ctx, &ctx->tr_snap, need) != UC_OK && adapt) {
                cudaGetLastError();           // a failed cudaMalloc leaves the context usable: clear the error
                ctx->tr_adapt_nomem = true;
                adapt = false;
                need = snaps(C);
            }
            RET_IF(dalloc(ctx, &ctx->tr_snap, need));   // no-op when the first allocation succeeded
            ctx->tr_snap_cap = need;
        }
        RET_IF(dalloc(ctx, &ctx->tr_partial, 2 * (size_t)TR_CHUNK_MAX * ctx->nsm));
        TrArgs t{ctx->tr_snap, ctx->tr_partial, C, ctx->status, adapt ? 1 : 0};
        RET_IF(encode_rc_map(ctx));
        void *targs[] = {&a, &t, &ctx->tr_map[0], &ctx->tr_map[1]};
        prof_begin(ctx, UC_K_UPDATE, slot);
        CK(cudaLaunchCooperativeKernel(tr_kernel(fs != nullptr || fn != nullptr, ctx->tr_lock), dim3(ctx->nsm),
                                       dim3(TR_WARPS * 32), targs, TR_SMEM, ctx->stream));
        prof_end(ctx, slot);
        if (passes) {
            CK(cudaMemcpyAsync(passes, ctx->passes, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
            RET_IF(check_status(ctx));
        }
        ctx->have_rc = false;
        ctx->rc_start = true;
        return UC_OK;
    }
    prof_begin(ctx, UC_K_UPDATE, slot);
    if (ctx->upd_ip) {
        const void *fn; size_t sm;
        ip_kernel(ctx->rc_prec == UC_MIXED, &fn, &sm);
        CK(cudaLaunchCooperativeKernel(fn, dim3(ctx->ip_grid), dim3(ctx->upd_ip * 32), args, sm, ctx->stream));
    } else {
        const void *kfn = ctx->rc_prec == UC_MIXED ? (const void *)update_kernel<float> : (const void *)update_kernel<double>;
        CK(cudaLaunchCooperativeKernel(kfn, dim3(ctx->upd_grid), dim3(UPD_THREADS), args, UPD_SMEM, ctx->stream));
    }
    prof_end(ctx, slot);
    if (passes) {
        CK(cudaMemcpyAsync(passes, ctx->passes, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    ctx->have_rc = false;   // the RC plane belongs to the state before the update
    ctx->rc_start = true;   // ... which the enthalpy equation uses (solveh.f:116-1145)
    return UC_OK;
}

extern "C" int uc_temperature_from_h(uc_ctx *ctx, const double *ht)
{
    if (!ctx || !ht) return set_err(ctx, UC_E_ARG, "uc_temperature_from_h: ht is required");
    if (!ctx->have_fields) return set_err(ctx, UC_E_STATE, "no fields uploaded");
    CK(cudaSetDevice(ctx->device));
    RET_IF(dalloc(ctx, &ctx->ht, ctx->npad));
    RET_IF(upload_rows(ctx, ctx->ht, ht, 1));
    TempArgs a{ctx->dP, ctx->y, ctx->ht, ctx->tk, ctx->status, ctx->n, ctx->npad, ctx->have_skip ? ctx->skip : nullptr};
    const int grid = std::min((ctx->n + 127) / 128, ctx->nsm * 16);
    int slot;
    prof_begin(ctx, UC_K_TEMP, slot);
    temperature_fp64_kernel<<<grid, 128, 0, ctx->stream>>>(a);
    prof_end(ctx, slot);
    CK(cudaGetLastError());
    ctx->have_rc = false;
    return check_status(ctx);
}

extern "C" int uc_sweep(uc_ctx *ctx, int precision, double dt, int isor, double relx, double tol, double spnorm,
                        const double *face_sum, const double *face_nbr, int *passes)
{
    if (!ctx) return UC_E_ARG;
    if (!ctx->have_fields) return set_err(ctx, UC_E_STATE, "uc_sweep before uc_upload_fields");
    if (precision != UC_FP64 && precision != UC_MIXED) return set_err(ctx, UC_E_ARG, "unknown precision %d", precision);
    RET_IF(props_impl(ctx, precision, nullptr, nullptr, nullptr));
    if (ctx->have_grid && ctx->have_flow && !face_sum && !face_nbr)
        RET_IF(uc_assemble_faces(ctx, dt, nullptr, nullptr, nullptr, nullptr));
    RET_IF(cp_h_impl(ctx, precision, nullptr, nullptr));
    CK(cudaSetDevice(ctx->device));
    RET_IF(launch_chem(ctx, precision, true, true));
    ctx->have_rc = true;
    ctx->rc_start = false;
    return uc_species_update(ctx, dt, isor, relx, tol, spnorm, face_sum, face_nbr, passes);
}

extern "C" int uc_sweep_host(uc_ctx *ctx, int precision, double dt, int isor, double relx, double tol,
                             double spnorm, const double *face_sum, const double *face_nbr, const uc_host_io *io,
                             int *passes)
{
    if (!ctx) return UC_E_ARG;
    if (!io) return set_err(ctx, UC_E_ARG, "uc_sweep_host: io is required");
    if (precision != UC_FP64 && precision != UC_MIXED) return set_err(ctx, UC_E_ARG, "unknown precision %d", precision);
    RET_IF(uc_upload_fields(ctx, io->tk, io->rho, io->fsp, io->stmf, io->stnd));
    RET_IF(props_impl(ctx, precision, nullptr, nullptr, nullptr));
    if (ctx->have_grid && ctx->have_flow && !face_sum && !face_nbr)
        RET_IF(uc_assemble_faces(ctx, dt, nullptr, nullptr, nullptr, nullptr));
    RET_IF(cp_h_impl(ctx, precision, nullptr, nullptr));
    CK(cudaSetDevice(ctx->device));
    RET_IF(launch_chem(ctx, precision, true, true));
    ctx->have_rc = true;
    ctx->rc_start = false;
    if (!ctx->io_stream) {
        CK(cudaStreamCreateWithFlags(&ctx->io_stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&ctx->io_event, cudaEventDisableTiming));
    }
    // the properties, cp/h, omega and d(omega)/dY are final here: the side stream copies them after this
    // point while the update (which writes only Y and soot) runs on the context's stream
    CK(cudaEventRecord(ctx->io_event, ctx->stream));
    RET_IF(uc_species_update(ctx, dt, isor, relx, tol, spnorm, face_sum, face_nbr, nullptr));
    CK(cudaStreamWaitEvent(ctx->io_stream, ctx->io_event, 0));
    struct { double *dst; const double *src; int rows; } o[] = {
        {io->qdsp, ctx->qdsp, LSP}, {io->qdot, ctx->qdot, 1}, {io->domega_dy, ctx->dwdy, LSP}, {io->vmu, ctx->vmu, 1},
        {io->vtc, ctx->vtc, 1}, {io->vdf, ctx->vdf, LSP}, {io->cp, ctx->cp, 1}, {io->h, ctx->h, 1}};
    cudaError_t ce = cudaSuccess;
    for (auto &x : o)
        if (x.dst && x.src && ce == cudaSuccess)
            ce = cudaMemcpy2DAsync(x.dst, (size_t)ctx->n * sizeof(double), x.src, (size_t)ctx->npad * sizeof(double),
                                   (size_t)ctx->n * sizeof(double), x.rows, cudaMemcpyDeviceToHost, ctx->io_stream);
    // the updated state and the pass count after the update, on the context's stream
    if (ce == cudaSuccess) {
        if (io->fsp_out) ce = cudaMemcpy2DAsync(io->fsp_out, (size_t)ctx->n * sizeof(double), ctx->y,
                                                (size_t)ctx->npad * sizeof(double), (size_t)ctx->n * sizeof(double), LSP,
                                                cudaMemcpyDeviceToHost, ctx->stream);
        if (ce == cudaSuccess && io->stmf_out)
            ce = cudaMemcpyAsync(io->stmf_out, ctx->soot, (size_t)ctx->n * sizeof(double), cudaMemcpyDeviceToHost,
                                 ctx->stream);
        if (ce == cudaSuccess && io->stnd_out)
            ce = cudaMemcpyAsync(io->stnd_out, ctx->soot + ctx->npad, (size_t)ctx->n * sizeof(double),
                                 cudaMemcpyDeviceToHost, ctx->stream);
        if (ce == cudaSuccess && passes)
            ce = cudaMemcpyAsync(passes, ctx->passes, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    }
    // both streams drained before returning, also after an error (the host buffers must not be written later)
    const cudaError_t e1 = cudaStreamSynchronize(ctx->io_stream), e2 = cudaStreamSynchronize(ctx->stream);
    if (ce == cudaSuccess) ce = e1 != cudaSuccess ? e1 : e2;
    if (ce != cudaSuccess) return set_err(ctx, UC_E_CUDA, "uc_sweep_host: %s", cudaGetErrorString(ce));
    return check_status(ctx);
}

extern "C" int uc_download_outputs(uc_ctx *ctx, double *qdsp, double *qdot, double *domega_dy, double *vmu,
                                   double *vtc, double *vdf, double *cp, double *h)
{
    if (!ctx) return UC_E_ARG;
    CK(cudaSetDevice(ctx->device));
    struct { double *dst; double *src; int rows; const char *name; } o[] = {
        {qdsp, ctx->qdsp, LSP, "qdsp"}, {qdot, ctx->qdot, 1, "qdot"}, {domega_dy, ctx->dwdy, LSP, "domega_dy"},
        {vmu, ctx->vmu, 1, "vmu"}, {vtc, ctx->vtc, 1, "vtc"}, {vdf, ctx->vdf, LSP, "vdf"},
        {cp, ctx->cp, 1, "cp"}, {h, ctx->h, 1, "h"}};
    for (auto &x : o) {
        if (!x.dst) continue;
        if (!x.src) return set_err(ctx, UC_E_STATE, "%s has not been computed yet", x.name);
        RET_IF(download_rows(ctx, x.dst, x.src, x.rows));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return check_status(ctx);
}

extern "C" int uc_profile(uc_ctx *ctx, int on)
{
    if (!ctx) return UC_E_ARG;
    ctx->prof = on != 0;
    ctx->ev_used.clear();
    return UC_OK;
}

extern "C" int uc_profile_read(uc_ctx *ctx, double *ms, int *launches)
{
    if (!ctx || !ms || !launches) return UC_E_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k < UC_K_COUNT; ++k) { ms[k] = 0.0; launches[k] = 0; }
    for (auto &u : ctx->ev_used) {
        float t = 0.f;
        CK(cudaEventElapsedTime(&t, ctx->ev_pool[u.second], ctx->ev_pool[u.second + 1]));
        ms[u.first] += t;
        launches[u.first] += 1;
    }
    ctx->ev_used.clear();
    return UC_OK;
}

extern "C" int uc_stat(uc_ctx *ctx, const char *name, double *value)
{
    if (!ctx || !name || !value) return UC_E_ARG;
    if (!strcmp(name, "tiles")) { *value = ctx->ntile; return UC_OK; }
    if (!strcmp(name, "int_warps")) { *value = ctx->int_warps; return UC_OK; }
    if (!strcmp(name, "update_ip_warps")) { *value = ctx->upd_ip; return UC_OK; }
    if (!strcmp(name, "update_kind")) { *value = ctx->upd_kind; return UC_OK; }
    if (!strcmp(name, "update_chunk")) { *value = ctx->tr_chunk; return UC_OK; }
    if (!strcmp(name, "update_lockstep")) { *value = ctx->tr_lock; return UC_OK; }
    if (!strcmp(name, "update_flops_per_cell_pass")) { *value = UC_UPDATE_FLOPS_PER_CELL_PASS; return UC_OK; }
    if (!strcmp(name, "int_sorted")) { *value = ctx->int_sorted; return UC_OK; }
    if (!strcmp(name, "int_tune_best_ms")) { *value = ctx->tune_best; return UC_OK; }
    if (!strcmp(name, "int_tune_worst_ms")) { *value = ctx->tune_worst; return UC_OK; }
    if (!strcmp(name, "mixed_fp64_tiles")) {
        int c = 0;
        if (ctx->tile_count) {
            CK(cudaMemcpyAsync(&c, ctx->tile_count, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
        }
        *value = c;
        return UC_OK;
    }
    return set_err(ctx, UC_E_ARG, "unknown statistic '%s'", name);
}

extern "C" int uc_sync(uc_ctx *ctx)
{
    if (!ctx) return UC_E_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    return check_status(ctx);
}

extern "C" const char *uc_last_error(const uc_ctx *ctx)
{
    return ctx ? ctx->err : "null context";
}

extern "C" void uc_destroy(uc_ctx *ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    free_ctx(ctx);
    delete ctx;
}

extern "C" int uc_device_view_get(uc_ctx *ctx, uc_device_view *v)
{
    if (!ctx || !v) return UC_E_ARG;
    v->tk = ctx->tk; v->rho = ctx->rho; v->fsp = ctx->y; v->fsp_old = ctx->y0;
    v->stmf = ctx->soot; v->stnd = ctx->soot + ctx->npad;
    v->rc = ctx->rc; v->qdsp = ctx->qdsp; v->qdot = ctx->qdot; v->domega_dy = ctx->dwdy;
    v->vmu = ctx->vmu; v->vtc = ctx->vtc; v->vdf = ctx->vdf; v->cp = ctx->cp; v->h = ctx->h;
    v->n = ctx->n; v->npad = ctx->npad;
    v->stream = (void *)ctx->stream;
    return UC_OK;
}

// ------------------------------------------------------------------ species-equation faces

static int upload_vec(uc_ctx *ctx, double **dst, const double *src, size_t n)
{
    RET_IF(dalloc(ctx, dst, n));
    CK(cudaMemcpyAsync(*dst, src, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    return UC_OK;
}

extern "C" int uc_set_grid(uc_ctx *ctx, const uc_grid *g)
{
    if (!ctx) return UC_E_ARG;
    if (!g) {
        ctx->have_grid = ctx->faces_ready = false;
        return UC_OK;
    }
    if (g->lj < 3 || g->li < 3 || (long)g->lj * g->li != ctx->n || !g->xxs || !g->xxc || !g->yys || !g->yyc || !g->yr)
        return set_err(ctx, UC_E_ARG, "uc_set_grid: the context's cells must be the lj x li grid (lj, li >= 3)");
    CK(cudaSetDevice(ctx->device));
    ctx->lj = g->lj;
    ctx->li = g->li;
    ctx->isym = g->isym;
    RET_IF(upload_vec(ctx, &ctx->g_xxs, g->xxs, g->li));
    RET_IF(upload_vec(ctx, &ctx->g_xxc, g->xxc, g->li));
    RET_IF(upload_vec(ctx, &ctx->g_yys, g->yys, g->lj));
    RET_IF(upload_vec(ctx, &ctx->g_yyc, g->yyc, g->lj));
    RET_IF(dalloc(ctx, &ctx->g_yr, ctx->npad));
    RET_IF(upload_rows(ctx, ctx->g_yr, g->yr, 1));
    if (!ctx->hold) {
        if (cudaMalloc((void **)&ctx->hold, ctx->npad) != cudaSuccess) { ctx->hold = nullptr; return set_err(ctx, UC_E_NOMEM, "hold mask"); }
    }
    hold_mask_kernel<<<ctx->nsm, 256, 0, ctx->stream>>>(g->lj, g->li, ctx->npad, ctx->hold);
    CK(cudaGetLastError());
    ctx->have_grid = true;
    ctx->faces_ready = false;
    return UC_OK;
}

extern "C" int uc_set_flow(uc_ctx *ctx, const double *u, const double *v, const double *tmu, double sigsp)
{
    if (!ctx) return UC_E_ARG;
    if (!u || !v || !tmu || !(sigsp > 0.0)) return set_err(ctx, UC_E_ARG, "uc_set_flow: u, v, tmu and sigsp > 0 are required");
    CK(cudaSetDevice(ctx->device));
    RET_IF(dalloc(ctx, &ctx->f_u, ctx->npad));
    RET_IF(dalloc(ctx, &ctx->f_v, ctx->npad));
    RET_IF(dalloc(ctx, &ctx->f_tmu, ctx->npad));
    RET_IF(upload_rows(ctx, ctx->f_u, u, 1));
    RET_IF(upload_rows(ctx, ctx->f_v, v, 1));
    RET_IF(upload_rows(ctx, ctx->f_tmu, tmu, 1));
    ctx->sigsp = sigsp;
    ctx->have_flow = true;
    return UC_OK;
}

extern "C" int uc_assemble_faces(uc_ctx *ctx, double dt, double *e, double *w, double *n, double *s)
{
    if (!ctx) return UC_E_ARG;
    if (!ctx->have_grid || !ctx->have_flow) return set_err(ctx, UC_E_STATE, "uc_set_grid and uc_set_flow first");
    if (!ctx->vdf) return set_err(ctx, UC_E_STATE, "the faces need the diffusivities of uc_props");
    CK(cudaSetDevice(ctx->device));
    const size_t rows = (size_t)(LSP - 1) * ctx->npad;
    RET_IF(dalloc(ctx, &ctx->fe, rows));
    RET_IF(dalloc(ctx, &ctx->fw, rows));
    RET_IF(dalloc(ctx, &ctx->fn, rows));
    RET_IF(dalloc(ctx, &ctx->fs, rows));
    if (!ctx->faces_ready)
        for (double *b : {ctx->fe, ctx->fw, ctx->fn, ctx->fs}) CK(cudaMemsetAsync(b, 0, rows * sizeof(double), ctx->stream));
    FaceArgs a{};
    a.P = ctx->dP; a.lj = ctx->lj; a.li = ctx->li; a.npad = ctx->npad; a.isym = ctx->isym;
    a.rho = ctx->rho; a.vdf = ctx->vdf; a.u = ctx->f_u; a.v = ctx->f_v; a.tmu = ctx->f_tmu; a.yr = ctx->g_yr;
    a.xxs = ctx->g_xxs; a.xxc = ctx->g_xxc; a.yys = ctx->g_yys; a.yyc = ctx->g_yyc;
    a.dt = dt; a.sigsp = ctx->sigsp; a.e = ctx->fe; a.w = ctx->fw; a.n = ctx->fn; a.s = ctx->fs;
    faces_kernel<<<std::max(1, std::min((ctx->n + 127) / 128, ctx->nsm * 8)), 128, 0, ctx->stream>>>(a);
    CK(cudaGetLastError());
    ctx->faces_ready = true;
    if (e || w || n || s) {
        RET_IF(download_rows(ctx, e, ctx->fe, LSP - 1));
        RET_IF(download_rows(ctx, w, ctx->fw, LSP - 1));
        RET_IF(download_rows(ctx, n, ctx->fn, LSP - 1));
        RET_IF(download_rows(ctx, s, ctx->fs, LSP - 1));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return UC_OK;
}

// ------------------------------------------------------------------ enthalpy equation (SOLVEH)

// Cells of the skewed plane of the relaxation: (ni + nj - 1) steps x nj rows.
static __host__ __device__ size_t relax_plane(int lj, int li) { return (size_t)((li - 2) + (lj - 2) - 1) * (lj - 2); }

// The relaxation on coefficients already in the skewed layout (cf, f0s) and
// FPZ on entry f0 (natural layout). Writes fpz (natural layout), the pass
// count and its own error word (rb.flags[2 isor + 1], [2 isor + 2]); isor >= 1.
static int launch_relax(uc_ctx *ctx, cudaStream_t st, int nsm, RelaxBuffers &rb, int lj, int li, const double *cf,
                        const double *f0, const double *f0s, int isor, double relx, double tol, double hnorm,
                        double *fpz)
{
    const int nj = lj - 2, ni = li - 2;
    const size_t plane = relax_plane(lj, li);
    // ring of pass results: every pass when it fits in 1 GiB, else as many as fit (at least 2)
    const size_t budget = (size_t)1 << 30;
    int R = (int)std::min<size_t>((size_t)isor, std::max<size_t>(2, budget / (plane * sizeof(double))));
    if (const char *e = getenv("UNICHEM_RELAX_RING")) {     // cap on the ring (memory); 2 is the least
        const int cap = atoi(e);
        if (cap >= 2) R = std::min(R, cap);
    }
    R = std::max(R, 2);
    if ((size_t)R * plane > rb.ring_cap) {
        if (rb.ring) cudaFree(rb.ring);
        rb.ring = nullptr;
        rb.ring_cap = 0;
        if (cudaMalloc((void **)&rb.ring, (size_t)R * plane * sizeof(double)) != cudaSuccess)
            return set_err(ctx, UC_E_NOMEM, "relaxation ring of %d x %zu doubles", R, plane);
        rb.ring_cap = (size_t)R * plane;
    }
    if ((size_t)isor > rb.isor_cap) {
        if (rb.rsdz) cudaFree(rb.rsdz);
        if (rb.flags) cudaFree(rb.flags);
        rb.rsdz = nullptr;
        rb.flags = nullptr;
        rb.isor_cap = 0;
        if (cudaMalloc((void **)&rb.rsdz, (size_t)isor * sizeof(double)) != cudaSuccess ||
            cudaMalloc((void **)&rb.flags, (2 * (size_t)isor + 3) * sizeof(int)) != cudaSuccess)
            return set_err(ctx, UC_E_NOMEM, "relaxation flags");
        rb.isor_cap = isor;
    }
    int *progress = rb.flags, *done = rb.flags + isor, *stop = rb.flags + 2 * isor, *passes = stop + 1, *status = stop + 2;
    CK(cudaMemsetAsync(rb.flags, 0, 2 * (size_t)isor * sizeof(int), st));
    CK(cudaMemsetAsync(passes, 0, 2 * sizeof(int), st));
    CK(cudaMemcpyAsync(stop, &isor, sizeof(int), cudaMemcpyHostToDevice, st));
    RelaxArgs a{};
    a.lj = lj; a.li = li; a.nj = nj; a.ni = ni; a.nstep = ni + nj - 1;
    a.cf = cf; a.f0 = f0; a.f0s = f0s; a.ring = rb.ring; a.rsdz = rb.rsdz;
    a.progress = progress; a.done = done; a.stop_at = stop; a.status = status;
    a.isor = isor; a.R = R;
    a.sor1 = relx; a.sor2 = (double)1.0f - relx; a.tol = tol; a.hnorm = hnorm;
    // the bounded waits between passes give up after UNICHEM_RELAX_WAIT_NS nanoseconds of wall clock (2 s)
    a.timeout_ns = 2000000000LL;
    if (const char *e = getenv("UNICHEM_RELAX_WAIT_NS")) a.timeout_ns = std::max(0LL, atoll(e));
    const int threads = (nj + 31) / 32 * 32;
    const size_t smem = 3 * (size_t)nj * sizeof(double);
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, enth_relax_kernel, threads, smem));
    if (per_sm < 1) return set_err(ctx, UC_E_CUDA, "relaxation kernel does not fit on an SM");
    const int grid = std::min(isor, per_sm * nsm);
    void *args[] = {&a};
    CK(cudaLaunchCooperativeKernel((const void *)enth_relax_kernel, dim3(grid), dim3(threads), args, smem, st));
    enth_relax_final_kernel<<<std::max(1, std::min((lj * li + 255) / 256, nsm * 4)), 256, 0, st>>>(a, fpz, passes);
    CK(cudaGetLastError());
    return UC_OK;
}

// skewed coefficient planes from natural-layout arrays: RHSZ, PPP = RHO - (ZE + ZW + ZN + ZS)
// (solveh.f:1155), ZN, ZS, ZE, ZW, and the interior of FPZ on entry
__global__ void enth_skew_kernel(int lj, int li, const double *rho, const double *rhsz, const double *ze,
                                 const double *zw, const double *zn, const double *zs, const double *f0, double *cf,
                                 double *f0s)
{
    const int nj = lj - 2;
    const size_t plane = relax_plane(lj, li);
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < lj * li; idx += gridDim.x * blockDim.x) {
        const int j = idx % lj, i = idx / lj;
        if (j == 0 || j == lj - 1 || i == 0 || i == li - 1) continue;
        const size_t k = skew_index(j - 1, i - 1, nj);
        cf[CF_RHSZ * plane + k] = rhsz[idx];
        cf[CF_PPP * plane + k] = rho[idx] - (ze[idx] + zw[idx] + zn[idx] + zs[idx]);
        cf[CF_ZN * plane + k] = zn[idx];
        cf[CF_ZS * plane + k] = zs[idx];
        cf[CF_ZE * plane + k] = ze[idx];
        cf[CF_ZW * plane + k] = zw[idx];
        f0s[k] = f0[idx];
    }
}

static int check_relax_grid(uc_ctx *ctx, int lj, int li)
{
    if (lj < 3 || li < 3) return set_err(ctx, UC_E_ARG, "enthalpy relaxation: lj, li >= 3");
    if (lj - 2 > RELAX_MAX_ROWS)
        return set_err(ctx, UC_E_ARG, "enthalpy relaxation: at most %d interior rows (lj - 2), got %d", RELAX_MAX_ROWS,
                       lj - 2);
    return UC_OK;
}

extern "C" int uc_enthalpy_relax(int device, int lj, int li, const double *rho, const double *rhsz, const double *ze,
                                 const double *zw, const double *zn, const double *zs, double *fpz, int isor,
                                 double relx, double tol, double hnorm, int *passes)
{
    if (!rho || !rhsz || !ze || !zw || !zn || !zs || !fpz) return UC_E_ARG;
    RET_IF(check_relax_grid(nullptr, lj, li));
    if (!(relx > 0.0)) return UC_E_ARG;
    const size_t n = (size_t)lj * li, plane = relax_plane(lj, li);
    if (isor < 1) {                   // zero-trip DO loop: FPZ unchanged, ISOR2 = 1 (solveh.f:1149-1167)
        if (passes) *passes = 1;
        return UC_OK;
    }
    if (cudaSetDevice(device) != cudaSuccess) return UC_E_CUDA;
    int nsm = 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return UC_E_CUDA;
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return UC_E_CUDA;
    double *buf = nullptr;
    RelaxBuffers rb;
    int rc = UC_OK;
    int hp[2] = {0, 0};
    do {
        if (cudaMalloc((void **)&buf, (8 * n + 7 * plane) * sizeof(double)) != cudaSuccess) { rc = UC_E_NOMEM; break; }
        double *d_rho = buf, *d_rhsz = d_rho + n, *d_ze = d_rhsz + n, *d_zw = d_ze + n, *d_zn = d_zw + n,
               *d_zs = d_zn + n, *d_f0 = d_zs + n, *d_out = d_f0 + n, *d_cf = d_out + n, *d_f0s = d_cf + 6 * plane;
        const double *src[7] = {rho, rhsz, ze, zw, zn, zs, fpz};
        double *dst[7] = {d_rho, d_rhsz, d_ze, d_zw, d_zn, d_zs, d_f0};
        bool ok = true;
        for (int q = 0; q < 7 && ok; ++q)
            ok = cudaMemcpyAsync(dst[q], src[q], n * sizeof(double), cudaMemcpyHostToDevice, st) == cudaSuccess;
        if (!ok) { rc = UC_E_CUDA; break; }
        enth_skew_kernel<<<std::max(1, std::min((int)((n + 255) / 256), nsm * 4)), 256, 0, st>>>(
            lj, li, d_rho, d_rhsz, d_ze, d_zw, d_zn, d_zs, d_f0, d_cf, d_f0s);
        if (cudaGetLastError() != cudaSuccess) { rc = UC_E_CUDA; break; }
        rc = launch_relax(nullptr, st, nsm, rb, lj, li, d_cf, d_f0, d_f0s, isor, relx, tol,
                          hnorm > 0.0 ? hnorm : (double)n, d_out);
        if (rc != UC_OK) break;
        if (cudaMemcpyAsync(hp, rb.flags + 2 * isor + 2, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaMemcpyAsync(hp + 1, rb.flags + 2 * isor + 1, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) { rc = UC_E_CUDA; break; }
        if (hp[0] == ST_OK &&
            (cudaMemcpyAsync(fpz, d_out, n * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
             cudaStreamSynchronize(st) != cudaSuccess)) { rc = UC_E_CUDA; break; }
        if (hp[0] == ST_RELAX_TIMEOUT) { rc = UC_E_TIMEOUT; break; }
        if (passes) *passes = hp[1];
    } while (0);
    cudaStreamSynchronize(st);
    rb.release();
    if (buf) cudaFree(buf);
    cudaStreamDestroy(st);
    return rc;
}

extern "C" int uc_set_enthalpy(uc_ctx *ctx, const double *ht, const double *w)
{
    if (!ctx) return UC_E_ARG;
    if (!ht) return set_err(ctx, UC_E_ARG, "uc_set_enthalpy: ht is required");
    CK(cudaSetDevice(ctx->device));
    RET_IF(dalloc(ctx, &ctx->ht, ctx->npad));
    RET_IF(upload_rows(ctx, ctx->ht, ht, 1));
    RET_IF(dalloc(ctx, &ctx->e_w, ctx->npad));
    RET_IF(upload_rows(ctx, ctx->e_w, w, 1));       // NULL: no swirl (zeros)
    ctx->have_ht = true;
    return UC_OK;
}

extern "C" int uc_enthalpy_update(uc_ctx *ctx, const uc_enthalpy_opts *o, int *passes, double *resdh)
{
    if (!ctx || !o) return UC_E_ARG;
    if (!ctx->have_grid || !ctx->have_flow) return set_err(ctx, UC_E_STATE, "uc_enthalpy_update: uc_set_grid and uc_set_flow first");
    if (!ctx->have_ht) return set_err(ctx, UC_E_STATE, "uc_enthalpy_update: uc_set_enthalpy first");
    if (!ctx->rc_start) return set_err(ctx, UC_E_STATE, "uc_enthalpy_update needs the rate plane of a species update (uc_sweep)");
    if (!ctx->vtc || !ctx->vdf || !ctx->cp) return set_err(ctx, UC_E_STATE, "uc_enthalpy_update needs the properties and cp of uc_sweep");
    if (!(o->dt >= 0.0) || !(o->relx > 0.0) || !(o->sigh > 0.0)) return set_err(ctx, UC_E_ARG, "invalid dt/relx/sigh");
    RET_IF(check_relax_grid(ctx, ctx->lj, ctx->li));
    CK(cudaSetDevice(ctx->device));
    const size_t np = ctx->npad, plane = relax_plane(ctx->lj, ctx->li);
    for (double **b : {&ctx->e_ekt, &ctx->e_prod, &ctx->e_fpz, &ctx->e_ze, &ctx->e_zw, &ctx->e_zn, &ctx->e_zs, &ctx->e_rhsz})
        RET_IF(dalloc(ctx, b, np));
    RET_IF(dalloc(ctx, &ctx->e_rdhsp, (size_t)LSP * np));
    RET_IF(dalloc(ctx, &ctx->e_cf, CF_N * plane));
    RET_IF(dalloc(ctx, &ctx->e_f0s, plane));
    const int tgrid = ctx->nsm * 4;
    RET_IF(dalloc(ctx, &ctx->e_part, tgrid));
    int slot;
    prof_begin(ctx, UC_K_ENTHALPY, slot);
    // heat release of the start-state RC and the updated Y (solveh.f:116-1145)
    {
        EnthSrcArgs a{};
        a.P = ctx->dP; a.rc = ctx->rc; a.rc32 = ctx->rc32; a.tile_flag = ctx->tile_flag;
        a.tk = ctx->tk; a.y = ctx->y; a.hold = ctx->hold; a.qdsp = ctx->qdsp; a.qdot = ctx->qdot; a.prod = ctx->e_prod;
        a.npad = ctx->npad; a.ntile = ctx->ntile;
        const bool mixed = ctx->rc_prec == UC_MIXED;
        const void *fn = mixed ? (const void *)enth_source_kernel<float> : (const void *)enth_source_kernel<double>;
        CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ENTH_SRC_SMEM));
        if (mixed)
            enth_source_kernel<float><<<std::min(ctx->ntile, 2 * ctx->nsm), CHEM_THREADS, ENTH_SRC_SMEM, ctx->stream>>>(a);
        else
            enth_source_kernel<double><<<std::min(ctx->ntile, 2 * ctx->nsm), CHEM_THREADS, ENTH_SRC_SMEM, ctx->stream>>>(a);
        CK(cudaGetLastError());
    }
    // EKT and the species-enthalpy diffusion factors of every cell
    {
        EnthCoefArgs a{};
        a.P = ctx->dP; a.tk = ctx->tk; a.rho = ctx->rho; a.cp = ctx->cp; a.vtc = ctx->vtc; a.vdf = ctx->vdf;
        a.tmu = ctx->f_tmu; a.sigsp = ctx->sigsp; a.sigh = o->sigh; a.beta2 = ctx->sc.beta2;
        a.ekt = ctx->e_ekt; a.rdhsp = ctx->e_rdhsp; a.n = ctx->n; a.npad = ctx->npad;
        enth_coef_kernel<<<std::max(1, std::min((ctx->n + 127) / 128, ctx->nsm * 8)), 128, 0, ctx->stream>>>(a);
        CK(cudaGetLastError());
    }
    // coefficients and right-hand side of the interior cells
    {
        EnthRhsArgs a{};
        a.P = ctx->dP; a.lj = ctx->lj; a.li = ctx->li; a.npad = ctx->npad; a.isym = ctx->isym;
        a.tk = ctx->tk; a.rho = ctx->rho; a.y = ctx->y; a.ht = ctx->ht; a.stmf = ctx->soot0; a.u = ctx->f_u; a.v = ctx->f_v;
        a.ekt = ctx->e_ekt; a.rdhsp = ctx->e_rdhsp; a.prod = ctx->e_prod;
        a.yr = ctx->g_yr; a.xxs = ctx->g_xxs; a.xxc = ctx->g_xxc; a.yys = ctx->g_yys; a.yyc = ctx->g_yyc;
        a.dt = o->dt; a.crad = ctx->sc.alstr / ctx->sc.rstr / ctx->sc.vstr / ctx->sc.vstr / ctx->sc.vstr;
        a.rsoot = 1.9000e+03;
        a.ze = ctx->e_ze; a.zw = ctx->e_zw; a.zn = ctx->e_zn; a.zs = ctx->e_zs; a.rhsz = ctx->e_rhsz;
        a.cf = ctx->e_cf; a.f0s = ctx->e_f0s;
        enth_rhs_kernel<<<std::max(1, std::min((ctx->n + 127) / 128, ctx->nsm * 8)), 128, 0, ctx->stream>>>(a);
        CK(cudaGetLastError());
    }
    // relaxation of FPZ (solveh.f:1146-1167)
    const double hnorm = o->hnorm > 0.0 ? o->hnorm : (double)ctx->lj * ctx->li;
    int hpass = 1;
    if (o->isor >= 1) {
        RET_IF(launch_relax(ctx, ctx->stream, ctx->nsm, ctx->e_rb, ctx->lj, ctx->li, ctx->e_cf, ctx->ht, ctx->e_f0s,
                            o->isor, o->relx, o->tol, hnorm, ctx->e_fpz));
    } else {
        CK(cudaMemcpyAsync(ctx->e_fpz, ctx->ht, np * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    }
    // T from FPZ, HT := FPZ (solveh.f:1170-1234, spgsolv.f:1304,1358)
    {
        EnthTempArgs a{};
        a.P = ctx->dP; a.lj = ctx->lj; a.li = ctx->li; a.npad = ctx->npad;
        a.y = ctx->y; a.fpz = ctx->e_fpz; a.u = ctx->f_u; a.v = ctx->f_v; a.w = ctx->e_w;
        a.tk = ctx->tk; a.ht = ctx->ht; a.partial = ctx->e_part; a.status = ctx->status;
        a.relax_status = o->isor >= 1 ? ctx->e_rb.flags + 2 * o->isor + 2 : nullptr;
        enth_temp_kernel<<<tgrid, 256, 0, ctx->stream>>>(a);
        CK(cudaGetLastError());
    }
    prof_end(ctx, slot);
    std::vector<double> part(tgrid);
    int st = 0;
    CK(cudaMemcpyAsync(part.data(), ctx->e_part, tgrid * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (o->isor >= 1) {
        CK(cudaMemcpyAsync(&hpass, ctx->e_rb.flags + 2 * o->isor + 1, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(&st, ctx->e_rb.flags + 2 * o->isor + 2, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->rc_start = false;
    if (st != ST_OK)          // T and HT were left as they were
        return set_err(ctx, UC_E_TIMEOUT, "enthalpy relaxation: a wait between passes timed out on the device");
    double r = 0.0;
    for (double v : part) r += v;
    if (passes) *passes = hpass;
    if (resdh) *resdh = r / hnorm;
    return check_status(ctx);
}

extern "C" int uc_density(uc_ctx *ctx)
{
    if (!ctx) return UC_E_ARG;
    if (!ctx->have_fields) return set_err(ctx, UC_E_STATE, "no fields uploaded");
    if (!ctx->have_grid || ctx->li < 3) return set_err(ctx, UC_E_STATE, "uc_density needs the grid of uc_set_grid (li >= 3)");
    CK(cudaSetDevice(ctx->device));
    density_kernel<<<std::max(1, std::min((ctx->n + 255) / 256, ctx->nsm * 4)), 256, 0, ctx->stream>>>(
        ctx->dP, ctx->sc.pback, ctx->n, ctx->npad, ctx->tk, ctx->y, ctx->rho);
    density_edges_kernel<<<1, 1024, 0, ctx->stream>>>(ctx->lj, ctx->li, ctx->rho);
    CK(cudaGetLastError());
    ctx->have_rc = false;
    ctx->rc_start = false;
    return UC_OK;
}

extern "C" int uc_enthalpy_get(uc_ctx *ctx, double *ht, double *rhsz, double *ze, double *zw, double *zn, double *zs)
{
    if (!ctx) return UC_E_ARG;
    CK(cudaSetDevice(ctx->device));
    if (ht) {
        if (!ctx->have_ht) return set_err(ctx, UC_E_STATE, "no enthalpy field");
        RET_IF(download_rows(ctx, ht, ctx->ht, 1));
    }
    const double *src[5] = {ctx->e_rhsz, ctx->e_ze, ctx->e_zw, ctx->e_zn, ctx->e_zs};
    double *dst[5] = {rhsz, ze, zw, zn, zs};
    for (int q = 0; q < 5; ++q) {
        if (!dst[q]) continue;
        if (!src[q]) return set_err(ctx, UC_E_STATE, "no enthalpy update yet");
        RET_IF(download_rows(ctx, dst[q], src[q], 1));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return UC_OK;
}

// ------------------------------------------------------------------ FDETAIL fields

extern "C" int uc_fdetail(uc_ctx *ctx, int lj, int li, const double *x, const double *y, const double *u,
                          const double *v, double *out)
{
    if (!ctx) return UC_E_ARG;
    if (lj < 2 || li < 2 || (long)lj * li != ctx->n || !x || !y || !u || !v || !out)
        return set_err(ctx, UC_E_ARG, "uc_fdetail: the context's cells must be the lj x li grid; x, y, u, v, out required");
    if (!ctx->qdsp || !ctx->qdot || !ctx->vmu || !ctx->vtc || !ctx->vdf)
        return set_err(ctx, UC_E_STATE, "uc_fdetail needs omega and the properties of the state (uc_sweep)");
    CK(cudaSetDevice(ctx->device));
    RET_IF(dalloc(ctx, &ctx->fd_x, ctx->npad));
    RET_IF(dalloc(ctx, &ctx->fd_y, ctx->npad));
    RET_IF(dalloc(ctx, &ctx->fd_u, ctx->npad));
    RET_IF(dalloc(ctx, &ctx->fd_v, ctx->npad));
    RET_IF(dalloc(ctx, &ctx->fd_out, (size_t)FD_ROWS * ctx->npad));
    RET_IF(upload_rows(ctx, ctx->fd_x, x, 1));
    RET_IF(upload_rows(ctx, ctx->fd_y, y, 1));
    RET_IF(upload_rows(ctx, ctx->fd_u, u, 1));
    RET_IF(upload_rows(ctx, ctx->fd_v, v, 1));
    FdArgs a{};
    a.P = ctx->dP; a.lj = lj; a.li = li; a.npad = ctx->npad;
    a.x = ctx->fd_x; a.y = ctx->fd_y; a.u = ctx->fd_u; a.v = ctx->fd_v;
    a.rho = ctx->rho; a.tk = ctx->tk; a.qdot = ctx->qdot; a.vmu = ctx->vmu; a.vtc = ctx->vtc;
    a.fsp = ctx->y; a.vdf = ctx->vdf; a.qdsp = ctx->qdsp;
    a.ALSTR = ctx->sc.alstr; a.RSTR = ctx->sc.rstr; a.TSTR = ctx->sc.tstr; a.AMSTR = ctx->sc.amstr;
    a.ACSTR = ctx->sc.acstr; a.VSTR = ctx->sc.vstr; a.DSTR = ctx->sc.dstr;
    a.out = ctx->fd_out;
    fdetail_kernel<<<std::max(1, std::min((ctx->n + 255) / 256, ctx->nsm * 8)), 256, 0, ctx->stream>>>(a);
    CK(cudaGetLastError());
    RET_IF(download_rows(ctx, out, ctx->fd_out, FD_ROWS));
    CK(cudaStreamSynchronize(ctx->stream));
    return UC_OK;
}

// ------------------------------------------------------------------ batched stiff integration

static bool same_opts(const uc_integrate_opts &a, const uc_integrate_opts &b)
{
    return a.dt == b.dt && a.isor == b.isor && a.relx == b.relx && a.tol == b.tol && a.c_tau == b.c_tau &&
           a.y_tau == b.y_tau && a.nsub_max == b.nsub_max;
}

static int check_opts(uc_ctx *ctx, const uc_integrate_opts *o)
{
    if (!o) return set_err(ctx, UC_E_ARG, "integration options are required");
    if (!(o->dt > 0.0) || o->isor < 1 || !(o->relx > 0.0 && o->relx <= 1.0) || !(o->tol >= 0.0) || !(o->c_tau > 0.0) ||
        !(o->y_tau >= 0.0) || o->nsub_max < 1 || o->nsub_max > SORT_MAXBIN)
        return set_err(ctx, UC_E_ARG, "integration options out of range (dt>0, isor>=1, 0<relx<=1, tol>=0, c_tau>0, "
                                      "y_tau>=0, 1<=nsub_max<=%d)", SORT_MAXBIN);
    return UC_OK;
}

static int ensure_pressure(uc_ctx *ctx)
{
    if (ctx->pnd) return UC_OK;
    RET_IF(dalloc(ctx, &ctx->pnd, ctx->npad));
    std::vector<double> pb(ctx->npad, ctx->sc.pback);
    CK(cudaMemcpy(ctx->pnd, pb.data(), ctx->npad * sizeof(double), cudaMemcpyHostToDevice));
    return UC_OK;
}

static int integrate_buffers(uc_ctx *ctx)
{
    const size_t np = ctx->npad;
    const int nchunk = (ctx->n + SORT_CHUNK - 1) / SORT_CHUNK;
    RET_IF(ensure_pressure(ctx));
    RET_IF(dalloc(ctx, &ctx->qdsp, (size_t)LSP * np));
    int **bufs[] = {&ctx->nsub, &ctx->order, &ctx->cpasses, &ctx->hist, &ctx->next_tile};
    const size_t counts[] = {np, np, np, (size_t)(SORT_MAXBIN + 1) * nchunk, 1};
    for (int i = 0; i < 5; ++i)
        if (!*bufs[i]) {
            cudaError_t e = cudaMalloc((void **)bufs[i], counts[i] * sizeof(int));
            if (e != cudaSuccess) {
                *bufs[i] = nullptr;
                return set_err(ctx, UC_E_NOMEM, "integration buffers: %s", cudaGetErrorString(e));
            }
        }
    return UC_OK;
}

extern "C" int uc_set_pressure(uc_ctx *ctx, const double *pnd)
{
    if (!ctx || !pnd) return set_err(ctx, UC_E_ARG, "uc_set_pressure: pressures are required");
    CK(cudaSetDevice(ctx->device));
    RET_IF(dalloc(ctx, &ctx->pnd, ctx->npad));
    RET_IF(upload_rows(ctx, ctx->pnd, pnd, 1));
    return UC_OK;
}

extern "C" int uc_hold_enthalpy(uc_ctx *ctx)
{
    if (!ctx) return UC_E_ARG;
    if (!ctx->have_fields) return set_err(ctx, UC_E_STATE, "no fields uploaded");
    CK(cudaSetDevice(ctx->device));
    RET_IF(dalloc(ctx, &ctx->enth, ctx->npad));
    hold_enthalpy_kernel<<<ctx->nsm * 4, 256, 0, ctx->stream>>>(ctx->dP, ctx->tk, ctx->y, ctx->npad, ctx->enth);
    CK(cudaGetLastError());
    return UC_OK;
}

extern "C" int uc_temperature_from_held(uc_ctx *ctx)
{
    if (!ctx) return UC_E_ARG;
    if (!ctx->enth) return set_err(ctx, UC_E_STATE, "uc_hold_enthalpy first");
    CK(cudaSetDevice(ctx->device));
    RET_IF(ensure_pressure(ctx));
    int slot;
    prof_begin(ctx, UC_K_TEMP, slot);
    temperature_held_kernel<<<ctx->nsm * 4, 128, 0, ctx->stream>>>(ctx->dP, ctx->enth, ctx->y, ctx->pnd, ctx->npad,
                                                                    ctx->tk, ctx->rho, ctx->status);
    prof_end(ctx, slot);
    CK(cudaGetLastError());
    return UC_OK;
}

template <int NW>
static bool set_integrate_attr()
{
    return cudaFuncSetAttribute(integrate_fp64_kernel<NW, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)INT_SMEM) == cudaSuccess &&
           cudaFuncSetAttribute(integrate_fp64_kernel<NW, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)INT_SMEM) == cudaSuccess;
}

// The rounds form's arrays inside rnd_state / rnd_int: two state buffers b = 0, 1, then (ints) the sort
// keys and permutation of a round, the cells and tiles of each round and the tile list 0..ntile-1
static RoundState round_state(uc_ctx *ctx, int b)
{
    const size_t np = ctx->npad;
    RoundState r;
    r.y = ctx->rnd_state + (size_t)b * (LSP + 6) * np;
    r.tk = r.y + (size_t)LSP * np;
    r.rho = r.tk + np;
    r.pnd = r.rho + np;
    r.soot = r.pnd + np;
    r.enth = r.soot + 2 * np;
    r.nsub = ctx->rnd_int + (size_t)b * 4 * np;
    r.passes = r.nsub + np;
    r.last = r.passes + np;
    r.ord = r.last + np;
    return r;
}
static size_t round_state_doubles(uc_ctx *ctx) { return 2 * (size_t)(LSP + 6) * ctx->npad; }
static size_t round_ints(uc_ctx *ctx) { return 10 * (size_t)ctx->npad + 2 * SORT_MAXBIN + ctx->ntile; }
static int *round_key(uc_ctx *ctx) { return ctx->rnd_int + 8 * (size_t)ctx->npad; }
static int *round_perm(uc_ctx *ctx) { return round_key(ctx) + ctx->npad; }
static int *round_cells(uc_ctx *ctx) { return round_perm(ctx) + ctx->npad; }
static int *round_tiles(uc_ctx *ctx) { return round_cells(ctx) + SORT_MAXBIN; }
static int *round_tile_list(uc_ctx *ctx) { return round_tiles(ctx) + SORT_MAXBIN; }

// Rounds form of the integration step (FP64; after the sub-step counts and the sort): the state is gathered
// in n_sub order, then round r advances the cells with n_sub > r (a prefix of the positions) by one sub-step
// with the field kernels -- chem_fp64_kernel for RC and SOUR of those tiles, the per-cell tile-resident
// update (own dt, own stop, closure), T from the held enthalpy and rho -- and re-orders the prefix for the
// next round (the cells that go on first, by the passes of their last sub-step; a stable counting sort and
// a permutation into the other state buffer); at the end the state is scattered back to cell order. Every
// kernel reads its round's cell or tile count from device memory, so the step is one graph whatever the
// counts are.
static int enqueue_rounds(uc_ctx *ctx, const uc_integrate_opts &o)
{
    const int np = ctx->npad;
    const int nchunk = (ctx->n + SORT_CHUNK - 1) / SORT_CHUNK;
    int *cells = round_cells(ctx), *tiles = round_tiles(ctx), *key = round_key(ctx), *perm = round_perm(ctx);
    const int eg = std::max(1, std::min((np + 255) / 256, ctx->nsm * 8));
    round_counts_kernel<<<(o.nsub_max + 255) / 256, 256, 0, ctx->stream>>>(ctx->hist, nchunk, o.nsub_max, cells, tiles);
    CK(cudaGetLastError());
    RoundState rs = round_state(ctx, 0), other = round_state(ctx, 1);
    gather_state_kernel<<<eg, 256, 0, ctx->stream>>>(ctx->order, ctx->n, np, ctx->y, ctx->tk, ctx->rho, ctx->pnd,
                                                     ctx->soot, ctx->nsub, rs);
    CK(cudaGetLastError());
    hold_enthalpy_kernel<<<ctx->nsm * 4, 256, 0, ctx->stream>>>(ctx->dP, rs.tk, rs.y, np, rs.enth);
    CK(cudaGetLastError());
    ChemArgs c{};
    c.P = ctx->dP; c.tab = ctx->dTab;
    c.rc = ctx->rc; c.sour = ctx->sour;
    c.n = ctx->n; c.npad = np; c.ntile = ctx->ntile; c.status = ctx->status;
    c.tile_list = round_tile_list(ctx);
    UpdArgs u{};
    u.P = ctx->dP; u.rc = ctx->rc; u.sour = ctx->sour;
    u.dt = o.dt; u.sor1 = o.relx; u.tol = o.tol; u.isor = o.isor;
    u.n = ctx->n; u.npad = np; u.ntile = ctx->ntile;
    for (int r = 0; r < o.nsub_max; ++r) {
        c.tk = rs.tk; c.rho = rs.rho; c.y = rs.y; c.stmf = rs.soot; c.stnd = rs.soot + np;
        c.tile_count = tiles + r;
        chem_fp64_kernel<<<std::min(ctx->ntile, ctx->nsm), CHEM_THREADS, CHEM_SMEM, ctx->stream>>>(c);
        CK(cudaGetLastError());
        u.rho = rs.rho;
        u.y0 = rs.y; u.soot0 = rs.soot; u.y = rs.y; u.soot = rs.soot;     // old level = the sub-step's start state
        update_cells_kernel<<<ctx->nsm, TR_WARPS * 32, TR_SMEM, ctx->stream>>>(u, cells + r, rs.nsub, rs.passes,
                                                                               rs.last, ctx->status, ctx->tr_map[0],
                                                                               ctx->tr_map[1]);
        CK(cudaGetLastError());
        temperature_held_kernel<<<ctx->nsm * 4, 128, 0, ctx->stream>>>(ctx->dP, rs.enth, rs.y, rs.pnd, np, rs.tk,
                                                                        rs.rho, ctx->status, cells + r);
        CK(cudaGetLastError());
        if (r + 1 == o.nsub_max) break;
        round_key_kernel<<<eg, 256, 0, ctx->stream>>>(rs.nsub, rs.last, cells + r, r, key);
        CK(cudaGetLastError());
        key_count_kernel<<<nchunk, 256, 0, ctx->stream>>>(key, cells + r, ROUND_KEYS, nchunk, ctx->hist);
        CK(cudaGetLastError());
        sort_scan_kernel<<<1, 1024, 0, ctx->stream>>>(ctx->hist, ROUND_KEYS * nchunk);
        CK(cudaGetLastError());
        key_scatter_kernel<<<nchunk, 32, 0, ctx->stream>>>(key, cells + r, ROUND_KEYS, nchunk, ctx->hist, perm);
        CK(cudaGetLastError());
        permute_state_kernel<<<eg, 256, 0, ctx->stream>>>(perm, cells + r, np, rs, other);
        CK(cudaGetLastError());
        std::swap(rs, other);
    }
    scatter_state_kernel<<<eg, 256, 0, ctx->stream>>>(ctx->n, np, rs, ctx->y, ctx->tk, ctx->rho, ctx->soot,
                                                      ctx->cpasses);
    CK(cudaGetLastError());
    return UC_OK;
}

// Enqueue one integration step on the context's stream (graph capture or not). warps 16 or 8: the
// persistent kernel with that many warps; 3: the rounds form (FP64; the mixed form takes 16 warps).
static int enqueue_integrate(uc_ctx *ctx, int precision, const uc_integrate_opts &o, int warps, int sorted)
{
    const int np = ctx->npad;
    if (warps == 3 && precision != UC_FP64) warps = 16;
    if (warps == 3) sorted = 1;
    // omega of the start state (QDSP rows) for the sub-step counts
    if (precision == UC_MIXED) {
        ChemMArgs m{};
        m.P = ctx->dP; m.tab = ctx->dTabM;
        m.tk = ctx->tk; m.rho = ctx->rho; m.y = ctx->y; m.stmf = ctx->soot; m.stnd = ctx->soot + np;
        m.qdsp = ctx->qdsp; m.tile_flag = ctx->tile_flag;
        m.n = ctx->n; m.npad = np; m.ntile = ctx->ntile; m.status = ctx->status;
        chem_mixed_kernel<<<std::min(ctx->ntile, ctx->nsm), CHEM_THREADS, CHEMM_SMEM, ctx->stream>>>(m);
        CK(cudaGetLastError());
        compact_tiles_kernel<<<1, 1024, 0, ctx->stream>>>(ctx->tile_flag, ctx->ntile, ctx->tile_list, ctx->tile_count);
        CK(cudaGetLastError());
    }
    ChemArgs c{};
    c.P = ctx->dP; c.tab = ctx->dTab;
    c.tk = ctx->tk; c.rho = ctx->rho; c.y = ctx->y; c.stmf = ctx->soot; c.stnd = ctx->soot + np;
    c.qdsp = ctx->qdsp;
    c.n = ctx->n; c.npad = np; c.ntile = ctx->ntile; c.status = ctx->status;
    if (precision == UC_MIXED) { c.tile_list = ctx->tile_list; c.tile_count = ctx->tile_count; }
    chem_fp64_kernel<<<std::min(ctx->ntile, ctx->nsm), CHEM_THREADS, CHEM_SMEM, ctx->stream>>>(c);
    CK(cudaGetLastError());
    nsub_kernel<<<std::max(1, std::min((np + 255) / 256, ctx->nsm * 8)), 256, 0, ctx->stream>>>(
        ctx->dP, ctx->rho, ctx->y, ctx->qdsp, ctx->n, np, o.dt, o.c_tau, o.y_tau, o.nsub_max, ctx->nsub);
    CK(cudaGetLastError());
    if (sorted) {
        const int nchunk = (ctx->n + SORT_CHUNK - 1) / SORT_CHUNK;
        sort_count_kernel<<<nchunk, 256, 0, ctx->stream>>>(ctx->nsub, ctx->n, o.nsub_max, nchunk, ctx->hist);
        CK(cudaGetLastError());
        sort_scan_kernel<<<1, 1024, 0, ctx->stream>>>(ctx->hist, (o.nsub_max + 1) * nchunk);
        CK(cudaGetLastError());
        sort_scatter_kernel<<<nchunk, 32, 0, ctx->stream>>>(ctx->nsub, ctx->n, np, o.nsub_max, nchunk, ctx->hist,
                                                           ctx->order);
        CK(cudaGetLastError());
    }
    if (warps == 3) return enqueue_rounds(ctx, o);
    CK(cudaMemsetAsync(ctx->next_tile, 0, sizeof(int), ctx->stream));
    IntArgs a{};
    a.P = ctx->dP; a.tab = ctx->dTab; a.tabm = ctx->dTabM;
    a.tk = ctx->tk; a.rho = ctx->rho; a.y = ctx->y; a.soot = ctx->soot; a.pnd = ctx->pnd;
    a.nsub = ctx->nsub; a.order = sorted ? ctx->order : nullptr; a.next_tile = ctx->next_tile;
    a.passes = ctx->cpasses; a.status = ctx->status;
    a.dt = o.dt; a.sor1 = o.relx; a.tol = o.tol; a.isor = o.isor;
    a.n = ctx->n; a.npad = np; a.ntile = ctx->ntile;
    const int grid = std::min(ctx->ntile, ctx->nsm);
    const bool mixed = precision == UC_MIXED;
    if (warps == 16 && mixed)
        integrate_fp64_kernel<16, true><<<grid, 16 * 32, INT_SMEM, ctx->stream>>>(a);
    else if (warps == 16)
        integrate_fp64_kernel<16, false><<<grid, 16 * 32, INT_SMEM, ctx->stream>>>(a);
    else if (warps == 8 && mixed)
        integrate_fp64_kernel<8, true><<<grid, 8 * 32, INT_SMEM, ctx->stream>>>(a);
    else if (warps == 8)
        integrate_fp64_kernel<8, false><<<grid, 8 * 32, INT_SMEM, ctx->stream>>>(a);
    else
        return set_err(ctx, UC_E_ARG, "integration kernel shape %d warps is not built", warps);
    CK(cudaGetLastError());
    return UC_OK;
}

static int integrate_prepare(uc_ctx *ctx, int precision, const uc_integrate_opts *o)
{
    if (!ctx) return UC_E_ARG;
    if (precision != UC_FP64 && precision != UC_MIXED)
        return set_err(ctx, UC_E_ARG, "integration precision %d is not available", precision);
    RET_IF(check_opts(ctx, o));
    if (!ctx->have_fields) return set_err(ctx, UC_E_STATE, "no fields uploaded");
    CK(cudaSetDevice(ctx->device));
    RET_IF(integrate_buffers(ctx));
    if (precision == UC_MIXED && !ctx->tile_flag) {
        if (cudaMalloc((void **)&ctx->tile_flag, ctx->ntile * sizeof(int)) != cudaSuccess ||
            cudaMalloc((void **)&ctx->tile_list, ctx->ntile * sizeof(int)) != cudaSuccess ||
            cudaMalloc((void **)&ctx->tile_count, sizeof(int)) != cudaSuccess)
            return set_err(ctx, UC_E_NOMEM, "tile flag buffers");
    }
    if (!set_integrate_attr<16>() || !set_integrate_attr<8>())
        return set_err(ctx, UC_E_CUDA, "integration kernel shared-memory attribute");
    if (precision == UC_FP64) {
        // the rounds form: its state copy in n_sub order, the RC plane and its tensor maps
        const size_t np = ctx->npad;
        if (!ctx->rnd_state) RET_IF(dalloc(ctx, &ctx->rnd_state, round_state_doubles(ctx)));
        if (!ctx->rnd_int) {
            cudaError_t e = cudaMalloc((void **)&ctx->rnd_int, round_ints(ctx) * sizeof(int));
            if (e != cudaSuccess) {
                ctx->rnd_int = nullptr;
                return set_err(ctx, UC_E_NOMEM, "integration rounds buffers: %s", cudaGetErrorString(e));
            }
            iota_kernel<<<std::max(1, std::min((ctx->ntile + 255) / 256, ctx->nsm * 4)), 256, 0, ctx->stream>>>(
                round_tile_list(ctx), ctx->ntile);
            CK(cudaGetLastError());
        }
        if (!ctx->rc) RET_IF(dalloc(ctx, &ctx->rc, (size_t)LRX * np));
        RET_IF(encode_rc_map(ctx));
        if (cudaFuncSetAttribute(update_cells_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TR_SMEM) !=
            cudaSuccess)
            return set_err(ctx, UC_E_CUDA, "integration rounds: update kernel shared-memory attribute");
        if (cudaFuncSetAttribute(chem_fp64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CHEM_SMEM) !=
            cudaSuccess)
            return set_err(ctx, UC_E_CUDA, "integration rounds: rate kernel shared-memory attribute");
    }
    return UC_OK;
}

extern "C" int uc_integrate(uc_ctx *ctx, int precision, const uc_integrate_opts *o)
{
    RET_IF(integrate_prepare(ctx, precision, o));
    ctx->rc_start = false;
    ctx->have_rc = false;          // the state moves on (and the rounds form uses the RC plane)
    const bool fresh = ctx->int_exec && ctx->int_prec == precision && ctx->int_gwarps == ctx->int_warps &&
                       ctx->int_gsorted == ctx->int_sorted && same_opts(ctx->int_opts, *o);
    if (!fresh) {
        if (ctx->int_exec) { cudaGraphExecDestroy(ctx->int_exec); ctx->int_exec = nullptr; }
        if (ctx->int_graph) { cudaGraphDestroy(ctx->int_graph); ctx->int_graph = nullptr; }
        CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        const int rc = enqueue_integrate(ctx, precision, *o, ctx->int_warps, ctx->int_sorted);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
        if (rc != UC_OK) { if (g) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) return set_err(ctx, UC_E_CUDA, "graph capture: %s", cudaGetErrorString(e));
        e = cudaGraphInstantiate(&ctx->int_exec, g, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(g);
            return set_err(ctx, UC_E_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
        }
        ctx->int_graph = g;
        ctx->int_prec = precision;
        ctx->int_gwarps = ctx->int_warps;
        ctx->int_gsorted = ctx->int_sorted;
        ctx->int_opts = *o;
    }
    int slot;
    prof_begin(ctx, UC_K_INTEGRATE, slot);
    CK(cudaGraphLaunch(ctx->int_exec, ctx->stream));
    prof_end(ctx, slot);
    return UC_OK;
}

extern "C" int uc_integrate_tune(uc_ctx *ctx, int precision, const uc_integrate_opts *o)
{
    RET_IF(integrate_prepare(ctx, precision, o));
    const size_t np = ctx->npad;
    // save the state, run each shape once from it, keep the fastest
    double *save = nullptr;
    const size_t nd = (size_t)(LSP + 4) * np;
    cudaError_t e = cudaMalloc((void **)&save, nd * sizeof(double));
    if (e != cudaSuccess) return set_err(ctx, UC_E_NOMEM, "tuning copy of the state: %s", cudaGetErrorString(e));
    auto copy_state = [&](bool to_save) -> cudaError_t {
        double *src[4] = {ctx->tk, ctx->rho, ctx->y, ctx->soot};
        const size_t cnt[4] = {np, np, (size_t)LSP * np, 2 * np};
        size_t off = 0;
        for (int i = 0; i < 4; ++i) {
            cudaError_t r = to_save ? cudaMemcpyAsync(save + off, src[i], cnt[i] * sizeof(double),
                                                      cudaMemcpyDeviceToDevice, ctx->stream)
                                    : cudaMemcpyAsync(src[i], save + off, cnt[i] * sizeof(double),
                                                      cudaMemcpyDeviceToDevice, ctx->stream);
            if (r != cudaSuccess) return r;
            off += cnt[i];
        }
        return cudaSuccess;
    };
    // persistent kernel (16 or 8 warps, sorted or natural queue order); the rounds form (FP64)
    const int shapes[5][2] = {{16, 1}, {8, 1}, {16, 0}, {8, 0}, {3, 1}};
    const int nshape = precision == UC_FP64 ? 5 : 4;
    double best = 1e300, worst = 0.0;
    int bw = 16, bs = 1, rc = UC_OK;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    if (copy_state(true) != cudaSuccess) rc = set_err(ctx, UC_E_CUDA, "tuning: state copy failed");
    for (int i = 0; i < nshape && rc == UC_OK; ++i) {
        cudaEventRecord(e0, ctx->stream);
        rc = enqueue_integrate(ctx, precision, *o, shapes[i][0], shapes[i][1]);
        cudaEventRecord(e1, ctx->stream);
        if (rc != UC_OK) break;
        if (cudaEventSynchronize(e1) != cudaSuccess) { rc = set_err(ctx, UC_E_CUDA, "tuning run failed"); break; }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) { best = ms; bw = shapes[i][0]; bs = shapes[i][1]; }
        if (ms > worst) worst = ms;
        if (copy_state(false) != cudaSuccess) rc = set_err(ctx, UC_E_CUDA, "tuning: state restore failed");
    }
    cudaStreamSynchronize(ctx->stream);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(save);
    if (rc != UC_OK) return rc;
    ctx->int_warps = bw;
    ctx->int_sorted = bs;
    ctx->tune_best = best;
    ctx->tune_worst = worst;
    const int st = check_status(ctx);
    return st == UC_E_NOCONV ? UC_OK : st;   // a Newton that ran out of steps is reported by uc_integrate_counts
}

extern "C" int uc_integrate_counts(uc_ctx *ctx, int *nsub, int *passes)
{
    if (!ctx) return UC_E_ARG;
    if (!ctx->nsub) return set_err(ctx, UC_E_STATE, "no integration has run");
    if (nsub) CK(cudaMemcpyAsync(nsub, ctx->nsub, (size_t)ctx->n * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    if (passes)
        CK(cudaMemcpyAsync(passes, ctx->cpasses, (size_t)ctx->n * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return check_status(ctx);
}

// ------------------------------------------------------------------ tensor-core GEMM

// A row-major BF16 matrix [rows][ld] (its first `cols` columns) as a TMA tensor map: boxes of 64 columns
// (128 B) x box_rows rows, 128-byte swizzle (the K-major operand layout of the tensor-core kernels), rows
// beyond `rows` read as zeros.
static bool encode_bf16_map(CUtensorMap *m, const void *base, int cols, int rows, int ld, int box_rows)
{
    uc_encode_tiled_fn encode = tensor_map_encoder();
    if (!encode || ((uintptr_t)base & 15) || ld % 8 || cols % GK || box_rows < 1 || box_rows > 256) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {(cuuint32_t)GK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// multiprocessors of the current device (cached per device)
static int device_sms()
{
    static thread_local int nsm = 0, nsm_dev = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (nsm_dev != dev) {
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        nsm_dev = dev;
    }
    return nsm;
}

// split-K factor of the tiled GEMM: FP32 outputs only, enough CTAs to cover the SMs, at least four K
// chunks per split, and no more partial tiles than `ws_floats` holds
static int gemm_splits(const GemmArgs &g, size_t ws_floats)
{
    if (g.epi != EPI_F32 || !ws_floats) return 1;
    const int tiles = ((g.M + GM - 1) / GM) * ((g.N + GN_MAX - 1) / GN_MAX), nk = g.K / GK;
    int sp = std::min(nk / 4, (device_sms() + tiles - 1) / tiles);
    sp = (int)std::min<size_t>((size_t)sp, ws_floats / ((size_t)g.M * g.N));
    if (sp <= 1) return 1;
    const int per = (nk + sp - 1) / sp;
    return (nk + per - 1) / per;                 // no empty split
}

// Launch C = A * B^T on the stream (mlp_gemm.cuh gives the shapes it takes); FP32 outputs are split
// along K over the workspace `ws` ([splits][M][N]) when that fills more SMs, then reduced in order.
static cudaError_t launch_gemm(const GemmArgs &g, cudaStream_t st, float *ws, size_t ws_floats)
{
    static thread_local int attr_done = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (attr_done != dev) {
        cudaError_t e = cudaFuncSetAttribute(gemm_bf16_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)GEMM_SMEM_LAUNCH);
        if (e != cudaSuccess) return e;
        attr_done = dev;
    }
    const int sp = gemm_splits(g, ws_floats);
    // without a split, narrower column tiles where 256-column ones would leave SMs idle (one row per
    // thread in the epilogue: more CTAs, more rows in flight)
    GemmArgs gt = g;
    gt.ntile = GN_MAX;
    const int mt = (g.M + GM - 1) / GM;
    while (sp == 1 && gt.ntile > 64 && mt * ((g.N + gt.ntile - 1) / gt.ntile) < device_sms() && gt.ntile / 2 < g.N)
        gt.ntile /= 2;
    CUtensorMap map_a, map_b;
    if (!encode_bf16_map(&map_a, g.A, g.K, g.M, g.lda, GM) ||
        !encode_bf16_map(&map_b, g.B, g.K, g.N, g.ldb, std::min(g.N, gt.ntile)))
        return cudaErrorInvalidValue;
    dim3 grid(mt, (g.N + gt.ntile - 1) / gt.ntile, sp);
    if (sp == 1) {
        gemm_bf16_tc_kernel<<<grid, GEMM_THREADS, GEMM_SMEM_LAUNCH, st>>>(gt, map_a, map_b);
        return cudaGetLastError();
    }
    GemmArgs gs = gt;
    gs.out_f32 = ws;
    gs.ldo = g.N;
    gs.split_stride = (size_t)g.M * g.N;
    gemm_bf16_tc_kernel<<<grid, GEMM_THREADS, GEMM_SMEM_LAUNCH, st>>>(gs, map_a, map_b);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    splitk_reduce_kernel<<<device_sms() * 2, 256, 0, st>>>(ws, sp, g.M, g.N, g.out_f32, g.ldo);
    return cudaGetLastError();
}

// One network layer over M rows with the weights resident in shared memory (mlp_gemm.cuh):
// N and K multiples of 64 up to 256.
static cudaError_t launch_layer(const GemmArgs &g, int nsm, cudaStream_t st)
{
    if (g.N % 64 || g.N > 256 || g.K % GK || g.K > 256 || g.M <= 0) return cudaErrorInvalidValue;
    if (g.epi == EPI_DECODE && (!g.dec_out || g.dec_n > g.N || g.dec_n > 64)) return cudaErrorInvalidValue;
    static thread_local int attr_done = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (attr_done != dev) {
        cudaError_t e = cudaFuncSetAttribute(gemm_w_resident_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)LW_SMEM);
        if (e != cudaSuccess) return e;
        attr_done = dev;
    }
    CUtensorMap map_a, map_w;
    if (!encode_bf16_map(&map_a, g.A, g.K, g.M, g.lda, GM) || !encode_bf16_map(&map_w, g.B, g.K, g.N, g.ldb, g.N))
        return cudaErrorInvalidValue;
    const int ntiles = (g.M + GM - 1) / GM;
    gemm_w_resident_kernel<<<std::min(ntiles, nsm), LW_THREADS, LW_SMEM, st>>>(g, map_a, map_w);
    return cudaGetLastError();
}

static bool gemm_shape_ok(int M, int N, int K, int lda, int ldb)
{
    return M > 0 && N > 0 && K > 0 && N % 16 == 0 && K % GK == 0 && lda % 8 == 0 && ldb % 8 == 0 && lda >= K &&
           ldb >= K;
}

extern "C" int uc_gemm_bf16(int device, int kernel, int M, int N, int K, const uint16_t *a, const uint16_t *b, float *c)
{
    if (!a || !b || !c || !gemm_shape_ok(M, N, K, K, K)) return UC_E_ARG;
    if (kernel != 0 && (kernel != 1 || N > 256 || N % 64 != 0 || K > 256)) return UC_E_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return UC_E_CUDA;
    __nv_bfloat16 *dA = nullptr, *dB = nullptr;
    float *dC = nullptr;
    int *dst = nullptr, st = 0, rc = UC_OK;
    if (cudaMalloc((void **)&dA, (size_t)M * K * 2) != cudaSuccess || cudaMalloc((void **)&dB, (size_t)N * K * 2) != cudaSuccess ||
        cudaMalloc((void **)&dC, (size_t)M * N * 4) != cudaSuccess || cudaMalloc((void **)&dst, sizeof(int)) != cudaSuccess)
        rc = UC_E_NOMEM;
    if (rc == UC_OK) {
        cudaMemcpy(dA, a, (size_t)M * K * 2, cudaMemcpyHostToDevice);
        cudaMemcpy(dB, b, (size_t)N * K * 2, cudaMemcpyHostToDevice);
        cudaMemset(dst, 0, sizeof(int));
        GemmArgs g{};
        g.A = dA; g.B = dB; g.lda = K; g.ldb = K; g.M = M; g.N = N; g.K = K;
        g.epi = EPI_F32; g.out_f32 = dC; g.ldo = N; g.status = dst;
        float *zb = nullptr;
        cudaError_t e;
        if (kernel == 1) {                 // the layer kernel adds a bias: give it zeros
            g.epi = EPI_BIAS_F32;
            if (cudaMalloc((void **)&zb, N * sizeof(float)) != cudaSuccess) rc = UC_E_NOMEM;
            else cudaMemset(zb, 0, N * sizeof(float));
            g.bias = zb;
            cudaDeviceProp prop;
            cudaGetDeviceProperties(&prop, device);
            e = rc == UC_OK ? launch_layer(g, prop.multiProcessorCount, 0) : cudaSuccess;
        } else {
            const size_t wsf = (size_t)M * N * std::max(1, K / GK / 4);   // the largest split gemm_splits may take
            float *ws = nullptr;
            if (cudaMalloc((void **)&ws, wsf * sizeof(float)) != cudaSuccess) rc = UC_E_NOMEM;
            e = rc == UC_OK ? launch_gemm(g, 0, ws, wsf) : cudaSuccess;
            if (rc == UC_OK && e == cudaSuccess) e = cudaDeviceSynchronize();
            cudaFree(ws);
        }
        if (rc == UC_OK && (e != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)) rc = UC_E_CUDA;
        cudaFree(zb);
        if (rc == UC_OK) {
            cudaMemcpy(c, dC, (size_t)M * N * 4, cudaMemcpyDeviceToHost);
            cudaMemcpy(&st, dst, sizeof(int), cudaMemcpyDeviceToHost);
            if (st == ST_MMA_TIMEOUT) rc = UC_E_TIMEOUT;
        }
    }
    cudaFree(dA); cudaFree(dB); cudaFree(dC); cudaFree(dst);
    return rc;
}

// ------------------------------------------------------------------ learned surrogate

// split-K workspace of the weight-gradient GEMMs: 32 partial tiles of the largest layer (256 x 256)
constexpr size_t MLP_WS_FLOATS = (size_t)32 * MLP_H * MLP_H;

struct uc_mlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    MlpNorm hnorm{};
    MlpNorm *dnorm = nullptr;
    bool have_norm = false;
    int in[MLP_LAYERS] = {MLP_IN, MLP_H, MLP_H, MLP_H, MLP_H};
    int out[MLP_LAYERS] = {MLP_H, MLP_H, MLP_H, MLP_H, MLP_OUT};
    int woff[MLP_LAYERS], boff[MLP_LAYERS], bfoff[MLP_LAYERS];
    int np = 0, nw = 0;
    float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    __nv_bfloat16 *wb = nullptr, *wbt = nullptr;
    // data set
    __nv_bfloat16 *Xall = nullptr;
    float *Tall = nullptr;
    long ndata = 0, cap = 0;
    // training buffers
    int bcap = 0;
    __nv_bfloat16 *H[MLP_LAYERS] = {}, *G[MLP_LAYERS] = {}, *Ht = nullptr, *Gt = nullptr;
    float *Z[MLP_LAYERS - 1] = {}, *Out = nullptr, *T = nullptr;
    float *ws = nullptr;           // split-K partial tiles of the weight gradients (MLP_WS_FLOATS)
    double *partial = nullptr;
    int *d_iter = nullptr, *d_t = nullptr, *idx = nullptr;
    long idx_cap = 0;
    float *loss_hist = nullptr;
    int loss_cap = 0;
    cudaGraphExec_t train_exec = nullptr;
    cudaGraph_t train_graph = nullptr;
    // inference buffers
    long icap = 0;
    __nv_bfloat16 *IX = nullptr, *IH0 = nullptr, *IH1 = nullptr;
    int *outside = nullptr, *list = nullptr, *count = nullptr, *tlist = nullptr, *tcount = nullptr, *pass_s = nullptr;
    double *pred_s = nullptr, *err_s = nullptr;
    uc_ctx *sample = nullptr;      // compact field of the cells recomputed exactly
    unsigned ncall = 0;
    // statistics of the last uc_mlp_omega with statistics (uc_mlp_stat)
    double st_exact = 0, st_outside = 0, st_sample_med = 0, st_acc = 0, st_acc_ok = 0, st_acc_p50 = 0, st_acc_p99 = 0;
    int *status = nullptr;
    char err[256] = {0};
};

static int mlp_err(uc_mlp *m, int code, const char *msg)
{
    if (m) snprintf(m->err, sizeof(m->err), "%s", msg);
    return code;
}

#define MCK(call)                                                                             \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return mlp_err(mlp, UC_E_CUDA, cudaGetErrorString(e_));        \
    } while (0)

template <typename T>
static int mlp_alloc(uc_mlp *mlp, T **p, size_t count)
{
    if (*p) return UC_OK;
    if (cudaMalloc((void **)p, count * sizeof(T)) != cudaSuccess) {
        *p = nullptr;
        return mlp_err(mlp, UC_E_NOMEM, "device allocation for the surrogate failed");
    }
    return UC_OK;
}

static uint64_t splitmix(uint64_t &s)
{
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

extern "C" int uc_mlp_create(int device, unsigned long long seed, long capacity, uc_mlp **out)
{
    if (!out || capacity < 0) return UC_E_ARG;
    *out = nullptr;
    uc_mlp *mlp = new (std::nothrow) uc_mlp();
    if (!mlp) return UC_E_NOMEM;
    mlp->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&mlp->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete mlp;
        return UC_E_CUDA;
    }
    int off = 0, bo = 0;
    for (int l = 0; l < MLP_LAYERS; ++l) {
        mlp->woff[l] = off;
        off += mlp->out[l] * mlp->in[l];
        mlp->boff[l] = off;
        off += mlp->out[l];
        mlp->bfoff[l] = bo;
        bo += mlp->out[l] * mlp->in[l];
    }
    mlp->np = off;
    mlp->nw = bo;
    // initial weights: uniform in +-1/sqrt(fan_in) (fan_in of the first layer: the 54 real
    // features), zero for the padded rows and columns
    std::vector<float> hw(mlp->np, 0.0f);
    uint64_t st = seed;
    for (int l = 0; l < MLP_LAYERS; ++l) {
        const int fan = l == 0 ? MLP_NF : mlp->in[l];
        const float bound = 1.0f / sqrtf((float)fan);
        const int rows = l == MLP_LAYERS - 1 ? MLP_NO : mlp->out[l];
        const int cols = l == 0 ? MLP_NF : mlp->in[l];
        for (int o = 0; o < rows; ++o) {
            for (int i = 0; i < cols; ++i) {
                const double u = (double)(splitmix(st) >> 11) * (1.0 / 9007199254740992.0);
                hw[mlp->woff[l] + o * mlp->in[l] + i] = (float)((2.0 * u - 1.0) * bound);
            }
            const double u = (double)(splitmix(st) >> 11) * (1.0 / 9007199254740992.0);
            hw[mlp->boff[l] + o] = (float)((2.0 * u - 1.0) * bound);
        }
    }
    int rc = UC_OK;
    if ((rc = mlp_alloc(mlp, &mlp->w, mlp->np)) || (rc = mlp_alloc(mlp, &mlp->g, mlp->np)) ||
        (rc = mlp_alloc(mlp, &mlp->m, mlp->np)) || (rc = mlp_alloc(mlp, &mlp->v, mlp->np)) ||
        (rc = mlp_alloc(mlp, &mlp->wb, mlp->nw)) || (rc = mlp_alloc(mlp, &mlp->wbt, mlp->nw)) ||
        (rc = mlp_alloc(mlp, &mlp->dnorm, 1)) || (rc = mlp_alloc(mlp, &mlp->status, 1)) ||
        (rc = mlp_alloc(mlp, &mlp->d_iter, 1)) || (rc = mlp_alloc(mlp, &mlp->d_t, 1))) {
        uc_mlp_destroy(mlp);
        return rc;
    }
    if (capacity > 0 && ((rc = mlp_alloc(mlp, &mlp->Xall, (size_t)capacity * MLP_IN)) ||
                         (rc = mlp_alloc(mlp, &mlp->Tall, (size_t)capacity * MLP_OUT)))) {
        uc_mlp_destroy(mlp);
        return rc;
    }
    mlp->cap = capacity;
    cudaMemcpy(mlp->w, hw.data(), mlp->np * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemset(mlp->m, 0, mlp->np * sizeof(float));
    cudaMemset(mlp->v, 0, mlp->np * sizeof(float));
    cudaMemset(mlp->g, 0, mlp->np * sizeof(float));
    cudaMemset(mlp->status, 0, sizeof(int));
    cudaMemset(mlp->d_iter, 0, sizeof(int));
    cudaMemset(mlp->d_t, 0, sizeof(int));
    *out = mlp;
    return uc_mlp_params(mlp, nullptr, hw.data());   // also writes the BF16 copies
}

extern "C" int uc_mlp_nparams(const uc_mlp *mlp) { return mlp ? mlp->np : 0; }

// get (if get != NULL) then set (if set != NULL) the flat FP32 parameter vector:
// for each layer W [out][in] then b [out]; set also rewrites the BF16 copies
extern "C" int uc_mlp_params(uc_mlp *mlp, float *get, const float *set)
{
    if (!mlp) return UC_E_ARG;
    MCK(cudaSetDevice(mlp->device));
    MCK(cudaStreamSynchronize(mlp->stream));
    if (get) MCK(cudaMemcpy(get, mlp->w, mlp->np * sizeof(float), cudaMemcpyDeviceToHost));
    if (set) {
        MCK(cudaMemcpy(mlp->w, set, mlp->np * sizeof(float), cudaMemcpyHostToDevice));
        std::vector<__nv_bfloat16> b(mlp->nw), bt(mlp->nw);
        for (int l = 0; l < MLP_LAYERS; ++l)
            for (int o = 0; o < mlp->out[l]; ++o)
                for (int i = 0; i < mlp->in[l]; ++i) {
                    const __nv_bfloat16 x = __float2bfloat16_rn(set[mlp->woff[l] + o * mlp->in[l] + i]);
                    b[mlp->bfoff[l] + o * mlp->in[l] + i] = x;
                    bt[mlp->bfoff[l] + i * mlp->out[l] + o] = x;
                }
        MCK(cudaMemcpy(mlp->wb, b.data(), mlp->nw * 2, cudaMemcpyHostToDevice));
        MCK(cudaMemcpy(mlp->wbt, bt.data(), mlp->nw * 2, cudaMemcpyHostToDevice));
    }
    return UC_OK;
}

extern "C" int uc_mlp_set_norm(uc_mlp *mlp, const float *feat_mu, const float *feat_sd, const float *hull_lo,
                               const float *hull_hi, const float *tgt_mu, const float *tgt_sd, const float *tgt_scale)
{
    if (!mlp || !feat_mu || !feat_sd || !hull_lo || !hull_hi || !tgt_mu || !tgt_sd || !tgt_scale) return UC_E_ARG;
    for (int f = 0; f < MLP_NF; ++f) {
        if (!(feat_sd[f] > 0.0f)) return mlp_err(mlp, UC_E_ARG, "feature scales must be positive");
        mlp->hnorm.feat_mu[f] = feat_mu[f];
        mlp->hnorm.feat_sd[f] = feat_sd[f];
        mlp->hnorm.hull_lo[f] = hull_lo[f];
        mlp->hnorm.hull_hi[f] = hull_hi[f];
    }
    for (int k = 0; k < MLP_NO; ++k) {
        if (!(tgt_sd[k] > 0.0f) || !(tgt_scale[k] > 0.0f)) return mlp_err(mlp, UC_E_ARG, "target scales must be positive");
        mlp->hnorm.tgt_mu[k] = tgt_mu[k];
        mlp->hnorm.tgt_sd[k] = tgt_sd[k];
        mlp->hnorm.tgt_scale[k] = tgt_scale[k];
    }
    MCK(cudaSetDevice(mlp->device));
    MCK(cudaMemcpy(mlp->dnorm, &mlp->hnorm, sizeof(MlpNorm), cudaMemcpyHostToDevice));
    mlp->have_norm = true;
    return UC_OK;
}

// Appends the context's cells to the training set: features of its fields and
// the exact FP64 omega of that state (uc_omega) as targets.
extern "C" int uc_mlp_add_data(uc_mlp *mlp, uc_ctx *ctx)
{
    if (!mlp || !ctx) return UC_E_ARG;
    if (!mlp->have_norm) return mlp_err(mlp, UC_E_STATE, "uc_mlp_set_norm first");
    if (!ctx->have_fields || !ctx->pnd) return mlp_err(mlp, UC_E_STATE, "the context needs fields and pressures");
    if (ctx->device != mlp->device) return mlp_err(mlp, UC_E_ARG, "context and surrogate on different devices");
    if (mlp->ndata + ctx->n > mlp->cap) return mlp_err(mlp, UC_E_ARG, "training set capacity exceeded");
    CK(cudaSetDevice(ctx->device));
    RET_IF(launch_chem(ctx, UC_FP64, false, true));
    const int grid = ctx->nsm * 8;
    mlp_features_kernel<<<grid, 256, 0, ctx->stream>>>(ctx->dP, mlp->dnorm, ctx->tk, ctx->pnd, ctx->y, ctx->npad, 0,
                                                       ctx->n, mlp->Xall, (int)mlp->ndata, nullptr);
    CK(cudaGetLastError());
    mlp_targets_kernel<<<grid, 256, 0, ctx->stream>>>(mlp->dnorm, ctx->qdsp, ctx->npad, 0, ctx->n, mlp->Tall,
                                                      (int)mlp->ndata);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    mlp->ndata += ctx->n;
    return UC_OK;
}

static int mlp_gemm(uc_mlp *mlp, cudaStream_t st, const __nv_bfloat16 *A, int lda, const __nv_bfloat16 *B, int ldb,
                    int M, int N, int K, int epi, const float *bias, const float *z_in, float *z_save, int ldz,
                    float *of, __nv_bfloat16 *ob, int ldo)
{
    GemmArgs g{};
    g.A = A; g.B = B; g.lda = lda; g.ldb = ldb; g.M = M; g.N = N; g.K = K; g.epi = epi;
    g.bias = bias; g.z_in = z_in; g.z_save = z_save; g.ldz = ldz; g.out_f32 = of; g.out_bf16 = ob; g.ldo = ldo;
    g.status = mlp->status;
    MCK(launch_gemm(g, st, mlp->ws, MLP_WS_FLOATS));
    return UC_OK;
}

static void mlp_free_batch(uc_mlp *mlp)
{
    for (int l = 0; l < MLP_LAYERS; ++l) {
        cudaFree(mlp->H[l]);
        cudaFree(mlp->G[l]);
        mlp->H[l] = mlp->G[l] = nullptr;
        if (l < MLP_LAYERS - 1) { cudaFree(mlp->Z[l]); mlp->Z[l] = nullptr; }
    }
    void **bufs[] = {(void **)&mlp->Ht, (void **)&mlp->Gt, (void **)&mlp->Out, (void **)&mlp->T, (void **)&mlp->partial,
                     (void **)&mlp->ws};
    for (auto b : bufs) { cudaFree(*b); *b = nullptr; }
    mlp->bcap = 0;
}

// forward layer l over M rows (weights resident in shared memory)
static int mlp_layer(uc_mlp *mlp, cudaStream_t st, const __nv_bfloat16 *A, int lda, int l, int M, int epi,
                     float *z_save, float *of, __nv_bfloat16 *ob, double *dec_out = nullptr, int dec_ld = 0)
{
    GemmArgs g{};
    if (epi == EPI_DECODE) {           // the output layer decoded into omega [52][dec_ld] (FP64)
        const char *nb = reinterpret_cast<const char *>(mlp->dnorm);
        g.dec_sd = reinterpret_cast<const float *>(nb + offsetof(MlpNorm, tgt_sd));
        g.dec_mu = reinterpret_cast<const float *>(nb + offsetof(MlpNorm, tgt_mu));
        g.dec_scale = reinterpret_cast<const float *>(nb + offsetof(MlpNorm, tgt_scale));
        g.dec_out = dec_out;
        g.dec_ld = dec_ld;
        g.dec_n = MLP_NO;
    }
    g.A = A; g.lda = lda; g.B = mlp->wb + mlp->bfoff[l]; g.ldb = mlp->in[l];
    g.M = M; g.N = mlp->out[l]; g.K = mlp->in[l]; g.epi = epi; g.bias = mlp->w + mlp->boff[l];
    g.z_save = z_save; g.ldz = MLP_H; g.out_f32 = of; g.out_bf16 = ob; g.ldo = mlp->out[l];
    g.status = mlp->status;
    MCK(launch_layer(g, device_sms(), st));
    return UC_OK;
}

static int mlp_batch_buffers(uc_mlp *mlp, int B)
{
    if (B <= mlp->bcap) return UC_OK;
    cudaStreamSynchronize(mlp->stream);
    mlp_free_batch(mlp);
    int rc;
    for (int l = 0; l < MLP_LAYERS; ++l) {
        if ((rc = mlp_alloc(mlp, &mlp->H[l], (size_t)B * mlp->in[l])) || (rc = mlp_alloc(mlp, &mlp->G[l], (size_t)B * mlp->out[l])))
            return rc;
        if (l < MLP_LAYERS - 1 && (rc = mlp_alloc(mlp, &mlp->Z[l], (size_t)B * MLP_H))) return rc;
    }
    if ((rc = mlp_alloc(mlp, &mlp->Ht, (size_t)B * MLP_H)) || (rc = mlp_alloc(mlp, &mlp->Gt, (size_t)B * MLP_H)) ||
        (rc = mlp_alloc(mlp, &mlp->Out, (size_t)B * MLP_OUT)) || (rc = mlp_alloc(mlp, &mlp->T, (size_t)B * MLP_OUT)) ||
        (rc = mlp_alloc(mlp, &mlp->partial, 1024)) || (rc = mlp_alloc(mlp, &mlp->ws, MLP_WS_FLOATS)))
        return rc;
    mlp->bcap = B;
    return UC_OK;
}

// forward and backward of one batch already in H[0] (features) and T (targets); gradients in g
static int mlp_enqueue_fwd_bwd(uc_mlp *mlp, int B, float *loss_hist)
{
    cudaStream_t st = mlp->stream;
    for (int l = 0; l < MLP_LAYERS; ++l) {
        const bool last = l == MLP_LAYERS - 1;
        RET_IF(mlp_layer(mlp, st, mlp->H[l], mlp->in[l], l, B, last ? EPI_BIAS_F32 : EPI_BIAS_GELU,
                         last ? nullptr : mlp->Z[l], last ? mlp->Out : nullptr, last ? nullptr : mlp->H[l + 1]));
    }
    const int lblk = 256;
    mlp_loss_grad_kernel<<<lblk, 256, 0, st>>>(mlp->Out, mlp->T, B, mlp->G[MLP_LAYERS - 1], mlp->partial);
    MCK(cudaGetLastError());
    if (loss_hist) {
        mlp_loss_final_kernel<<<1, 32, 0, st>>>(mlp->partial, lblk, B, mlp->d_iter, loss_hist);
        MCK(cudaGetLastError());
    }
    for (int l = MLP_LAYERS - 1; l >= 0; --l) {
        const int in = mlp->in[l], out = mlp->out[l];
        dim3 tb(32, 8);
        transpose_bf16_kernel<<<dim3((out + 31) / 32, (B + 31) / 32), tb, 0, st>>>(mlp->G[l], B, out, mlp->Gt);
        transpose_bf16_kernel<<<dim3((in + 31) / 32, (B + 31) / 32), tb, 0, st>>>(mlp->H[l], B, in, mlp->Ht);
        MCK(cudaGetLastError());
        // dW[out][in] = G^T H over the batch
        RET_IF(mlp_gemm(mlp, st, mlp->Gt, B, mlp->Ht, B, out, in, B, EPI_F32, nullptr, nullptr, nullptr, 0,
                        mlp->g + mlp->woff[l], nullptr, in));
        bias_grad_kernel<<<(out + 7) / 8, 256, 0, st>>>(mlp->Gt, B, out, mlp->g + mlp->boff[l]);
        MCK(cudaGetLastError());
        if (l > 0)   // gradient w.r.t. the previous pre-activation: (G W) * gelu'(z)
            RET_IF(mlp_gemm(mlp, st, mlp->G[l], out, mlp->wbt + mlp->bfoff[l], out, B, in, out, EPI_DGELU, nullptr,
                            mlp->Z[l - 1], nullptr, MLP_H, nullptr, mlp->G[l - 1], in));
    }
    return UC_OK;
}

static int mlp_enqueue_adam(uc_mlp *mlp, float lr, int total)
{
    AdamArgs a{};
    a.w = mlp->w; a.g = mlp->g; a.m = mlp->m; a.v = mlp->v; a.n = mlp->np;
    a.lr = lr; a.b1 = 0.9f; a.b2 = 0.999f; a.eps = 1e-8f; a.step = mlp->d_t;
    a.iter = mlp->d_iter; a.total = total;
    a.wb = mlp->wb; a.wbt = mlp->wbt;
    for (int l = 0; l < MLP_LAYERS; ++l) {
        a.woff[l] = mlp->woff[l]; a.wout[l] = mlp->out[l]; a.win[l] = mlp->in[l]; a.bfoff[l] = mlp->bfoff[l];
    }
    adam_kernel<<<592, 256, 0, mlp->stream>>>(a);
    MCK(cudaGetLastError());
    return UC_OK;
}

// Adam training (beta 0.9/0.999, eps 1e-8; the learning rate starts at lr and
// decays to lr/100 along a half cosine over the call's steps) for `steps` batches of `batch`
// rows drawn without replacement from the training set (reshuffled every
// pass over it, generator seeded by `seed`). The whole step is one CUDA graph.
// loss (host [steps], may be NULL) receives each batch's mean squared error.
extern "C" int uc_mlp_train(uc_mlp *mlp, int steps, int batch, float lr, unsigned long long seed, float *loss)
{
    if (!mlp || steps <= 0 || batch <= 0 || batch % GK != 0 || !(lr > 0.0f)) return UC_E_ARG;
    if (mlp->ndata < batch) return mlp_err(mlp, UC_E_STATE, "training set smaller than one batch");
    MCK(cudaSetDevice(mlp->device));
    RET_IF(mlp_batch_buffers(mlp, batch));
    // index list: consecutive permutations of the data set
    const long need = (long)steps * batch;
    if (need > mlp->idx_cap) {
        if (mlp->idx) cudaFree(mlp->idx);
        mlp->idx = nullptr;
        RET_IF(mlp_alloc(mlp, &mlp->idx, (size_t)need));
        mlp->idx_cap = need;
    }
    if (steps > mlp->loss_cap) {
        if (mlp->loss_hist) cudaFree(mlp->loss_hist);
        mlp->loss_hist = nullptr;
        RET_IF(mlp_alloc(mlp, &mlp->loss_hist, (size_t)steps));
        mlp->loss_cap = steps;
    }
    {
        std::vector<int> idx((size_t)need), perm((size_t)mlp->ndata);
        uint64_t st = seed;
        long pos = mlp->ndata;
        for (long i = 0; i < need; ++i) {
            if (pos == mlp->ndata) {
                for (long j = 0; j < mlp->ndata; ++j) perm[j] = (int)j;
                for (long j = mlp->ndata - 1; j > 0; --j) std::swap(perm[j], perm[splitmix(st) % (uint64_t)(j + 1)]);
                pos = 0;
            }
            idx[i] = perm[pos++];
        }
        MCK(cudaMemcpy(mlp->idx, idx.data(), need * sizeof(int), cudaMemcpyHostToDevice));
    }
    MCK(cudaMemsetAsync(mlp->d_iter, 0, sizeof(int), mlp->stream));
    {   // captured afresh on every call: the buffers it names may have been reallocated
        if (mlp->train_exec) { cudaGraphExecDestroy(mlp->train_exec); mlp->train_exec = nullptr; }
        if (mlp->train_graph) { cudaGraphDestroy(mlp->train_graph); mlp->train_graph = nullptr; }
        MCK(cudaStreamBeginCapture(mlp->stream, cudaStreamCaptureModeThreadLocal));
        mlp_gather_kernel<<<256, 256, 0, mlp->stream>>>(mlp->Xall, mlp->Tall, mlp->idx, mlp->d_iter, batch, mlp->H[0], mlp->T);
        int rc = cudaGetLastError() == cudaSuccess ? UC_OK : mlp_err(mlp, UC_E_CUDA, "gather launch");
        if (rc == UC_OK) rc = mlp_enqueue_fwd_bwd(mlp, batch, mlp->loss_hist);
        if (rc == UC_OK) rc = mlp_enqueue_adam(mlp, lr, steps);
        if (rc == UC_OK) {
            step_incr_kernel<<<1, 32, 0, mlp->stream>>>(mlp->d_iter);
            step_incr_kernel<<<1, 32, 0, mlp->stream>>>(mlp->d_t);
        }
        cudaGraph_t gph = nullptr;
        cudaError_t e = cudaStreamEndCapture(mlp->stream, &gph);
        if (rc != UC_OK) { if (gph) cudaGraphDestroy(gph); return rc; }
        if (e != cudaSuccess) return mlp_err(mlp, UC_E_CUDA, cudaGetErrorString(e));
        if (cudaGraphInstantiate(&mlp->train_exec, gph, 0) != cudaSuccess) {
            cudaGraphDestroy(gph);
            return mlp_err(mlp, UC_E_CUDA, "train graph instantiate");
        }
        mlp->train_graph = gph;
    }
    for (int s = 0; s < steps; ++s) MCK(cudaGraphLaunch(mlp->train_exec, mlp->stream));
    MCK(cudaStreamSynchronize(mlp->stream));
    if (loss) MCK(cudaMemcpy(loss, mlp->loss_hist, steps * sizeof(float), cudaMemcpyDeviceToHost));
    int st = 0;
    MCK(cudaMemcpy(&st, mlp->status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st == ST_MMA_TIMEOUT) return mlp_err(mlp, UC_E_TIMEOUT, "a tensor-core wait timed out");
    return UC_OK;
}

// One forward and backward pass on given rows (no update): x [M][64] BF16 bit
// patterns (features), t [M][64] targets; grad (host [nparams]) receives the
// gradient of the mean squared error, loss its value. M a multiple of 64.
extern "C" int uc_mlp_grad(uc_mlp *mlp, int M, const uint16_t *x, const float *t, float *grad, float *loss)
{
    if (!mlp || M <= 0 || M % GK != 0 || !x || !t) return UC_E_ARG;
    MCK(cudaSetDevice(mlp->device));
    RET_IF(mlp_batch_buffers(mlp, M));
    MCK(cudaMemcpyAsync(mlp->H[0], x, (size_t)M * MLP_IN * 2, cudaMemcpyHostToDevice, mlp->stream));
    MCK(cudaMemcpyAsync(mlp->T, t, (size_t)M * MLP_OUT * 4, cudaMemcpyHostToDevice, mlp->stream));
    if (!mlp->loss_hist) {
        RET_IF(mlp_alloc(mlp, &mlp->loss_hist, 1));
        mlp->loss_cap = 1;
    }
    MCK(cudaMemsetAsync(mlp->d_iter, 0, sizeof(int), mlp->stream));
    RET_IF(mlp_enqueue_fwd_bwd(mlp, M, mlp->loss_hist));
    MCK(cudaStreamSynchronize(mlp->stream));
    if (grad) MCK(cudaMemcpy(grad, mlp->g, mlp->np * sizeof(float), cudaMemcpyDeviceToHost));
    if (loss) MCK(cudaMemcpy(loss, mlp->loss_hist, sizeof(float), cudaMemcpyDeviceToHost));
    return UC_OK;
}

// Omega of the context's state from the surrogate, with fallback to the exact
// FP64 kernel per 32-cell tile: a tile is recomputed exactly if one of its
// cells lies outside the training hull, or if the surrogate's relative error
// on one sampled cell of the tile exceeds tol (species with Y > 1e-8).
// The result is the context's QDSP (as uc_omega leaves it; download with
// uc_download_outputs). stats (host [3], may be NULL): fraction of tiles
// recomputed, fraction of cells outside the hull, median sampled residual.
extern "C" int uc_mlp_omega(uc_mlp *mlp, uc_ctx *ctx, double tol, double *stats)
{
    if (!mlp || !ctx || !(tol >= 0.0)) return UC_E_ARG;
    if (!mlp->have_norm) return mlp_err(mlp, UC_E_STATE, "uc_mlp_set_norm first");
    if (!ctx->have_fields || !ctx->pnd) return mlp_err(mlp, UC_E_STATE, "the context needs fields and pressures");
    if (ctx->device != mlp->device) return mlp_err(mlp, UC_E_ARG, "context and surrogate on different devices");
    CK(cudaSetDevice(ctx->device));
    const int n = ctx->n, np = ctx->npad, nt = ctx->ntile, ns = (n + 31) / 32;
    int rc;
    if (mlp->icap < np) {
        // grown to the largest field seen (the buffers of a smaller one are released first)
        CK(cudaStreamSynchronize(ctx->stream));
        void *old[] = {mlp->IX, mlp->IH0, mlp->IH1, mlp->outside, mlp->list, mlp->count, mlp->tlist,
                       mlp->tcount, mlp->pass_s, mlp->pred_s, mlp->err_s};
        for (void *b : old)
            if (b) cudaFree(b);
        mlp->IX = mlp->IH0 = mlp->IH1 = nullptr;
        mlp->outside = mlp->list = mlp->count = mlp->tlist = mlp->tcount = mlp->pass_s = nullptr;
        mlp->pred_s = mlp->err_s = nullptr;
        if (mlp->sample) { uc_destroy(mlp->sample); mlp->sample = nullptr; }
        mlp->icap = 0;
        if ((rc = mlp_alloc(mlp, &mlp->IX, (size_t)np * MLP_IN)) || (rc = mlp_alloc(mlp, &mlp->IH0, (size_t)np * MLP_H)) ||
            (rc = mlp_alloc(mlp, &mlp->IH1, (size_t)np * MLP_H)) ||
            (rc = mlp_alloc(mlp, &mlp->outside, (size_t)np)) || (rc = mlp_alloc(mlp, &mlp->list, (size_t)np)) ||
            (rc = mlp_alloc(mlp, &mlp->count, 1)) || (rc = mlp_alloc(mlp, &mlp->tlist, (size_t)nt)) ||
            (rc = mlp_alloc(mlp, &mlp->tcount, 1)) || (rc = mlp_alloc(mlp, &mlp->pass_s, (size_t)ns)) ||
            (rc = mlp_alloc(mlp, &mlp->pred_s, (size_t)ns * LSP)) || (rc = mlp_alloc(mlp, &mlp->err_s, (size_t)ns)))
            return rc;
        mlp->icap = np;
        // the compact field of the cells recomputed exactly: at most every cell of the field
        if ((rc = uc_init(&ctx->inputs, n, ctx->device, &mlp->sample)) != UC_OK)
            return mlp_err(mlp, rc, "set-up of the compact field of the recomputed cells failed");
    }
    RET_IF(dalloc(ctx, &ctx->qdsp, (size_t)LSP * np));
    cudaStream_t st = ctx->stream;
    const int grid = ctx->nsm * 8;
    // surrogate for every cell
    mlp_features_kernel<<<grid, 256, 0, st>>>(ctx->dP, mlp->dnorm, ctx->tk, ctx->pnd, ctx->y, np, 0, np, mlp->IX, 0,
                                              mlp->outside);
    CK(cudaGetLastError());
    __nv_bfloat16 *hin = mlp->IX, *hb[2] = {mlp->IH0, mlp->IH1};
    for (int l = 0; l < MLP_LAYERS; ++l) {
        const bool last = l == MLP_LAYERS - 1;
        RET_IF(mlp_layer(mlp, st, hin, mlp->in[l], l, np, last ? EPI_DECODE : EPI_BIAS_GELU, nullptr, nullptr,
                         last ? nullptr : hb[l & 1], last ? ctx->qdsp : nullptr, np));
        if (!last) hin = hb[l & 1];
    }
    if (std::isinf(tol)) {          // the network alone: no checks, no fallback
        if (stats) {
            CK(cudaStreamSynchronize(st));
            stats[0] = stats[1] = stats[2] = 0.0;
            mlp->st_exact = mlp->st_outside = mlp->st_sample_med = mlp->st_acc = mlp->st_acc_p50 = mlp->st_acc_p99 = 0.0;
            mlp->st_acc_ok = 0.0;
        }
        return UC_OK;
    }
    // per-cell checks; the flagged and the sampled cells recomputed by the exact kernel
    const int off = (int)((mlp->ncall++ * 7u + 3u) & 31u);
    CK(cudaMemsetAsync(mlp->count, 0, sizeof(int), st));
    mlp_cell_check_kernel<<<grid, 256, 0, st>>>(ctx->dP, ctx->qdsp, mlp->outside, n, np, tol, off, mlp->list,
                                                 mlp->count, mlp->pred_s, mlp->pass_s);
    CK(cudaGetLastError());
    uc_ctx *S = mlp->sample;
    mlp_gather_cells_kernel<<<grid, 256, 0, st>>>(mlp->list, mlp->count, ctx->tk, ctx->rho, ctx->y, ctx->soot, np,
                                                   S->tk, S->rho, S->y, S->soot, S->npad, mlp->tlist, mlp->tcount);
    CK(cudaGetLastError());
    RET_IF(dalloc(S, &S->qdsp, (size_t)LSP * S->npad));
    RET_IF(dalloc(S, &S->qdot, S->npad));
    ChemArgs c{};
    c.P = ctx->dP; c.tab = ctx->dTab;
    c.tk = S->tk; c.rho = S->rho; c.y = S->y; c.stmf = S->soot; c.stnd = S->soot + S->npad;
    c.qdsp = S->qdsp; c.qdot = S->qdot;
    c.n = S->n; c.npad = S->npad; c.ntile = S->ntile; c.status = ctx->status;
    c.tile_list = mlp->tlist; c.tile_count = mlp->tcount;
    int slot;
    prof_begin(ctx, UC_K_CHEM, slot);
    chem_fp64_kernel<<<std::min(S->ntile, ctx->nsm), CHEM_THREADS, CHEM_SMEM, st>>>(c);
    prof_end(ctx, slot);
    CK(cudaGetLastError());
    mlp_scatter_cells_kernel<<<grid, 256, 0, st>>>(mlp->list, mlp->count, S->qdsp, S->qdot, S->npad, ctx->qdsp,
                                                    ctx->qdot, np);
    CK(cudaGetLastError());
    if (stats) {
        mlp_sample_error_kernel<<<(ns + 255) / 256, 256, 0, st>>>(mlp->pred_s, ctx->qdsp, ctx->y, n, np, off, ns,
                                                                    mlp->err_s);
        CK(cudaGetLastError());
        int cnt = 0;
        std::vector<int> outs(n), pass(ns);
        std::vector<double> err(ns);
        CK(cudaMemcpyAsync(&cnt, mlp->count, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(outs.data(), mlp->outside, n * sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(pass.data(), mlp->pass_s, ns * sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(err.data(), mlp->err_s, ns * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        long no = 0;
        for (int v : outs) no += v;
        std::vector<double> all, acc;
        for (int i = 0; i < ns; ++i) {
            if (err[i] < 0.0) continue;
            all.push_back(err[i]);
            if (pass[i]) acc.push_back(err[i]);
        }
        auto quant = [](std::vector<double> v, double q) {
            if (v.empty()) return 0.0;
            const size_t k = std::min(v.size() - 1, (size_t)(q * (double)(v.size() - 1) + 0.5));
            std::nth_element(v.begin(), v.begin() + k, v.end());
            return v[k];
        };
        long ok = 0;
        for (double e : acc) ok += e <= tol;
        mlp->st_exact = (double)cnt / n;
        mlp->st_outside = (double)no / n;
        mlp->st_sample_med = quant(all, 0.5);
        mlp->st_acc = all.empty() ? 0.0 : (double)acc.size() / all.size();
        mlp->st_acc_ok = acc.empty() ? 1.0 : (double)ok / acc.size();
        mlp->st_acc_p50 = quant(acc, 0.5);
        mlp->st_acc_p99 = quant(acc, 0.99);
        stats[0] = mlp->st_exact;
        stats[1] = mlp->st_outside;
        stats[2] = mlp->st_sample_med;
    }
    int s2 = 0;
    CK(cudaMemcpyAsync(&s2, mlp->status, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (s2 == ST_MMA_TIMEOUT) return set_err(ctx, UC_E_TIMEOUT, "a tensor-core wait timed out");
    return UC_OK;
}

extern "C" int uc_mlp_stat(const uc_mlp *mlp, const char *name, double *value)
{
    if (!mlp || !name || !value) return UC_E_ARG;
    const struct { const char *k; double v; } t[] = {
        {"cells_exact", mlp->st_exact}, {"cells_outside_hull", mlp->st_outside},
        {"sample_error_p50", mlp->st_sample_med}, {"sample_accepted", mlp->st_acc},
        {"sample_accepted_within_tol", mlp->st_acc_ok}, {"sample_accepted_error_p50", mlp->st_acc_p50},
        {"sample_accepted_error_p99", mlp->st_acc_p99}};
    for (auto &e : t)
        if (!strcmp(name, e.k)) { *value = e.v; return UC_OK; }
    return UC_E_ARG;
}

extern "C" const char *uc_mlp_last_error(const uc_mlp *mlp) { return mlp ? mlp->err : "null surrogate"; }

extern "C" void uc_mlp_destroy(uc_mlp *mlp)
{
    if (!mlp) return;
    cudaSetDevice(mlp->device);
    if (mlp->stream) cudaStreamSynchronize(mlp->stream);
    if (mlp->train_exec) cudaGraphExecDestroy(mlp->train_exec);
    if (mlp->train_graph) cudaGraphDestroy(mlp->train_graph);
    void *bufs[] = {mlp->dnorm, mlp->w, mlp->g, mlp->m, mlp->v, mlp->wb, mlp->wbt, mlp->Xall, mlp->Tall,
                    mlp->d_iter, mlp->d_t, mlp->idx, mlp->loss_hist, mlp->IX, mlp->IH0, mlp->IH1,
                    mlp->outside, mlp->list, mlp->count, mlp->tlist, mlp->tcount, mlp->pass_s, mlp->pred_s,
                    mlp->err_s, mlp->status};
    for (void *b : bufs)
        if (b) cudaFree(b);
    mlp_free_batch(mlp);
    if (mlp->sample) uc_destroy(mlp->sample);
    if (mlp->stream) cudaStreamDestroy(mlp->stream);
    delete mlp;
}

// ------------------------------------------------------------------ no-allocation update

// Scratch of uc_species_update_noalloc: residual partial sums of the
// cooperating blocks (two halves, alternating by pass) and the pass counter.
// It lives in the library image, so the call never allocates device memory.
static __device__ __align__(256) double uc_noalloc_partial[2 * UC_NOALLOC_MAX_BLOCKS];
static __device__ __align__(256) int uc_noalloc_passes;

// Device addresses of the two arrays, looked up once per device (host code
// may not use the symbols themselves as device pointers).
static std::mutex g_noalloc_mu;
static double *g_noalloc_partial[64];
static int *g_noalloc_passes[64];

static int noalloc_scratch(uc_ctx *ctx, double **partial, int **passes)
{
    const int dev = ctx->device;
    if (dev < 0 || dev >= 64) return set_err(ctx, UC_E_ARG, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_partial[dev]) {
        CK(cudaSetDevice(dev));
        double *p = nullptr;
        int *q = nullptr;
        CK(cudaGetSymbolAddress((void **)&p, uc_noalloc_partial));
        CK(cudaGetSymbolAddress((void **)&q, uc_noalloc_passes));
        g_noalloc_partial[dev] = p;
        g_noalloc_passes[dev] = q;
    }
    *partial = g_noalloc_partial[dev];
    *passes = g_noalloc_passes[dev];
    return UC_OK;
}

extern "C" int uc_species_update_noalloc(uc_ctx *ctx, const uc_update_arrays *arr, double dt, int isor,
                                         double relx, double tol, double spnorm, int *passes)
{
    if (!ctx) return UC_E_ARG;
    if (!arr || !arr->rc || !arr->sour || !arr->rho || !arr->y0 || !arr->soot0 || !arr->y || !arr->soot)
        return set_err(ctx, UC_E_ARG, "uc_species_update_noalloc: a required device array is NULL");
    if (arr->n <= 0 || arr->npad < arr->n || arr->npad % TILE != 0)
        return set_err(ctx, UC_E_ARG, "uc_species_update_noalloc: need 0 < n <= npad and npad a multiple of %d "
                                      "(n=%d, npad=%d)", TILE, arr->n, arr->npad);
    if (isor < 1 || !(relx > 0.0) || !(dt >= 0.0)) return set_err(ctx, UC_E_ARG, "invalid isor/relx/dt");
    CK(cudaSetDevice(ctx->device));
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, update_kernel<double>, UPD_THREADS, UPD_SMEM));
    const int max_grid = std::max(1, per_sm) * ctx->nsm;
    if (max_grid > UC_NOALLOC_MAX_BLOCKS)
        return set_err(ctx, UC_E_ARG, "uc_species_update_noalloc: this device needs %d cooperating blocks, "
                                      "more than the %d the fixed scratch holds", max_grid, UC_NOALLOC_MAX_BLOCKS);
    double *partial = nullptr;
    int *dpasses = nullptr;
    RET_IF(noalloc_scratch(ctx, &partial, &dpasses));
    CK(cudaSetDevice(ctx->device));
    const int ntile = arr->npad / TILE;
    UpdArgs a{};
    a.P = ctx->dP; a.rc = arr->rc; a.sour = arr->sour; a.rho = arr->rho; a.y0 = arr->y0; a.soot0 = arr->soot0;
    a.face_sum = arr->face_sum; a.face_nbr = arr->face_nbr; a.y = arr->y; a.soot = arr->soot;
    a.partial = partial;
    a.passes = dpasses;
    a.dt = dt; a.sor1 = relx; a.tol = tol; a.spnorm = spnorm > 0.0 ? spnorm : (double)arr->n * (LSP - 1);
    a.isor = isor; a.n = arr->n; a.npad = arr->npad; a.ntile = ntile;
    const int grid = std::min(max_grid, std::max(1, (ntile + UPD_THREADS / 32 - 1) / (UPD_THREADS / 32)));
    void *args[] = {&a};
    CK(cudaLaunchCooperativeKernel((void *)update_kernel<double>, dim3(grid), dim3(UPD_THREADS), args, UPD_SMEM,
                                   ctx->stream));
    if (passes) {
        CK(cudaMemcpyAsync(passes, dpasses, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return UC_OK;
}
