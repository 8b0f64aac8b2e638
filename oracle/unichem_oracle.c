/*
 * ORACLE (test infrastructure only) -- FP64 CPU restatement of UNICORN's
 * per-cell chemistry and property hot path.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
 * this file, as the checker. The product (unicorn_b200/csrc) never links it.
 *
 * It follows the reference's evaluation order so that its results can be
 * compared bit for bit with the reference routines themselves (translated
 * mechanically to C under oracle/_ref by oracle/build_ref.py):
 *   orc_setup            src/unicornd-mild-sd-5.f:327-483 (tables and scales)
 *   orc_rates            src/lib/ckrates.f:92-1352        (CKRATES, per cell)
 *   orc_omega            src/lib/solveh.f:39-57,116-1145  (h_k, RA, PRD, QDSP, QDOT)
 *   orc_cp               src/lib/spgsolv.f:102-173        (mixture cp, TCP)
 *   orc_props            src/unicornd-mild-sd-5.f:821-1006 (Y clip, mu, lambda, D_k)
 *   orc_species_update   src/lib/solvesp.f:82-2915        (point-implicit update)
 *   orc_temperature      src/lib/solveh.f:1170-1234       (T from h, Newton)
 *   orc_nsub, orc_integrate  batched stiff integration: the functions above
 *                        chained per cell and sub-step (no single reference routine)
 * The mechanism arrives as flat tables built from the reference sources by
 * unicorn_b200/mech/extract.py and packed by oracle/oracle.py.
 *
 * Literal constants keep their Fortran kind: a default-REAL literal such as
 * 82.06 in the reference is the single-precision value promoted to double,
 * written here as F(82.06).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define LSP 52
#define LRX 544
#define F(x) ((double)(float)(x))

/* ------------------------------------------------------------- tables */

/* factor kinds of the product chains in the packed program tables */
enum { FK_NUM = 0, FK_A = 1, FK_RC = 2, FK_Y = 3, FK_Y0 = 4, FK_SOUR = 5, FK_RA = 6, FK_SRA = 7 };

typedef struct {
    /* species data (1-based species numbers are stored 0-based here) */
    const double *wsp, *cdia, *tlj;     /* [52] */
    const double *poly;                 /* [52][14] NASA coefficients, POLSP(14,LSP) */
    const double *om22;                 /* [52][12] Omega(2,2) fits, CISP(12,LSP) */
    const double *ci11;                 /* [4][5]  CI11(4,5) stored row-major [K][n] */
    double tpol1, tpol2;
    /* reactions, raw DATA values (Ea in cal/mol) */
    const double *akf, *alf, *exaf, *aklow, *allow, *ealow, *troe; /* troe [544][4] */
    /* reverse formulas for even slots: rut (-1,0,+1), q chain (op, species) */
    const int *rev_has, *rev_rut, *rev_off, *rev_len, *rev_op, *rev_sp;
    /* third-body groups: g=0 TBODY, g=1..10 TB001..TB010 */
    const int *tb_off, *tb_len, *tb_sign, *tb_sp; const double *tb_coef; const int *tb_hascoef;
    const int *dmole_grp;               /* [544] group used by DMOLE (0 = TBODY) */
    /* RC assembly */
    const int *rc_has, *rc_order, *rc_tb, *rc_off, *rc_len, *rc_op, *rc_kind, *rc_idx;
    /* SOLVEH: RA reactant lists, PRD term lists */
    const int *ra_has, *ra_off, *ra_len, *ra_sp;
    const int *prd_has, *prd_off, *prd_len;         /* per species, terms */
    /* generic term store: term t has sign term_sign[t] and factors
       [term_foff[t], term_foff[t]+term_flen[t]) in (fac_kind, fac_idx, fac_val) */
    const int *term_sign, *term_foff, *term_flen;
    const int *fac_kind, *fac_idx; const double *fac_val;
    /* SOLVESP blocks (species 1..51): recompute (r, factor list), sums, multiplies */
    const int *blk_rec_off, *blk_rec_len, *rec_r, *rec_foff, *rec_flen;
    const int *blk_prod_has, *blk_prod_off, *blk_prod_len;
    const int *blk_extra_off, *blk_extra_len;
    const int *blk_loss_has, *blk_loss_off, *blk_loss_len;
    const int *blk_mul_off, *blk_mul_len, *mul_r;
    /* loss lists used for d(omega)/dY: from the PRD negative RA terms */
} orc_tables;

typedef struct {
    double RTIN, RTOT, VREF, TREF, PREF, RREF, FO2IN;
} orc_inputs;

typedef struct {
    /* /CB06/ scales and derived constants (src/unicornd-mild-sd-5.f:421-459) */
    double ALSTR, VSTR, RSTR, PSTR, TSTR, TMSTR, AMSTR, ACSTR, DSTR, HSTR, CPSTR, AKSTR, EPSTR,
           WMSTR, GASC, BETA1, BETA2, BETA3, BETA4, REI, PBACK, HCONV, CONVRC, CONVRM, CONVRD;
    double WM[LSP], HFO[LSP];
    double AKF[LRX], ALF[LRX], EXAF[LRX], AKLOW[LRX], ALLOW[LRX], EALOW[LRX], TROE[LRX][4];
    int NRLIND, LREV;
    double WMIK[LSP][LSP], DWMIK[LSP][LSP], WMCD[LSP][LSP];
    double ETLJ1[LSP][LSP], ETLJ2[LSP][LSP], ETLJ3[LSP][LSP], ETLJ4[LSP][LSP];
} orc_state;

static orc_tables T;
static orc_state S;

/* ------------------------------------------------------------- set-up */

/* src/unicornd-mild-sd-5.f:327-483: unit conversions, reverse slots,
 * reference scales, non-dimensional molar masses, formation enthalpies and
 * pair constants of the transport model. All reactions switched on (IRSW=1). */
int orc_setup(const orc_tables *tab, const orc_inputs *in, double *scales_out)
{
    T = *tab;
    const double RUCAL = F(1.9872), GASC = F(8.3144), GAMA = F(1.4);
    S.LREV = 2;
    S.NRLIND = 0;
    for (int r = 0; r < LRX; ++r) {
        S.AKF[r] = T.akf[r]; S.ALF[r] = T.alf[r]; S.EXAF[r] = T.exaf[r];
        S.AKLOW[r] = T.aklow[r]; S.ALLOW[r] = T.allow[r]; S.EALOW[r] = T.ealow[r];
        for (int c = 0; c < 4; ++c) S.TROE[r][c] = T.troe[r * 4 + c];
    }
    for (int i = 0; i < LRX; i += 2) {          /* DO 10 I=1,LRX,LREV  (main:364-413) */
        S.EXAF[i] = S.EXAF[i] / RUCAL;
        if (S.AKF[i] < 0) {
            S.NRLIND += 1;
            S.AKF[i] = -S.AKF[i];
            S.EALOW[i] = S.EALOW[i] / RUCAL;
        } else {
            S.EALOW[i] = 0.0; S.AKLOW[i] = 0.0; S.ALLOW[i] = 0.0;
            for (int c = 0; c < 4; ++c) S.TROE[i][c] = 0.0;
        }
        S.AKF[i + 1] = 1.0;
        S.EXAF[i + 1] = 0.0; S.ALF[i + 1] = 0.0; S.EALOW[i + 1] = 0.0; S.AKLOW[i + 1] = 0.0;
        S.ALLOW[i + 1] = 0.0;
        for (int c = 0; c < 4; ++c) S.TROE[i + 1][c] = 0.0;
    }
    /* freestream properties and scales (main:421-453) */
    double WMREF = 1.0 / (in->FO2IN / T.wsp[1] + (1.0 - in->FO2IN) / T.wsp[LSP - 1]) / 1000.0;
    double AMREF = 5.69428e-07 * pow(in->TREF, F(0.62245));
    double ACREF = 2.78763e-04 * pow(in->TREF, F(0.796783));
    double DREF = 1.2e-04;
    double RREF = in->PREF / (GASC / WMREF) / in->TREF;
    S.GASC = GASC;
    S.ALSTR = in->RTOT - in->RTIN;
    S.VSTR = in->VREF;
    S.RSTR = RREF;
    S.PSTR = RREF * in->VREF * in->VREF;
    S.PBACK = in->PREF / S.PSTR;
    S.TSTR = in->TREF;
    S.HSTR = in->VREF * in->VREF;
    S.AKSTR = in->VREF * in->VREF;
    S.EPSTR = in->VREF * in->VREF * in->VREF / S.ALSTR;
    S.CPSTR = in->VREF * in->VREF / in->TREF;
    S.ACSTR = ACREF;
    S.TMSTR = S.ALSTR / in->VREF;
    S.AMSTR = AMREF;
    S.DSTR = DREF;
    S.WMSTR = WMREF;
    S.REI = AMREF / RREF / in->VREF / S.ALSTR;
    S.BETA1 = GASC * S.RSTR * S.TSTR / S.PSTR / S.WMSTR;
    S.BETA2 = S.TSTR * S.ACSTR / S.AMSTR / S.VSTR / S.VSTR;
    S.BETA3 = S.RSTR * S.DSTR / S.AMSTR;
    S.BETA4 = 0.0;
    S.HCONV = GASC / S.WMSTR / S.HSTR;
    /* main:457-459 */
    S.CONVRC = F(418.68) * 1.9891e-04 * sqrt(S.TSTR / 1000.0 / S.WMSTR) / S.ACSTR;
    S.CONVRM = F(0.1) * 2.6693e-05 * sqrt(1000.0 * S.WMSTR * S.TSTR) / S.AMSTR;
    S.CONVRD = F(0.02628) * S.TSTR * sqrt(S.TSTR) / S.PSTR / sqrt(S.WMSTR * 1000.0) / S.DSTR;
    /* main:461-464 */
    for (int k = 0; k < LSP; ++k) {
        S.WM[k] = T.wsp[k] / 1000.0 / S.WMSTR;
        S.HFO[k] = S.HCONV * T.poly[k * 14 + 5] / S.WM[k];
    }
    /* main:471-483 pair constants */
    for (int i = 0; i < LSP; ++i)
        for (int j = 0; j < LSP; ++j) {
            S.WMIK[i][j] = pow(S.WM[i] / S.WM[j], F(0.25));
            if (i == j) S.WMIK[i][j] = sqrt(S.WM[i]);
            S.DWMIK[i][j] = F(2.828427125) * sqrt(1.0 + S.WM[i] / S.WM[j]);
            double ECDIA = F(0.5) * (T.cdia[i] + T.cdia[j]);
            S.WMCD[i][j] = sqrt((S.WM[i] + S.WM[j]) / 2.0 / S.WM[i] / S.WM[j]) / ECDIA / ECDIA;
            S.ETLJ1[i][j] = sqrt(T.tlj[i] * T.tlj[j]);
            S.ETLJ2[i][j] = S.ETLJ1[i][j] * S.ETLJ1[i][j];
            S.ETLJ3[i][j] = S.ETLJ2[i][j] * S.ETLJ1[i][j];
            S.ETLJ4[i][j] = S.ETLJ3[i][j] * S.ETLJ1[i][j];
        }
    if (scales_out) {
        double v[] = {S.ALSTR, S.VSTR, S.RSTR, S.PSTR, S.TSTR, S.TMSTR, S.AMSTR, S.ACSTR, S.DSTR,
                      S.HSTR, S.CPSTR, S.AKSTR, S.EPSTR, S.WMSTR, S.GASC, S.BETA1, S.BETA2,
                      S.BETA3, S.BETA4, S.REI, S.PBACK, S.HCONV, S.CONVRC, S.CONVRM, S.CONVRD};
        memcpy(scales_out, v, sizeof(v));
    }
    return 0;
}

void orc_get_tables(double *wm, double *hfo, double *akf, double *exaf, double *ealow,
                    double *pair /* [7][52][52] */)
{
    memcpy(wm, S.WM, sizeof(S.WM));
    memcpy(hfo, S.HFO, sizeof(S.HFO));
    memcpy(akf, S.AKF, sizeof(S.AKF));
    memcpy(exaf, S.EXAF, sizeof(S.EXAF));
    memcpy(ealow, S.EALOW, sizeof(S.EALOW));
    memcpy(pair + 0 * LSP * LSP, S.WMIK, sizeof(S.WMIK));
    memcpy(pair + 1 * LSP * LSP, S.DWMIK, sizeof(S.DWMIK));
    memcpy(pair + 2 * LSP * LSP, S.WMCD, sizeof(S.WMCD));
    memcpy(pair + 3 * LSP * LSP, S.ETLJ1, sizeof(S.ETLJ1));
    memcpy(pair + 4 * LSP * LSP, S.ETLJ2, sizeof(S.ETLJ2));
    memcpy(pair + 5 * LSP * LSP, S.ETLJ3, sizeof(S.ETLJ3));
    memcpy(pair + 6 * LSP * LSP, S.ETLJ4, sizeof(S.ETLJ4));
}

/* ------------------------------------------------------------- CKRATES */

typedef struct {
    double sprf[LRX];
    double rc[LRX];
    double sour[6];
    double tbody;
} cell_rates;

static double tb_value(int g, const double *y, double tbody)
{
    /* ckrates.f:706-731 TBnnn = TBODY + sum(coef*Y/W) (left to right) */
    int o = T.tb_off[g], n = T.tb_len[g];
    double acc = tbody;
    for (int t = 0; t < n; ++t) {
        int k = T.tb_sp[o + t];
        double term = T.tb_hascoef[o + t] ? (T.tb_coef[o + t] * y[k]) / S.WM[k] : y[k] / S.WM[k];
        acc = T.tb_sign[o + t] > 0 ? acc + term : acc - term;
    }
    return acc;
}

/* ckrates.f:92-1352 for one cell; y[k] are the 52 mass fractions */
static void rates_cell(double tk, double rho, const double *y, double stmf, double stnd,
                       cell_rates *o)
{
    double *SPRF = o->sprf;
    memset(SPRF, 0, sizeof(o->sprf));       /* slots never written stay 0 (static local) */
    const double C1ST = S.ALSTR / S.VSTR;
    const double C2ND = S.ALSTR / S.VSTR * (S.RSTR / S.WMSTR * 1.0e-06);
    const double C3RD = S.ALSTR / S.VSTR * (S.RSTR * S.RSTR / S.WMSTR / S.WMSTR * 1.0e-12);
    double TKD = tk * S.TSTR;
    double ELOGT = log(TKD);
    /* forward specific rates, ckrates.f:95-101 */
    for (int ir = 0; ir < LRX; ir += S.LREV) {
        double ACTV = S.ALF[ir] * ELOGT - S.EXAF[ir] / TKD;
        SPRF[ir] = S.AKF[ir] * exp(ACTV);
    }
    /* Gibbs functions, ckrates.f:103-115 */
    double TKD1 = TKD / 2.0;
    double TKD2 = TKD * TKD / 6.0;
    double TKD3 = TKD1 * TKD2;
    double TKD4 = F(1.2) * TKD1 * TKD3;
    int ip = TKD > T.tpol1 ? 7 : 0;
    double GSP[LSP];
    for (int k = 0; k < LSP; ++k) {
        const double *a = T.poly + k * 14 + ip;
        double g0 = a[0] * (ELOGT - 1.0) + a[1] * TKD1 + a[2] * TKD2 + a[3] * TKD3 + a[4] * TKD4
                    - a[5] / TKD + a[6];
        GSP[k] = exp(g0);
    }
    double RUT = F(82.06) * TKD;
    /* reverse rates, ckrates.f:116-642: k_r = AKF*k_f [/RUT|*RUT] / q */
    for (int r = 1; r < LRX; r += 2) {
        if (!T.rev_has[r]) continue;        /* Q1: SPRF(116),(254),(472),(502..) never set */
        int o2 = T.rev_off[r], n = T.rev_len[r];
        double q = GSP[T.rev_sp[o2]];
        for (int t = 1; t < n; ++t)
            q = T.rev_op[o2 + t] == '*' ? q * GSP[T.rev_sp[o2 + t]] : q / GSP[T.rev_sp[o2 + t]];
        double v = S.AKF[r] * SPRF[r - 1];
        if (T.rev_rut[r] < 0) v = v / RUT;
        else if (T.rev_rut[r] > 0) v = v * RUT;
        SPRF[r] = v / q;
    }
    /* third bodies, ckrates.f:643-731 */
    double RHO1 = rho, RHO2 = rho * rho, RHO3 = rho * rho * rho;
    double TBODY = y[0] / S.WM[0];
    for (int k = 1; k < LSP; ++k) TBODY = TBODY + y[k] / S.WM[k];
    double TB[11];
    TB[0] = TBODY;
    for (int g = 1; g <= 10; ++g) TB[g] = tb_value(g, y, TBODY);
    o->tbody = TBODY;
    /* fall-off blending, ckrates.f:740-794 */
    if (S.NRLIND != 0) {
        double DMOLEA = rho * S.RSTR / S.WMSTR * 1.0e-06;
        for (int ir = 0; ir < LRX; ir += S.LREV) {
            double DMOLE = TB[T.dmole_grp[ir]] * DMOLEA;
            if (S.AKLOW[ir] == 0.0) continue;
            const double *TR = S.TROE[ir];
            if (S.AKLOW[ir] < 0.0) {            /* Tseng form (no reaction of this data uses it) */
                double AK0M = pow(10.0, TR[0] + (TR[1] + (TR[2] + TR[3] * TKD) * TKD) * TKD) * DMOLE;
                double AFP = AK0M / (1.0 + AK0M);
                SPRF[ir] = AFP * SPRF[ir];
                SPRF[ir + 1] = AFP * SPRF[ir + 1];
                continue;
            }
            double ACTV = S.ALLOW[ir] * ELOGT - S.EALOW[ir] / TKD;
            double AK0M = S.AKLOW[ir] * exp(ACTV) * DMOLE / (SPRF[ir] + 1.0e-20);
            double RFACT;
            if (TR[0] > 0.0) {
                double FCLOG;
                if (TR[1] == 0.0) FCLOG = log10(TR[0]);
                else FCLOG = log10((1.0 - TR[0]) * exp(-(TKD / TR[1])) + TR[0] * exp(-(TKD / TR[2]))
                                   + exp(-(TR[3] / TKD)));   /* Q2: exp(-T4/T) always added */
                double CPLOG = log10(AK0M) - (F(0.4) + F(0.67) * FCLOG);
                double z = CPLOG / (F(0.75) - F(1.27) * FCLOG - F(0.14) * CPLOG);
                RFACT = pow(10.0, FCLOG / (1.0 + z * z));
            } else if (TR[0] == 0.0) {
                RFACT = 1.0;
            } else {                             /* SRI form */
                double l = log10(AK0M);
                double XFACT = 1.0 / (1.0 + l * l);
                RFACT = pow(-(TR[0] * exp(-(TR[1] / TKD))) + exp(-(TKD / TR[2])), XFACT);
            }
            double AFP = (AK0M / (1.0 + AK0M)) * RFACT;
            SPRF[ir] = AFP * SPRF[ir];
            SPRF[ir + 1] = AFP * SPRF[ir + 1];
        }
    }
    /* rate-coefficient plane, ckrates.f:796-1333 */
    const double CC[4] = {0, C1ST, C2ND, C3RD};
    const double RR[4] = {0, RHO1, RHO2, RHO3};
    for (int r = 0; r < LRX; ++r) {
        if (!T.rc_has[r]) { o->rc[r] = 0.0; continue; }   /* slots 502..518: zero COMMON */
        int od = T.rc_order[r];
        double v = CC[od] * RR[od];
        if (T.rc_tb[r] >= 0) v = v * TB[T.rc_tb[r]];
        v = v * SPRF[r];
        int oo = T.rc_off[r];
        for (int t = 0; t < T.rc_len[r]; ++t) {
            int k = T.rc_idx[oo + t];
            if (T.rc_kind[oo + t] == FK_Y) v = v * y[k];
            else v = v / S.WM[k];
        }
        o->rc[r] = v;
    }
    /* soot source terms, ckrates.f:1337-1352 */
    {
        const double PI = 3.1415927e+00, RSOOT = 1.9000e+03, SIGB = 1.38e-23, AVNO = 6.0232e+23;
        const double CMIN = F(100.0), CAGL = F(9.0);
        const double AKST1 = 1.000e+04, EAST1 = 2.0632e+04, AKST2 = 3.468e+03, EAST2 = 1.2077e+04;
        const double AKST3 = 1.000e+04, ALST3 = F(0.5), EAST3 = 1.9626e+04;
        const double AKST4 = 1.060e+02, ALST4 = F(-0.5), EAST4 = F(0.0);
        const double AKST5 = 5.54e+00, ALST5 = F(-0.5), EAST5 = F(0.0);
        double DPST = 0.0;
        if (stnd >= 1.0) DPST = pow(6.0 * stmf / (PI * RSOOT * stnd), F(0.333333));
        double ASST = PI * DPST * DPST * S.RSTR * rho * stnd;
        double SOURNU = C1ST * RHO1 * AKST1 * exp(-(EAST1 / TKD)) / S.WM[21];
        o->sour[0] = SOURNU + C1ST * RHO1 * ASST * AKST2 * exp(-(EAST2 / TKD)) / S.WM[21];
        o->sour[1] = 2.0 * SOURNU * AVNO / CMIN / S.WMSTR;
        o->sour[2] = C1ST * RHO1 * ASST * AKST3 * pow(TKD, ALST3) * exp(-(EAST3 / TKD)) / S.WM[1];
        o->sour[3] = F(0.13) * C1ST * ASST * AKST4 * pow(TKD, ALST4) * exp(-(EAST4 / TKD)) / S.WM[4] / TBODY;
        o->sour[4] = F(0.5) * C1ST * ASST * AKST5 * pow(TKD, ALST5) * exp(-(EAST5 / TKD)) / S.WM[3] / TBODY;
        o->sour[5] = 2.0 * C1ST * S.RSTR * CAGL * sqrt(DPST * 6.0 * SIGB * TKD / RSOOT) * rho * rho * stnd;
    }
}

/* n cells, SoA inputs: y[k*n + c]. Outputs rc[r*n + c], sour[m*n + c]. */
void orc_rates(int n, const double *tk, const double *rho, const double *y, const double *stmf,
               const double *stnd, double *rc, double *sour)
{
    cell_rates cr;
    double yc[LSP];
    for (int c = 0; c < n; ++c) {
        for (int k = 0; k < LSP; ++k) yc[k] = y[(size_t)k * n + c];
        rates_cell(tk[c], rho[c], yc, stmf ? stmf[c] : 0.0, stnd ? stnd[c] : 0.0, &cr);
        if (rc) for (int r = 0; r < LRX; ++r) rc[(size_t)r * n + c] = cr.rc[r];
        if (sour) for (int m = 0; m < 6; ++m) sour[(size_t)m * n + c] = cr.sour[m];
    }
}

/* ------------------------------------------------------------- products */

/* value of a product chain; A = current A-terms, RA = reaction rates */
static double chain_value(int foff, int flen, const double *A, const double *RC, const double *Y,
                          const double *Y0, const double *SOUR, const double *RA)
{
    double v = 0.0;
    for (int f = 0; f < flen; ++f) {
        int kd = T.fac_kind[foff + f], ix = T.fac_idx[foff + f];
        double x;
        switch (kd) {
        case FK_NUM: x = T.fac_val[foff + f]; break;
        case FK_A: x = A[ix]; break;
        case FK_RC: x = RC[ix]; break;
        case FK_Y: x = Y[ix]; break;
        case FK_Y0: x = Y0[ix]; break;
        case FK_SOUR: x = SOUR[ix]; break;
        case FK_RA: x = RA[ix]; break;
        default: x = 0.0; break;           /* FK_SRA: SRA(1..6)=0.0, solveh.f:671-676 */
        }
        v = f == 0 ? x : v * x;
    }
    return v;
}

static double sum_terms(int off, int len, const double *A, const double *RC, const double *Y,
                        const double *Y0, const double *SOUR, const double *RA)
{
    double acc = 0.0;
    for (int t = 0; t < len; ++t) {
        int ti = off + t;
        double v = chain_value(T.term_foff[ti], T.term_flen[ti], A, RC, Y, Y0, SOUR, RA);
        if (t == 0) acc = T.term_sign[ti] > 0 ? v : -v;
        else acc = T.term_sign[ti] > 0 ? acc + v : acc - v;
    }
    return acc;
}

/* ------------------------------------------------------------- SOLVEH rates */

static void henth_cell(double tk, double *henth)
{
    /* solveh.f:39-57 */
    double HCONVR = S.GASC / S.WMSTR / S.HSTR;
    double TKD = tk * S.TSTR;
    double TKD2 = TKD * TKD, TKD3 = TKD * TKD2, TKD4 = TKD * TKD3, TKD5 = TKD * TKD4;
    int ip = TKD > T.tpol1 ? 7 : 0;
    for (int k = 0; k < LSP; ++k) {
        const double *a = T.poly + k * 14 + ip;
        double HSSP = (a[0] * TKD + a[1] * TKD2 / 2.0 + a[2] * TKD3 / 3.0 + a[3] * TKD4 / 4.0
                       + a[4] * TKD5 / 5.0) / S.WM[k] * HCONVR;
        henth[k] = HSSP * S.WMSTR * S.HSTR + a[5] / S.WM[k] * S.GASC;
    }
}

/* CKRATES followed by SOLVEH's rate part (solveh.f:116-1145) per cell.
 * qdsp[k*n+c] = -RCONV*PRD/HFO (the reference's sign: minus omega),
 * qdot[c] = -HRR*RCONV, henth[k*n+c] species enthalpies, and
 * domega_dy[k*n+c] = -RCONV*W_k*L_k, the diagonal linearisation of omega_k
 * (L_k = sum of the loss rate terms of PRD(k) with one Y_k factored out). */
void orc_omega(int n, const double *tk, const double *rho, const double *y, const double *stmf,
               const double *stnd, double *qdsp, double *qdot, double *henth, double *domega_dy)
{
    cell_rates cr;
    double yc[LSP], RA[LRX], H[LSP], PRD[LSP];
    const double RCONV = S.VSTR / S.WMSTR / S.ALSTR * 1.0e-06;
    for (int c = 0; c < n; ++c) {
        for (int k = 0; k < LSP; ++k) yc[k] = y[(size_t)k * n + c];
        rates_cell(tk[c], rho[c], yc, stmf ? stmf[c] : 0.0, stnd ? stnd[c] : 0.0, &cr);
        henth_cell(tk[c], H);
        for (int r = 0; r < LRX; ++r) {     /* solveh.f:116-664 RA(r)=RC*Y*Y... */
            if (!T.ra_has[r]) { RA[r] = 0.0; continue; }
            double v = cr.rc[r];
            for (int t = 0; t < T.ra_len[r]; ++t) v = v * yc[T.ra_sp[T.ra_off[r] + t]];
            RA[r] = v;
        }
        for (int k = 0; k < LSP; ++k) {     /* solveh.f:677-1133 */
            if (!T.prd_has[k]) { PRD[k] = 0.0; continue; }
            double s = sum_terms(T.prd_off[k], T.prd_len[k], NULL, cr.rc, yc, NULL, cr.sour, RA);
            PRD[k] = S.WM[k] * S.HFO[k] * s;
        }
        double HRR = 0.0;
        for (int k = 0; k < LSP; ++k) {     /* solveh.f:1134-1140 */
            HRR = HRR + PRD[k] * H[k] / S.HFO[k];
            if (qdsp) qdsp[(size_t)k * n + c] = -(RCONV * PRD[k] / S.HFO[k]);
            if (henth) henth[(size_t)k * n + c] = H[k];
        }
        if (qdot) qdot[c] = -(HRR * RCONV);
        if (domega_dy) {
            for (int k = 0; k < LSP; ++k) {
                double L = 0.0;
                if (T.prd_has[k]) {
                    int o = T.prd_off[k];
                    for (int t = 0; t < T.prd_len[k]; ++t) {
                        int ti = o + t;
                        if (T.term_sign[ti] > 0) continue;
                        /* loss term -RA(r): RC(r) times the reactants but one Y_k */
                        int fo = T.term_foff[ti];
                        if (T.fac_kind[fo + T.term_flen[ti] - 1] != FK_RA) continue;
                        int r = T.fac_idx[fo + T.term_flen[ti] - 1];
                        double v = cr.rc[r];
                        int skipped = 0;
                        for (int q = 0; q < T.ra_len[r]; ++q) {
                            int sp = T.ra_sp[T.ra_off[r] + q];
                            if (sp == k && !skipped) { skipped = 1; continue; }
                            v = v * yc[sp];
                        }
                        L = L + v;
                    }
                }
                domega_dy[(size_t)k * n + c] = -(RCONV * S.WM[k] * L);
            }
        }
    }
}

/* ------------------------------------------------------------- cp, h */

/* spgsolv.f:102-173: TCP, the non-dimensional mixture cp */
void orc_cp(int n, const double *tk, const double *y, double *cp)
{
    for (int c = 0; c < n; ++c) {
        double TKD = tk[c] * S.TSTR;
        double TKD2 = TKD * TKD, TKD3 = TKD * TKD2, TKD4 = TKD * TKD3;
        int ip = TKD > T.tpol1 ? 7 : 0;
        double TCP = 0.0;
        for (int k = 0; k < LSP; ++k) {
            const double *a = T.poly + k * 14 + ip;
            double t = (a[0] + a[1] * TKD + a[2] * TKD2 + a[3] * TKD3 + a[4] * TKD4) / S.WM[k];
            TCP = TCP + t * y[(size_t)k * n + c];
        }
        cp[c] = TCP / S.WMSTR * S.GASC * S.TSTR / S.HSTR;
    }
}

/* species enthalpies (solveh.f:39-57) and the mixture value sum_k Y_k h_k */
void orc_enthalpy(int n, const double *tk, const double *y, double *henth, double *hmix)
{
    double H[LSP];
    for (int c = 0; c < n; ++c) {
        henth_cell(tk[c], H);
        double s = 0.0;
        for (int k = 0; k < LSP; ++k) {
            if (henth) henth[(size_t)k * n + c] = H[k];
            s = s + y[(size_t)k * n + c] * H[k];
        }
        if (hmix) hmix[c] = s;
    }
}

/* ------------------------------------------------------------- transport */

static double ci11t(int K, double TKDS, double TKD2, double TKD3, double TKD4, int i, int j)
{
    const double *c = T.ci11 + K * 5;
    return c[0] + c[1] * TKDS + c[2] * TKD2 / S.ETLJ2[i][j] + c[3] * TKD3 / S.ETLJ3[i][j]
           + c[4] * TKD4 / S.ETLJ4[i][j];
}

static int ci_range(double TKDS)
{
    int K = 0;
    if (TKDS >= 2.0) K = 1;
    if (TKDS > 5.0) K = 2;
    if (TKDS > 70.0) K = 3;
    return K;
}

/* main:821-1006 for n cells. y is clipped in place (Y<0 -> 0, N2 = 1 - sum).
 * Outputs are the reference's non-dimensional VMU, VTC and VDFSP. nsub[c]
 * (optional) receives the sub-mixture size LSPT. */
void orc_props(int n, const double *tk, double *y, double *vmu, double *vtc, double *vdf,
               int *nsub)
{
    const double FLMT = 1.0e-03;
    int ISPQ[LSP], ISPQR[LSP + 1];
    double XSP[LSP], ATC[LSP], AMU[LSP], PHIK[LSP], PHDIK[LSP], EFDIK[LSP], VDFQ[LSP];
    static double DIF[LSP][LSP];   /* DIFSP: diagonal never assigned (static zero) */
    for (int c = 0; c < n; ++c) {
        double yc[LSP];
        for (int k = 0; k < LSP; ++k) yc[k] = y[(size_t)k * n + c];
        /* main:821-828 */
        double TMASS = 0.0;
        for (int k = 0; k < LSP - 1; ++k) {
            if (yc[k] < 0.0) yc[k] = 0.0;
            TMASS = TMASS + yc[k];
        }
        yc[LSP - 1] = 1.0 - TMASS;
        for (int k = 0; k < LSP; ++k) y[(size_t)k * n + c] = yc[k];
        /* sub-mixture, main:842-915 */
        int IA = 0;
        TMASS = 0.0;
        double TMOLE = 0.0;
        for (int k = 0; k < LSP - 1; ++k) {
            ISPQ[k] = -1;
            if (yc[k] < FLMT) continue;
            ISPQ[k] = IA;
            ISPQR[IA] = k;
            TMASS = TMASS + yc[k];
            XSP[IA] = yc[k] / S.WM[k];
            TMOLE = TMOLE + XSP[IA];
            IA += 1;
        }
        ISPQ[LSP - 1] = -1;                /* ISPQ(LSP) is never assigned (static 0) */
        int LSPT = IA + 1;
        if (LSPT >= LSP) LSPT = LSP;
        ISPQR[LSPT - 1] = LSP - 1;
        XSP[LSPT - 1] = (1.0 - TMASS) / S.WM[LSP - 1];
        TMOLE = TMOLE + XSP[LSPT - 1];
        if (nsub) nsub[c] = LSPT;
        double TKRT = sqrt(tk[c]);
        double TKD1 = tk[c] * S.TSTR;
        double TKD2 = TKD1 * TKD1, TKD3 = TKD2 * TKD1, TKD4 = TKD3 * TKD1, TKD5 = TKD4 * TKD1;
        int IPL1 = 0, IPL2 = 0;
        if (TKD1 >= T.tpol1) { IPL1 = 7; IPL2 = 6; }
        double TKBP = tk[c] * TKRT / S.PBACK;
        /* main:929-955 */
        for (int a = 0; a < LSPT; ++a) {
            int k = ISPQR[a];
            const double *p = T.poly + k * 14 + IPL1;
            const double *q = T.om22 + k * 12 + IPL2;
            double EUKEN = F(0.115) + F(0.354) * (p[0] + p[1] * TKD1 + p[2] * TKD2 + p[3] * TKD3
                                                  + p[4] * TKD4);
            double SIOME = T.cdia[k] * T.cdia[k] * (q[0] + q[1] * TKD1 + q[2] * TKD2 + q[3] * TKD3
                                                   + q[4] * TKD4 + q[5] * TKD5);
            ATC[a] = S.CONVRC * EUKEN * TKRT / S.WMIK[k][k] / SIOME;
            AMU[a] = S.CONVRM * TKRT * S.WMIK[k][k] / SIOME;
            for (int b = a + 1; b < LSPT; ++b) {
                int kb = ISPQR[b];
                double TKDS = TKD1 / S.ETLJ1[k][kb];
                int K = ci_range(TKDS);
                double CI = ci11t(K, TKDS, TKD2, TKD3, TKD4, k, kb);
                DIF[a][b] = S.WMCD[k][kb] * TKBP / CI;
                DIF[b][a] = S.WMCD[kb][k] * TKBP / CI;
            }
        }
        /* main:957-979 */
        for (int a = 0; a < LSPT; ++a) {
            int k = ISPQR[a];
            PHIK[a] = 0.0; PHDIK[a] = 0.0; EFDIK[a] = 0.0;
            for (int b = 0; b < LSPT; ++b) {
                if (b == a) continue;
                int kb = ISPQR[b];
                double t1 = 1.0 + sqrt(ATC[a] / ATC[b]) * S.WMIK[k][kb];
                double t2 = 1.0 + sqrt(AMU[a] / AMU[b]) * S.WMIK[k][kb];
                PHIK[a] = PHIK[a] + XSP[b] * (t1 * t1) / S.DWMIK[k][kb];
                PHDIK[a] = PHDIK[a] + XSP[b] * (t2 * t2) / S.DWMIK[k][kb];
                EFDIK[a] = EFDIK[a] + XSP[b] / DIF[a][b];
            }
        }
        double VTC = 0.0, VMU = 0.0;
        for (int a = 0; a < LSPT; ++a) {
            VTC = VTC + ATC[a] * XSP[a] / (XSP[a] + F(1.065) * PHIK[a]);
            VMU = VMU + AMU[a] * XSP[a] / (XSP[a] + PHDIK[a]);
            double AA = TMOLE - XSP[a];
            if (AA <= 1.0e-10) VDFQ[a] = S.CONVRD * DIF[a][LSPT - 1];
            else VDFQ[a] = S.CONVRD * (TMOLE - XSP[a]) / EFDIK[a];
        }
        vtc[c] = VTC;
        vmu[c] = VMU;
        /* main:981-1003 */
        for (int k = 0; k < LSP; ++k) {
            double v;
            if (ISPQ[k] < 0) {
                double EFD = 0.0;
                for (int b = 0; b < LSPT; ++b) {
                    int nb = ISPQR[b];
                    double TKDS = TKD1 / S.ETLJ1[k][nb];
                    int K = ci_range(TKDS);
                    double CI = ci11t(K, TKDS, TKD2, TKD3, TKD4, k, nb);
                    EFD = EFD + XSP[b] / (S.WMCD[k][nb] * TKBP / CI);
                }
                v = S.CONVRD * TMOLE / EFD;
            } else {
                v = VDFQ[ISPQ[k]];
            }
            vdf[(size_t)k * n + c] = v;
        }
    }
}

/* ------------------------------------------------------------- SOLVESP */

/* Point-implicit relaxation of species 1..51 and the two soot scalars
 * (solvesp.f:82-2836), then the N2 closure (solvesp.f:2837-2915).
 *
 * Cells are independent here: the face coefficients of the reference
 * (EA..QA, ``nbr``) enter through face_sum[k*n+c] = E+W+N+S and
 * face_nbr[k*n+c] = P*Y(J+1)+Q*Y(J-1)+E*Y(I+1)+W*Y(I-1) evaluated on a frozen
 * neighbour field (both may be NULL: no transport). The pass loop stops when
 * sum|dY|/spnorm <= tol (solvesp.f:2833), over all n cells.
 * y0: old-time mass fractions (FA..), y: current values (SA..), updated in
 * place; rc, sour: CKRATES outputs; soot[2*n]: mass fraction, number density
 * (updated in place; old-time values in soot0). Returns the pass count as
 * the reference reports it in ISOR1. */
int orc_species_update(int n, const double *rho, const double *y0, double *y, const double *rc,
                       const double *sour, const double *soot0, double *soot,
                       const double *face_sum, const double *face_nbr, double dt, int isor,
                       double relx, double tol, double spnorm)
{
    const double SOR1 = relx, SOR2 = 1.0 - SOR1;
    double *A = (double *)calloc(LRX + 1, sizeof(double));
    double Y[LSP], Y0[LSP], RC[LRX], SO[6];
    int ISORP;
    for (ISORP = 1; ISORP <= isor; ++ISORP) {
        double RSD = 0.0;
        for (int c = 0; c < n; ++c) {
            for (int k = 0; k < LSP; ++k) { Y[k] = y[(size_t)k * n + c]; Y0[k] = y0[(size_t)k * n + c]; }
            for (int r = 0; r < LRX; ++r) RC[r] = rc[(size_t)r * n + c];
            for (int m = 0; m < 6; ++m) SO[m] = sour[(size_t)m * n + c];
            double RHO = rho[c];
            double RHS1A = 0.0;
            for (int b = 0; b < LSP - 1; ++b) {
                /* A-term (re)computations */
                int ro = T.blk_rec_off[b];
                for (int t = 0; t < T.blk_rec_len[b]; ++t) {
                    int r = T.rec_r[ro + t];
                    A[r] = chain_value(T.rec_foff[ro + t], T.rec_flen[ro + t], A, RC, Y, Y0, SO, NULL);
                }
                /* Q3: a block without an RHS1A statement reuses the previous value */
                if (T.blk_prod_has[b])
                    RHS1A = sum_terms(T.blk_prod_off[b], T.blk_prod_len[b], A, RC, Y, Y0, SO, NULL);
                double RHS1B = sum_terms(T.blk_extra_off[b], T.blk_extra_len[b], A, RC, Y, Y0, SO, NULL);
                int k = b;   /* block b updates species b+1 (0-based b) */
                double RHS1 = RHO * Y0[k] + dt * S.WM[k] * (RHS1A + RHS1B);
                double RHS2 = 0.0;
                if (T.blk_loss_has[b])
                    RHS2 = -(dt * S.WM[k] * sum_terms(T.blk_loss_off[b], T.blk_loss_len[b], A, RC, Y, Y0, SO, NULL));
                double fs = face_sum ? face_sum[(size_t)k * n + c] : 0.0;
                double fn = face_nbr ? face_nbr[(size_t)k * n + c] : 0.0;
                double PPP = RHO - fs;
                double FNEW = SOR2 * Y[k] + (RHS1 - fn) * SOR1 / (PPP - RHS2);
                RSD = RSD + fabs(Y[k] - FNEW);
                if (FNEW < 0.0) FNEW = 0.0;
                Y[k] = FNEW;
                int mo = T.blk_mul_off[b];
                for (int t = 0; t < T.blk_mul_len[b]; ++t) A[T.mul_r[mo + t]] = FNEW * A[T.mul_r[mo + t]];
            }
            /* soot mass fraction, solvesp.f:2807-2820 (molar mass of C) */
            {
                double RHS1 = RHO * soot0[c] + dt * (F(0.012011) / S.WMSTR) *
                              (2.0 * SO[0] * Y[21] - SO[2] * Y[1] - SO[3] * Y[4] - SO[4] * Y[3]);
                double PPP = RHO - 0.0;
                double FNEW = SOR2 * soot[c] + RHS1 * SOR1 / (PPP - 0.0);
                RSD = RSD + fabs(soot[c] - FNEW);
                if (FNEW < 0.0) FNEW = 0.0;
                soot[c] = FNEW;
            }
            /* soot number density, solvesp.f:2822-2832 */
            {
                double RHS1 = RHO * soot0[n + c] + dt * SO[1] * Y[21];
                double RHS2 = -(dt * SO[5]);
                double PPP = RHO - 0.0;
                double FNEW = SOR2 * soot[n + c] + RHS1 * SOR1 / (PPP - RHS2);
                if (FNEW < 0.0) FNEW = 0.0;
                soot[n + c] = FNEW;
            }
            for (int k = 0; k < LSP - 1; ++k) y[(size_t)k * n + c] = Y[k];
        }
        if (RSD / spnorm <= tol) break;
    }
    /* solvesp.f:2834-2838: the reference reports ISORP (ISOR1+1 if not converged) */
    int passes = ISORP;
    /* N2 closure and renormalisation, solvesp.f:2839-2915 (Q5: only if sum > 1) */
    for (int c = 0; c < n; ++c) {
        double FTOT = y[c];
        for (int k = 1; k < LSP - 1; ++k) FTOT = FTOT + y[(size_t)k * n + c];
        FTOT = FTOT + soot[c];
        double N2 = 1.0 - FTOT;
        if (FTOT > 1.0) {
            for (int k = 0; k < LSP - 1; ++k) y[(size_t)k * n + c] = y[(size_t)k * n + c] / FTOT;
            soot[c] = soot[c] / FTOT;
            N2 = 0.0;
        }
        y[(size_t)(LSP - 1) * n + c] = N2;
    }
    free(A);
    return passes;
}

/* ------------------------------------------------------------- T from h */

/* solveh.f:1170-1234: temperature from the non-dimensional sensible
 * enthalpy ht (FPZ) and the mass fractions; tk holds the guess on entry. */
/* Newton for T at the total enthalpy ENTH (solveh.f:1186-1234); y has
 * stride ys between species. Returns the new non-dimensional tk. */
static double temperature_cell_conv(double tk, const double *y, size_t ys, double ENTH, int *conv);
static double temperature_cell(double tk, const double *y, size_t ys, double ENTH)
{
    return temperature_cell_conv(tk, y, ys, ENTH, NULL);
}

/* conv (optional) receives 1 when the Newton met its step rule within 100 steps */
static double temperature_cell_conv(double tk, const double *y, size_t ys, double ENTH, int *conv)
{
    const double TKDMIN = S.TSTR - 1.0;
    int IPL = 0;
    double TPOLY = T.tpol1;
    double TKD = tk * S.TSTR;
    double A1, A2, A3, A4, A5, A6;
    for (;;) {
        if (TKD > TPOLY) TKD = TPOLY / 2.0;
        A1 = A2 = A3 = A4 = A5 = A6 = 0.0;
        for (int k = 0; k < LSP; ++k) {
            const double *a = T.poly + k * 14 + IPL;
            double yk = y[(size_t)k * ys];
            A1 = A1 + a[0] * yk / S.WM[k];
            A2 = A2 + a[1] * yk / S.WM[k] / 2.0;
            A3 = A3 + a[2] * yk / S.WM[k] / 3.0;
            A4 = A4 + a[3] * yk / S.WM[k] / 4.0;
            A5 = A5 + a[4] * yk / S.WM[k] / 5.0;
            A6 = A6 + a[5] * yk / S.WM[k];
        }
        double FUNT = ((A1 + (A2 + (A3 + (A4 + A5 * TPOLY) * TPOLY) * TPOLY) * TPOLY) * TPOLY + A6)
                      * S.GASC / S.WMSTR - ENTH;
        if (FUNT >= 1.0e-07) break;
        if (IPL >= 7) break;
        IPL = 7;
        if (TKD <= TPOLY) TKD = T.tpol2 / 2.0;
        TPOLY = T.tpol2;
    }
    if (conv) *conv = 0;
    for (int it = 1; it <= 100; ++it) {
        double DTKD = ((A1 + (A2 + (A3 + (A4 + A5 * TKD) * TKD) * TKD) * TKD) * TKD + A6
                       - ENTH * S.WMSTR / S.GASC)
                      / (A1 + (2.0 * A2 + (3.0 * A3 + (4.0 * A4 + 5.0 * A5 * TKD) * TKD) * TKD) * TKD);
        if (fabs(DTKD) <= F(0.001)) {
            if (conv) *conv = 1;
            break;
        }
        TKD = TKD - DTKD;
    }
    if (TKD > T.tpol2) TKD = T.tpol2;
    if (TKD < TKDMIN) TKD = TKDMIN;
    return TKD / S.TSTR;
}

void orc_temperature(int n, double *tk, const double *y, const double *ht)
{
    for (int c = 0; c < n; ++c) {
        double ENTH = (ht[c] - F(0.5) * 0.0) * S.HSTR;
        for (int k = 0; k < LSP; ++k) ENTH = ENTH + y[(size_t)k * n + c] * S.HFO[k] * S.HSTR;
        tk[c] = temperature_cell(tk[c], y + c, (size_t)n, ENTH);
    }
}

/* ------------------------------------------------------------- batched stiff integration */

/* Total enthalpy of a cell at its own temperature, in the units of ENTH in
 * solveh.f:1186-1205 (the polynomial of the T-from-h Newton at T, range by
 * T > TPOL1 as in the kinetics). */
static double enthalpy_total(double tk, const double *y, size_t ys)
{
    double TKD = tk * S.TSTR;
    int ip = TKD > T.tpol1 ? 7 : 0;
    double A1 = 0.0, A2 = 0.0, A3 = 0.0, A4 = 0.0, A5 = 0.0, A6 = 0.0;
    for (int k = 0; k < LSP; ++k) {
        const double *a = T.poly + k * 14 + ip;
        double yk = y[(size_t)k * ys];
        A1 = A1 + a[0] * yk / S.WM[k];
        A2 = A2 + a[1] * yk / S.WM[k] / 2.0;
        A3 = A3 + a[2] * yk / S.WM[k] / 3.0;
        A4 = A4 + a[3] * yk / S.WM[k] / 4.0;
        A5 = A5 + a[4] * yk / S.WM[k] / 5.0;
        A6 = A6 + a[5] * yk / S.WM[k];
    }
    return ((A1 + (A2 + (A3 + (A4 + A5 * TKD) * TKD) * TKD) * TKD) * TKD + A6) * S.GASC / S.WMSTR;
}

/* The in-loop T update of the sweep loop (uc_hold_enthalpy, uc_temperature_from_held):
 * each cell's total enthalpy at its own T is held; after the species update T
 * follows from the held enthalpy and the new mass fractions by the Newton of
 * solveh.f:1186-1234 (T clamped to [TSTR-1, TPOL2] as there), and rho from the
 * ideal gas at the cell pressure (main:1056-1062, RHO = P/(BETA1 TK sum Y/W)).
 * The same step that orc_integrate takes per sub-step; conv (optional) [n]
 * receives 1 where the Newton met its step rule (the reference prints a
 * message where it did not, and carries on). */
void orc_enthalpy_total(int n, const double *tk, const double *y, double *enth)
{
    for (int c = 0; c < n; ++c) enth[c] = enthalpy_total(tk[c], y + c, (size_t)n);
}

void orc_temperature_held(int n, double *tk, double *rho, const double *y, const double *pnd, const double *enth,
                          int *conv)
{
    for (int c = 0; c < n; ++c) {
        const double t = temperature_cell_conv(tk[c], y + c, (size_t)n, enth[c], conv ? conv + c : NULL);
        double rbar = 0.0;
        for (int k = 0; k < LSP; ++k) rbar = rbar + y[(size_t)k * n + c] / S.WM[k];
        tk[c] = t;
        rho[c] = pnd[c] / (S.BETA1 * t * rbar);
    }
}

/* Sub-step count of each cell from its chemical time scale:
 *   x = max over species with Y_k > y_tau of dt*|QDSP_k| / (RCONV*rho*Y_k)
 * (dY_k/dt = -QDSP_k/(RCONV*rho) in the reference's units, solveh.f:1138),
 *   n_sub = clamp(ceil(x / c_tau), 1, nsub_max);  x_out (optional) gets x. */
void orc_nsub(int n, const double *rho, const double *y, const double *qdsp, double dt, double c_tau,
              double y_tau, int nsub_max, int *nsub, double *x_out)
{
    const double RCONV = S.VSTR / S.WMSTR / S.ALSTR * 1.0e-06;
    for (int c = 0; c < n; ++c) {
        double x = 0.0;
        for (int k = 0; k < LSP; ++k) {
            double yk = y[(size_t)k * n + c];
            if (yk > y_tau) {
                double v = dt * fabs(qdsp[(size_t)k * n + c]) / (RCONV * rho[c] * yk);
                if (!(v <= x)) x = v;       /* NaN propagates */
            }
        }
        double m = ceil(x / c_tau);
        int ns = (m != m || m >= (double)nsub_max) ? nsub_max : (m < 1.0 ? 1 : (int)m);
        nsub[c] = ns;
        if (x_out) x_out[c] = x;
    }
}

/* Batched stiff point-implicit integration of independent cells over dt.
 * Each cell is its own one-cell field advanced n_sub times by dt/n_sub with
 * the reference's own steps: rates (ckrates.f), the species update with its
 * closure (solvesp.f; SPNORM = LSP-1, no face terms; each cell converges on
 * its own residual), T from the cell's constant total enthalpy
 * (solveh.f:1186-1234) and rho from the ideal gas at the cell's pressure
 * pnd = p/PSTR (main:1056-1062). State arrays are [52][n], [n] and soot
 * [2][n], updated in place. nsub holds the per-cell counts (orc_nsub).
 * passes (optional) receives the update passes summed over the sub-steps. */
void orc_integrate(int n, double *tk, double *rho, double *y, double *soot, const double *pnd,
                   const int *nsub, double dt, int isor, double relx, double tol, int *passes)
{
#pragma omp parallel for schedule(dynamic, 1)
    for (int c = 0; c < n; ++c) {
        cell_rates cr;
        double yc[LSP], y0[LSP], s[2], s0[2];
        for (int k = 0; k < LSP; ++k) yc[k] = y[(size_t)k * n + c];
        s[0] = soot[c];
        s[1] = soot[(size_t)n + c];
        double t = tk[c], r = rho[c];
        const double ENTH0 = enthalpy_total(t, yc, 1);
        const double dts = dt / (double)nsub[c];
        int np = 0;
        for (int st = 0; st < nsub[c]; ++st) {
            rates_cell(t, r, yc, s[0], s[1], &cr);
            memcpy(y0, yc, sizeof(y0));
            s0[0] = s[0];
            s0[1] = s[1];
            int p = orc_species_update(1, &r, y0, yc, cr.rc, cr.sour, s0, s, NULL, NULL, dts, isor, relx, tol,
                                       (double)(LSP - 1));
            np += p > isor ? isor : p;
            t = temperature_cell(t, yc, 1, ENTH0);
            double rbar = 0.0;
            for (int k = 0; k < LSP; ++k) rbar = rbar + yc[k] / S.WM[k];
            r = pnd[c] / (S.BETA1 * t * rbar);
        }
        for (int k = 0; k < LSP; ++k) y[(size_t)k * n + c] = yc[k];
        soot[c] = s[0];
        soot[(size_t)n + c] = s[1];
        tk[c] = t;
        rho[c] = r;
        if (passes) passes[c] = np;
    }
}

/* ------------------------------------------------------------- species face coefficients */

/* E/W/N/S coefficients of the species equations (spgsolv.f:233-348 face
 * conductances, :350-1290 hybrid convection-diffusion coefficients) for the
 * interior cells J=2..LJ-1, I=2..LI-1 of an lj x li grid (J fastest; cell
 * c = (I-1)*lj + (J-1)). rho, u, v, tmu, yr [lj*li]; vdf [52][lj*li];
 * xxs, xxc [li]; yys, yyc [lj]. Outputs e, w, n, s [51][lj*li]; boundary
 * entries are left untouched. Every cell is assembled (no ISKIP). */
void orc_faces(int lj, int li, const double *rho, const double *vdf, const double *u, const double *v,
               const double *tmu, const double *yr, const double *xxs, const double *xxc, const double *yys,
               const double *yyc, int isym, double dt, double sigsp, double *e, double *w, double *n, double *s)
{
    const size_t ne = (size_t)lj * li;
    const double SYM = (double)isym;
#define CI(j, i) ((size_t)(i) * lj + (j))          /* 0-based (j, i) */
#define EMU(j, i) (S.REI * S.BETA3 * rho[CI(j, i)])
    for (int i = 1; i < li - 1; ++i) {
        for (int j = 1; j < lj - 1; ++j) {
            const size_t c = CI(j, i);
            const double DTBRX = dt / xxc[i], DTBRY = dt / yyc[j];
            const double RHOUE = 0.5 * (rho[CI(j, i + 1)] + rho[c]) * u[CI(j, i + 1)];
            const double RHOUW = 0.5 * (rho[c] + rho[CI(j, i - 1)]) * u[c];
            const double RHOVN = 0.5 * (rho[CI(j + 1, i)] + rho[c]) * v[CI(j + 1, i)];
            const double RHOVS = 0.5 * (rho[c] + rho[CI(j - 1, i)]) * v[c];
            const double SYM1 = SYM * dt * 0.5 * EMU(j, i) / yr[c];
            const double SYM2 = SYM * dt * 0.5 * S.REI * tmu[c] / sigsp / yr[c];
            /* turbulent parts of the conductances of the faces E (= W of I+1), W, N (= S of J+1), S */
            const double TURE = S.REI * (tmu[CI(j, i + 1)] + tmu[c]) / sigsp;
            const double TURW = S.REI * (tmu[c] + tmu[CI(j, i - 1)]) / sigsp;
            const double TURN = S.REI * (tmu[CI(j + 1, i)] + tmu[c]) / sigsp;
            const double TURS = S.REI * (tmu[c] + tmu[CI(j - 1, i)]) / sigsp;
            for (int k = 0; k < LSP - 1; ++k) {
                const double *d = vdf + (size_t)k * ne;
                const double DE = (EMU(j, i + 1) * d[CI(j, i + 1)] + EMU(j, i) * d[c] + TURE) / xxs[i + 1];
                const double DW = (EMU(j, i) * d[c] + EMU(j, i - 1) * d[CI(j, i - 1)] + TURW) / xxs[i];
                const double DN = (EMU(j + 1, i) * d[CI(j + 1, i)] + EMU(j, i) * d[c] + TURN) / yys[j + 1];
                const double DS = (EMU(j, i) * d[c] + EMU(j - 1, i) * d[CI(j - 1, i)] + TURS) / yys[j];
                const double SYMA = SYM1 * d[c] + SYM2;
                double cv;
                cv = fabs(RHOUE); if (DE >= cv) cv = DE;
                e[(size_t)k * ne + c] = DTBRX * 0.5 * (RHOUE - cv);
                cv = fabs(RHOUW); if (DW >= cv) cv = DW;
                w[(size_t)k * ne + c] = DTBRX * 0.5 * (-RHOUW - cv);
                cv = fabs(RHOVN); if (DN >= cv) cv = DN;
                n[(size_t)k * ne + c] = DTBRY * 0.5 * (RHOVN - cv) - SYMA / yys[j + 1];
                cv = fabs(RHOVS); if (DS >= cv) cv = DS;
                s[(size_t)k * ne + c] = DTBRY * 0.5 * (-RHOVS - cv) + SYMA / yys[j];
            }
        }
    }
#undef CI
#undef EMU
}

/* ------------------------------------------------------------- FDETAIL fields */

/* stdata.f:26-118: corner averages of an lj x li grid (J fastest), the last
 * row and column copied, dimensional scales; cp and h_k at the corner T.
 * out [10 + 4*52][lj*li] in the order of the FDETAIL record. */
void orc_fdetail(int lj, int li, const double *x, const double *y, const double *rho, const double *u,
                 const double *v, const double *tk, const double *qdot, const double *vmu, const double *vtc,
                 const double *fsp, const double *vdf, const double *qdsp, double *out)
{
    const size_t ne = (size_t)lj * li;
    const double XSHIFT = 0.5 * (x[0] + x[lj]), YSHIFT = 0.5 * (y[0] + y[1]);
#define O(r, p) out[(size_t)(r) * ne + (p)]
    /* interior corners (stdata.f:1320-1326) */
    for (int i = 0; i < li - 1; ++i)
        for (int j = 0; j < lj - 1; ++j) {
            const size_t c = (size_t)i * lj + j, cN = c + 1, cE = c + lj, cNE = c + lj + 1;
            O(0, c) = (0.5 * (x[c] + x[cE]) - XSHIFT) * S.ALSTR;
            O(1, c) = (0.5 * (y[c] + y[cN]) - YSHIFT) * S.ALSTR;
            O(2, c) = 0.25 * (rho[c] + rho[cN] + rho[cE] + rho[cNE]) * S.RSTR;
            O(5, c) = 0.25 * (tk[c] + tk[cN] + tk[cE] + tk[cNE]) * S.TSTR;
            O(6, c) = 0.25 * (qdot[c] + qdot[cN] + qdot[cE] + qdot[cNE]);
            O(7, c) = 0.25 * (vmu[c] + vmu[cN] + vmu[cE] + vmu[cNE]) * S.AMSTR;
            O(8, c) = 0.25 * (vtc[c] + vtc[cN] + vtc[cE] + vtc[cNE]) * S.ACSTR;
            O(3, c) = 0.5 * (u[cE] + u[cNE]) * S.VSTR;
            O(4, c) = 0.5 * (v[cN] + v[cNE]) * S.VSTR;
            double FTOT = 0.0;
            for (int k = 0; k < LSP; ++k) {
                const size_t kk = (size_t)k * ne;
                O(10 + 4 * k + 1, c) = 0.25 * (vdf[kk + c] + vdf[kk + cN] + vdf[kk + cE] + vdf[kk + cNE]) * S.DSTR;
                O(10 + 4 * k + 2, c) = 0.25 * (qdsp[kk + c] + qdsp[kk + cN] + qdsp[kk + cE] + qdsp[kk + cNE]);
                if (k < LSP - 1) {
                    O(10 + 4 * k, c) = 0.25 * (fsp[kk + c] + fsp[kk + cN] + fsp[kk + cE] + fsp[kk + cNE]);
                    FTOT = FTOT + O(10 + 4 * k, c);
                }
            }
            O(10 + 4 * (LSP - 1), c) = 1.0 - FTOT;
        }
    /* last row, then last column (stdata.f:1322-1325) */
    for (int i = 0; i < li; ++i) {
        const size_t p = (size_t)i * lj + (lj - 1), q = p - 1;
        for (int r = 0; r < 10 + 4 * LSP; ++r) O(r, p) = O(r, q);
        O(1, p) = y[p] * S.ALSTR;
    }
    for (int j = 0; j < lj; ++j) {
        const size_t p = (size_t)(li - 1) * lj + j, q = p - lj;
        for (int r = 0; r < 10 + 4 * LSP; ++r) O(r, p) = O(r, q);
        O(0, p) = x[p] * S.ALSTR;
    }
    /* cp and h_k at the corner temperature (stdata.f:91-118) */
    for (size_t p = 0; p < ne; ++p) {
        const double TKD = O(5, p);
        const double TKD2 = TKD * TKD, TKD3 = TKD * TKD2, TKD4 = TKD * TKD3, TKD5 = TKD * TKD4;
        const int ip = TKD > T.tpol1 ? 7 : 0;
        double TCP = 0.0;
        for (int k = 0; k < LSP; ++k) {
            const double *a = T.poly + k * 14 + ip;
            TCP = TCP + (a[0] + a[1] * TKD + a[2] * TKD2 + a[3] * TKD3 + a[4] * TKD4) * O(10 + 4 * k, p) * S.GASC
                        / S.WM[k] / S.WMSTR;
            O(10 + 4 * k + 3, p) = (a[0] * TKD + a[1] * TKD2 / 2.0 + a[2] * TKD3 / 3.0 + a[3] * TKD4 / 4.0
                                    + a[4] * TKD5 / 5.0 + a[5]) * S.GASC / S.WM[k] / S.WMSTR;
        }
        O(9, p) = TCP;
    }
#undef O
}

/* ------------------------------------------------------------- enthalpy equation */

static inline double powi5(double x) { double t = x * x; double u = t * x; return u * t; }

/* Enthalpy-equation coefficients ZE, ZW, ZN, ZS (spgsolv.f:233-348 and the
 * Z lines of :350-1290) and EKT = REI (BETA2 VTC/TCP + TMU/SIGH)
 * (spgsolv.f:174) of every cell; tcp is the mixture cp of orc_cp. */
void orc_zfaces(int lj, int li, const double *rho, const double *tcp, const double *vtc, const double *tmu,
                const double *u, const double *v, const double *yr, const double *xxs, const double *xxc,
                const double *yys, const double *yyc, int isym, double dt, double sigh, double *ze, double *zw,
                double *zn, double *zs, double *ekt)
{
    const size_t ne = (size_t)lj * li;
    const double SYM = (double)isym;
    for (size_t c = 0; c < ne; ++c) ekt[c] = S.REI * (S.BETA2 * vtc[c] / tcp[c] + tmu[c] / sigh);
#define CI(j, i) ((size_t)(i) * lj + (j))
    for (int i = 1; i < li - 1; ++i)
        for (int j = 1; j < lj - 1; ++j) {
            const size_t c = CI(j, i);
            const double DTBRX = dt / xxc[i], DTBRY = dt / yyc[j];
            const double RHOUE = 0.5 * (rho[CI(j, i + 1)] + rho[c]) * u[CI(j, i + 1)];
            const double RHOUW = 0.5 * (rho[c] + rho[CI(j, i - 1)]) * u[c];
            const double RHOVN = 0.5 * (rho[CI(j + 1, i)] + rho[c]) * v[CI(j + 1, i)];
            const double RHOVS = 0.5 * (rho[c] + rho[CI(j - 1, i)]) * v[c];
            const double SYMZ = SYM * dt * 0.5 * ekt[c] / yr[c];
            const double DE = (ekt[CI(j, i + 1)] + ekt[c]) / xxs[i + 1];
            const double DW = (ekt[c] + ekt[CI(j, i - 1)]) / xxs[i];
            const double DN = (ekt[CI(j + 1, i)] + ekt[c]) / yys[j + 1];
            const double DS = (ekt[c] + ekt[CI(j - 1, i)]) / yys[j];
            double cv;
            cv = fabs(RHOUE); if (DE >= cv) cv = DE;
            ze[c] = DTBRX * 0.5 * (RHOUE - cv);
            cv = fabs(RHOUW); if (DW >= cv) cv = DW;
            zw[c] = DTBRX * 0.5 * (-RHOUW - cv);
            cv = fabs(RHOVN); if (DN >= cv) cv = DN;
            zn[c] = DTBRY * 0.5 * (RHOVN - cv) - SYMZ / yys[j + 1];
            cv = fabs(RHOVS); if (DS >= cv) cv = DS;
            zs[c] = DTBRY * 0.5 * (-RHOVS - cv) + SYMZ / yys[j];
        }
    (void)ne;
}

/* Right-hand side of the enthalpy equation (solveh.f:34-1145) for the
 * interior cells: species-enthalpy diffusion (RDHSP of every cell), the
 * radiation loss of CH4, CO2, CO, H2O and soot, RHO HT and the heat release
 * DT PROD from RA = RC (start state) x Y (after the species update); also
 * QDSP and QDOT of that state. y_new [52][n]; rc [544][n]. */
void orc_enthalpy_rhs(int lj, int li, const double *tk, const double *rho, const double *y_new, const double *ht,
                      const double *stmf, const double *vdf, const double *tmu, const double *ekt, const double *rc,
                      const double *yr, const double *xxs, const double *xxc, const double *yys, const double *yyc,
                      int isym, double dt, double sigsp, double *rhsz, double *qdsp, double *qdot)
{
    const size_t ne = (size_t)lj * li;
    const double SYM = (double)isym, HCONVR = S.GASC / S.WMSTR / S.HSTR;
    const double CRAD = S.ALSTR / S.RSTR / S.VSTR / S.VSTR / S.VSTR;
    const double RCONV = S.VSTR / S.WMSTR / S.ALSTR * 1.0e-06;
    const double RSOOT = 1.9000e+03;
    double *RDHSP = (double *)malloc(ne * LSP * sizeof(double));
    double *HENTH = (double *)malloc(ne * LSP * sizeof(double));
    /* solveh.f:39-57 */
    for (size_t c = 0; c < ne; ++c) {
        const double TKD = tk[c] * S.TSTR;
        const double TKD2 = TKD * TKD, TKD3 = TKD * TKD2, TKD4 = TKD * TKD3, TKD5 = TKD * TKD4;
        const int ip = TKD > T.tpol1 ? 7 : 0;
        const double EMU = S.REI * S.BETA3 * rho[c];
        for (int k = 0; k < LSP; ++k) {
            const double *a = T.poly + k * 14 + ip;
            const double HSSP = (a[0] * TKD + a[1] * TKD2 / 2.0 + a[2] * TKD3 / 3.0 + a[3] * TKD4 / 4.0
                                 + a[4] * TKD5 / 5.0) / S.WM[k] * HCONVR;
            RDHSP[(size_t)k * ne + c] = (EMU * vdf[(size_t)k * ne + c] + S.REI * tmu[c] / sigsp - ekt[c]) * HSSP;
            HENTH[(size_t)k * ne + c] = HSSP * S.WMSTR * S.HSTR + a[5] / S.WM[k] * S.GASC;
        }
    }
#define CI(j, i) ((size_t)(i) * lj + (j))
#define RD(k, p) RDHSP[(size_t)(k) * ne + (p)]
#define YS(k, p) y_new[(size_t)(k) * ne + (p)]
    /* solveh.f:59-115 */
    for (int j = 1; j < lj - 1; ++j)
        for (int i = 1; i < li - 1; ++i) {
            const size_t c = CI(j, i), cE = c + lj, cW = c - lj, cN = c + 1, cS = c - 1;
            double RDHE = 0.0, RDHW = 0.0, RDHN = 0.0, RDHS = 0.0, RDHP = 0.0, TMOLE = 0.0;
            for (int k = 0; k < LSP; ++k) {
                TMOLE = TMOLE + YS(k, c) / S.WM[k];
                RDHE = RDHE + (RD(k, cE) + RD(k, c)) * (YS(k, cE) - YS(k, c));
                RDHW = RDHW + (RD(k, c) + RD(k, cW)) * (YS(k, c) - YS(k, cW));
                RDHN = RDHN + (RD(k, cN) + RD(k, c)) * (YS(k, cN) - YS(k, c));
                RDHS = RDHS + (RD(k, c) + RD(k, cS)) * (YS(k, c) - YS(k, cS));
                RDHP = RDHP + (RD(k, c)) * (YS(k, cN) - YS(k, cS));
            }
            const double TKD = tk[c] * S.TSTR;
            const double TKDI = 1000.0 / TKD, TKDIS = TKDI * TKDI;
            const double PLANK1 = F(6.6334) + TKD * (-3.5686e-03 + TKD * (1.6682e-08 + TKD * (2.5611e-10 - 2.6558e-14 * TKD)));
            const double PLANK2 = 1.8741e+01 - TKDI * (1.2131e+02 - 2.7350e+02 * TKDI + 1.9405e+02 * TKDIS
                                                      - 5.6310e+01 * TKDIS * TKDI + F(5.81690) * TKDIS * TKDIS);
            double PLANK3;
            if (TKD <= F(750.0))
                PLANK3 = F(4.7869) + TKD * (-6.953e-02 + TKD * (2.95775e-04 + TKD * (-4.25732e-07 + 2.02894e-10 * TKD)));
            else
                PLANK3 = 1.009e+01 + TKD * (-1.183e-02 + TKD * (4.7753e-06 + TKD * (-5.87209e-10 - 2.5334e-14 * TKD)));
            const double PLANK4 = -F(0.23093) - TKDI * (F(1.12390) - F(9.41530) * TKDI + F(2.99880) * TKDIS
                                                       - F(0.51382) * TKDIS * TKDI + 1.86840e-05 * TKDIS * TKDIS);
            const double PLANKC = (PLANK1 * YS(12, c) / S.WM[12] + PLANK2 * YS(9, c) / S.WM[9]
                                   + PLANK3 * YS(8, c) / S.WM[8] + PLANK4 * YS(5, c) / S.WM[5]) / TMOLE;
            const double QRAD = CRAD * F(0.4) * (F(4.0) * 5.669e-08 * PLANKC * (pow(TKD, F(4.0)) - 8.1e+09)
                                                + 3.334e-04 * stmf[c] * (rho[c] / RSOOT) * powi5(TKD));
            rhsz[c] = dt * F(0.5) * ((RDHE / xxs[i + 1] - RDHW / xxs[i]) / xxc[i]
                                     + (RDHN / yys[j + 1] - RDHS / yys[j]) / yyc[j]
                                     + SYM * RDHP / yr[c] / yyc[j]) - QRAD * dt;
        }
    /* solveh.f:117-1145 */
    double RA[LRX], PRD[LSP], yc[LSP], rcc[LRX], so0[6] = {0, 0, 0, 0, 0, 0};
    for (int j = 1; j < lj - 1; ++j)
        for (int i = 1; i < li - 1; ++i) {
            const size_t c = CI(j, i);
            for (int k = 0; k < LSP; ++k) yc[k] = YS(k, c);
            for (int r = 0; r < LRX; ++r) rcc[r] = rc[(size_t)r * ne + c];
            for (int r = 0; r < LRX; ++r) {
                if (!T.ra_has[r]) { RA[r] = 0.0; continue; }
                double v = rcc[r];
                for (int t = 0; t < T.ra_len[r]; ++t) v = v * yc[T.ra_sp[T.ra_off[r] + t]];
                RA[r] = v;
            }
            double PROD = 0.0, HRR = 0.0;
            for (int k = 0; k < LSP; ++k) {
                PRD[k] = T.prd_has[k] ? S.WM[k] * S.HFO[k] * sum_terms(T.prd_off[k], T.prd_len[k], NULL, rcc, yc, NULL,
                                                                       so0, RA) : 0.0;
            }
            for (int k = 0; k < LSP; ++k) {
                PROD = PROD + PRD[k];
                HRR = HRR + PRD[k] * HENTH[(size_t)k * ne + c] / S.HFO[k];
                if (qdsp) qdsp[(size_t)k * ne + c] = -(RCONV * PRD[k] / S.HFO[k]);
            }
            rhsz[c] = rhsz[c] + rho[c] * ht[c] - dt * PROD;
            if (qdot) qdot[c] = -(HRR * RCONV);
        }
#undef CI
#undef RD
#undef YS
    free(RDHSP);
    free(HENTH);
}

/* Point relaxation of the enthalpy equation (solveh.f:1146-1167): up to isor
 * lexicographic Gauss-Seidel passes (J outer, I inner) over the interior
 * cells, over-relaxed by relx, until sum|dFPZ| / hnorm <= tol. fpz [lj*li]
 * holds HT on entry (boundary cells stay). Returns the pass count in the
 * reference's convention (the converging pass, or isor + 1). */
int orc_enthalpy_relax(int lj, int li, const double *rho, const double *rhsz, const double *ze, const double *zw,
                       const double *zn, const double *zs, double *fpz, int isor, double relx, double tol,
                       double hnorm)
{
    const double SOR1 = relx, SOR2 = F(1.0) - SOR1;
    int p;
    for (p = 1; p <= isor; ++p) {
        double RSDZ = F(0.0);
        for (int j = 1; j < lj - 1; ++j)
            for (int i = 1; i < li - 1; ++i) {
                const size_t c = (size_t)i * lj + j;
                const double PPP = rho[c] - (ze[c] + zw[c] + zn[c] + zs[c]);
                const double FNEW = SOR2 * fpz[c] + (rhsz[c] - zn[c] * fpz[c + 1] - zs[c] * fpz[c - 1]
                                                     - ze[c] * fpz[c + lj] - zw[c] * fpz[c - lj]) * SOR1 / PPP;
                RSDZ = RSDZ + fabs(fpz[c] - FNEW);
                fpz[c] = FNEW;
            }
        if (RSDZ / hnorm <= tol) return p;
    }
    return p;
}

/* Temperature of the interior cells from FPZ less the kinetic energy
 * (solveh.f:1170-1234): ENTH = (FPZ - (U^2 + V^2 + W^2)/2) HSTR + sum Y_k HFO_k HSTR.
 * y [52][lj*li]; w may be NULL (no swirl). tk holds the guess on entry. */
void orc_temperature_ke(int lj, int li, double *tk, const double *y, const double *fpz, const double *u,
                        const double *v, const double *w)
{
    const size_t ne = (size_t)lj * li;
    for (int i = 1; i < li - 1; ++i)
        for (int j = 1; j < lj - 1; ++j) {
            const size_t c = (size_t)i * lj + j;
            const double wc = w ? w[c] : 0.0;
            double ENTH = (fpz[c] - F(0.5) * (u[c] * u[c] + v[c] * v[c] + wc * wc)) * S.HSTR;
            for (int k = 0; k < LSP; ++k) ENTH = ENTH + y[(size_t)k * ne + c] * S.HFO[k] * S.HSTR;
            tk[c] = temperature_cell(tk[c], y + c, ne, ENTH);
        }
}

/* Density from the gas law at the back pressure (src/unicornd-mild-sd-5.f:1056-1068):
 * RHONP = PBACK / (BETA1 TK RBAR), RBAR = sum Y_k / W_k, on every cell of the
 * lj x li grid; the last column (I = LI) extrapolated linearly from the two
 * before it, then the first row (J = 1) copied from the second. y [52][lj*li]. */
void orc_density(int lj, int li, const double *tk, const double *y, double *rho)
{
    const size_t ne = (size_t)lj * li;
    for (size_t c = 0; c < ne; ++c) {
        double RBAR = F(0.0);
        for (int k = 0; k < LSP; ++k) RBAR = RBAR + y[(size_t)k * ne + c] / S.WM[k];
        rho[c] = S.PBACK / (S.BETA1 * tk[c] * RBAR);
    }
    for (size_t c = ne - lj; c < ne; ++c) rho[c] = F(2.0) * rho[c - lj] - rho[c - 2 * (size_t)lj];
    for (size_t c = 0; c < ne; c += lj) rho[c] = rho[c + 1];
}
