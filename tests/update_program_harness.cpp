// Test-only harness: runs the generated species-update program
// (unicorn_b200/csrc/generated/update_program.cuh) on the host, so that the
// symbolic resolution of the reference's A-terms can be checked against the
// oracle without a GPU. Not part of the product.
#include <cmath>
#include <cstring>
#define LSP 52
#define LRX 544

extern "C" int harness_update(int n, const double *rho_a, const double *y0_a, double *y_a,
                              const double *rc_a, const double *sour_a, const double *wm,
                              double dt, int isor, double relx, double tol, double spnorm)
{
    const double sor1 = relx, sor2 = 1.0 - relx;
    double yo[LSP], yn[LSP], y0[LSP], sour[6];
    int pass;
    for (pass = 1; pass <= isor; ++pass) {
        double rsd = 0.0;
        for (int c = 0; c < n; ++c) {
            for (int k = 0; k < LSP; ++k) { yo[k] = y_a[k * n + c]; y0[k] = y0_a[k * n + c]; yn[k] = 0.0; }
            for (int m = 0; m < 6; ++m) sour[m] = sour_a[m * n + c];
            const double rho = rho_a[c];
#define RC(r) rc_a[(r) * n + c]
#define RC_LAST(r) rc_a[(r) * n + c]
#define YO(k) yo[k]
#define YN(k) yn[k]
#define Y0(k) y0[k]
#define SOUR(m) sour[m]
#define WM(k) wm[k]
#define FACE_SUM(k) 0.0
#define FACE_NBR(k) 0.0
#define UC_UPDATE_SYNC() do { } while (0)
#define UC_UPDATE_BLOCK_BEGIN(b) do { } while (0)
#define UC_UPDATE_TAIL(k) do { if (fnew < 0.0) fnew = 0.0; yn[k] = fnew; } while (0)
#include "../unicorn_b200/csrc/generated/update_program.cuh"
            UC_UPDATE_PROGRAM();
            for (int k = 0; k < LSP - 1; ++k) y_a[k * n + c] = yn[k];
        }
        if (rsd / spnorm <= tol) break;
    }
    return pass;
}

// The in-place form (UC_UPDATE_PROGRAM_IP): one Y array per cell, overwritten
// species by species; the species read at their start-of-pass value after
// their own update come from the cell's row in y_a, which still holds the
// start-of-pass values while the program runs (as on the device).
extern "C" int harness_update_ip(int n, const double *rho_a, const double *y0_a, double *y_a,
                                 const double *rc_a, const double *sour_a, const double *wm,
                                 double dt, int isor, double relx, double tol, double spnorm)
{
    const double sor1 = relx, sor2 = 1.0 - relx;
    static const int shadow[UC_IP_NSHADOW] = UC_IP_SHADOW_LIST;
    double y[LSP], y0[LSP], sour[6];
    int pass;
    for (pass = 1; pass <= isor; ++pass) {
        double rsd = 0.0;
        for (int c = 0; c < n; ++c) {
            for (int k = 0; k < LSP; ++k) { y[k] = y_a[k * n + c]; y0[k] = y0_a[k * n + c]; }
            for (int m = 0; m < 6; ++m) sour[m] = sour_a[m * n + c];
            const double rho = rho_a[c];
#undef YO
#undef YN
#undef UC_UPDATE_TAIL
#define YO(k) y[k]
#define YN(k) y[k]
#define YOS(m) y_a[shadow[m] * n + c]
#define UC_UPDATE_TAIL(k) do { if (fnew < 0.0) fnew = 0.0; y[k] = fnew; } while (0)
            UC_UPDATE_PROGRAM_IP();
            for (int k = 0; k < LSP - 1; ++k) y_a[k * n + c] = y[k];
        }
        if (rsd / spnorm <= tol) break;
    }
    return pass;
}

// The tile-resident form (UC_UPDATE_PROGRAM_TR): the in-place program with its
// RC operands split between "shared-memory rows" and "tensor-memory rows"
// loaded into two register banks segment by segment; here both stores are
// host arrays holding the cell's RC values in the program's row order.
#include "../unicorn_b200/csrc/generated/update_program_tr.cuh"
extern "C" int harness_update_tr(int n, const double *rho_a, const double *y0_a, double *y_a,
                                 const double *rc_a, const double *sour_a, const double *wm,
                                 double dt, int isor, double relx, double tol, double spnorm)
{
    const double sor1 = relx, sor2 = 1.0 - relx;
    double y[LSP], y0[LSP], sour[6], ysh[UC_IP_NSHADOW], srows[UC_TR_NS], trows[UC_TR_NT], bank[2][UC_TR_SEG];
    double y0s[2], fss[2], fns[2];
    int pass;
    for (pass = 1; pass <= isor; ++pass) {
        double rsd = 0.0;
        for (int c = 0; c < n; ++c) {
            for (int k = 0; k < LSP; ++k) { y[k] = y_a[k * n + c]; y0[k] = y0_a[k * n + c]; }
            for (int m = 0; m < 6; ++m) sour[m] = sour_a[m * n + c];
            for (int i = 0; i < UC_TR_NS; ++i) srows[i] = rc_a[uc_tr_srow[i] * n + c];
            for (int i = 0; i < UC_TR_NT; ++i) trows[i] = rc_a[uc_tr_trow[i] * n + c];
            const double rho = rho_a[c];
#undef YOS
#define YOS(m) ysh[m]
#define RCS(i) srows[i]
#define TM_LD(b, q, col) bank[b][q] = trows[(col) / 2]
#define TM_WAIT(b) do { } while (0)
#define RCT(b, q) bank[b][q]
#define UC_TR_PF(s, k) do { y0s[s] = y0[k]; fss[s] = 0.0; fns[s] = 0.0; } while (0)
#define Y0S(s) y0s[s]
#define FSS(s) fss[s]
#define FNS(s) fns[s]
#define UC_TR_SYNC() do { } while (0)
            UC_TR_SHADOW_SAVE();
            UC_UPDATE_PROGRAM_TR();
            for (int k = 0; k < LSP - 1; ++k) y_a[k * n + c] = y[k];
        }
        if (rsd / spnorm <= tol) break;
    }
    return pass;
}
