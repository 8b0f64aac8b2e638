/*
 * unichem: B200 (sm_100a) implementation of UNICORN's per-cell chemistry and
 * property hot path, behind a C ABI that a Fortran host binds with
 * ISO_C_BINDING.
 *
 * Data layout: the host's COMMON arrays as they are. A field of n cells is
 * passed as Fortran arrays over the (J,I) grid flattened column-major, i.e.
 * cell c = (I-1)*LJ + (J-1); species fields are FSP(LJ,LI,LSP), which is
 * [52][n] in C terms. All quantities are the reference's non-dimensional
 * ones (TK = T/TSTR, RHO = rho/RSTR, ...; the scales follow from uc_inputs).
 *
 * Fields stay resident on the device between calls: uc_upload_fields copies
 * host arrays in, the compute calls work on the device copies, and results
 * are copied out only when a host pointer is given. The library never keeps
 * a host pointer after a call returns.
 *
 * Every call returns 0 on success or a negative UC_E* code; uc_last_error()
 * gives the message. Calls on one context are not re-entrant; use one context
 * per host thread (each context owns one CUDA stream).
 */
#ifndef UNICHEM_H
#define UNICHEM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UC_LSP 52   /* species, src/unicornd-mild-sd-5.f:3 (LSP) */
#define UC_LRX 544  /* reaction slots, src/unicornd-mild-sd-5.f:3 (LRX) */

/* precision of uc_rates / uc_omega */
#define UC_FP64 0   /* all-FP64, the drop-in form */
#define UC_MIXED 1  /* FP32 exponentials, power laws and sums; FP64 Kc and update */

/* error codes */
#define UC_OK 0
#define UC_E_ARG -1        /* invalid argument (null pointer, size out of range) */
#define UC_E_CUDA -2       /* CUDA runtime error (message in uc_last_error) */
#define UC_E_STATE -3      /* call order: e.g. update before fields were uploaded */
#define UC_E_TIMEOUT -4    /* a device-side bounded wait gave up */
#define UC_E_NOCONV -5     /* a bounded iteration did not converge (reported, not fatal) */
/* The device kernels record UC_E_NOCONV (a cell's T Newton ran out of its 100
 * steps, as the reference reports and carries on from) in a status word that
 * the next call which synchronises the stream reads and clears: a call that
 * returns UC_E_NOCONV has completed its own work, the non-convergence may come
 * from an earlier asynchronous call (e.g. uc_temperature_from_held). */
#define UC_E_NOMEM -6      /* device allocation failed */

typedef struct uc_ctx uc_ctx;

/* Input-card values the reference reads from cfg/input.uni
 * (src/unicornd-mild-sd-5.f:154-155; sample values docs/input.uni:4-5). */
typedef struct {
    double rtin, rtot;   /* inner/outer radius [m]: ALSTR = RTOT - RTIN */
    double vref;         /* reference velocity [m/s] */
    double tref;         /* reference temperature [K] */
    double pref;         /* reference pressure [Pa] */
    double rref;         /* density card value (recomputed from the gas law, as the reference does) */
    double fo2in;        /* O2 mass fraction of the air stream */
} uc_inputs;

/* Reference scales after set-up (/CB06/ of the reference, main:421-459). */
typedef struct {
    double alstr, vstr, rstr, pstr, tstr, tmstr, amstr, acstr, dstr, hstr, cpstr, akstr, epstr,
           wmstr, gasc, beta1, beta2, beta3, beta4, rei, pback, hconv, convrc, convrm, convrd;
} uc_scales;

/* Set-up: replaces the reference's table preparation (main:327-483) and
 * allocates device storage for n cells on CUDA device `device`.
 * Replaces: the start-up section of PROGRAM UNICORN, src/unicornd-mild-sd-5.f:327-483. */
int uc_init(const uc_inputs *in, int ncell, int device, uc_ctx **out);

/* Scales and non-dimensional molar masses WM(52), formation enthalpies HFO(52). */
int uc_get_scales(const uc_ctx *ctx, uc_scales *sc, double *wm, double *hfo);

/* Copy fields to the device. tk[n], rho[n], fsp[52*n] required; stmf, stnd
 * (soot mass fraction and number density) may be NULL (= 0). The uploaded
 * mass fractions also become the "old time level" (FA.. of SOLVESP).
 * Replaces: the COMMON /CB04/ and /SOOT/ state read by CKRATES/SOLVESP. */
int uc_upload_fields(uc_ctx *ctx, const double *tk, const double *rho, const double *fsp,
                     const double *stmf, const double *stnd);

/* The same from arrays already in device memory (a host whose fields live on
 * the GPU: CUDA Fortran / OpenACC device arrays): tk, rho [ld], fsp [52][ld],
 * stmf, stnd [ld] or NULL, with row stride ld >= n elements. Asynchronous on
 * the context's stream (uc_device_view_get().stream): writes to the source
 * arrays made on other streams must be complete or ordered before the call,
 * and the sources must not change until the copies have run (uc_sync).
 * Replaces: the same COMMON state as uc_upload_fields. */
int uc_upload_fields_device(uc_ctx *ctx, const double *tk, const double *rho, const double *fsp,
                            const double *stmf, const double *stnd, int ld);

/* The reference's skip flags ISKIP(LJ,LI) [n] (src/lib/skipdf.f: 3 marks
 * injection cells, 10 and above body cells); NULL clears them. As the
 * reference does, cells with ISKIP >= 3 keep their RC and SOUR in the rate
 * calls (ckrates.f:94), keep Y and stay out of the residual and the N2
 * closure in the species update (solvesp.f:89,2842), and keep T in
 * uc_temperature_from_h (solveh.f:1173); cells with ISKIP >= 10 also keep
 * omega, QDOT and d(omega)/dY (solveh.f:119), while those below 10 take them
 * from the RC they kept. Planes never computed start at zero, like the
 * reference's COMMON blocks. The transport properties are computed for every
 * cell (the property block has no skip test); the batched integration, the
 * face assembly and the enthalpy equation do not read ISKIP.
 * Replaces: ISKIP of COMMON /CB01/ as CKRATES, SOLVESP and SOLVEH read it. */
int uc_set_iskip(uc_ctx *ctx, const int *iskip);

/* Copy the device-resident state back (any pointer may be NULL). */
int uc_download_fields(uc_ctx *ctx, double *tk, double *rho, double *fsp, double *stmf,
                       double *stnd);

/* Rate coefficients of all 544 slots, kept on the device for uc_species_update.
 * Replaces: CALL CKRATES, src/lib/spgsolv.f:1293 (src/lib/ckrates.f). If rc is
 * not NULL the RC plane RC(n,544) ([544][n]) is also copied to the host. */
int uc_rates(uc_ctx *ctx, int precision, double *rc);

/* Species source terms from the device-resident state: qdsp[52*n] is the
 * reference's QDSP (= -omega_k), qdot[n] its QDOT, domega_dy[52*n] the
 * diagonal linearisation d(omega_k)/dY_k = -RCONV*W_k*L_k (same units as
 * omega). NULL outputs stay on the device.
 * Replaces: the rate part of CALL SOLVEH, src/lib/solveh.f:116-1145. */
int uc_omega(uc_ctx *ctx, int precision, double *qdsp, double *qdot, double *domega_dy);

/* Y clip and N2 closure (applied to the device state, as main:821-828 does)
 * and mixture-averaged transport: vmu[n], vtc[n], vdf[52*n].
 * Replaces: the inline property block of PROGRAM UNICORN, src/unicornd-mild-sd-5.f:821-1006. */
int uc_props(uc_ctx *ctx, double *vmu, double *vtc, double *vdf);

/* Mixture cp (the reference's TCP, non-dimensional) and mixture enthalpy
 * h = sum_k Y_k h_k with h_k the reference's HENTH.
 * Replaces: src/lib/spgsolv.f:102-173 (TCP) and src/lib/solveh.f:39-57 (HENTH). */
int uc_cp_h(uc_ctx *ctx, double *cp, double *h);

/* Point-implicit species update of species 1..51 and the two soot scalars,
 * up to isor passes until sum|dY|/spnorm <= tol (spnorm <= 0 means
 * 51*n), then the N2 closure. Uses the RC plane of the last uc_rates call.
 * face_sum[51*n] (E+W+N+S) and face_nbr[51*n] (sum of coefficient times the
 * neighbour value) are the frozen transport terms; NULL means none. passes
 * receives the count the reference reports in ISOR1.
 * Replaces: CALL SOLVESP(ISOR1,RELXSP,TOLRSP,SPNORM), src/lib/spgsolv.f:1295. */
int uc_species_update(uc_ctx *ctx, double dt, int isor, double relx, double tol, double spnorm,
                      const double *face_sum, const double *face_nbr, int *passes);

/* Temperature from the non-dimensional sensible enthalpy ht[n] (FPZ) by
 * Newton's method; updates the device temperature (initial guess = current).
 * Replaces: src/lib/solveh.f:1170-1234. */
int uc_temperature_from_h(uc_ctx *ctx, const double *ht);

/* One species sweep on the device-resident state, in the order of the
 * reference's time step: Y clip + transport properties (main:821-1006), cp
 * and h, rate coefficients with omega and d(omega)/dY at the start-of-step
 * state (CKRATES + SOLVEH rates), then the point-implicit update (SOLVESP)
 * with the arguments of uc_species_update. Outputs stay on the device
 * (uc_device_view_get / the download calls). With UC_MIXED the per-pair
 * terms of the transport sums (square roots, divisions, products) also run in
 * FP32; the polynomials in T, the sums over species, cp and h, the state's
 * clip and closure, Kc and the update stay FP64.
 * Replaces: CALL SPGSOLV's chemistry part (src/lib/spgsolv.f:102-176,1291-1298)
 * preceded by the property block of main:821-1006. */
int uc_sweep(uc_ctx *ctx, int precision, double dt, int isor, double relx, double tol, double spnorm,
             const double *face_sum, const double *face_nbr, int *passes);

/* Host buffers of one uc_sweep_host call (each [n] or [52][n] like the
 * upload and download calls; any output may be NULL = not copied; stmf/stnd
 * in may be NULL = zero). */
typedef struct {
    const double *tk, *rho, *fsp, *stmf, *stnd;             /* state in */
    double *qdsp, *qdot, *domega_dy, *vmu, *vtc, *vdf, *cp, *h;   /* outputs of the sweep's first steps */
    double *fsp_out, *stmf_out, *stnd_out;                  /* state after the update */
} uc_host_io;

/* One species sweep on host buffers: uc_upload_fields(tk, rho, fsp, stmf,
 * stnd), uc_sweep(...), uc_download_outputs(...) and the updated Y and soot,
 * with the same results as those calls in that order. The outputs of the
 * properties, cp/h and the rates are final before the species update starts,
 * so they are copied to the host on a second stream while the update runs;
 * only the updated state is copied after it. The host buffers may be pinned
 * (copies asynchronous) or pageable. Returns when every copy has landed. */
int uc_sweep_host(uc_ctx *ctx, int precision, double dt, int isor, double relx, double tol, double spnorm,
                  const double *face_sum, const double *face_nbr, const uc_host_io *io, int *passes);

/* The chemistry and properties of the device-resident state without the
 * update: the Y clip with transport properties, cp and h, then omega and
 * d(omega)/dY (the first three steps of uc_sweep, in its order; no RC plane is
 * kept). Asynchronous; read the outputs with uc_download_outputs.
 * Replaces: the property block of main:821-1006, the TCP loop of
 * spgsolv.f:102-173 and the rate part of SOLVEH (solveh.f:116-1145). */
int uc_chem_props(uc_ctx *ctx, int precision);

/* ---------------------------------------------------------------------------
 * The species equations' face coefficients on the device.
 * Replaces: the coefficient assembly of SPGSOLV, src/lib/spgsolv.f:233-1290
 * (face conductances from EMU, VDFSP and the eddy viscosity; hybrid
 * convection-diffusion coefficients E, W, N, S with the axisymmetric terms).
 * The context's n cells must be the whole lj x li grid (J fastest), boundary
 * cells included. Geometry: XXS, XXC [li], YYS, YYC [lj], the radial
 * coordinate Y(J,I) [n], ISYM. Flow: U, V, TMU [n] and SIGSP.
 * Once a grid and a flow are set, uc_sweep assembles the faces after the
 * properties (with its dt) and the update uses them whenever no face arrays
 * are passed: face_sum = E+W+N+S, face_nbr = N Y(J+1) + S Y(J-1) + E Y(I+1)
 * + W Y(I-1) with the neighbours' Y at the start of the update (Jacobi over
 * cells; the reference's lexicographic Gauss-Seidel has no parallel form),
 * and the grid's boundary cells keep their state, as SOLVESP updates only
 * J = 2..LJ-1, I = 2..LI-1. Every interior cell is assembled (no ISKIP).
 * uc_set_grid(ctx, NULL) returns to the face-less update.
 */
typedef struct {
    int lj, li, isym;
    const double *xxs, *xxc, *yys, *yyc, *yr;
} uc_grid;
int uc_set_grid(uc_ctx *ctx, const uc_grid *g);
int uc_set_flow(uc_ctx *ctx, const double *u, const double *v, const double *tmu, double sigsp);
/* Assemble now (needs uc_props of the current state); e, w, n, s [51*n] host copies (may be NULL). */
int uc_assemble_faces(uc_ctx *ctx, double dt, double *e, double *w, double *n, double *s);

/* ---------------------------------------------------------------------------
 * The enthalpy equation on the device.
 * Replaces: CALL SOLVEH(ISOR2,RELXH,TOLRH,SIGSP,HNORM) at src/lib/spgsolv.f:1298
 * (src/lib/solveh.f:34-1234) with the enthalpy coefficients of SPGSOLV
 * (EKT spgsolv.f:174; ZE, ZW, ZN, ZS of spgsolv.f:240-1290) and the
 * HT := FPZ copy and residual RESDH of spgsolv.f:1299-1415.
 *
 * uc_set_enthalpy uploads HT [n] (the reference's non-dimensional FPZ/HT) and
 * the swirl velocity W [n] of the kinetic-energy term (NULL: none).
 * uc_enthalpy_update runs, after a uc_sweep (whose species update leaves the
 * rate plane of its start state, the properties and cp on the device) and on
 * the grid and flow of uc_set_grid / uc_set_flow (SIGSP of the flow is the
 * SIGSP of RDHSP):
 *  - QDSP and QDOT from the start-state rates and the updated Y, overwriting
 *    the context's omega as SOLVEH overwrites /DUMD/ and /HRLS/ (interior cells);
 *  - RHSZ: species-enthalpy diffusion, radiation of CH4, CO2, CO, H2O and soot
 *    (40%, with the soot mass fraction of the start of the update), RHO HT and
 *    DT PROD; coefficients from EKT = REI (BETA2 VTC/TCP + TMU/SIGH);
 *  - up to isor relaxation passes over the interior cells in the reference's
 *    lexicographic Gauss-Seidel order (J outer, I inner: the same iterates),
 *    until sum|dFPZ| / hnorm <= tol (hnorm <= 0 means lj*li, the reference's LE);
 *  - T of the interior cells from FPZ less (U^2+V^2+W^2)/2 by the Newton of
 *    solveh.f:1170-1234, then HT := FPZ.
 * passes receives ISOR2 as the reference returns it (the converging pass, or
 * isor + 1); resdh = sum|FPZ - HT| / hnorm. At most 1024 interior rows (lj - 2).
 * Returns UC_E_NOCONV (not fatal) when a cell's Newton did not converge and
 * UC_E_TIMEOUT when a bounded wait between passes gave up (T and HT are then
 * left unchanged); the waits give up after the number of nanoseconds in the
 * environment variable UNICHEM_RELAX_WAIT_NS, read at each call (2 s when unset). */
typedef struct {
    double dt;      /* DT */
    int isor;       /* ISOR2: passes at most */
    double relx;    /* RELXH */
    double tol;     /* TOLRH */
    double hnorm;   /* HNORM (<= 0: lj*li) */
    double sigh;    /* SIGH of EKT */
} uc_enthalpy_opts;
int uc_set_enthalpy(uc_ctx *ctx, const double *ht, const double *w);
int uc_enthalpy_update(uc_ctx *ctx, const uc_enthalpy_opts *o, int *passes, double *resdh);
/* HT [n] and the last update's RHSZ, ZE, ZW, ZN, ZS [n] to the host (NULL = skip). */
int uc_enthalpy_get(uc_ctx *ctx, double *ht, double *rhsz, double *ze, double *zw, double *zn, double *zs);

/* Density of every cell from the gas law at the back pressure PBACK,
 * RHO = PBACK / (BETA1 TK sum Y_k/W_k), with the reference's edge rules (last
 * column extrapolated linearly, first row copied from the second); needs the
 * grid of uc_set_grid. The reference stores this as RHONP and makes it RHO in
 * steady runs (ISTDY = 1).
 * Replaces: src/unicornd-mild-sd-5.f:1056-1073. */
int uc_density(uc_ctx *ctx);

/* The relaxation alone, on host arrays of an lj x li grid (J fastest):
 * fpz [lj*li] holds HT on entry and FPZ on return; rho, rhsz and the
 * coefficients ze, zw, zn, zs are read on the interior cells. Same ordering,
 * rounding and pass count as the loop of solveh.f:1146-1167.
 * Replaces: src/lib/solveh.f:1146-1167. */
int uc_enthalpy_relax(int device, int lj, int li, const double *rho, const double *rhsz, const double *ze,
                      const double *zw, const double *zn, const double *zs, double *fpz, int isor, double relx,
                      double tol, double hnorm, int *passes);

/* FDETAIL fields of the current state on the cell corners of the lj x li grid
 * (the context's cells): out [218][n] in the order of the reference's record
 * z, r, RHO, v, u, T, QDOT, VMU, VTC, CP, then Y_k, D_k, QDSP_k, h_k per species,
 * dimensional as the reference writes them. x, y: node coordinates [n]; u, v [n].
 * Needs omega and the properties of the state (after uc_sweep).
 * Replaces: the field computation of SUBROUTINE STDATA, src/lib/stdata.f:26-118
 * (the host writes the file; unicorn_b200/fdetail.py writes the reference's layout). */
int uc_fdetail(uc_ctx *ctx, int lj, int li, const double *x, const double *y, const double *u,
               const double *v, double *out);

/* Outputs of the last uc_sweep/uc_omega/uc_props/uc_cp_h to the host (NULL = skip). */
int uc_download_outputs(uc_ctx *ctx, double *qdsp, double *qdot, double *domega_dy, double *vmu,
                        double *vtc, double *vdf, double *cp, double *h);

/* Kernel timing with CUDA events on the context's stream (tracing).
 * uc_profile(ctx, 1) starts recording every launch; uc_profile_read
 * synchronises and returns, per kernel kind (UC_K_*), the summed device time
 * in ms and the launch count since the last read. */
#define UC_K_CHEM 0
#define UC_K_UPDATE 1
#define UC_K_PROPS 2
#define UC_K_CPH 3
#define UC_K_TEMP 4
#define UC_K_INTEGRATE 5   /* one uc_integrate graph launch */
#define UC_K_ENTHALPY 6    /* one uc_enthalpy_update (all its kernels) */
#define UC_K_COUNT 7
int uc_profile(uc_ctx *ctx, int on);
int uc_profile_read(uc_ctx *ctx, double *ms, int *launches);

/* Counters of the last calls (synchronises the stream):
 *   "tiles"               32-cell tiles of the context
 *   "mixed_fp64_tiles"    tiles the last UC_MIXED rate call sent to FP64 because a
 *                         rate left the FP32 range
 *   "update_kind"         species update kernel: 0 tile-resident (default; RC on chip
 *                         across chunks of passes), 1 per pass with Y in place
 *                         (UNICHEM_UPDATE=inplace), 2 per pass with two Y sets
 *                         (UNICHEM_UPDATE=twoset), chosen at uc_init
 *   "update_chunk"        passes per chunk of the tile-resident update (UNICHEM_TR_CHUNK, 16)
 *   "update_lockstep"     1 if its warps run species by species in step (UNICHEM_TR_LOCKSTEP)
 *   "update_flops_per_cell_pass"  floating-point operations of one cell and pass of the
 *                         update (each multiplication, addition and division one)
 *   "update_ip_warps"     warps per CTA of the species update with Y in place
 *                         (14); 0 when UNICHEM_UPDATE=twoset was set at uc_init and
 *                         the two-Y-set kernel (8 warps) runs instead
 * Returns UC_E_ARG for an unknown name. */
int uc_stat(uc_ctx *ctx, const char *name, double *value);

/* Synchronise the context's stream. */
int uc_sync(uc_ctx *ctx);

/* Message of the last error on this context (static storage, valid until the next call). */
const char *uc_last_error(const uc_ctx *ctx);

/* Release all device memory of the context. */
void uc_destroy(uc_ctx *ctx);

/* Device pointers of the resident state, for callers that keep their own
 * device data (all [k][n] SoA, FP64). */
typedef struct {
    double *tk, *rho, *fsp, *fsp_old, *stmf, *stnd, *rc, *qdsp, *qdot, *domega_dy, *vmu, *vtc,
           *vdf, *cp, *h;
    int n, npad;
    void *stream;   /* cudaStream_t */
} uc_device_view;
int uc_device_view_get(uc_ctx *ctx, uc_device_view *v);

/* ---------------------------------------------------------------------------
 * Batched stiff integration of independent cells.
 *
 * No single reference routine corresponds: every cell of the context is a
 * one-cell field advanced over o->dt by n_sub sub-steps of dt/n_sub, each
 * the reference's own chain - CKRATES (src/lib/ckrates.f), SOLVESP with its
 * closure (src/lib/solvesp.f, SPNORM = LSP-1 so that each cell converges on
 * its own residual, no face terms), T from the cell's constant total
 * enthalpy (src/lib/solveh.f:1186-1234) and rho from the ideal gas at the
 * cell's pressure (src/unicornd-mild-sd-5.f:1056-1062). The state (TK, RHO,
 * FSP, STMF, STND) is advanced in place; read it with uc_download_fields.
 *
 * n_sub = clamp(ceil(x / c_tau), 1, nsub_max), x = max over species with
 * Y_k > y_tau of dt*|QDSP_k| / (RCONV*rho*Y_k), QDSP of the start state.
 * The whole step (rates of the start state, n_sub, a stable sort of the
 * cells by n_sub, then the sub-steps) is one CUDA graph launch; the graph is
 * captured on the first call and again when an option or the tuned kernel
 * shape changes. Two shapes run the sub-steps: the persistent work-queue
 * kernel (each CTA advances one 32-cell tile through all its sub-steps) and,
 * for UC_FP64, the rounds form (the cells gathered in n_sub order; round r
 * advances the cells with n_sub > r by one sub-step with the field kernels:
 * rates, a per-cell form of the tile-resident species update, T and rho;
 * between rounds the cells that go on are re-ordered by the passes of their
 * last sub-step). The rounds form holds two copies of the state in its own
 * order on the device (116 doubles and 10 ints per cell) and uses the
 * context's RC plane.
 *
 * precision: UC_FP64 (everything FP64) or UC_MIXED (the rates of every
 * sub-step and of the start state in the mixed form of uc_rates, stored as
 * doubles; a tile with a rate beyond the FP32 range is recomputed in FP64; the
 * update, closure, T and rho stay FP64); other values return UC_E_ARG.
 */
typedef struct {
    double dt;          /* non-dimensional step (DT = 1e-3 is 1e-5 s) */
    int isor;           /* update passes per sub-step, at most */
    double relx, tol;   /* relaxation (RELXSP) and per-cell tolerance */
    double c_tau;       /* time-scale factor of the sub-step count */
    double y_tau;       /* species above this mass fraction set the time scale */
    int nsub_max;       /* 1..1024 */
} uc_integrate_opts;
/* Cell pressures p/PSTR [n] (host); cells default to PBACK. */
int uc_set_pressure(uc_ctx *ctx, const double *pnd);
/* Record each cell's total enthalpy h(T, Y) (the polynomial of solveh.f:1186-1205 at the
 * cell's T); uc_temperature_from_held then re-solves T from it for the current Y
 * (the Newton of src/lib/solveh.f:1170-1234) and sets rho from the ideal gas at the
 * cell's pressure (src/unicornd-mild-sd-5.f:1056-1062): the in-loop T update of a
 * sweep with enthalpy transport frozen. */
int uc_hold_enthalpy(uc_ctx *ctx);
int uc_temperature_from_held(uc_ctx *ctx);
int uc_integrate(uc_ctx *ctx, int precision, const uc_integrate_opts *o);
/* Times each kernel shape on the current state (restored after each trial)
 * and keeps the fastest for uc_integrate; uc_stat "int_warps" (16 or 8: the
 * persistent kernel with that many warps per CTA; 3: the rounds form),
 * "int_sorted", "int_tune_best_ms", "int_tune_worst_ms" report the outcome. */
int uc_integrate_tune(uc_ctx *ctx, int precision, const uc_integrate_opts *o);
/* Per-cell sub-step counts and update passes of the last uc_integrate (host [n], either may be NULL). */
int uc_integrate_counts(uc_ctx *ctx, int *nsub, int *passes);

/* ---------------------------------------------------------------------------
 * The BF16 tensor-core GEMMs of the surrogate network, on host buffers (no
 * reference counterpart; the surrogate is not part of the reference):
 * c[M][N] (FP32) = a[M][K] * b[N][K]^T with a, b BF16 bit patterns, row-major.
 * kernel 0: the tiled GEMM (N a multiple of 16, K of 64); kernel 1: the
 * layer kernel with b resident in shared memory (N and K multiples of 64 up
 * to 256). Allocates and frees its own device buffers; meant for checking the
 * kernels, not for speed. */
int uc_gemm_bf16(int device, int kernel, int M, int N, int K, const uint16_t *a, const uint16_t *b, float *c);

/* ---------------------------------------------------------------------------
 * Learned surrogate of omega (no reference counterpart: the reference always
 * evaluates the mechanism). A 54 -> 256 x 4 (GELU) -> 52 network with BF16
 * weights and FP32 accumulation; inputs T, ln p and ln max(Y_k, 1e-12) scaled
 * by uc_mlp_set_norm, outputs asinh(QDSP_k / s_k) scaled likewise. Trained
 * with Adam on states whose targets the exact FP64 kernel computes, run with
 * a per-cell fallback to that kernel (uc_mlp_omega). All matrix products run
 * on the tensor cores (uc_gemm_bf16's kernel).
 */
typedef struct uc_mlp uc_mlp;
/* capacity: rows of the training set kept on the device (64 features + 64 targets each). */
int uc_mlp_create(int device, unsigned long long seed, long capacity, uc_mlp **out);
int uc_mlp_nparams(const uc_mlp *mlp);
/* Flat FP32 parameters, per layer W[out][in] then b[out] (layers 64->256, 3 x 256->256,
 * 256->64; padded rows/columns are zero): get (if not NULL), then set (if not NULL). */
int uc_mlp_params(uc_mlp *mlp, float *get, const float *set);
/* Feature means, scales and training hull [54]; target means, scales and s_k [52]. */
int uc_mlp_set_norm(uc_mlp *mlp, const float *feat_mu, const float *feat_sd, const float *hull_lo,
                    const float *hull_hi, const float *tgt_mu, const float *tgt_sd, const float *tgt_scale);
/* Append the context's cells (fields and uc_set_pressure pressures) with their exact omega. */
int uc_mlp_add_data(uc_mlp *mlp, uc_ctx *ctx);
/* Adam (beta 0.9/0.999, eps 1e-8) over `steps` batches, the learning rate decaying from lr to lr/100
 * along a half cosine over the call; loss[steps] (may be NULL). batch % 64 == 0. */
int uc_mlp_train(uc_mlp *mlp, int steps, int batch, float lr, unsigned long long seed, float *loss);
/* One forward+backward pass on given rows (M % 64 == 0): x [M][64] BF16 bits, t [M][64];
 * grad [nparams] and loss receive the mean-squared-error gradient and value. */
int uc_mlp_grad(uc_mlp *mlp, int M, const uint16_t *x, const float *t, float *grad, float *loss);
/* Omega of the context's state (its QDSP, as uc_omega leaves it) from the surrogate with
 * per-cell fallback to the exact FP64 kernel. A cell is recomputed exactly when it lies
 * outside the training hull, or when the surrogate's omega breaks element conservation
 * (max over C, H, O of |sum_k a_ek omega_k/W_k| / sum_k |a_ek omega_k/W_k|, which is 1e-16
 * for the exact omega) by more than tol; every 32nd cell is recomputed as well, as a
 * sample of the surrogate's true error. The flagged cells are gathered into a compact
 * field, the exact kernel runs on it and the results go back to their cells. QDOT is
 * written for the recomputed cells only. stats[3] (may be NULL; giving it synchronises):
 * fraction of cells recomputed, fraction outside the training hull, median error of the
 * surrogate on the sampled cells (max over species with Y_k > 1e-8 of the error relative to
 * max(|omega_k|, 1e-6 max_j |omega_j|)). tol = +infinity gives the network's output alone
 * (no checks, no fallback). */
int uc_mlp_omega(uc_mlp *mlp, uc_ctx *ctx, double tol, double *stats);
/* Statistics of the last uc_mlp_omega that was given stats: "cells_exact",
 * "cells_outside_hull", "sample_error_p50", "sample_accepted" (fraction of the sampled
 * cells the checks accepted), "sample_accepted_within_tol" (of those, the fraction whose
 * true error is at most tol: the estimate for the accepted cells of the field),
 * "sample_accepted_error_p50", "sample_accepted_error_p99". UC_E_ARG for another name. */
int uc_mlp_stat(const uc_mlp *mlp, const char *name, double *value);
const char *uc_mlp_last_error(const uc_mlp *mlp);
void uc_mlp_destroy(uc_mlp *mlp);

/* ---------------------------------------------------------------------------
 * Species update on caller-owned device arrays, with no device allocation.
 *
 * This entry point has no counterpart in the reference; it exists for callers
 * that cannot let a library call cudaMalloc: hosts whose device memory all
 * comes from their own allocator or pool (a Fortran code with CUDA Fortran or
 * OpenACC device arrays, a solver held to a fixed memory budget), or code on
 * a path where allocation is not allowed. It runs the same point-implicit
 * update as uc_species_update, but every array is the caller's and the only
 * scratch (the per-block residual partial sums and the pass counter) is a
 * fixed array inside the library: UC_NOALLOC_MAX_BLOCKS doubles x 2 plus one
 * int (16 KiB + 4 B per GPU that loads the library, held until process exit).
 *
 *  - ctx supplies the mechanism tables, scales and the CUDA stream; it must
 *    come from uc_init (which is where allocation happens, once, at set-up).
 *  - a->n cells with row stride a->npad (npad >= n, a multiple of 32);
 *    rc [544][npad] as written by uc_rates, sour [6][npad], rho [npad],
 *    y0 [52][npad] and soot0 [2][npad] the old time level, y [52][npad] and
 *    soot [2][npad] updated in place, face_sum/face_nbr [51][npad] or NULL.
 *    Padding cells (n..npad-1) are read and must hold finite values.
 *  - Returns UC_E_ARG if npad is not a multiple of 32 or below n, or if the
 *    device would need more than UC_NOALLOC_MAX_BLOCKS cooperating blocks.
 *  - The first call on a device looks up the scratch array's device address
 *    (cudaGetSymbolAddress, with that device current); make that first call
 *    before any stream capture.
 *  - All calls share the one scratch array and it keeps the last call's
 *    contents; nothing in it has to start at zero (every partial sum is written
 *    before it is read). Calls that overlap on the GPU, from any context or
 *    stream, race on it: serialise them.
 *  - The update runs on the context's stream (uc_device_view_get().stream),
 *    which is created non-blocking: writes to the input arrays made on other
 *    streams must be complete, or ordered before the call (an event the
 *    caller records and makes that stream wait on), when the call is made.
 *  - passes (host pointer, may be NULL) receives the pass count; giving it
 *    makes the call wait for the update to finish. With passes == NULL the
 *    call returns once the update is queued: synchronise (uc_sync, or a wait
 *    on the context's stream) before reading y or soot.
 *  - It runs the two-Y-set form of the update kernel (8 warps per block, the
 *    kernel UNICHEM_UPDATE=twoset selects for uc_species_update), whose only
 *    scratch is the per-block partial sums; the tile-resident kernel that
 *    uc_species_update runs by default would need Y snapshots and tensor maps
 *    of the caller's RC array. Same pass count as uc_species_update, Y within
 *    1e-12 relative (bit for bit against UNICHEM_UPDATE=twoset).
 */
#define UC_NOALLOC_MAX_BLOCKS 1024
typedef struct {
    int n, npad;
    const double *rc, *sour, *rho, *y0, *soot0, *face_sum, *face_nbr;
    double *y, *soot;
} uc_update_arrays;
int uc_species_update_noalloc(uc_ctx *ctx, const uc_update_arrays *a, double dt, int isor, double relx,
                              double tol, double spnorm, int *passes);

#ifdef __cplusplus
}
#endif
#endif
