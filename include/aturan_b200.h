/*
 * aturan_b200 — B200 (sm_100a) kernels for ATURAN's dynamical-core time step, behind a C ABI.
 *
 * The reference has no plugin or FFI layer for this path: its call sites are member and friend
 * calls on one cUranusModel object. Each entry point below replaces one of those calls and says
 * which. A maintainer binds them from the reference's driver (planet/cUranusModel.cpp:Run) with a
 * compile-time switch around those calls, or from Python with ctypes (aturan_b200/api.py).
 *
 * Conventions
 *   - Every function returns an int status: 0 = ATURAN_OK, negative = error (nothing was
 *     changed on the device unless the function says otherwise), positive = completed but not
 *     converged. aturan_last_error() returns a message for the last error on a context.
 *   - Fields are exchanged as contiguous FP64 blocks in the reference's logical order x[i][j][k]
 *     (i = radius 0..im-1, j = colatitude 0..jm-1, k = longitude 0..km-1, k fastest), i.e. the
 *     jagged Array of lib/Array.cpp:58-67 flattened. On the device each row is padded to a
 *     pitch of 32 elements; the padding never crosses this interface.
 *   - State stays resident on the device between calls. A context owns one CUDA stream; calls on
 *     one context are not thread-safe, separate contexts may be used from separate threads.
 *   - There is no CPU fallback: without a usable CUDA device every call returns ATURAN_E_CUDA.
 */
#ifndef ATURAN_B200_H
#define ATURAN_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ATURAN_ABI_VERSION 1

enum aturan_status {
    ATURAN_OK              =  0,
    ATURAN_NOT_CONVERGED   =  1,   /* iterative solve stopped at its cap above tolerance */
    ATURAN_E_INVALID       = -1,   /* bad argument: null pointer, size, id, version */
    ATURAN_E_UNSUPPORTED   = -2,   /* a parameter value this build does not implement */
    ATURAN_E_CUDA          = -3,   /* CUDA runtime error (message in aturan_last_error) */
    ATURAN_E_NOMEM         = -4,   /* device allocation failed */
    ATURAN_E_NONFINITE     = -5    /* a NaN/Inf was found where the path forbids it */
};

enum aturan_precision {
    ATURAN_FP64  = 0,   /* state, stencils and solves in FP64: the parity path */
    ATURAN_MIXED = 1    /* FP32 state and stencils; FP64 Poisson refinement and SatAdj Newton */
};

/* Field ids. The first 19 are the prognostic fields in the order RHS_Uran_Turb.cpp assembles
 * them; the next 19 their start-of-step copies (tn, un, ...; cUranusModel.h:1377-1393). */
enum aturan_field {
    ATURAN_T = 0, ATURAN_U, ATURAN_V, ATURAN_W,
    ATURAN_CH4, ATURAN_CH4_CLOUD, ATURAN_CH4_ICE,
    ATURAN_H2O, ATURAN_H2O_CLOUD, ATURAN_H2O_ICE,
    ATURAN_H2S, ATURAN_H2S_CLOUD, ATURAN_H2S_ICE,
    ATURAN_NH3, ATURAN_NH3_CLOUD, ATURAN_NH3_ICE,
    ATURAN_NH4SH, ATURAN_TKE, ATURAN_DIS,                       /* 0..18 */
    ATURAN_TN, ATURAN_UN, ATURAN_VN, ATURAN_WN,
    ATURAN_CH4N, ATURAN_CH4_CLOUDN, ATURAN_CH4_ICEN,
    ATURAN_H2ON, ATURAN_H2O_CLOUDN, ATURAN_H2O_ICEN,
    ATURAN_H2SN, ATURAN_H2S_CLOUDN, ATURAN_H2S_ICEN,
    ATURAN_NH3N, ATURAN_NH3_CLOUDN, ATURAN_NH3_ICEN,
    ATURAN_NH4SHN, ATURAN_TKEN, ATURAN_DISN,                    /* 19..37 */
    ATURAN_P_DYN, ATURAN_P_HYDRO, ATURAN_P_STAT,                /* 38..40 */
    /* pointwise inputs of the RHS, held fixed through a step */
    ATURAN_NUE, ATURAN_THERMALMASSFLUX, ATURAN_Q_PRECIP,
    ATURAN_S_PRECIP_CH4, ATURAN_S_PRECIP_CH4_CLOUD, ATURAN_S_PRECIP_CH4_ICE,
    ATURAN_S_PRECIP_H2O, ATURAN_S_PRECIP_H2O_CLOUD, ATURAN_S_PRECIP_H2O_ICE,
    ATURAN_S_PRECIP_H2S, ATURAN_S_PRECIP_H2S_CLOUD, ATURAN_S_PRECIP_H2S_ICE,
    ATURAN_S_PRECIP_NH3, ATURAN_S_PRECIP_NH3_CLOUD, ATURAN_S_PRECIP_NH3_ICE,
    ATURAN_MASSFLUX_H2S, ATURAN_MASSFLUX_NH3, ATURAN_MASSFLUX_NH4SH, ATURAN_FLUXLIM_NH4SH,
    ATURAN_RHO_MIX, ATURAN_TKE_SOURCE, ATURAN_DIS_SOURCE,       /* 41..62 */
    /* hydrostatic split state (cUranusModel.h:1482-1495, flat [(i*jm + j)*km + k] there) */
    ATURAN_P_BARO, ATURAN_P_B0, ATURAN_P_BFOLLOW,               /* 63..65 */
    /* projection fields: last RK stage's tendencies and aux = rhs + grad p_dyn */
    ATURAN_RHS_U, ATURAN_RHS_V, ATURAN_RHS_W,
    ATURAN_AUX_U, ATURAN_AUX_V, ATURAN_AUX_W,                   /* 66..71 */
    /* the chemistry's diffusive tendencies D lap(c) (cUranusModel.h:1401-1403): persistent state
     * whose boundary rows the boundary passes set and whose neighbours the chemistry's filters read */
    ATURAN_DIFFLUX_H2S, ATURAN_DIFFLUX_NH3, ATURAN_DIFFLUX_NH4SH, /* 72..74 */
    /* the turbulence closure's shear production P_k (cUranusModel.h:358), a diagnostic */
    ATURAN_PROD,                                                /* 75 */
    ATURAN_NFIELDS
};

#define ATURAN_NPROG 19

/* One condensable's constants, exactly the arguments SaturationAdjustmentUran::run passes to the
 * shared SaturationAdjustment<Planet>::run (SaturationAdjustmentUran.cpp:222-238). */
typedef struct aturan_gas {
    double t_0, t_00;                   /* [K] melting point, all-ice temperature */
    double ep, lv, ls;                  /* gas-constant ratio, latent heats [J/kg] */
    double C, L0, R, del_alf, del_bet;  /* liquid saturation-pressure set (ATPhys.h:49-53) */
    double C_i, L0_i, del_alf_i, del_bet_i;   /* ice set */
} aturan_gas;

/* Everything the path reads besides the fields: the grid, the config scalars
 * (UranusParams.h.inc), the mixture properties of the initialised model and the resolved knobs.
 * aturan_params_default() fills the reference's defaults after its initialisation. */
typedef struct aturan_params {
    int32_t abi_version;         /* = ATURAN_ABI_VERSION */
    int32_t im, jm, km;          /* stored grid; k = km-1 is the copy of k = 0 */
    int32_t precision;           /* enum aturan_precision */
    int32_t turb_active;         /* k*, omega* prognostic (cUranusModel::turb_active) */
    int32_t coriolis_full;       /* ATURAN_CORIOLIS_FULL: scale L_atm in metres */
    int32_t cp_h2_mode;          /* ATURAN_CP_H2: 0 constant, 1 normal, 2 equilibrium H2 */
    int32_t cp_gas;              /* ATURAN_CP_GAS */
    int32_t cp_dyn;              /* cp(T) in the RHS pressure-work term (CpH2::dyn_on) */
    int32_t press_consistent;    /* ATURAN_PRESS_CONSISTENT (PressureSolverUran.h:68) */
    int32_t press_incr;          /* ATURAN_PRESS_INCR of PressureSolverUran (:139) */
    int32_t rigid_lid;           /* ATURAN_BC_RIGID_LID for the shared solver */
    int32_t satadj_conserve, satadj_newton, satadj_evap, satadj_ice_entry;
    int32_t satadj_bergeron, satadj_freeze, satadj_dry_exit, local_rho;
    int32_t nh4sh_sync;          /* RK_SCALAR_SYNC also copies nh4sh (ATURAN_NH4SH_EQ) */
    int32_t exact_reductions;    /* FP64 only. 1 (default): the level means of the buoyancy
                                    reference are summed in the reference's serial order, so the
                                    RK4 step is bit-equal to the CPU's; 0: a fixed tree order
                                    (deterministic run to run, within ~1e-12 of the serial sums).
                                    The mixed form always uses the tree order. */
    int32_t reserved_i[7];

    double r0, dr, the0, dthe, phi0, dphi, dt;
    double metric_R_km;          /* ATURAN_METRIC_RADIUS; <= 0 keeps the unshifted rad.z */
    double sinthe_min;           /* polar metric floor (cUranusModel.h:675) */
    double L_atm, u_0, t_ref, g, omega, re, pr;
    double Coriolis, centrifugal, buoyancy, chemical_reaction, R_ref, p_ref;
    double r_mix, R_mix, cp_mix, mue_mix;
    double r_h2, r_he, r_ch4, cp_h2, cp_he, cp_ch4;
    double sc_ch4, sc_h2o, sc_h2s, sc_nh3, sc_nh4sh;
    double alpha_sponge, r_p_nh4sh, rho_cond_nh4sh;
    double turb_coupling;        /* ATURAN_TURB_COUPLING */
    double precip_coupling;      /* ATURAN_PRECIP_COUPLING */
    double tmf_scale;            /* ATURAN_THERMAL_MASSFLUX */
    double cent_mom;             /* ATURAN_CENTRIFUGAL_MOM (0 or 1) */
    double pbaro_follow;         /* ATURAN_PBARO_FOLLOW tau [RK steps]; 0 = p_baro frozen */
    double t_min_K, t_max_K;     /* integrator temperature guards */
    double p_dyn_cap;            /* shared solver source clamp (PressureSolver.h:168) */
    double satadj_stop_tol;      /* the adjustment's stopping test on |q_v - q_hyp| / q_hyp
                                    (SaturationAdjustment.h:551): the reference's 1e-3 (default;
                                    <= 0 reads as 1e-3); smaller values take the passes nearer the
                                    root (within the 15-pass cap), as a finite-difference check of
                                    the implicit adjoint needs */
    double satadj_entry_tol;     /* the entry test (SaturationAdjustment.h:446): a cell whose vapour
                                    lies within this fraction of its entry saturation is left
                                    alone. 0 (default): the reference's 1e-3; < 0: no band (only
                                    exact equality is left alone), which makes the adjustment a
                                    continuous map, as a finite-difference check needs */
    double reserved_d[6];
    aturan_gas gas[4];           /* H2O, H2S, NH3, CH4: the loop's order */
} aturan_params;

enum aturan_pressure_kind {
    ATURAN_PRESS_GS_LEX    = 0, /* PressureSolverUran::run, one lexicographic GS sweep (default) */
    ATURAN_PRESS_RB_SHARED = 1, /* PressureSolver<cUranusModel>::run, max_sweeps red-black sweeps */
    ATURAN_PRESS_RB_SOR    = 2, /* the shared solver's equation solved to a relative residual with
                                   point red-black SOR at omega (new behaviour, no reference oracle) */
    ATURAN_PRESS_RB_LINE   = 3  /* the same equation and tolerance with red-black radial-line SOR,
                                   each column solved exactly in r (the reference's PRESS_LINE) */
};

typedef struct aturan_ctx aturan_ctx;

/* Fill *p with the reference's resolved defaults on the 41 x 181 x 361 grid. */
int aturan_params_default(aturan_params* p);

/* Create a context: allocate the device state for p->im x p->jm x p->km, build the geometry and
 * cp(T) tables on the host in FP64 and upload them. Replaces nothing in the reference (its state
 * is allocated by cUranusModel::resetArrays, cUranusModel.cpp:1416). */
int aturan_ctx_create(const aturan_params* p, aturan_ctx** out);
int aturan_ctx_destroy(aturan_ctx* ctx);
const char* aturan_last_error(const aturan_ctx* ctx);   /* NULL: the last error of the calls
                                                          without a context, on this thread */

/* Copy one field between host memory (contiguous FP64 [i][j][k], im*jm*km values) and the
 * device. Both return when the host buffer may be reused (upload) or holds the data (download).
 * In a mixed context t and tn are stored as the FP32 pair hi + lo (FP64 to ~2^-48), so they come
 * back as uploaded; every other FP32 field comes back rounded to FP32. */
int aturan_upload(aturan_ctx* ctx, int field, const double* host);
int aturan_download(aturan_ctx* ctx, int field, double* host);
/* As upload/download for a field on a device pointer (contiguous [i][j][k] FP64). The upload is
 * asynchronous on the context's stream. */
int aturan_upload_device(aturan_ctx* ctx, int field, const double* dev);
int aturan_download_device(aturan_ctx* ctx, int field, double* dev);
/* n fields in one call: fields[q] from src[q] (to dst[q]); host buffers (pinned for overlap), or
 * device buffers with on_device = 1. The host copies of field q overlap the on-device layout
 * change of field q-1, and the call waits once instead of once per field (what a driver that
 * exchanges the fields its CPU modules touch each iteration uses). Same return conditions as the
 * one-field calls, except that a device upload is asynchronous. */
int aturan_upload_many(aturan_ctx* ctx, int n, const int* fields, const double* const* src, int on_device);
int aturan_download_many(aturan_ctx* ctx, int n, const int* fields, double* const* dst, int on_device);
/* buoy_ref_level[im] of the last RK4 step (cUranusModel.h:1431). */
int aturan_download_buoy_ref(aturan_ctx* ctx, double* host_im);

/* One RK4 step: computeBuoyancyRefLevel + computeHydrostaticPressure(true) + the four stages
 * with their fused RHS evaluation and the final update.
 * Replaces cUranusModel::RungeKuttaUran() (RungeKutta_Uran_Turb.cpp:179-404). */
int aturan_rk4_step(aturan_ctx* ctx);

/* Adjoint of one RK4 step of the dry dynamics, FP64 contexts. No counterpart in the reference,
 * which has no adjoint; it differentiates RungeKutta_Uran_Turb.cpp:18-403 with RHS_Uran_Turb.cpp's
 * tendencies of t, u, v, w.
 * aturan_tape(ctx, 1): every later aturan_rk4_step and RB_SOR / RB_LINE aturan_pressure keeps what
 *   its adjoint needs (the stage inputs of t, u, v, w, the new T, p_dyn, the clamped pressure
 *   source and the level means: 19 fields, plus 56 fields of work arrays, of device memory);
 *   aturan_tape(ctx, 2): the moist tape (aturan_moist_adjoint); aturan_tape(ctx, 0) frees either.
 *   ATURAN_E_UNSUPPORTED on a mixed context.
 * aturan_rk4_adjoint(ctx, ybar, xbar): ybar[4] and xbar[4] are device pointers to contiguous
 *   [im][jm][km] FP64 arrays in the order t, u, v, w. Given the adjoint ybar of those fields after
 *   the last taped aturan_rk4_step, writes xbar = J^T ybar, J the step's Jacobian with respect to
 *   the fields before it, taken as the state and its start-of-step copies together (as after
 *   aturan_sync_ncopies). p_dyn, p_stat, p_baro, p_b0, p_bfollow, the forcing and the other
 *   prognostic fields are held fixed. The T clamp and cp(T)'s 0.5 K table are differentiated
 *   piecewise (0 where clamped, the interval's slope). Synchronous. */
int aturan_tape(aturan_ctx* ctx, int on);
int aturan_rk4_adjoint(aturan_ctx* ctx, const double* const* ybar, double* const* xbar);

/* The same with the two links to the pressure solve (no counterpart in the reference):
 * auxbar[3] (or NULL) is the adjoint of the step's projection outputs aux_u, aux_v, aux_w (the
 * stage-3 tendencies of u, v, w without the p_dyn gradient, which the next pressure solve reads;
 * RHS_Uran_Turb.cpp:1020-1022), and pbar (or NULL) receives the adjoint of the p_dyn the step
 * read, all [im][jm][km] FP64 device arrays; heatbar (or NULL) receives the adjoint of the
 * heating field of aturan_set_heating, a [jm][km] FP64 device array. */
int aturan_rk4_adjoint_ex(aturan_ctx* ctx, const double* const* ybar, const double* const* auxbar,
                          double* const* xbar, double* pbar, double* heatbar);

/* The moist step's adjoint (no counterpart in the reference). aturan_tape(ctx, 2) switches on the
 * moist tape (the dry one's contents over sixteen fields -- t, u, v, w and the twelve condensable
 * species ATURAN_CH4 .. ATURAN_NH3_ICE -- plus the state an aturan_satadj of all four gases, or
 * aturan_step's adjustment, had on entry: 16 more fields and 84 more work fields; replaces a dry
 * tape). Given ybar[16], the adjoint of those sixteen fields after the last taped
 * aturan_rk4_step, writes xbar[16]: the RK4 step's adjoint over the sixteen fields (the species'
 * transport and diffusion by the taped u, v, w, their forcing held fixed) and, when an adjustment
 * ran between the previous taped RK4 step and this one, then the implicit adjoint of the
 * converged saturation adjustment (SaturationAdjustment.h:255-746): per cell and gas the
 * derivative of the root of the closure q_v = H(T, q_c, q_i) on the adjustment's invariants (total
 * water, and the moist enthalpy cp rho T - L_v q_c - L_s q_i), the phases present at convergence
 * frozen; a gas that was not adjusted contributes its entry melt / freeze, piecewise linear. xbar
 * is then the adjoint with respect to the state before the adjustment. auxbar, pbar and heatbar
 * as for aturan_rk4_adjoint_ex. FP64 contexts. Synchronous. */
int aturan_moist_adjoint(aturan_ctx* ctx, const double* const* ybar, const double* const* auxbar,
                         double* const* xbar, double* pbar, double* heatbar);

/* A heating rate H(theta, phi) in K/s added to the temperature tendency at every interior level,
 * rhs_t += H (L_atm 1e3 / u_0) / t_ref (no counterpart in the reference, whose heating enters as
 * Q_rad in W/m^3, RHS_Uran_Turb.cpp:503-526). H: [jm][km] FP64, host or device (on_device);
 * NULL removes the term (the default: the step is then the reference's, bit for bit). */
int aturan_set_heating(aturan_ctx* ctx, const double* H, int on_device);

/* Adjoint of the last taped ATURAN_PRESS_RB_SOR / RB_LINE pressure call (no counterpart in the
 * reference): given pbar, the adjoint of the p_dyn it produced (boundary rows included), writes
 * auxbar[3], the adjoint of the aux_u, aux_v, aux_w it read. The chain reversed: the boundary
 * passes, the solve (a solve with the transposed operator, kind/omega/max_sweeps/tol as for the
 * forward; ATURAN_NOT_CONVERGED at the cap), the compatibility shift, the source clamp (0 where the
 * forward clamped) and the divergence (PressureSolver.h:370-487 with prepareProjectionBoundaries,
 * Pressure_Uran.cpp:30-146). The free constant of p_dyn is taken as not differentiated (its
 * adjoint is made zero-mean). FP64 contexts with the tape on. Synchronous. */
int aturan_pressure_adjoint(aturan_ctx* ctx, int kind, double omega, int max_sweeps, double tol,
                            const double* pbar, double* const* auxbar, int* sweeps_done, double* resid);

/* The pressure solve.
 *   GS_LEX:    replaces PressureSolverUran(m).run() (PressureSolverUran.h:33-250); omega,
 *              max_sweeps and tol are ignored (exactly one sweep, as the reference).
 *   RB_SHARED: replaces PressureSolver<cUranusModel>(m).run() (PressureSolver.h:145-766) with
 *              ATURAN_PRESS_SWEEPS = max_sweeps; omega and tol ignored.
 *   RB_SOR:    the shared solver's equation (its source, clamp and boundary folds) solved with
 *              point red-black SOR at omega until the relative L2 residual <= tol or max_sweeps.
 *   RB_LINE:   the same with red-black radial-line SOR; max_sweeps counts line sweeps.
 *   Both to-residual kinds add an exact correction of the column-uniform mode every few sweeps,
 *   return ATURAN_NOT_CONVERGED at the cap, and compute in FP64, or in the mixed form as FP32
 *   correction solves inside FP64 iterative refinement.
 * sweeps_done and resid (relative L2 residual at exit; RB_SOR only, else 0) may be NULL. */
int aturan_pressure(aturan_ctx* ctx, int kind, double omega, int max_sweeps, double tol,
                    int* sweeps_done, double* resid);

/* The sweeps and the residual of the context's last pressure solve, whether aturan_pressure or
 * aturan_step ran it (aturan_step has no out-parameters); 0 and 0.0 before any. No counterpart in
 * the reference, which prints no solver diagnostics for its single sweep. Either pointer may be
 * NULL. */
int aturan_pressure_last(aturan_ctx* ctx, int* sweeps_done, double* resid);

/* Solve the pressure equation's folded operator, or its transpose, on caller buffers: the linear
 * solve inside ATURAN_PRESS_RB_SOR / RB_LINE, and with transposed = 1 the adjoint of that solve
 * (no counterpart in the reference, which has no adjoint). b and x are device pointers to
 * contiguous [im][jm][km] FP64 arrays; x holds the initial guess and receives the solution on the
 * interior (i = 1..im-2, j = 1..jm-2, k = 0..km-2; its other entries are left as given).
 *   transposed = 0: Lc x = b, b first made compatible by removing its component along Lc's left
 *     null vector y_i y_j, y = (3/2, 1, ..., 1, 3/2); x is then defined up to a constant.
 *   transposed = 1: Lc^T x = b, b first made zero-mean (Lc^T's left null vector is the constant);
 *     x is defined up to a multiple of y_i y_j. For compatible s and g,
 *     <solve(s), g> = <s, solve^T(g)>: the adjoint of the pressure solve.
 * kind is ATURAN_PRESS_RB_SOR or ATURAN_PRESS_RB_LINE, in the context's precision as
 * aturan_pressure: FP64 relaxation in an FP64 context; in a mixed context FP32 correction solves
 * inside FP64 iterative refinement (residual, its norm and x += e in FP64; b and x stay FP64).
 * ATURAN_NOT_CONVERGED at the cap. Synchronous. */
int aturan_pressure_solve(aturan_ctx* ctx, int kind, int transposed, double omega, int max_sweeps, double tol,
                          const double* b, double* x, int* sweeps_done, double* resid);

/* The saturation adjustment of every gas whose bit is set in gas_mask (bit 0 H2O, 1 H2S, 2 NH3,
 * 3 CH4), in that order, fused per cell. Replaces the four
 * SaturationAdjustmentUran(m).run(...) calls of cUranusModel.cpp:998-1027 (and each one alone).
 * n_adjusted / n_noconv (may be NULL) receive the reference's per-call counters summed over
 * the gases (SaturationAdjustment.h:592-593). */
int aturan_satadj(aturan_ctx* ctx, int gas_mask, long* n_adjusted, long* n_noconv);

/* The ATURAN_RK_SCALAR_SYNC=2 copy of the condensables and T (and NH4SH when nh4sh_sync) into
 * their start-of-step copies, cUranusModel.cpp:1049-1073. */
int aturan_sync_ncopies(aturan_ctx* ctx);

/* restoreVar(coeff) at the end of an iteration (cUranusModel.cpp:1264, :1638-1680): every
 * prognostic field's start-of-step copy set to coeff times the field (p_dynn and chromn, which the
 * library does not hold, excepted). A driver running several steps on the device calls it after
 * each step, where the reference's loop does. */
int aturan_restore_ncopies(aturan_ctx* ctx, double coeff);

/* The in-scope part of one even iteration of cUranusModel::Run (cUranusModel.cpp:967-1123):
 * pressure (kind/omega/max_sweeps/tol as aturan_pressure), the four saturation adjustments,
 * the n-copy sync and the RK4 step. */
int aturan_step(aturan_ctx* ctx, int press_kind, double omega, int max_sweeps, double tol);

/* The knobs of the part of an iteration that follows RungeKuttaUran (cUranusModel.cpp:1218-1248):
 * the t filter, the velocity filter, the three boundary passes (BC_Uran.h:140-173 over
 * BoundaryConditions.h:152-518) and the species clamp. The reference reads each from an
 * ATURAN_* environment variable once per process; the caller resolves them.
 * aturan_post_params_default gives the values they take with the environment unset. A form is
 * BCForm's (BoundaryConditions.h): 0 the model default (Neumann), 1 copy, 2 Neumann
 * c43 a - c13 b, anything else the cubic c - 3 b + 3 a. */
typedef struct aturan_post_params {
    int32_t abi_version;      /* = ATURAN_ABI_VERSION */
    int32_t damp_t_j;         /* ATURAN_DAMP_T_J: the t filter's latitude pass (default !GEO_BALANCE = 0) */
    int32_t radius_form;      /* ATURAN_BC_RADIUS_COPY (0): i = 0 and im-1 of the radius list */
    int32_t bottom_form;      /* ATURAN_BC_BOTTOM_FORM (0 = radius_form): i = 0 of every field but u */
    int32_t pole_form;        /* ATURAN_BC_POLE_COPY (0): j = 0 and jm-1 of the theta list */
    int32_t lid_u;            /* ATURAN_BC_LID_U (= ATURAN_BC_RIGID_LID = 1): u = 0 on i = 0, im-1 */
    int32_t top_taper;        /* ATURAN_BC_TOP_TAPER (0; 1 or 2): v, w toward zero at the top */
    int32_t lid_vw;           /* ATURAN_BC_LID_VW (2 with GEO_BALANCE): v, w at im-1; 2 linear, 3 cubic */
    int32_t radius_positive;  /* ATURAN_BC_RADIUS_POSITIVE (1): species floor on i = 0, im-1; 2 copy */
    int32_t phi_periodic;     /* ATURAN_BC_PHI_PERIODIC (1): k = km-1 copies k = 0; 0 = averaged ends */
    int32_t species_clamp;    /* ATURAN_SPECIES_CLAMP (1): negative and NaN species values -> 0 */
    int32_t reserved_i[5];
    double damp_t_horiz;      /* ATURAN_DAMP_T_HORIZ (1.0): strength of the t filter's horizontal passes */
    double damp_t_vert;       /* ATURAN_DAMP_T_VERT (0.0): strength of its radial pass */
    double vel_shapiro;       /* ATURAN_VEL_SHAPIRO (0.0 with GEO_BALANCE): 1-2-1 pass on u, v, w */
    double reserved_d[5];
} aturan_post_params;

#define ATURAN_NSPECIES 13    /* h2o, h2o_cloud, h2o_ice, h2s.., nh3.., ch4.., nh4sh (BC_Uran.h:83-89) */

int aturan_post_params_default(aturan_post_params* pp);

/* What cUranusModel.cpp:1218-1248 does to the state after RungeKuttaUran, in its order:
 *   damp_wiggles(t, along k [and j]) with damp_t_horiz, damp_wiggles(t, along i) with damp_t_vert
 *   (lib/Utils.cpp:224-317), damp_wiggles(u / v / w, along k, j, i) with vel_shapiro, then
 *   BC_Uran::bcRadius (with floorRadialSpecies and the lid v, w), bcTheta, bcPhi, and
 *   clampNegativeSpecies (BC_Uran.h:91-128).
 * The boundary passes apply to the fields of the reference's lists (BC_Uran.cpp) that the
 * context holds: t, u, v, w, the twelve condensables, nh4sh, massflux_h2s/nh3/nh4sh,
 * fluxlim_nh4sh, thermalmassflux and difflux_h2s/nh3/nh4sh. The other listed arrays (chrom, the
 * j_/jT_/w_ fluxes, the force and heat diagnostics) are not held; a driver applies the passes to
 * those on the host. clamp_added / clamp_cells (may be NULL; ATURAN_NSPECIES entries each, in the order
 * above) receive this call's clipped sum and count per species, what the reference adds to its
 * cumulative clamp_added / clamp_cells; passing them synchronizes the stream.
 * Not implemented (the reference's defaults leave them off; the host keeps them): BC_T_LID_PIN,
 * BC_SEAM_DAMP, VEL_SHAPIRO_ORDER=4, the turbulence fields' floors (bc_turb_active is false for
 * Uranus) and pole fill rows (bc_pole_open_rows is 0 for Uranus). */
int aturan_post_step(aturan_ctx* ctx, const aturan_post_params* pp, double* clamp_added, long* clamp_cells);

/* MoistConvectiveAdjustment<cUranusModel>::run (planet/ConvectiveAdjustment.h:402-849) as the
 * model's loop calls it (cUranusModel.cpp:1272-1292, every iteration by default), with the
 * reference's default knobs (MCA_LEDOUX 1, MCA_LOADING 1, MCA_RELAX 1, MCA_SMOOTH 0, MCA_PASSES 64,
 * no phase split, interior levels): per (j, k) column, the unstable pairs' segments mixed to their
 * mass-weighted liquid-water static energy and total mixing ratios and settled to equilibrium;
 * t, the twelve condensables and nh4sh written where touched. FP64 contexts with im <= 64; other
 * contexts return ATURAN_E_UNSUPPORTED. The first call allocates 24 KB on the device. */
int aturan_mca(aturan_ctx* ctx);

/* The chemistry of the iteration loop (planet/ChemistryUran.h, FluxLimiter.h) as the model calls
 * it (cUranusModel.cpp:1034 and 1074-1087) with the reference's default knobs. Constants the
 * params struct does not carry come from aturan_params (r_mix, R_mix, cp_mix, mue_mix, sc_h2s,
 * sc_nh3, sinthe_min, metric_R_km, t_ref). */
typedef struct aturan_chem_params {
    int32_t abi_version;          /* = ATURAN_ABI_VERSION */
    int32_t nh4sh_eq;             /* ATURAN_NH4SH_EQ (ChemistryUran.h:143): only 1 (the default) */
    int32_t difflux_plus;         /* ATURAN_CHEM_DIFFLUX_PLUS: 1 (default) massflux = +difflux, 0: minus */
    int32_t difflux_laplacian;    /* ATURAN_CHEM_DIFFLUX_LAPLACIAN: only 1 (the default) */
    int32_t phi_periodic;         /* ATURAN_BC_PHI_PERIODIC (ATPhys.h:125): 1 (default) or 0 */
    int32_t reserved_i[3];
    double m_nh3, m_h2s, m_nh4sh;      /* molar masses [kg/kmol] (cUranusModel.h:997-999) */
    double c_mix;                      /* mixture molar density [kmol/m3] (ThermalPropertiesUran) */
    double D_nh4sh, DT_nh4sh;          /* NH4SH diffusion coefficients (cUranusModel.h:1135-1140) */
    double cp_nh3, cp_h2s, cp_nh4sh;   /* [J/(kg K)] (cUranusModel.h:1085-1087) */
    double k_nh3, k_h2s, k_nh4sh;      /* [W/(m K)] (cUranusModel.h:1076-1078) */
    double polar_floor;                /* ATPhys::polar_divisor_floor (ATPhys.h:104): 0.4 */
    double reserved_d[5];
} aturan_chem_params;

/* Fill the reference's defaults. */
int aturan_chem_params_default(aturan_chem_params* cp);

#define ATURAN_CHEM_NH4SH_EQ 1    /* ChemistryUran::EquilibriumNH4SH("loop") (ChemistryUran.h:222-280) */
#define ATURAN_CHEM_FORCING 2     /* DiffMassFluxUran, the 1-2-1 filters, ChemMassRateUran,
                                     FluxLimiterNH4SH, the filters (cUranusModel.cpp:1074-1087) */

/* Run the parts of the chemistry selected in `what` (a mask of the two flags above; NH4SH_EQ runs
 * first when both are set, as the loop orders them: it follows the saturation adjustment and
 * precedes the precipitation, FORCING follows the n-copy sync).
 * NH4SH_EQ: every cell to the NH3 + H2S <-> NH4SH(s) equilibrium of K_p(T) (Lewis 1969), solved
 * with T by bisection; writes nh3, h2s, nh4sh and t where x != 0; n_formed / n_decomposed (may be
 * NULL; passing either synchronizes the stream) receive the cells that formed / decomposed NH4SH.
 * FORCING: rho_mix (every cell), thermalmassflux, difflux_h2s/nh3/nh4sh = D lap(c), the filters
 * on those four, massflux_* = w_* + sign difflux_* with w_* = 0 (equilibrium form), the Superbee
 * limiter's fluxlim_nh4sh, the filters on those four. The interior rows are written, the
 * boundary rows of the persistent fields are read as the last boundary passes left them.
 * Knob values other than those supported return ATURAN_E_UNSUPPORTED. */
int aturan_chemistry(aturan_ctx* ctx, const aturan_chem_params* cp, int what, long* n_formed,
                     long* n_decomposed);

/* The turbulence closure (planet/Turbulence.h, Turbulence<cUranusModel>::run, :307-331) as the
 * model's loop calls it (cUranusModel.cpp:1270, every iteration when the closure is on, which is
 * the default) with the reference's default knobs. */
typedef struct aturan_turb_params {
    int32_t abi_version;         /* = ATURAN_ABI_VERSION */
    int32_t model;               /* ATURAN_TURB_MODEL: 2 = k_omega_SST (the default; the only one implemented) */
    int32_t turb_free;           /* ATURAN_TURB_FREE (Turbulence.h:141): only 1 (the default) */
    int32_t clamp_pass;          /* ATURAN_TURB_CLAMP_PASS (:175): only 1 (the default) */
    int32_t curv;                /* ATURAN_TURB_CURV: 1 (default) the curvature terms of the velocity gradient */
    int32_t buoy;                /* ATURAN_TURB_BUOY: only 0 (Uranus's default) */
    int32_t abl_taper;           /* ATURAN_ABL_TAPER: only 0 (the default) */
    int32_t phi_periodic;        /* ATURAN_BC_PHI_PERIODIC: 1 (default) or 0 */
    double nue_max;              /* ATURAN_NUE_MAX [m2/s] (:123): 1e5 */
    double k_bg;                 /* ATURAN_TURB_K_BG [m2/s2] (:156): 1 */
    double nue_air;              /* the gas's kinematic viscosity [m2/s] (constructor default): 1.8e-5 */
    double reserved_d[5];
} aturan_turb_params;

/* Fill the reference's defaults. */
int aturan_turb_params_default(aturan_turb_params* tp);

/* compute_sources (clamp pass, SST production, eddy viscosity and sources, floors and caps on the
 * interior), apply_wall_bc (zero-gradient copy at i = 0), clamp_nue, seam_copy and
 * fill_lid_corners (lid and pole rows copied from their neighbours): tke, dis, nue, prod,
 * tke_source, dis_source written, tken and disn copied at the seam and the edges. Knob values
 * other than those supported return ATURAN_E_UNSUPPORTED. */
int aturan_turbulence(aturan_ctx* ctx, const aturan_turb_params* tp);

/* The precipitation microphysics (planet/Precipitation.h, Precipitation<cUranusModel>::run,
 * :192-277, and its column solver, :280-446) as the model's loop calls it (cUranusModel.cpp:1037,
 * after the NH4SH equilibrium and
 * before the n-copy sync, on by default): per (j, k) column, top down, the three-category
 * (rain / snow / graupel) scheme of each condensable in the order H2O, NH3, CH4 and then H2S
 * (cUranusModel.h:280-297). */
typedef struct aturan_precip_params {
    int32_t abi_version;         /* = ATURAN_ABI_VERSION */
    int32_t coupling;            /* ATURAN_PRECIP_COUPLING (Precipitation.h:164): 1 (default) the depletion
                                    as rates in S_precip_*; 0 written into the condensate fields */
    int32_t h2s;                 /* ATURAN_PRECIP_H2S (cUranusModel.h:276): 1 (default) H2S runs too */
    int32_t reserved_i[5];
    double rate_scale;           /* ATURAN_PRECIP_SCALE: the factor on the five rate coefficients,
                                    Uranus's default 0.00071 (cUranusModel.h:610) */
    double reserved_d[7];
} aturan_precip_params;

/* Fill the reference's defaults. */
int aturan_precip_params_default(aturan_precip_params* pp);

/* Q_precip and the twelve S_precip_* zeroed, then every column of every species: Q_precip gains
 * each species' latent heating; with coupling, S_precip_<gas>, _cloud, _ice receive the vapour
 * source and the cloud and ice depletion rates (nondimensional); without it the vapour, cloud and
 * ice fields are updated in place. The precipitation fluxes themselves (P_rain, ..., the NH4SH
 * settling flux and the surface maps) are the reference's diagnostics and are not kept. */
int aturan_precipitation(aturan_ctx* ctx, const aturan_precip_params* pp);

/* One iteration of the model's loop (cUranusModel.cpp:952-1296) with the reference's default
 * knobs, all on the device. Even iter_n (the loop's `iter_n % 2 == 0` branch): the pressure solve,
 * the p_dyn filter (:975-984), the four saturation adjustments, the NH4SH equilibrium, the
 * precipitation, the n-copy sync, the chemistry forcing; every iteration: the RK4 step, the passes
 * after it (aturan_post_step), restoreVar(1.0), the turbulence closure, the moist convective
 * adjustment every mca_stride-th iteration. The diagnostics of the loop (forces, latent heat,
 * radiation with its default RAD_COUPLING 0, the budgets and reports) change no field the step
 * reads and are not run. */
typedef struct aturan_iter_params {
    int32_t abi_version;         /* = ATURAN_ABI_VERSION */
    int32_t press_kind;          /* enum aturan_pressure_kind; GS_LEX = PressureSolverUran (the default) */
    int32_t max_sweeps;          /* as aturan_pressure */
    int32_t chemistry;           /* 1 (default): aturan_chemistry's two parts on even iterations */
    int32_t precipitation;       /* ATURAN_PRECIP (cUranusModel.cpp:105-108): 1 (default) */
    int32_t turbulence;          /* turb_active (cUranusModel.cpp:482): 1 (default) */
    int32_t mca_stride;          /* ATURAN_MCA (cUranusModel.cpp:131-134): 1 (default); 0 = off */
    int32_t reserved_i[5];
    double omega, tol;           /* as aturan_pressure (RB_SOR / RB_LINE) */
    double damp_p_horiz;         /* ATURAN_DAMP_P_HORIZ (:979-980): 0 (default with GEO_BALANCE) = the radial
                                    pass of the p_dyn filter only; 1 = all three axes; else horizontal
                                    passes of that strength, then the radial one */
    double reserved_d[5];
    aturan_post_params post;
    aturan_chem_params chem;
    aturan_turb_params turb;
    aturan_precip_params precip;
} aturan_iter_params;

/* Fill the reference's defaults. */
int aturan_iter_params_default(aturan_iter_params* ip);

/* One iteration number iter_n (1-based, as the reference counts) of the loop above. Parts whose
 * knob values are not implemented return ATURAN_E_UNSUPPORTED before any launch. */
int aturan_iteration(aturan_ctx* ctx, const aturan_iter_params* ip, int iter_n);

/* Kernel classes for the per-class launch counts and timings below. */
enum aturan_kernel_kind {
    ATURAN_K_RK_STAGE = 0,   /* fused RHS + RK4 stage update */
    ATURAN_K_SATADJ,         /* fused 4-gas saturation adjustment */
    ATURAN_K_GS,             /* PressureSolverUran sweep (incl. its source and boundary passes) */
    ATURAN_K_RB,             /* red-black sweeps, source, boundary passes, residual checks */
    ATURAN_K_HYDRO,          /* buoyancy reference level + hydrostatic column integral */
    ATURAN_K_COPY,           /* n-copy sync and layout conversions */
    ATURAN_K_ADJOINT,        /* the RK4 step's adjoint (aturan_rk4_adjoint) */
    ATURAN_K_POST,           /* filters, boundary passes and species clamp (aturan_post_step) */
    ATURAN_K_MCA,            /* moist convective adjustment (aturan_mca) */
    ATURAN_K_CHEM,           /* NH4SH equilibrium and chemistry forcing (aturan_chemistry) */
    ATURAN_K_TURB,           /* turbulence closure (aturan_turbulence) */
    ATURAN_K_PRECIP,         /* precipitation microphysics (aturan_precipitation) */
    ATURAN_K_NKINDS
};

/* Reset the per-class counters; enable = 1 also brackets every class's launches with CUDA events
 * on the context's stream (a few microseconds per bracket), enable = 0 counts launches only. */
int aturan_profile(aturan_ctx* ctx, int enable);
/* Read the counters since the last aturan_profile: launches[n] kernels of class n and, when timing
 * was enabled, ms[n] their summed device time. Synchronizes the stream. Either pointer may be NULL. */
int aturan_profile_read(aturan_ctx* ctx, double* ms, long* launches, int nkinds);

/* The buoyancy reference level of RungeKutta_Uran_Turb.cpp:18-37 computed without allocating any
 * device memory; no counterpart in the reference, which has no device. It is for callers that may
 * not allocate: an application whose memory pool owns the whole GPU and hands this library only
 * the buffers it holds, or a plugin run under a fixed device-memory budget. t and p_stat are the
 * caller's device arrays, contiguous FP64 [i][j][k] with k fastest (im*jm*km values); ref_out
 * receives im doubles on the device.
 * The scratch (block partial sums and the sin(theta) weights, both written by the call's own
 * kernels) is a fixed array inside the library image, so every GPU that loads the library holds
 * 288 KiB until the process exits; it bounds the grid to im <= ATURAN_STATIC_MAX_IM,
 * jm <= ATURAN_STATIC_MAX_JM and jm * km <= ATURAN_STATIC_MAX_LEVEL_CELLS; larger grids are
 * rejected with ATURAN_E_INVALID (message in aturan_last_error(NULL)). The first call on a device
 * looks the array's address up (cudaGetSymbolAddress) with that device current; make it before any
 * stream capture. The call is asynchronous on `stream` (a cudaStream_t, NULL for the legacy default
 * stream). All calls on a device share the array and each overwrites what it reads: calls whose
 * kernels may overlap on the GPU (on unordered streams) race and must not be issued. The result
 * agrees with aturan_rk4_step's level means with exact_reductions = 0 (the same tree order) to
 * rounding: the weights' sin is the device's here, the host's there. */
#define ATURAN_STATIC_MAX_IM 512
#define ATURAN_STATIC_MAX_JM 4096
#define ATURAN_STATIC_MAX_LEVEL_CELLS 1073741824
int aturan_buoy_ref_level_static(const aturan_params* p, const double* t, const double* p_stat,
                                 double* ref_out, void* stream);

/* Wait for all work queued on the context's stream. */
int aturan_sync(aturan_ctx* ctx);

/* The context's CUDA stream (a cudaStream_t), for callers that time or order work around it. */
void* aturan_stream(aturan_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif /* ATURAN_B200_H */
