/*
 * CPU ORACLE for the aturan_b200 hot path — TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.
 *
 * A plain-C restatement of the reference's FP64 algorithm for the dynamical-core step, written
 * from the reference's sources with the same expression order so that, compiled without FMA
 * contraction, it reproduces the reference bit for bit. Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load it, and only as the checker.
 *
 * Parity pinned: tests/test_oracle_vs_ref.py runs every function below against the compiled
 * reference (oracle/_ref, built from the reference's own sources by oracle/Makefile) on the
 * reference's initialised state and on seeded perturbations of it, and requires bit equality;
 * tests/golden/ holds fixtures made the same way for machines without the reference tree.
 *
 * Fields: f[id] for id in enum aturan_field, each a contiguous FP64 block [i][j][k] of
 * im*jm*km values (NULL where a function does not read it). Grid sizes come from the params.
 */
#ifndef ATURAN_ORACLE_H
#define ATURAN_ORACLE_H
#include "aturan_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

void   oracle_coords(const aturan_params* p, double* rad_z, double* the_z);
double oracle_cp_lapse(const aturan_params* p, double T_K);

int oracle_buoy_ref(const aturan_params* p, double* const* f, double* ref_level);
int oracle_hydro(const aturan_params* p, double* const* f, const double* ref_level, int advance_follow);
int oracle_rhs_cell(const aturan_params* p, double* const* f, int i, int j, int k, double* rhs22);
int oracle_rk4(const aturan_params* p, double* const* f, double* ref_level_out);
int oracle_pressure_gs(const aturan_params* p, double* const* f);
int oracle_pressure_rb(const aturan_params* p, double* const* f, int sweeps);
int oracle_pressure_sor(const aturan_params* p, double* const* f, double omega, int max_sweeps,
                        double tol, int check_every, int* sweeps_done, double* resid);
int oracle_pressure_line(const aturan_params* p, double* const* f, double omega, int max_iter,
                         double tol, int* iters_done, double* resid);
double oracle_pressure_residual(const aturan_params* p, double* const* f, const double* src);
int oracle_laplace_apply(const aturan_params* p, const double* x, double* out, int transposed);
int oracle_solve(const aturan_params* p, const double* b, double* x, int transposed, int line, double omega,
                 int max_iter, double tol, int* iters_done, double* resid);
int oracle_pressure_source(const aturan_params* p, double* const* f, double* src);
int oracle_pressure_source_compat(const aturan_params* p, double* const* f, double* src);
int oracle_satadj(const aturan_params* p, double* const* f, int gas, long* n_adjusted, long* n_noconv);
int oracle_sync_ncopies(const aturan_params* p, double* const* f);
int oracle_step(const aturan_params* p, double* const* f, int press_kind, double omega,
                int max_sweeps, double tol, double* ref_level_out);
void oracle_set_threads(int n);
/* cUranusModel.cpp:1218-1248 after RK4: filters, boundary passes, species clamp */
/* ConvectiveAdjustment.h:402-849 with the reference's default knobs, the gas list of
 * cUranusModel.cpp:1276-1290 */
int oracle_mca(const aturan_params* p, double* const* f);
int oracle_post_step(const aturan_params* p, double* const* f, const aturan_post_params* pp,
                     double* clamp_added, long* clamp_cells);
/* ChemistryUran.h:210-275, EquilibriumNH4SH("loop"); counts[2] = cells formed, decomposed */
int oracle_nh4sh_eq(const aturan_params* p, const aturan_chem_params* cp, double* const* f, long* counts);
/* cUranusModel.cpp:1074-1087: DiffMassFluxUran, filters, ChemMassRateUran, FluxLimiterNH4SH, filters */
int oracle_chem_forcing(const aturan_params* p, const aturan_chem_params* cp, double* const* f);
/* Turbulence.h:307-331, Turbulence<cUranusModel>::run with the default knobs (k-omega SST) */
int oracle_turbulence(const aturan_params* p, const aturan_turb_params* tp, double* const* f);
/* Precipitation.h:192-446 for H2O, NH3, CH4, H2S (cUranusModel.h:280-297) */
int oracle_precipitation(const aturan_params* p, const aturan_precip_params* pp, double* const* f);
/* cUranusModel.cpp:952-1296, one iteration (iter_n counted from 1) with the default knobs */
int oracle_iteration(const aturan_params* p, const aturan_iter_params* ip, double* const* f, int iter_n);

#ifdef __cplusplus
}
#endif
#endif
