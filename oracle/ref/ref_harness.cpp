// Test harness around the UNMODIFIED ATURAN reference (CPU, C++/OpenMP).
//
// This file is test infrastructure: it is compiled against the reference's own sources (see
// oracle/Makefile) into oracle/_ref/libaturan_ref*.so, and only the tests, the smoke check and the
// CPU-baseline leg of bench.py load it. It exposes a C ABI over one cUranusModel instance:
//
//   ref_create()         construct the model with its compiled defaults, nm = 0, and run Run():
//                        the initialisation sequence of planet/cUranusModel.cpp:435-708 without a
//                        single iteration (the loop at :952 does not execute for nm = 0).
//   ref_get / ref_set    copy a named 3-D field out of / into the model's jagged Array
//                        (lib/Array.cpp:58-67) as a contiguous [i][j][k] double block.
//   ref_rk4 / ref_hydro / ref_pressure_* / ref_satadj / ref_sync_ncopies
//                        call the reference's own routines on that state.
//
// The model's headers are included with `private` defined as `public` so the harness can reach
// the model's private members; that changes access, not layout. Nothing here re-implements any physics.

// Standard and library headers first, with their access specifiers intact; only the reference's
// own classes below are opened up.
#include <algorithm>
#include <cassert>
#include <chrono>
#include <cmath>
#include <csignal>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fenv.h>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <limits>
#include <map>
#include <numeric>
#include <omp.h>
#include <set>
#include <sstream>
#include <stdexcept>
#include <stdint.h>
#include <string>
#include <sys/stat.h>
#include <sys/types.h>
#include <tuple>
#include <utility>
#include <vector>
#include <fcntl.h>
#include <unistd.h>
#include "tinyxml2.h"

#define private public
#include "cUranusModel.h"
#include "PressureSolverUran.h"
#include "PressureSolver.h"
#include "SaturationAdjustmentUran.h"
#include "ChemistryUran.h"
#include "TurbulenceUran.h"
#include "PrecipitationUran.h"
#include "BC_Uran.h"
#include "ConvectiveAdjustmentUran.h"
#undef private

namespace {

cUranusModel* g_model = nullptr;
int g_saved_stdout = -1;

void quiet_begin(){
    fflush(stdout); std::cout.flush();
    g_saved_stdout = dup(1);
    int fd = open("/dev/null", O_WRONLY);
    if(fd >= 0){ dup2(fd, 1); close(fd); }
}
void quiet_end(){
    fflush(stdout); std::cout.flush();
    if(g_saved_stdout >= 0){ dup2(g_saved_stdout, 1); close(g_saved_stdout); g_saved_stdout = -1; }
}
int g_quiet = 1;
struct Quiet {
    Quiet(){ if(g_quiet) quiet_begin(); }
    ~Quiet(){ if(g_quiet) quiet_end(); }
};

Array* field(const char* name){
    cUranusModel& m = *g_model;
    struct E { const char* n; Array* a; };
    const E tab[] = {
        {"t", &m.t}, {"u", &m.u}, {"v", &m.v}, {"w", &m.w},
        {"ch4", &m.ch4}, {"ch4_cloud", &m.ch4_cloud}, {"ch4_ice", &m.ch4_ice},
        {"h2o", &m.h2o}, {"h2o_cloud", &m.h2o_cloud}, {"h2o_ice", &m.h2o_ice},
        {"h2s", &m.h2s}, {"h2s_cloud", &m.h2s_cloud}, {"h2s_ice", &m.h2s_ice},
        {"nh3", &m.nh3}, {"nh3_cloud", &m.nh3_cloud}, {"nh3_ice", &m.nh3_ice},
        {"nh4sh", &m.nh4sh}, {"tke", &m.tke}, {"dis", &m.dis},
        {"tn", &m.tn}, {"un", &m.un}, {"vn", &m.vn}, {"wn", &m.wn},
        {"ch4n", &m.ch4n}, {"ch4_cloudn", &m.ch4_cloudn}, {"ch4_icen", &m.ch4_icen},
        {"h2on", &m.h2on}, {"h2o_cloudn", &m.h2o_cloudn}, {"h2o_icen", &m.h2o_icen},
        {"h2sn", &m.h2sn}, {"h2s_cloudn", &m.h2s_cloudn}, {"h2s_icen", &m.h2s_icen},
        {"nh3n", &m.nh3n}, {"nh3_cloudn", &m.nh3_cloudn}, {"nh3_icen", &m.nh3_icen},
        {"nh4shn", &m.nh4shn}, {"tken", &m.tken}, {"disn", &m.disn},
        {"p_dyn", &m.p_dyn}, {"p_hydro", &m.p_hydro}, {"p_stat", &m.p_stat},
        {"nue", &m.nue}, {"thermalmassflux", &m.thermalmassflux}, {"Q_precip", &m.Q_precip},
        {"S_precip_ch4", &m.S_precip_ch4}, {"S_precip_ch4_cloud", &m.S_precip_ch4_cloud},
        {"S_precip_ch4_ice", &m.S_precip_ch4_ice},
        {"S_precip_h2o", &m.S_precip_h2o}, {"S_precip_h2o_cloud", &m.S_precip_h2o_cloud},
        {"S_precip_h2o_ice", &m.S_precip_h2o_ice},
        {"S_precip_h2s", &m.S_precip_h2s}, {"S_precip_h2s_cloud", &m.S_precip_h2s_cloud},
        {"S_precip_h2s_ice", &m.S_precip_h2s_ice},
        {"S_precip_nh3", &m.S_precip_nh3}, {"S_precip_nh3_cloud", &m.S_precip_nh3_cloud},
        {"S_precip_nh3_ice", &m.S_precip_nh3_ice},
        {"massflux_h2s", &m.massflux_h2s}, {"massflux_nh3", &m.massflux_nh3},
        {"massflux_nh4sh", &m.massflux_nh4sh}, {"fluxlim_nh4sh", &m.fluxlim_nh4sh},
        {"rho_mix", &m.rho_mix}, {"tke_source", &m.tke_source}, {"dis_source", &m.dis_source},
        {"difflux_h2s", &m.difflux_h2s}, {"difflux_nh3", &m.difflux_nh3}, {"difflux_nh4sh", &m.difflux_nh4sh},
        {"prod", &m.prod},
        {"rhs_t", &m.rhs_t}, {"rhs_u", &m.rhs_u}, {"rhs_v", &m.rhs_v}, {"rhs_w", &m.rhs_w},
        {"rhs_ch4", &m.rhs_ch4}, {"rhs_tke", &m.rhs_tke}, {"rhs_dis", &m.rhs_dis},
        {"rhs_nh4sh", &m.rhs_nh4sh},
        {"aux_u", &m.aux_u}, {"aux_v", &m.aux_v}, {"aux_w", &m.aux_w},
        {"acc_t", &m.acc_t}, {"acc_u", &m.acc_u},
    };
    for(const E& e : tab) if(std::strcmp(e.n, name) == 0) return e.a;
    return nullptr;
}

std::vector<double>* vec(const char* name){
    cUranusModel& m = *g_model;
    if(!std::strcmp(name, "p_baro"))         return &m.p_baro;
    if(!std::strcmp(name, "p_b0"))           return &m.p_b0;
    if(!std::strcmp(name, "p_bfollow"))      return &m.p_bfollow;
    if(!std::strcmp(name, "buoy_ref_level")) return &m.buoy_ref_level;
    return nullptr;
}

}  // namespace

extern "C" {

// The model, for the driver glue compiled beside this harness (b200_glue.cpp).
void* ref_model_ptr(){ return g_model; }

int ref_dims(int* im, int* jm, int* km){
    *im = cUranusModel::im; *jm = cUranusModel::jm; *km = cUranusModel::km;
    return 0;
}

void ref_set_quiet(int q){ g_quiet = q; }

// Construct the model and run its initialisation (Run() with nm = 0). outdir receives the
// directory the reference creates for its output files; nothing is written into it for nm = 0.
int ref_create(const char* outdir){
    if(g_model) return 0;
    Quiet q_;
    g_model = new cUranusModel();
    g_model->nm = 0;
    g_model->paraview_flag = false;
    g_model->output_path = std::string(outdir ? outdir : "/tmp/aturan_ref_out") + "/";
    g_model->Run();
    return 0;
}

// The same, then nm iterations of the model's own loop (planet/cUranusModel.cpp:952-1396) inside
// Run(); checkpoint is set past nm so that the loop writes no files and prints no reports.
int ref_create_loop(const char* outdir, int nm){
    if(g_model) return -1;
    Quiet q_;
    g_model = new cUranusModel();
    g_model->nm = nm;
    g_model->checkpoint = nm + 1000000;
    g_model->paraview_flag = false;
    g_model->output_path = std::string(outdir ? outdir : "/tmp/aturan_ref_out") + "/";
    g_model->Run();
    return 0;
}

int ref_get(const char* name, double* out){
    Array* a = field(name);
    if(!a || !a->x) return -1;
    const int im = cUranusModel::im, jm = cUranusModel::jm, km = cUranusModel::km;
    for(int i = 0; i < im; i++) for(int j = 0; j < jm; j++)
        std::memcpy(out + ((size_t)i * jm + j) * km, a->x[i][j], sizeof(double) * km);
    return 0;
}

int ref_set(const char* name, const double* in){
    Array* a = field(name);
    if(!a || !a->x) return -1;
    const int im = cUranusModel::im, jm = cUranusModel::jm, km = cUranusModel::km;
    for(int i = 0; i < im; i++) for(int j = 0; j < jm; j++)
        std::memcpy(a->x[i][j], in + ((size_t)i * jm + j) * km, sizeof(double) * km);
    return 0;
}

long ref_vec_size(const char* name){
    std::vector<double>* v = vec(name);
    return v ? (long)v->size() : -1;
}

int ref_get_vec(const char* name, double* out){
    std::vector<double>* v = vec(name);
    if(!v) return -1;
    std::memcpy(out, v->data(), sizeof(double) * v->size());
    return 0;
}

int ref_set_vec(const char* name, const double* in, long n){
    std::vector<double>* v = vec(name);
    if(!v) return -1;
    v->assign(in, in + n);
    return 0;
}

// Scalars of the initialised model that the hot path reads (the derived densities and heat
// capacities are set by ThermalPropertiesUran and the T-anchor rescale, cUranusModel.cpp:498-526).
int ref_scalar(const char* name, double* out){
    cUranusModel& m = *g_model;
    struct E { const char* n; double v; };
    const E tab[] = {
        {"r_mix", m.r_mix}, {"R_mix", m.R_mix}, {"cp_mix", m.cp_mix}, {"mue_mix", m.mue_mix},
        {"gam", m.gam}, {"dt", m.dt}, {"L_atm", m.L_atm}, {"u_0", m.u_0}, {"t_ref", m.t_ref},
        {"g", m.g}, {"omega", m.omega}, {"re", m.re}, {"pr", m.pr}, {"Coriolis", m.Coriolis},
        {"centrifugal", m.centrifugal}, {"buoyancy", m.buoyancy},
        {"chemical_reaction", m.chemical_reaction}, {"R_ref", m.R_ref}, {"p_ref", m.p_ref},
        {"r_h2", m.r_h2}, {"r_he", m.r_he}, {"r_ch4", m.r_ch4}, {"cp_h2", m.cp_h2},
        {"cp_he", m.cp_he}, {"cp_ch4", m.cp_ch4}, {"sc_ch4", m.sc_ch4}, {"sc_h2o", m.sc_h2o},
        {"sc_h2s", m.sc_h2s}, {"sc_nh3", m.sc_nh3}, {"sc_nh4sh", m.sc_nh4sh},
        {"alpha_sponge", m.alpha_sponge}, {"r_p_nh4sh", m.r_p_nh4sh},
        {"rho_cond_nh4sh", m.rho_cond_nh4sh},
        {"turb_active", m.turb_active ? 1.0 : 0.0},
        {"t_0_h2o", m.t_0_h2o}, {"t_00_h2o", m.t_00_h2o}, {"t_0_h2s", m.t_0_h2s},
        {"t_00_h2s", m.t_00_h2s}, {"t_0_nh3", m.t_0_nh3}, {"t_00_nh3", m.t_00_nh3},
        {"t_0_ch4", m.t_0_ch4}, {"t_00_ch4", m.t_00_ch4},
        {"ep_h2o", m.ep_h2o}, {"ep_h2s", m.ep_h2s}, {"ep_nh3", m.ep_nh3}, {"ep_ch4", m.ep_ch4},
        {"lv_h2o", m.lv_h2o}, {"lv_h2s", m.lv_h2s}, {"lv_nh3", m.lv_nh3}, {"lv_ch4", m.lv_ch4},
        {"ls_h2o", m.ls_h2o}, {"ls_h2s", m.ls_h2s}, {"ls_nh3", m.ls_nh3}, {"ls_ch4", m.ls_ch4},
        {"C_h2o", m.C_h2o}, {"C_h2s", m.C_h2s}, {"C_nh3", m.C_nh3}, {"C_ch4", m.C_ch4},
        {"L0_h2o", m.L0_h2o}, {"L0_h2s", m.L0_h2s}, {"L0_nh3", m.L0_nh3}, {"L0_ch4", m.L0_ch4},
        {"R_h2o", m.R_h2o}, {"R_h2s", m.R_h2s}, {"R_nh3", m.R_nh3}, {"R_ch4", m.R_ch4},
        {"del_alf_h2o", m.del_alf_h2o}, {"del_alf_h2s", m.del_alf_h2s},
        {"del_alf_nh3", m.del_alf_nh3}, {"del_alf_ch4", m.del_alf_ch4},
        {"del_bet_h2o", m.del_bet_h2o}, {"del_bet_h2s", m.del_bet_h2s},
        {"del_bet_nh3", m.del_bet_nh3}, {"del_bet_ch4", m.del_bet_ch4},
        {"C_h2o_ice", m.C_h2o_ice}, {"L0_h2o_ice", m.L0_h2o_ice},
        {"del_alf_h2o_ice", m.del_alf_h2o_ice}, {"del_bet_h2o_ice", m.del_bet_h2o_ice},
        {"C_nh3_ice", m.C_nh3_ice}, {"L0_nh3_ice", m.L0_nh3_ice},
        {"del_alf_nh3_ice", m.del_alf_nh3_ice}, {"del_bet_nh3_ice", m.del_bet_nh3_ice},
        {"C_ch4_ice", m.C_ch4_ice}, {"L0_ch4_ice", m.L0_ch4_ice},
        {"del_alf_ch4_ice", m.del_alf_ch4_ice}, {"del_bet_ch4_ice", m.del_bet_ch4_ice},
        {"nh4sh_eq", ChemistryUran::nh4sh_eq() ? 1.0 : 0.0},
    };
    for(const E& e : tab) if(std::strcmp(e.n, name) == 0){ *out = e.v; return 0; }
    return -1;
}

// The radial and colatitude coordinates as the model built them (Array_1D::Coordinates).
int ref_coords(double* rad, double* the){
    for(int i = 0; i < cUranusModel::im; i++) rad[i] = g_model->rad.z[i];
    for(int j = 0; j < cUranusModel::jm; j++) the[j] = g_model->the.z[j];
    return 0;
}

double ref_cp_lapse(double T){ return CpH2::cp_lapse(*g_model, T); }

// planet/RungeKutta_Uran_Turb.cpp:179-404 (which itself runs :18 and :62 first).
int ref_rk4(){ Quiet q_; g_model->RungeKuttaUran(); return 0; }

// planet/RungeKutta_Uran_Turb.cpp:18-37 and :62-177, as RungeKuttaUran calls them.
int ref_hydro(int advance_follow){
    Quiet q_;
    g_model->computeBuoyancyRefLevel();
    g_model->computeHydrostaticPressure(advance_follow != 0);
    return 0;
}

// The default solver, planet/PressureSolverUran.h:33-250.
int ref_pressure_uran(){ Quiet q_; PressureSolverUran(*g_model).run(); return 0; }

// The shared red-black solver, planet/PressureSolver.h:145-766, with ATURAN_PRESS_SWEEPS sweeps
// (that knob is read on every call, :174).
int ref_pressure_shared(int sweeps){
    Quiet q_;
    char buf[32]; snprintf(buf, sizeof buf, "%d", sweeps);
    setenv("ATURAN_PRESS_SWEEPS", buf, 1);
    PressureSolver<cUranusModel>(*g_model).run();
    unsetenv("ATURAN_PRESS_SWEEPS");
    return 0;
}

// One saturation adjustment with exactly the arguments of the iteration loop,
// planet/cUranusModel.cpp:998-1027. gas: 0 = H2O, 1 = H2S, 2 = NH3, 3 = CH4.
int ref_satadj(int gas){
    Quiet q_;
    cUranusModel& m = *g_model;
    SaturationAdjustmentUran s(m);
    switch(gas){
    case 0: s.run("H2O", m.coeff_h2o_A, m.coeff_h2o_B, m.coeff_h2o_A_i, m.coeff_h2o_B_i,
                  m.t_0_h2o, m.t_00_h2o, m.ep_h2o, m.lv_h2o, m.ls_h2o, m.cp_h2o, m.r_h2o,
                  m.C_h2o, m.L0_h2o, m.R_h2o, m.del_alf_h2o, m.del_bet_h2o, m.m_h2o,
                  m.h2o, m.h2o_cloud, m.h2o_ice); break;
    case 1: s.run("H2S", m.coeff_h2s_A, m.coeff_h2s_B, m.coeff_h2s_A_i, m.coeff_h2s_B_i,
                  m.t_0_h2s, m.t_00_h2s, m.ep_h2s, m.lv_h2s, m.ls_h2s, m.cp_h2s, m.r_h2s,
                  m.C_h2s, m.L0_h2s, m.R_h2s, m.del_alf_h2s, m.del_bet_h2s, m.m_h2s,
                  m.h2s, m.h2s_cloud, m.h2s_ice); break;
    case 2: s.run("NH3", m.coeff_nh3_A, m.coeff_nh3_B, m.coeff_nh3_A_i, m.coeff_nh3_B_i,
                  m.t_0_nh3, m.t_00_nh3, m.ep_nh3, m.lv_nh3, m.ls_nh3, m.cp_nh3, m.r_nh3,
                  m.C_nh3, m.L0_nh3, m.R_nh3, m.del_alf_nh3, m.del_bet_nh3, m.m_nh3,
                  m.nh3, m.nh3_cloud, m.nh3_ice); break;
    case 3: s.run("CH4", m.coeff_ch4_A, m.coeff_ch4_B, m.coeff_ch4_A_i, m.coeff_ch4_B_i,
                  m.t_0_ch4, m.t_00_ch4, m.ep_ch4, m.lv_ch4, m.ls_ch4, m.cp_ch4, m.r_ch4,
                  m.C_ch4, m.L0_ch4, m.R_ch4, m.del_alf_ch4, m.del_bet_ch4, m.m_ch4,
                  m.ch4, m.ch4_cloud, m.ch4_ice); break;
    default: return -1;
    }
    return 0;
}

// ATURAN_RK_SCALAR_SYNC=2 (its default) copy of the adjusted condensables and T into the n-level
// copies, planet/cUranusModel.cpp:1049-1073, written out here because it is inline in Run().
int ref_sync_ncopies(){
    cUranusModel& m = *g_model;
    const bool nh4 = ChemistryUran::nh4sh_eq();
    for(int i = 0; i < m.im; i++) for(int j = 0; j < m.jm; j++) for(int k = 0; k < m.km; k++){
        m.h2on.x[i][j][k] = m.h2o.x[i][j][k];  m.h2o_cloudn.x[i][j][k] = m.h2o_cloud.x[i][j][k];
        m.h2o_icen.x[i][j][k] = m.h2o_ice.x[i][j][k];
        m.h2sn.x[i][j][k] = m.h2s.x[i][j][k];  m.h2s_cloudn.x[i][j][k] = m.h2s_cloud.x[i][j][k];
        m.h2s_icen.x[i][j][k] = m.h2s_ice.x[i][j][k];
        m.nh3n.x[i][j][k] = m.nh3.x[i][j][k];  m.nh3_cloudn.x[i][j][k] = m.nh3_cloud.x[i][j][k];
        m.nh3_icen.x[i][j][k] = m.nh3_ice.x[i][j][k];
        m.ch4n.x[i][j][k] = m.ch4.x[i][j][k];  m.ch4_cloudn.x[i][j][k] = m.ch4_cloud.x[i][j][k];
        m.ch4_icen.x[i][j][k] = m.ch4_ice.x[i][j][k];
        m.tn.x[i][j][k] = m.t.x[i][j][k];
        if(nh4) m.nh4shn.x[i][j][k] = m.nh4sh.x[i][j][k];
    }
    return 0;
}

int ref_restore_var(){ g_model->restoreVar(1.0); return 0; }

// The calls cUranusModel.cpp:1218-1248 makes after RungeKuttaUran, each exposed alone so that a
// test composes them in the model's order. The boundary passes and the clamp read their knobs
// from the reference's own ATURAN_* environment variables (once per process); the filter takes
// its axes and strength as the model's call site passes them.
int ref_damp_wiggles(const char* name, int along_i, int along_j, int along_k, double strength){
    Array* a = field(name);
    if(!a || !a->x) return -1;
    AtomUtils::damp_wiggles(*a, nullptr, along_i != 0, along_j != 0, along_k != 0, strength);
    return 0;
}
int ref_bc_radius(){ BC_Uran(*g_model).bcRadius(); return 0; }
int ref_bc_theta(){ BC_Uran(*g_model).bcTheta(); return 0; }
int ref_bc_phi(){ BC_Uran(*g_model).bcPhi(); return 0; }
// clampNegativeSpecies with its cumulative sums reset first, so they hold this call's.
int ref_clamp_species(double* added, long* cells){
    cUranusModel& m = *g_model;
    m.clamp_added.clear();
    m.clamp_cells.clear();
    m.clampNegativeSpecies();
    for(size_t n = 0; n < m.clamp_added.size(); n++){ added[n] = m.clamp_added[n]; cells[n] = m.clamp_cells[n]; }
    return (int)m.clamp_added.size();
}
int ref_geo_balance(){ return cUranusModel::geo_balance() ? 1 : 0; }

// The moist convective adjustment as cUranusModel.cpp:1276-1292 calls it: the same gas list
// (H2O, NH3, H2S with its liquid set for both phases, CH4), NH4SH as a condensed tracer carrying
// its formation heat when the NH4SH equilibrium is on, and chrom when ATURAN_CHROM is set.
int ref_mca(){
    Quiet q_;
    cUranusModel& m = *g_model;
    typedef MoistConvectiveAdjustmentUran::Gas Gas_;
    typedef MoistConvectiveAdjustmentUran::Tracer Tr_;
    std::vector<Gas_> gases = {
        { "H2O", &m.h2o, &m.h2o_cloud, &m.h2o_ice, m.ep_h2o, m.lv_h2o, m.ls_h2o, m.t_0_h2o,
          m.C_h2o, m.L0_h2o, m.R_h2o, m.del_alf_h2o, m.del_bet_h2o,
          m.C_h2o_ice, m.L0_h2o_ice, m.del_alf_h2o_ice, m.del_bet_h2o_ice, m.t_00_h2o },
        { "NH3", &m.nh3, &m.nh3_cloud, &m.nh3_ice, m.ep_nh3, m.lv_nh3, m.ls_nh3, m.t_0_nh3,
          m.C_nh3, m.L0_nh3, m.R_nh3, m.del_alf_nh3, m.del_bet_nh3,
          m.C_nh3_ice, m.L0_nh3_ice, m.del_alf_nh3_ice, m.del_bet_nh3_ice, m.t_00_nh3 },
        { "H2S", &m.h2s, &m.h2s_cloud, &m.h2s_ice, m.ep_h2s, m.lv_h2s, m.ls_h2s, m.t_0_h2s,
          m.C_h2s, m.L0_h2s, m.R_h2s, m.del_alf_h2s, m.del_bet_h2s,
          m.C_h2s, m.L0_h2s, m.del_alf_h2s, m.del_bet_h2s, m.t_00_h2s },
        { "CH4", &m.ch4, &m.ch4_cloud, &m.ch4_ice, m.ep_ch4, m.lv_ch4, m.ls_ch4, m.t_0_ch4,
          m.C_ch4, m.L0_ch4, m.R_ch4, m.del_alf_ch4, m.del_bet_ch4,
          m.C_ch4_ice, m.L0_ch4_ice, m.del_alf_ch4_ice, m.del_bet_ch4_ice, m.t_00_ch4 } };
    const double L_nh4sh = ChemistryUran::nh4sh_eq() ? ChemistryUran::nh4sh_formation_heat() : 0.0;
    std::vector<Tr_> tracers = { { "NH4SH", &m.nh4sh, 0.0, true, L_nh4sh } };
    if(cUranusModel::chrom_on()) tracers.push_back({ "chrom", &m.chrom, 0.0, false, 0.0 });
    MoistConvectiveAdjustmentUran(m, gases, tracers).run();
    return 0;
}


// The chemistry as the loop calls it: EquilibriumNH4SH("loop") after the saturation adjustments
// (cUranusModel.cpp:1034) and the forcing sequence of :1074-1087, filters included.
int ref_chem_eq(){ Quiet q_; ChemistryUran(*g_model).EquilibriumNH4SH("loop"); return 0; }
int ref_chem_forcing(){
    Quiet q_;
    cUranusModel& m = *g_model;
    ChemistryUran(m).DiffMassFluxUran();
    AtomUtils::damp_wiggles(m.difflux_h2s,     nullptr, true, true, true);
    AtomUtils::damp_wiggles(m.difflux_nh3,     nullptr, true, true, true);
    AtomUtils::damp_wiggles(m.difflux_nh4sh,   nullptr, true, true, true);
    AtomUtils::damp_wiggles(m.thermalmassflux, nullptr, true, true, true);
    ChemistryUran(m).ChemMassRateUran();
    ChemistryUran(m).FluxLimiterNH4SH();
    AtomUtils::damp_wiggles(m.massflux_h2s,   nullptr, true, true, true);
    AtomUtils::damp_wiggles(m.massflux_nh3,   nullptr, true, true, true);
    AtomUtils::damp_wiggles(m.massflux_nh4sh, nullptr, true, true, true);
    AtomUtils::damp_wiggles(m.fluxlim_nh4sh,  nullptr, true, true, true);
    return 0;
}
// The chemistry's constants and resolved knobs.
int ref_chem_scalar(const char* name, double* out){
    cUranusModel& m = *g_model;
    struct E { const char* n; double v; };
    const E tab[] = {
        {"m_nh3", m.m_nh3}, {"m_h2s", m.m_h2s}, {"m_nh4sh", m.m_nh4sh}, {"c_mix", m.c_mix},
        {"D_nh4sh", m.D_nh4sh}, {"DT_nh4sh", m.DT_nh4sh},
        {"cp_nh3", m.cp_nh3}, {"cp_h2s", m.cp_h2s}, {"cp_nh4sh", m.cp_nh4sh},
        {"k_nh3", m.k_nh3}, {"k_h2s", m.k_h2s}, {"k_nh4sh", m.k_nh4sh},
        {"polar_floor", ATPhys::polar_divisor_floor<cUranusModel>()},
        {"nh4sh_eq", ChemistryUran::nh4sh_eq() ? 1.0 : 0.0},
        {"phi_periodic", ATPhys::phi_periodic<cUranusModel>() ? 1.0 : 0.0},
        {"coord_stretching", m.coord_stretching ? 1.0 : 0.0},
    };
    for(const E& e : tab) if(std::strcmp(e.n, name) == 0){ *out = e.v; return 0; }
    return -1;
}


// The turbulence closure as the loop calls it (cUranusModel.cpp:1270), and its resolved knobs.
int ref_turbulence(){ Quiet q_; TurbulenceUran(*g_model).run(); return 0; }
int ref_turb_scalar(const char* name, double* out){
    cUranusModel& m = *g_model;
    const std::string tm = m.turb_model;
    const char* curv_e = getenv("ATURAN_TURB_CURV");
    const char* buoy_e = getenv("ATURAN_TURB_BUOY");
    struct E { const char* n; double v; };
    const E tab[] = {
        {"active", m.turb_active ? 1.0 : 0.0},
        {"model", tm == "k_epsilon" ? 0.0 : (tm == "k_omega" ? 1.0 : 2.0)},
        {"turb_free", (double)TurbulenceUran::turb_free()},
        {"clamp_pass", (double)TurbulenceUran::turb_clamp_pass()},
        {"curv", (!curv_e || atoi(curv_e) != 0) ? 1.0 : 0.0},
        {"buoy", buoy_e ? (double)atoi(buoy_e) : (double)cUranusModel::turb_default_buoy()},
        {"abl_taper", (double)TurbulenceUran::abl_taper()},
        {"phi_periodic", ATPhys::phi_periodic<cUranusModel>() ? 1.0 : 0.0},
        {"nue_max", TurbulenceUran::nue_max_phys()},
        {"k_bg", TurbulenceUran::turb_k_bg()},
        {"bc_turb_active", m.bc_turb_active() ? 1.0 : 0.0},
    };
    for(const E& e : tab) if(std::strcmp(e.n, name) == 0){ *out = e.v; return 0; }
    return -1;
}


// The precipitation as the loop calls it (cUranusModel.cpp:1037), and its resolved knobs.
int ref_precipitation(){ Quiet q_; PrecipitationUran(*g_model).run(); return 0; }
int ref_precip_scalar(const char* name, double* out){
    struct E { const char* n; double v; };
    const E tab[] = {
        {"coupling", PrecipitationUran::coupling_on() ? 1.0 : 0.0},
        {"h2s", cUranusModel::precip_h2s_on() ? 1.0 : 0.0},
        {"rate_scale", PrecipitationUran::rate_scale()},
    };
    for(const E& e : tab) if(std::strcmp(e.n, name) == 0){ *out = e.v; return 0; }
    return -1;
}

}  // extern "C"
