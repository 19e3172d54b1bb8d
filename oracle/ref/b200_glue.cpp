// The driver glue a maintainer adds to the ATURAN reference to run its iteration loop through
// libaturan_b200 (include/aturan_b200.h), compiled here against the reference's unmodified headers
// and objects as TEST INFRASTRUCTURE (oracle/Makefile, target `glue`): tests/test_gpu_dropin.py
// runs the reference's own initialised model through it and compares the result with the oracle.
//
// What the glue does is what a `#ifdef ATURAN_USE_B200` block in cUranusModel::Run would do:
//   b200_params       the model's initialised constants -> aturan_params
//   b200_iter_params  the knobs, resolved as the reference's call sites resolve them
//   b200_transfer     every field the library holds, between the model's jagged Arrays (and the
//                     flat p_baro / p_b0 / p_bfollow vectors) and the device, in [i][j][k] order
//   glue_run          create a context, upload once, run iterations 1..n of the loop on the device
//                     (aturan_iteration), download once, back into the model's own fields
// The state stays on the device between the iterations; nothing of the loop runs on the host.

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
#include "ChemistryUran.h"
#include "TurbulenceUran.h"
#include "PrecipitationUran.h"
#undef private

#include "aturan_b200.h"

extern "C" void* ref_model_ptr();   // the harness's model (ref_harness.cpp)

namespace {

aturan_params b200_params(cUranusModel& m, int precision){
    aturan_params p;
    aturan_params_default(&p);
    p.im = cUranusModel::im; p.jm = cUranusModel::jm; p.km = cUranusModel::km;
    p.precision = precision;
    p.dt = m.dt;
    p.L_atm = m.L_atm; p.u_0 = m.u_0; p.t_ref = m.t_ref; p.g = m.g; p.omega = m.omega;
    p.re = m.re; p.pr = m.pr; p.Coriolis = m.Coriolis; p.centrifugal = m.centrifugal;
    p.buoyancy = m.buoyancy; p.chemical_reaction = m.chemical_reaction; p.R_ref = m.R_ref; p.p_ref = m.p_ref;
    p.r_mix = m.r_mix; p.R_mix = m.R_mix; p.cp_mix = m.cp_mix; p.mue_mix = m.mue_mix;
    p.r_h2 = m.r_h2; p.r_he = m.r_he; p.r_ch4 = m.r_ch4; p.cp_h2 = m.cp_h2; p.cp_he = m.cp_he; p.cp_ch4 = m.cp_ch4;
    p.sc_ch4 = m.sc_ch4; p.sc_h2o = m.sc_h2o; p.sc_h2s = m.sc_h2s; p.sc_nh3 = m.sc_nh3; p.sc_nh4sh = m.sc_nh4sh;
    p.alpha_sponge = m.alpha_sponge; p.r_p_nh4sh = m.r_p_nh4sh; p.rho_cond_nh4sh = m.rho_cond_nh4sh;
    p.turb_active = m.turb_active ? 1 : 0;
    p.nh4sh_sync = ChemistryUran::nh4sh_eq() ? 1 : 0;
    p.sinthe_min = cUranusModel::sinthe_min();
    // per gas, the arguments SaturationAdjustmentUran::run passes on (SaturationAdjustmentUran.cpp:
    // 222-238), in the library's order H2O, H2S, NH3, CH4; H2S has no ice set of its own
    const aturan_gas h2o = { m.t_0_h2o, m.t_00_h2o, m.ep_h2o, m.lv_h2o, m.ls_h2o, m.C_h2o, m.L0_h2o, m.R_h2o,
                             m.del_alf_h2o, m.del_bet_h2o, m.C_h2o_ice, m.L0_h2o_ice, m.del_alf_h2o_ice, m.del_bet_h2o_ice };
    const aturan_gas h2s = { m.t_0_h2s, m.t_00_h2s, m.ep_h2s, m.lv_h2s, m.ls_h2s, m.C_h2s, m.L0_h2s, m.R_h2s,
                             m.del_alf_h2s, m.del_bet_h2s, m.C_h2s, m.L0_h2s, m.del_alf_h2s, m.del_bet_h2s };
    const aturan_gas nh3 = { m.t_0_nh3, m.t_00_nh3, m.ep_nh3, m.lv_nh3, m.ls_nh3, m.C_nh3, m.L0_nh3, m.R_nh3,
                             m.del_alf_nh3, m.del_bet_nh3, m.C_nh3_ice, m.L0_nh3_ice, m.del_alf_nh3_ice, m.del_bet_nh3_ice };
    const aturan_gas ch4 = { m.t_0_ch4, m.t_00_ch4, m.ep_ch4, m.lv_ch4, m.ls_ch4, m.C_ch4, m.L0_ch4, m.R_ch4,
                             m.del_alf_ch4, m.del_bet_ch4, m.C_ch4_ice, m.L0_ch4_ice, m.del_alf_ch4_ice, m.del_bet_ch4_ice };
    p.gas[0] = h2o; p.gas[1] = h2s; p.gas[2] = nh3; p.gas[3] = ch4;
    return p;
}

aturan_iter_params b200_iter_params(cUranusModel& m){
    aturan_iter_params ip;
    aturan_iter_params_default(&ip);
    const bool geo = cUranusModel::geo_balance();
    ip.damp_p_horiz = geo ? 0.0 : 1.0;                              // cUranusModel.cpp:979-980
    ip.post.damp_t_j = !geo;                                        // :1216-1217
    ip.post.lid_vw = geo ? 2 : 0;                                   // BC_Uran.h:155
    ip.post.vel_shapiro = geo ? 0.0 : 1.0;                          // cUranusModel.cpp:1229-1230
    ip.chemistry = ChemistryUran::nh4sh_eq() ? 1 : 0;
    ip.turbulence = m.turb_active ? 1 : 0;
    ip.chem.m_nh3 = m.m_nh3; ip.chem.m_h2s = m.m_h2s; ip.chem.m_nh4sh = m.m_nh4sh; ip.chem.c_mix = m.c_mix;
    ip.chem.D_nh4sh = m.D_nh4sh; ip.chem.DT_nh4sh = m.DT_nh4sh;
    ip.chem.cp_nh3 = m.cp_nh3; ip.chem.cp_h2s = m.cp_h2s; ip.chem.cp_nh4sh = m.cp_nh4sh;
    ip.chem.k_nh3 = m.k_nh3; ip.chem.k_h2s = m.k_h2s; ip.chem.k_nh4sh = m.k_nh4sh;
    ip.chem.polar_floor = ATPhys::polar_divisor_floor<cUranusModel>();
    ip.turb.nue_max = TurbulenceUran::nue_max_phys(); ip.turb.k_bg = TurbulenceUran::turb_k_bg();
    ip.precip.rate_scale = PrecipitationUran::rate_scale();
    ip.precip.coupling = PrecipitationUran::coupling_on() ? 1 : 0;
    ip.precip.h2s = cUranusModel::precip_h2s_on() ? 1 : 0;
    return ip;
}

// aturan_field id -> the model's Array (or the flat vector of the hydrostatic split)
Array* b200_field(cUranusModel& m, int id){
    Array* tab[ATURAN_NFIELDS] = {
        &m.t, &m.u, &m.v, &m.w, &m.ch4, &m.ch4_cloud, &m.ch4_ice, &m.h2o, &m.h2o_cloud, &m.h2o_ice,
        &m.h2s, &m.h2s_cloud, &m.h2s_ice, &m.nh3, &m.nh3_cloud, &m.nh3_ice, &m.nh4sh, &m.tke, &m.dis,
        &m.tn, &m.un, &m.vn, &m.wn, &m.ch4n, &m.ch4_cloudn, &m.ch4_icen, &m.h2on, &m.h2o_cloudn, &m.h2o_icen,
        &m.h2sn, &m.h2s_cloudn, &m.h2s_icen, &m.nh3n, &m.nh3_cloudn, &m.nh3_icen, &m.nh4shn, &m.tken, &m.disn,
        &m.p_dyn, &m.p_hydro, &m.p_stat,
        &m.nue, &m.thermalmassflux, &m.Q_precip,
        &m.S_precip_ch4, &m.S_precip_ch4_cloud, &m.S_precip_ch4_ice,
        &m.S_precip_h2o, &m.S_precip_h2o_cloud, &m.S_precip_h2o_ice,
        &m.S_precip_h2s, &m.S_precip_h2s_cloud, &m.S_precip_h2s_ice,
        &m.S_precip_nh3, &m.S_precip_nh3_cloud, &m.S_precip_nh3_ice,
        &m.massflux_h2s, &m.massflux_nh3, &m.massflux_nh4sh, &m.fluxlim_nh4sh,
        &m.rho_mix, &m.tke_source, &m.dis_source,
        nullptr, nullptr, nullptr,                                   // p_baro, p_b0, p_bfollow: vectors
        &m.rhs_u, &m.rhs_v, &m.rhs_w, &m.aux_u, &m.aux_v, &m.aux_w,
        &m.difflux_h2s, &m.difflux_nh3, &m.difflux_nh4sh, &m.prod,
    };
    return (id >= 0 && id < ATURAN_NFIELDS) ? tab[id] : nullptr;
}
std::vector<double>* b200_vec(cUranusModel& m, int id){
    if(id == ATURAN_P_BARO) return &m.p_baro;
    if(id == ATURAN_P_B0) return &m.p_b0;
    if(id == ATURAN_P_BFOLLOW) return &m.p_bfollow;
    return nullptr;
}

// Every field between the model and the device; up = host -> device.
int b200_transfer(aturan_ctx* ctx, cUranusModel& m, bool up){
    const int im = cUranusModel::im, jm = cUranusModel::jm, km = cUranusModel::km;
    const size_t N = (size_t)im * jm * km;
    std::vector<double> buf(N);
    for(int id = 0; id < ATURAN_NFIELDS; id++){
        if(std::vector<double>* v = b200_vec(m, id)){
            if(v->size() != N){                                      // empty without the hydrostatic split
                if(up) continue;
                v->assign(N, 0.0);
            }
            const int rc = up ? aturan_upload(ctx, id, v->data()) : aturan_download(ctx, id, v->data());
            if(rc) return rc;
            continue;
        }
        Array* a = b200_field(m, id);
        if(!a || !a->x) return ATURAN_E_INVALID;
        if(up){
            for(int i = 0; i < im; i++) for(int j = 0; j < jm; j++)
                std::memcpy(&buf[((size_t)i * jm + j) * km], a->x[i][j], sizeof(double) * km);
            const int rc = aturan_upload(ctx, id, buf.data());
            if(rc) return rc;
        } else {
            const int rc = aturan_download(ctx, id, buf.data());
            if(rc) return rc;
            for(int i = 0; i < im; i++) for(int j = 0; j < jm; j++)
                std::memcpy(a->x[i][j], &buf[((size_t)i * jm + j) * km], sizeof(double) * km);
        }
    }
    return ATURAN_OK;
}

}  // namespace

extern "C" {

// Iterations 1..n of the model's loop on the device from the model's current state, the result
// written back into the model's fields. precision: enum aturan_precision. Returns an aturan_status.
int glue_run(int n, int precision){
    cUranusModel* m = static_cast<cUranusModel*>(ref_model_ptr());
    if(!m || n < 0) return ATURAN_E_INVALID;
    const aturan_params p = b200_params(*m, precision);
    aturan_ctx* ctx = nullptr;
    std::fprintf(stderr, "glue_run: creating the context\n");
    int rc = aturan_ctx_create(&p, &ctx);
    if(rc) return rc;
    const aturan_iter_params ip = b200_iter_params(*m);
    std::fprintf(stderr, "glue_run: uploading\n");
    rc = b200_transfer(ctx, *m, true);
    for(int it = 1; !rc && it <= n; it++){
        std::fprintf(stderr, "glue_run: iteration %d\n", it);
        rc = aturan_iteration(ctx, &ip, it);
    }
    if(!rc) rc = aturan_sync(ctx);
    std::fprintf(stderr, "glue_run: downloading (rc %d)\n", rc);
    if(!rc) rc = b200_transfer(ctx, *m, false);
    if(rc) std::fprintf(stderr, "glue_run: %s\n", aturan_last_error(ctx));
    aturan_ctx_destroy(ctx);
    return rc;
}

}  // extern "C"
