// The C ABI of include/aturan_b200.h: context, device layout, tables and the call sequences.
//
// Host logic only; the kernels live in fp64.cu / mixed.cu behind launch.h. Geometry, pressure
// weights and the cp(T) table are built here in FP64 with the reference's expressions and
// operand order (sources cited per table) and uploaded once, so the device reads the CPU's
// values rather than recomputing them.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <type_traits>
#include <vector>

#include "aturan_b200.h"
#include "common.cuh"
#include "launch.h"
#include "rk4.cuh"
#include "satadj.cuh"
#include "pressure.cuh"
#include "sor.cuh"
#include "adjoint.cuh"
#include "post.cuh"
#include "chem.cuh"
#include "turb.cuh"
#include "precip.cuh"
#include "mca.cuh"

using namespace aturan;

namespace aturan { const char* static_last_error(); }   // noalloc.cu: errors of calls without a context

struct aturan_ctx {
    aturan_params p;
    Grid g;
    int mixed;                 // 0: FP64 storage, 1: FP32 storage
    size_t esz;                // bytes per stored element
    int device;
    cudaStream_t st;           // every launch of the context, except:
    cudaStream_t st2;          // the saturation adjustment inside aturan_step (lower priority)
    cudaEvent_t ev_fork, ev_join;
    cudaEvent_t ev_xcopy[2], ev_xpack[2];   // the batched transfers' staging ring (aturan_upload_many)
    char* mem;                 // one device allocation for everything below
    size_t mem_bytes;
    // storage-type groups (each field fstride elements)
    void* state;               // 19 prognostic
    void* ncopy;               // 19 start-of-step copies
    void* ybuf[2];             // stage ping-pong, 19 each
    void* acc;                 // 19
    void* forc;                // 22 pointwise RHS inputs
    void* proj;                // rhs_u, rhs_v, rhs_w, aux_u, aux_v, aux_w
    void* chem;                // difflux_h2s, difflux_nh3, difflux_nh4sh, prod
    void* pstat;               // p_stat
    // FP64 always
    double *pdyn, *phydro, *pbaro, *pb0, *pbf;
    double* scratch;           // incr_src / clamped source
    double* stage64;           // one padded FP64 field, for conversions
    double* ref_level;         // im
    double *part_sum, *part_w; // im * nblk
    BuoyScratch bx;            // the exact level means' scratch (FP64 context with exact_reductions)
    int nblk;
    double *wsin, *rm_i, *cor_j, *cp_tab64;
    void* geo;                 // GeoIJ<C>[im*jm]
    void* cp_tab;              // C[CP_TABLE_N]
    GSW* gsw;
    RBW* rbw;
    unsigned long long* counters;
    // RB_SOR: Fourier tables, the 2-D correction's work arrays, FP32 correction fields
    SorConst sorc;
    double *sor_ct, *sor_st, *sor_ctT, *sor_stT, *sor_colR, *sor_Ac, *sor_As, *sor_part, *sor_q;
    double *mlu_a, *mlu_cf, *mlu_idn;            // per-mode theta factorisations
    double *llu_a, *llu_cf, *llu_idn;            // per-(i,j) radial-line factorisations
    double *mluT_a, *mluT_cf, *mluT_idn;         // the same for the transposed operator
    double *lluT_a, *lluT_cf, *lluT_idn;
    float *r32, *e32;
    float* tlo;                // mixed form: the low parts of t and of tn (two FP32 fields; common.cuh), else null
    int last_sweeps;           // the last aturan_pressure's sweeps and residual (aturan_pressure_last)
    double last_resid;
    int sor_nblk;
    int sor_pm;                // Fourier modes per block of the column correction's tridiagonal solves
    std::vector<double> host_part;
    // adjoint tape (aturan_tape): stage inputs of t, u, v, w, the step's T output and level means,
    // and the adjoint's work arrays; null when the tape is off
    double* tape;
    bool tape_valid;           // a taped RK4 step has run since the tape was switched on
    double *tX, *tTout, *tPd, *tSrc, *tref, *aslot, *aybar, *akbar, *ag0, *aphbar, *arbar, *apdbar, *aaux, *alev;
    bool tape_p_valid;         // a taped RB_SOR / RB_LINE pressure call has run since the tape was switched on
    double* ahacc;             // the T tendencies' adjoint summed over the stages (heating gradient)
    int tape_nf;               // fields taped per stage: ADJ_NF (dry) or ADJ_NF_MOIST (aturan_tape(ctx, 2))
    double* tPre;              // moist tape: the state (fields 0..15) before the saturation adjustment
    bool tape_sat_pending;     // moist tape: an adjustment has recorded its input since the last taped RK4 step
    bool tape_sat_valid;       // moist tape: the taped step's RK4 followed a recorded adjustment
    double* heat;              // aturan_set_heating: [jm][km] K/s, or null
    double* mca_H;             // aturan_mca: the cp table's running integral, made at the first call
    bool mca_H_ready;          // mca_H holds the integral (its kernel has launched)
    double* chem_tab;          // aturan_chemistry: radius, metric radius (im), sin, cos of the colatitude (jm)
    double* dz_tab;            // aturan_precipitation: layer thickness [m] per level (the float layer heights)
    // host-side constants
    RhsConst<double> k64;
    RhsConst<float> k32;
    HydroConst hc;
    SatConst sc;
    PressConst pc;
    cudaGraphExec_t gs_exec;
    long gs_launches;          // kernels in the captured GS graph
    // per-class launch counts and optional CUDA-event timing (aturan_profile)
    int prof_timing;
    long launches[ATURAN_K_NKINDS];
    struct EvPair { int kind; cudaEvent_t a, b; };
    std::vector<EvPair> evs;
    size_t ev_used;
    std::string err;
};

namespace {

constexpr int SOR_KSPLIT = 4;   // k-splits of the correction's transforms (more blocks in flight)

int fail(aturan_ctx* c, int code, const std::string& msg){
    if(c) c->err = msg;
    return code;
}

int cuda_check(aturan_ctx* c, cudaError_t e, const char* what){
    if(e == cudaSuccess) return ATURAN_OK;
    return fail(c, ATURAN_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call) do { int rc_ = cuda_check(ctx, (call), #call); if(rc_) return rc_; } while(0)
#define CK_LAUNCH(what) do { int rc_ = cuda_check(ctx, cudaGetLastError(), what); if(rc_) return rc_; } while(0)

size_t round_up(size_t x, size_t a){ return (x + a - 1) / a * a; }

// lib/Array_1D.cpp:50-60
void coords(const aturan_params& p, std::vector<double>& rad, std::vector<double>& the){
    rad.resize(p.im); the.resize(p.jm);
    rad[0] = p.r0;
    for(int l = 1; l < p.im; l++) rad[l] = rad[l - 1] + p.dr;
    the[0] = p.the0;
    for(int l = 1; l < p.jm; l++) the[l] = the[l - 1] + p.dthe;
}

// cUranusModel.h:641-647
double metric_radius(const aturan_params& p, double rm){
    if(!(p.metric_R_km > 0.0)) return rm;
    return rm + (p.metric_R_km / p.L_atm - 1.0);
}

double stdmax(double a, double b){ return (a < b) ? b : a; }

// CpH2.h:43-75: the H2 heat capacity table, 0.5 K steps from 5 K to 1500 K.
double cpR_exact(double T, int mode){
    auto moments = [T](int J0, double wgt, double& Z, double& E1, double& E2){
        for(int J = J0; J < 60; J += 2){
            const double e = 87.57 * J * (J + 1.0), b = wgt * (2.0 * J + 1.0) * std::exp(-e / T);
            Z += b; E1 += b * e; E2 += b * e * e;
        }
    };
    auto crot = [T](double Z, double E1, double E2){ const double m1 = E1 / Z, m2 = E2 / Z; return (m2 - m1 * m1) / (T * T); };
    double c;
    if(mode == 1){
        double Zp = 0, Ep = 0, Fp = 0, Zo = 0, Eo = 0, Fo = 0;
        moments(0, 1.0, Zp, Ep, Fp); moments(1, 1.0, Zo, Eo, Fo);
        c = 0.25 * crot(Zp, Ep, Fp) + 0.75 * crot(Zo, Eo, Fo);
    } else {
        double Z = 0, E1 = 0, E2 = 0;
        moments(0, 1.0, Z, E1, E2); moments(1, 3.0, Z, E1, E2);
        c = crot(Z, E1, E2);
    }
    const double x = 6332.0 / T, cv = (x < 700.0) ? x * x * std::exp(x) / ((std::exp(x) - 1.0) * (std::exp(x) - 1.0)) : 0.0;
    return 2.5 + c + cv;
}

template <typename C>
RhsConst<C> make_rhs_const(const aturan_params& p){
    RhsConst<double> k{};
    k.inv_2dr   = 1.0 / (2.0 * p.dr);
    k.inv_2dthe = 1.0 / (2.0 * p.dthe);
    k.inv_2dphi = 1.0 / (2.0 * p.dphi);
    k.inv_dr2   = 1.0 / (p.dr * p.dr);
    k.inv_dthe2 = 1.0 / (p.dthe * p.dthe);
    k.inv_dphi2 = 1.0 / (p.dphi * p.dphi);
    const double coeff_energy_p = p.u_0 * p.u_0 / (p.cp_mix * p.t_ref);          // RHS_Uran_Turb.cpp:280
    const double scale_p   = 1.0e5 / (p.r_mix * p.u_0 * p.u_0);                    // :283
    const double scale_Cor = (p.coriolis_full ? p.L_atm * 1.0e3 : p.L_atm) / p.u_0; // cUranusModel.h:1498
    const double scale_cen = p.L_atm * p.L_atm / (p.u_0 * p.u_0);                 // :285
    k.ce_sp = coeff_energy_p * scale_p;
    k.scale_p = scale_p;
    k.m2om = -2.0 * p.omega;
    k.p2om = +2.0 * p.omega;
    k.cor_sc = p.Coriolis * scale_Cor;
    k.cor_rad_f = 0.0 * p.Coriolis * scale_Cor;                                    // CORIOLIS_SPLIT = 1
    k.cen_f = 1.0 * p.centrifugal * p.cent_mom * scale_cen;
    k.re = p.re;
    k.re_pr = p.re * p.pr;
    k.re_eff = p.re / (1.0 + 2.5 * 0.0);
    k.inv_re = 1.0 / p.re;
    k.turb_coupling = p.turb_coupling;
    k.precip_coupling = p.precip_coupling;
    k.chemical_reaction = p.chemical_reaction;
    k.tmf = p.tmf_scale * p.chemical_reaction;
    k.precip_L = p.L_atm * 1.0e3;
    k.precip_den = p.r_mix * p.cp_mix * p.u_0 * p.t_ref;
    k.sc_re[0] = p.sc_ch4 * p.re; k.sc_re[1] = p.sc_h2o * p.re; k.sc_re[2] = p.sc_h2s * p.re;
    k.sc_re[3] = p.sc_nh3 * p.re; k.sc_re[4] = p.sc_nh4sh * p.re;
    k.stokes_a = (2.0 / 9.0) * p.r_p_nh4sh * p.r_p_nh4sh;
    k.rho_cond_nh4sh = p.rho_cond_nh4sh; k.g = p.g; k.mue_mix = p.mue_mix; k.u_0 = p.u_0;
    k.cp_mix = p.cp_mix; k.t_ref = p.t_ref;
    if(p.cp_gas){
        k.cp_rh2 = p.r_h2;
        k.cp_he_term = p.r_he * p.cp_he;
        k.cp_ch4_term = p.r_ch4 * p.cp_ch4;
        k.cp_rsum = p.r_h2 + p.r_he + p.r_ch4;
    } else {
        k.cp_rh2 = p.r_h2 / p.r_mix;
    }
    k.cp_h2_const = p.cp_h2;
    k.inv_re_eff = 1.0 / k.re_eff; k.inv_re_pr = 1.0 / k.re_pr;
    for(int n = 0; n < 5; n++) k.inv_sc_re[n] = 1.0 / k.sc_re[n];
    k.inv_mue_mix = 1.0 / k.mue_mix; k.inv_u_0 = 1.0 / k.u_0; k.inv_precip_den = 1.0 / k.precip_den;
    k.inv_cp_rsum = k.cp_rsum != 0.0 ? 1.0 / k.cp_rsum : 0.0;
    k.tke_max = 1000.0 / (p.u_0 * p.u_0);
    k.dis_min = 1.0e-10;
    k.t_min = p.t_min_K / p.t_ref;
    k.t_max = p.t_max_K / p.t_ref;
    k.dt = p.dt;
    k.heat_scale = (p.L_atm * 1.0e3 / p.u_0) / p.t_ref;
    k.cp_dyn = p.cp_dyn; k.cp_gas = p.cp_gas; k.cp_mode = p.cp_h2_mode; k.turb_active = p.turb_active;
    RhsConst<C> out;
    const double* src = reinterpret_cast<const double*>(&k);
    C* dst = reinterpret_cast<C*>(&out);
    const size_t nd = offsetof(RhsConst<double>, cp_dyn) / sizeof(double);
    for(size_t n = 0; n < nd; n++) dst[n] = (C)src[n];
    out.cp_dyn = k.cp_dyn; out.cp_gas = k.cp_gas; out.cp_mode = k.cp_mode; out.turb_active = k.turb_active;
    return out;
}

int validate(const aturan_params* p, std::string& why){
    if(p->abi_version != ATURAN_ABI_VERSION){ why = "abi_version mismatch"; return ATURAN_E_INVALID; }
    if(p->im < 5 || p->jm < 5 || p->km < 5 || p->im > 512 || p->jm > 4096 || p->km > 8192){ why = "grid size out of range"; return ATURAN_E_INVALID; }
    if((p->km - 1) % 2){ why = "km-1 must be even (the red-black colours must alternate across the seam)"; return ATURAN_E_UNSUPPORTED; }
    if(p->precision != ATURAN_FP64 && p->precision != ATURAN_MIXED){ why = "unknown precision"; return ATURAN_E_INVALID; }
    if(!(p->dt > 0.0) || !(p->dr > 0.0) || !(p->dthe > 0.0) || !(p->dphi > 0.0)){ why = "non-positive step"; return ATURAN_E_INVALID; }
    if(p->cp_h2_mode < 0 || p->cp_h2_mode > 2){ why = "cp_h2_mode must be 0, 1 or 2"; return ATURAN_E_INVALID; }
    if(p->pbaro_follow < 0.0){ why = "pbaro_follow must be >= 0"; return ATURAN_E_INVALID; }
    return ATURAN_OK;
}

// Brackets the launches of one kernel class: counts them and, with timing on, records a pair of
// CUDA events on the context's stream around them.
struct Region {
    aturan_ctx* c; int kind; long n; int slot; cudaStream_t s;
    Region(aturan_ctx* c_, int kind_, long n_, cudaStream_t s_ = nullptr)
        : c(c_), kind(kind_), n(n_), slot(-1), s(s_ ? s_ : c_->st){
        if(!c->prof_timing) return;
        if(c->ev_used == c->evs.size()){
            aturan_ctx::EvPair e{kind, nullptr, nullptr};
            if(cudaEventCreate(&e.a) != cudaSuccess || cudaEventCreate(&e.b) != cudaSuccess){ cudaGetLastError(); return; }
            c->evs.push_back(e);
        }
        slot = (int)c->ev_used++;
        c->evs[slot].kind = kind;
        cudaEventRecord(c->evs[slot].a, s);
    }
    ~Region(){
        c->launches[kind] += n;
        if(slot >= 0) cudaEventRecord(c->evs[slot].b, s);
    }
};

template <typename T>
T* carve(char*& cur, size_t n){
    T* r = reinterpret_cast<T*>(cur);
    cur += round_up(n * sizeof(T), 256);
    return r;
}

// field id -> (device pointer, is FP64)
void* field_ptr(aturan_ctx* c, int id, bool* is64){
    const size_t fs = c->g.fstride, e = c->esz;
    *is64 = !c->mixed;
    if(id >= 0 && id < ATURAN_NPROG) return (char*)c->state + (size_t)id * fs * e;
    if(id >= ATURAN_TN && id < ATURAN_TN + ATURAN_NPROG) return (char*)c->ncopy + (size_t)(id - ATURAN_TN) * fs * e;
    if(id >= ATURAN_NUE && id <= ATURAN_DIS_SOURCE) return (char*)c->forc + (size_t)(id - ATURAN_NUE) * fs * e;
    if(id >= ATURAN_RHS_U && id <= ATURAN_AUX_W) return (char*)c->proj + (size_t)(id - ATURAN_RHS_U) * fs * e;
    if(id >= ATURAN_DIFFLUX_H2S && id <= ATURAN_PROD) return (char*)c->chem + (size_t)(id - ATURAN_DIFFLUX_H2S) * fs * e;
    if(id == ATURAN_P_STAT) return c->pstat;
    *is64 = true;
    switch(id){
    case ATURAN_P_DYN: return c->pdyn;
    case ATURAN_P_HYDRO: return c->phydro;
    case ATURAN_P_BARO: return c->pbaro;
    case ATURAN_P_B0: return c->pb0;
    case ATURAN_P_BFOLLOW: return c->pbf;
    }
    return nullptr;
}

template <typename S> S* grp(void* base, int q, size_t fs){ return reinterpret_cast<S*>(base) + (size_t)q * fs; }

// The low part of the mixed form's temperature pair for field id t or tn, else null.
float* t_lo_of(aturan_ctx* c, int id){
    if(!c->tlo) return nullptr;
    if(id == ATURAN_T) return c->tlo;
    if(id == ATURAN_TN) return c->tlo + c->g.fstride;
    return nullptr;
}

template <typename S>
bool taping(const aturan_ctx* ctx){ return std::is_same<S, double>::value && ctx->tape != nullptr; }

// The RK4 prelude: the buoyancy level means and the hydrostatic integral from the state at the
// start of the step (RungeKutta_Uran_Turb.cpp:18-177), on stream st.
template <typename S>
int rk4_prelude(aturan_ctx* ctx, cudaStream_t st){
    const Grid g = ctx->g;
    const size_t fs = g.fstride;
    S* state = reinterpret_cast<S*>(ctx->state);
    const int exact = ctx->mixed ? 0 : ctx->p.exact_reductions;   // the mixed form always sums in tree order
    Region reg(ctx, ATURAN_K_HYDRO, exact ? 2 : 3, st);
    launch_buoy(g, grp<S>(state, ATURAN_T, fs), reinterpret_cast<const S*>(ctx->pstat), ctx->wsin, ctx->hc,
                ctx->part_sum, ctx->part_w, ctx->nblk, ctx->ref_level, exact, ctx->bx, st);
    CK_LAUNCH("buoyancy reference level");
    launch_hydro(g, grp<S>(state, ATURAN_T, fs), reinterpret_cast<const S*>(ctx->pstat), grp<S>(state, ATURAN_V, fs),
                 grp<S>(state, ATURAN_W, fs), ctx->ref_level, ctx->rm_i, ctx->cor_j, ctx->pbaro, ctx->pb0, ctx->pbf,
                 ctx->phydro, ctx->hc, 1, st);
    CK_LAUNCH("hydrostatic integral");
    return ATURAN_OK;
}

// The arguments of RK4 stage `stage` (RungeKutta_Uran_Turb.cpp:242-245: its input, output, the
// stage coefficient and the accumulator's weight).
template <typename S, typename C>
StageArgs<S, C> stage_args(aturan_ctx* ctx, const RhsConst<C>& K, int stage){
    const Grid g = ctx->g;
    const size_t fs = g.fstride;
    S* state = reinterpret_cast<S*>(ctx->state);
    StageArgs<S, C> a;
    a.g = g;
    a.St = state;
    a.Nc = reinterpret_cast<const S*>(ctx->ncopy);
    a.acc = reinterpret_cast<S*>(ctx->acc);
    a.pdyn = ctx->pdyn;
    a.phydro = ctx->phydro;
    a.forc = reinterpret_cast<const S*>(ctx->forc);
    a.proj = reinterpret_cast<S*>(ctx->proj);
    a.geo = reinterpret_cast<const GeoIJ<C>*>(ctx->geo);
    a.cp_tab = reinterpret_cast<const C*>(ctx->cp_tab);
    a.heat = ctx->heat;
    a.k = K;
    a.tlo = ctx->tlo;
    a.tnlo = ctx->tlo ? ctx->tlo + fs : nullptr;
    S* y0 = reinterpret_cast<S*>(ctx->ybuf[0]);
    S* y1 = reinterpret_cast<S*>(ctx->ybuf[1]);
    const double dt = ctx->p.dt;
    a.stage = stage;
    a.c_in = (C)((stage == 0 || stage == 1) ? 0.5 * dt : (stage == 2 ? dt : 0.0));
    a.wgt  = (C)((stage == 0 || stage == 3) ? 1.0 : 2.0);
    a.X = stage == 0 ? state : (stage == 1 ? y0 : (stage == 2 ? y1 : y0));
    a.Y = stage == 0 ? y0 : (stage == 1 ? y1 : (stage == 2 ? y0 : state));
    return a;
}

// One RK4 step; prelude_done: rk4_prelude has already run for this step (aturan_step runs it on
// the side stream, beside the pressure solve).
template <typename S, typename C>
int run_rk4(aturan_ctx* ctx, const RhsConst<C>& K, bool prelude_done = false){
    const Grid g = ctx->g;
    const size_t fs = g.fstride;
    S* state = reinterpret_cast<S*>(ctx->state);
    if(!prelude_done){ const int rc = rk4_prelude<S>(ctx, ctx->st); if(rc) return rc; }
    if(taping<S>(ctx)){
        CK(cudaMemcpyAsync(ctx->tref, ctx->ref_level, g.im * 8, cudaMemcpyDeviceToDevice, ctx->st));
        CK(cudaMemcpyAsync(ctx->tX, state, ctx->tape_nf * fs * 8, cudaMemcpyDeviceToDevice, ctx->st));
        CK(cudaMemcpyAsync(ctx->tPd, ctx->pdyn, fs * 8, cudaMemcpyDeviceToDevice, ctx->st));
    }
    for(int stage = 0; stage < 4; stage++){   // RungeKutta_Uran_Turb.cpp:242-245
        const StageArgs<S, C> a = stage_args<S, C>(ctx, K, stage);
        {
        Region reg(ctx, ATURAN_K_RK_STAGE, 2);
        // mixed form: the momentum launch on the side stream beside the scalar launch (they read
        // the stage input and write disjoint fields; measured 3 % faster RK4 at 41x181x361)
        if(ctx->mixed) launch_stage(a, ctx->st, ctx->st2, ctx->ev_fork, ctx->ev_join);
        else launch_stage(a, ctx->st);
        CK_LAUNCH("RK4 stage");
        }
        if(taping<S>(ctx)){      // the next stage's input of t, u, v, w; after stage 3 the new T
            if(stage < 3) CK(cudaMemcpyAsync(ctx->tX + (size_t)(stage + 1) * ctx->tape_nf * fs, a.Y, ctx->tape_nf * fs * 8,
                                             cudaMemcpyDeviceToDevice, ctx->st));
            else CK(cudaMemcpyAsync(ctx->tTout, state, fs * 8, cudaMemcpyDeviceToDevice, ctx->st));
        }
    }
    if(taping<S>(ctx)){
        ctx->tape_valid = true;
        ctx->tape_sat_valid = ctx->tape_sat_pending;   // this step's adjustment, if one ran before it
        ctx->tape_sat_pending = false;
    }
    return ATURAN_OK;
}

// with_sync: also perform aturan_sync_ncopies' copies, fused (the values are in registers).
template <typename S>
int run_satadj(aturan_ctx* ctx, int mask, bool count, cudaStream_t st, bool with_sync = false){
    const size_t fs = ctx->g.fstride;
    S* state = reinterpret_cast<S*>(ctx->state);
    SatArgs<S> a;
    a.g = ctx->g;
    a.t = grp<S>(state, ATURAN_T, fs);
    a.ps = reinterpret_cast<const S*>(ctx->pstat);
    a.rho_mix = grp<S>(ctx->forc, ATURAN_RHO_MIX - ATURAN_NUE, fs);
    static const int base[4] = {ATURAN_H2O, ATURAN_H2S, ATURAN_NH3, ATURAN_CH4};
    for(int gi = 0; gi < 4; gi++)
        for(int n = 0; n < 3; n++) a.spec[gi][n] = grp<S>(state, base[gi] + n, fs);
    a.k = ctx->sc;
    a.gas_mask = mask;
    a.counters = count ? ctx->counters : nullptr;
    a.nc_off = (long long)(reinterpret_cast<S*>(ctx->ncopy) - state);
    a.sync = with_sync ? (ctx->p.nh4sh_sync ? 2 : 1) : 0;
    a.nh4sh = grp<S>(state, ATURAN_NH4SH, fs);
    a.tlo = ctx->tlo;
    a.tnlo = ctx->tlo ? ctx->tlo + fs : nullptr;
    if(taping<S>(ctx) && ctx->tape_nf == ADJ_NF_MOIST){   // the moist tape: the adjustment's input
        if(mask != 0xF) return fail(ctx, ATURAN_E_UNSUPPORTED, "the moist tape records the adjustment of all four gases only");
        CK(cudaMemcpyAsync(ctx->tPre, state, (size_t)ADJ_NF_MOIST * fs * 8, cudaMemcpyDeviceToDevice, st));
        ctx->tape_sat_pending = true;
    }
    Region reg(ctx, ATURAN_K_SATADJ, 1, st);
    launch_satadj(a, st);
    CK_LAUNCH("saturation adjustment");
    return ATURAN_OK;
}

template <typename S>
int run_gs(aturan_ctx* ctx){
    const Grid g = ctx->g;
    const size_t fs = g.fstride;
    S* proj = reinterpret_cast<S*>(ctx->proj);
    if(!ctx->gs_exec){
        // The hyperplane sweep is (im-2)+(jm-2)+(km-2)-1 dependent launches; capture the whole
        // call once per context and replay it.
        cudaStream_t cs;
        CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaGraph_t graph;
        CK(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        launch_gs_pre(g, grp<S>(proj, 3, fs), grp<S>(proj, 4, fs), grp<S>(proj, 5, fs),
                      grp<S>(proj, 0, fs), grp<S>(proj, 1, fs), grp<S>(proj, 2, fs), ctx->pdyn, ctx->gsw,
                      ctx->pc, ctx->scratch, cs);
        const int s_lo = 2, s_hi = (g.im - 2) + (g.jm - 2) + (g.km - 2);
        ctx->gs_launches = 1 + (ctx->pc.press_incr ? 1 : 0) + (s_hi - s_lo + 1) + 3;
        for(int s = s_lo; s <= s_hi; s++)
            launch_gs_plane(g, ctx->pdyn, ctx->scratch, grp<S>(proj, 3, fs), grp<S>(proj, 4, fs),
                            grp<S>(proj, 5, fs), ctx->gsw, ctx->pc, s, cs);
        launch_pdyn_bcs(g, ctx->pdyn, cs);
        cudaError_t e1 = cudaGetLastError();
        cudaError_t e2 = cudaStreamEndCapture(cs, &graph);
        if(e1 != cudaSuccess || e2 != cudaSuccess){
            cudaStreamDestroy(cs);
            return fail(ctx, ATURAN_E_CUDA, std::string("capturing the GS sweep: ") +
                        cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
        }
        cudaError_t e3 = cudaGraphInstantiate(&ctx->gs_exec, graph, 0);
        cudaGraphDestroy(graph);
        cudaStreamDestroy(cs);
        CK(e3);
    }
    Region reg(ctx, ATURAN_K_GS, ctx->gs_launches);
    CK(cudaGraphLaunch(ctx->gs_exec, ctx->st));
    return ATURAN_OK;
}

template <typename S>
int run_rb(aturan_ctx* ctx, int sweeps, double omega){
    const Grid g = ctx->g;
    const size_t fs = g.fstride;
    S* proj = reinterpret_cast<S*>(ctx->proj);
    if(sweeps < 1) sweeps = 1;                                  // PressureSolver.h:174-175
    Region reg(ctx, ATURAN_K_RB, 3 + 5L * sweeps);
    launch_rb_prep(g, grp<S>(proj, 3, fs), grp<S>(proj, 4, fs), grp<S>(proj, 5, fs),
                   grp<S>(proj, 0, fs), grp<S>(proj, 1, fs), grp<S>(proj, 2, fs), ctx->p.rigid_lid,
                   ctx->rbw, ctx->pc, ctx->scratch, ctx->st);
    CK_LAUNCH("projection boundaries and source");
    for(int s = 0; s < sweeps; s++){
        launch_rb_colour(g, ctx->pdyn, ctx->scratch, ctx->rbw, 0, omega, ctx->st);
        launch_rb_colour(g, ctx->pdyn, ctx->scratch, ctx->rbw, 1, omega, ctx->st);
        launch_pdyn_bcs(g, ctx->pdyn, ctx->st);
        CK_LAUNCH("red-black sweep");
    }
    return ATURAN_OK;
}

// ---- RB_SOR: the shared solver's equation to a relative L2 residual (sor.cuh) ----

// Residual of P against src: relative L2 norm (host sum of the block partials, fixed order).
// TR: of the transposed operator. shift: apply the source's compatibility shift in this pass
// (after sor_compat with apply = false).
template <typename T, bool TR = false>
int sor_residual(aturan_ctx* ctx, const T* P, const T* src, bool want_col, double* rel, double* abs_rr,
                 bool fill32 = false, const double* shift = nullptr){
    const Grid g = ctx->g;
    double* src_w = nullptr;
    if constexpr(std::is_same<T, double>::value) src_w = shift ? const_cast<double*>(src) : nullptr;
    sor_colsum_kernel<T, TR><<<dim3((g.km - 1 + 31) / 32, g.jm - 2), dim3(32, 8), 0, ctx->st>>>(
        g, P, src, ctx->rbw, ctx->sor_colR, ctx->sor_part, want_col ? 1 : 0,
        fill32 ? ctx->r32 : nullptr, fill32 ? ctx->e32 : nullptr, src_w, src_w ? shift : nullptr);
    CK_LAUNCH("residual");
    if(!rel) return ATURAN_OK;                                 // column sums only: no host round trip
    CK(cudaMemcpyAsync(ctx->host_part.data(), ctx->sor_part, 2 * ctx->sor_nblk * 8, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    double rr = 0.0, ss = 0.0;
    for(int n = 0; n < ctx->sor_nblk; n++){ rr += ctx->host_part[2 * n]; ss += ctx->host_part[2 * n + 1]; }
    if(abs_rr) *abs_rr = std::sqrt(rr);
    *rel = ss > 0.0 ? std::sqrt(rr / ss) : std::sqrt(rr);
    return ATURAN_OK;
}

// The column-uniform correction (TR: the transposed system's y-shaped one) from the column sums
// left in sor_colR by the last residual.
template <typename T, bool TR = false>
int sor_correct(aturan_ctx* ctx, T* P){
    const Grid g = ctx->g;
    const SorConst& c = ctx->sorc;
    const MatRef R{ctx->sor_colR, c.N, 1};                        // (jj, k)
    const long sz_ac = (long)(c.NM + 1) * c.J, sz_q = (long)c.J * c.N;
    const int kcf = ((c.N + SOR_KSPLIT - 1) / SOR_KSPLIT + 31) / 32 * 32;
    const dim3 gf((c.NM + 1 + 31) / 32, (c.J + 31) / 32, SOR_KSPLIT);
    sor_gemm_kernel<<<gf, 256, 0, ctx->st>>>(c.J, c.NM + 1, c.N, R, MatRef{ctx->sor_ctT, c.NM + 1, 1},
                                            R, MatRef{ctx->sor_stT, c.NM + 1, 1}, 1.0 / c.A2y,
                                            ctx->sor_Ac, ctx->sor_As, 1, c.J, kcf, sz_ac);
    ModeLU lu = TR ? ModeLU{ctx->mluT_a, ctx->mluT_cf, ctx->mluT_idn} : ModeLU{ctx->mlu_a, ctx->mlu_cf, ctx->mlu_idn};
    const int pm = ctx->sor_pm;
    sor_tridiag_kernel<<<(c.NM + 1 + pm - 1) / pm, 128, (size_t)8 * c.J * (5 * pm + 4), ctx->st>>>(
        c, lu, ctx->sor_Ac, ctx->sor_As, pm, TR ? 1 : 0, SOR_KSPLIT, sz_ac);
    const int kci = ((c.NM + 1 + SOR_KSPLIT - 1) / SOR_KSPLIT + 31) / 32 * 32;
    const dim3 gi((c.N + 31) / 32, (c.J + 31) / 32, SOR_KSPLIT);
    sor_gemm_kernel<<<gi, 256, 0, ctx->st>>>(c.J, c.N, c.NM + 1, MatRef{ctx->sor_Ac, 1, c.J}, MatRef{ctx->sor_ct, c.N, 1},
                                            MatRef{ctx->sor_As, 1, c.J}, MatRef{ctx->sor_st, c.N, 1},
                                            1.0, ctx->sor_q, nullptr, c.N, 1, kci, sz_q);
    sor_add_kernel<T, TR><<<dim3((c.N + 127) / 128, g.jm - 2), 128, 0, ctx->st>>>(g, ctx->sor_q, P, SOR_KSPLIT, sz_q);
    CK_LAUNCH("column-uniform correction");
    return ATURAN_OK;
}

// Dynamic shared memory of sor_line_kernel: the right-hand sides of LINE_COLS columns and the
// row's three factor arrays, per level, in the kernel's arithmetic type.
template <typename T>
inline size_t line_smem(const Grid& g){ return (size_t)(g.im - 2) * (LINE_COLS + 3) * sizeof(typename LineArith<T>::A); }

// Allow sor_line_kernel above the default 48 KB of dynamic shared memory (once per instance).
template <typename T, bool TR>
bool line_smem_attr(){
    static const bool ok = cudaFuncSetAttribute(sor_line_kernel<T, TR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                227 * 1024) == cudaSuccess || (cudaGetLastError(), false);
    return ok;
}

// One relaxation sweep (both colours) of the folded operator (TR: its transpose): point
// (line = false) or radial line.
template <typename T, bool TR = false>
void sor_sweep(aturan_ctx* ctx, T* E, const T* R, double omega, bool line){
    const Grid g = ctx->g;
    if(line && line_smem<T>(g) > 48 * 1024) line_smem_attr<T, TR>();
    for(int colour = 0; colour < 2; colour++){
        if(line)
            sor_line_kernel<T, TR><<<dim3((g.km / 2 + LINE_COLS - 1) / LINE_COLS, g.jm - 2), 256, line_smem<T>(g), ctx->st>>>(
                g, E, R, ctx->rbw, TR ? ctx->lluT_a : ctx->llu_a, TR ? ctx->lluT_cf : ctx->llu_cf,
                TR ? ctx->lluT_idn : ctx->llu_idn, colour, omega);
        else
            sor_colour_kernel<T, TR><<<dim3((g.km / 2 + 127) / 128, g.jm - 2, g.im - 2), 128, 0, ctx->st>>>(
                g, E, R, ctx->rbw, colour, omega);
    }
}

int sor_check_sizes(aturan_ctx* ctx, double omega, bool line){
    const Grid& g = ctx->g;
    if(!(omega > 0.0 && omega < 2.0)) return fail(ctx, ATURAN_E_INVALID, "omega must lie in (0, 2)");
    if(8 * ctx->sorc.J * (5 * ctx->sor_pm + 4) > 227 * 1024)
        return fail(ctx, ATURAN_E_UNSUPPORTED, "the column correction needs jm <= 2900");
    if(line && line_smem<double>(g) > 227 * 1024)
        return fail(ctx, ATURAN_E_UNSUPPORTED, "line relaxation needs im <= 435");
    return ATURAN_OK;
}

// Sweeps between residual checks and between column-uniform corrections. Point SOR needs ~200
// sweeps and loses ~6 % of its rate with a correction every 16; line SOR needs 5-7 iterations
// and converges at the same rate with one correction per 8 as with one per iteration (the first
// correction removes the column-uniform error; oracle measurements at 41x181x361).
inline int sor_check_every(bool line){ return line ? 1 : 16; }
inline int sor_correct_every(bool line){ return line ? 8 : 16; }

// Remove src's component along the operator's left null vector (y_i y_j for Lc, the constant for
// Lc^T) by a shift of the interior, all on the device.
const double* sor_compat(aturan_ctx* ctx, double* src, bool transposed, bool apply = true){
    const Grid& g = ctx->g;
    const int ny = ((g.jm - 2) * (g.km - 1) + 255) / 256;
    // past the residual pass's block partials: the first residual reads it while writing those
    double* shift = ctx->sor_part + 2 * ctx->sor_nblk;
    sor_ysum_kernel<<<ny, 256, 0, ctx->st>>>(g, src, ctx->sor_part, transposed ? 1 : 0);
    sor_shift_finish_kernel<<<1, 256, 0, ctx->st>>>(ctx->sor_part, ny, shift);
    if(apply) sor_shift_kernel<<<148 * 4, 256, 0, ctx->st>>>(g, src, shift);
    return shift;
}

// FP64 red-black solve of Lc P = src (TR: Lc^T P = src) on the interior from the given P, src
// compatible. Returns ATURAN_OK at tol, ATURAN_NOT_CONVERGED at the cap; counts launches into nl.
template <bool TR>
int solve_fp64(aturan_ctx* ctx, double* P, const double* src, double omega, int max_sweeps, double tol, bool line,
               int* sweeps_done, double* resid, long& nl, const double* shift = nullptr){
    const int check_every = sor_check_every(line), every = sor_correct_every(line);
    double r = 0.0;
    int s = 0;
    int rc = sor_residual<double, TR>(ctx, P, src, true, &r, nullptr, false, shift); if(rc) return rc; nl++;
    while(s < max_sweeps && !(r <= tol)){
        if(s % every == 0){ rc = sor_correct<double, TR>(ctx, P); if(rc) return rc; nl += 4; }
        for(int n = 0; n < check_every && s < max_sweeps; n++, s++){ sor_sweep<double, TR>(ctx, P, src, omega, line); nl += 2; }
        CK_LAUNCH("SOR sweeps");
        rc = sor_residual<double, TR>(ctx, P, src, s % every == 0, &r, nullptr); if(rc) return rc; nl++;
    }
    if(sweeps_done) *sweeps_done = s;
    if(resid) *resid = r;
    return r <= tol ? ATURAN_OK : ATURAN_NOT_CONVERGED;
}

// The mixed form of the same solve: FP64 iterative refinement around FP32 correction solves,
// r = src - Lc p in FP64, Lc e = r by FP32 sweeps (with the column-uniform correction), p += e in
// FP64. Given shift, the first residual pass applies the source's compatibility shift.
template <bool TR>
int solve_mixed(aturan_ctx* ctx, double* P, const double* src, double omega, int max_sweeps, double tol, bool line,
                int* sweeps_done, double* resid, long& nl, const double* shift = nullptr){
    const size_t fs = ctx->g.fstride;
    const int every = sor_correct_every(line);
    // FP32 sweeps per refinement step: for line SOR 2 (measured at 41x181x361, warm: two
    // refinement steps of 2 reach 3e-8 against 6 sweeps with 3 per step, 0.53 vs 0.59 ms)
    const int inner = line ? 2 : 48;
    double r = 0.0;
    int s = 0;
    // Each FP64 residual also leaves r in FP32, e = 0 and the column sums of r: what the next
    // correction solve starts from (one pass over p and src per refinement step).
    int rc = sor_residual<double, TR>(ctx, P, src, true, &r, nullptr, true, shift); if(rc) return rc; nl++;
    while(s < max_sweeps && !(r <= tol)){
        for(int n = 0; n < inner && s < max_sweeps; n++, s++){
            // the correction on the same cadence as the FP64 solve (once per `every` sweeps,
            // counted over the whole solve): after the first one the column-uniform error is
            // gone and a later refinement step's correction changes nothing (measured: same
            // sweep count, 0.14 ms less at 41x181x361); with e = 0 its column sums are r's
            if(s % every == 0){
                if(n != 0){ rc = sor_residual<float, TR>(ctx, ctx->e32, ctx->r32, true, nullptr, nullptr); if(rc) return rc; nl++; }
                rc = sor_correct<float, TR>(ctx, ctx->e32); if(rc) return rc;
                nl += 4;
            }
            sor_sweep<float, TR>(ctx, ctx->e32, ctx->r32, omega, line);
            nl += 2;
        }
        sor_axpy_kernel<<<148 * 8, 256, 0, ctx->st>>>(fs, P, ctx->e32);
        CK_LAUNCH("SOR refinement");
        nl++;
        rc = sor_residual<double, TR>(ctx, P, src, true, &r, nullptr, true); if(rc) return rc; nl++;
    }
    if(sweeps_done) *sweeps_done = s;
    if(resid) *resid = r;
    return r <= tol ? ATURAN_OK : ATURAN_NOT_CONVERGED;
}

template <typename S>
int run_sor(aturan_ctx* ctx, double omega, int max_sweeps, double tol, bool line, int* sweeps_done, double* resid){
    const Grid g = ctx->g;
    const size_t fs = g.fstride;
    S* proj = reinterpret_cast<S*>(ctx->proj);
    int rc = sor_check_sizes(ctx, omega, line); if(rc) return rc;
    if(max_sweeps < 1) max_sweeps = 1;
    long nl = 0;
    Region reg(ctx, ATURAN_K_RB, 0);
    launch_rb_prep(g, grp<S>(proj, 3, fs), grp<S>(proj, 4, fs), grp<S>(proj, 5, fs),
                   grp<S>(proj, 0, fs), grp<S>(proj, 1, fs), grp<S>(proj, 2, fs), ctx->p.rigid_lid,
                   ctx->rbw, ctx->pc, ctx->scratch, ctx->st);
    if(taping<S>(ctx)){           // the clamped source, for the clamp mask of the adjoint
        CK(cudaMemcpyAsync(ctx->tSrc, ctx->scratch, fs * 8, cudaMemcpyDeviceToDevice, ctx->st));
        ctx->tape_p_valid = true;
    }
    // the shift itself is applied by the first residual pass
    const double* shift = sor_compat(ctx, ctx->scratch, false, false);
    CK_LAUNCH("SOR source");
    nl += 5;
    double* P = ctx->pdyn;
    const double* src = ctx->scratch;
    double r = 0.0;
    int s = 0;
    int status;
    status = ctx->mixed ? solve_mixed<false>(ctx, P, src, omega, max_sweeps, tol, line, &s, &r, nl, shift)
                        : solve_fp64<false>(ctx, P, src, omega, max_sweeps, tol, line, &s, &r, nl, shift);
    if(status < 0) return status;
    launch_pdyn_bcs(g, P, ctx->st);                            // the boundary rows of the solution
    CK_LAUNCH("SOR boundary rows");
    nl += 3;
    reg.n = nl;
    if(sweeps_done) *sweeps_done = s;
    if(resid) *resid = r;
    return status;
}

}  // namespace

// The passes after RK4 on the context's fields (aturan_post_step).
template <typename S>
int run_post(aturan_ctx* ctx, const aturan_post_params* pp, double* clamp_added, long* clamp_cells){
    const Grid& g = ctx->g;
    const size_t fs = g.fstride;
    S* X = reinterpret_cast<S*>(ctx->state);
    S* Fo = reinterpret_cast<S*>(ctx->forc);
    S* Ch = reinterpret_cast<S*>(ctx->chem);
    auto fld = [&](int id) -> S* {
        if(id >= ATURAN_DIFFLUX_H2S) return Ch + (size_t)(id - ATURAN_DIFFLUX_H2S) * fs;
        return id < ATURAN_NPROG ? X + (size_t)id * fs : Fo + (size_t)(id - ATURAN_NUE) * fs;
    };
    // the phi pass takes the first POST_NPHI: all but difflux_nh4sh (BC_Uran.cpp:73-88)
    static const int RAD[POST_NRAD] = { ATURAN_T, ATURAN_U, ATURAN_V, ATURAN_W,       // BC_Uran.cpp:21-41
        ATURAN_CH4, ATURAN_CH4_CLOUD, ATURAN_CH4_ICE, ATURAN_H2O, ATURAN_H2O_CLOUD, ATURAN_H2O_ICE,
        ATURAN_H2S, ATURAN_H2S_CLOUD, ATURAN_H2S_ICE, ATURAN_NH3, ATURAN_NH3_CLOUD, ATURAN_NH3_ICE,
        ATURAN_NH4SH, ATURAN_MASSFLUX_H2S, ATURAN_MASSFLUX_NH3, ATURAN_MASSFLUX_NH4SH,
        ATURAN_FLUXLIM_NH4SH, ATURAN_THERMALMASSFLUX, ATURAN_DIFFLUX_H2S, ATURAN_DIFFLUX_NH3,
        ATURAN_DIFFLUX_NH4SH };
    static const int THX[POST_NTHX] = { ATURAN_T, ATURAN_U,                             // BC_Uran.cpp:43-59
        ATURAN_CH4, ATURAN_CH4_CLOUD, ATURAN_CH4_ICE, ATURAN_H2O, ATURAN_H2O_CLOUD, ATURAN_H2O_ICE,
        ATURAN_H2S, ATURAN_H2S_CLOUD, ATURAN_H2S_ICE, ATURAN_NH3, ATURAN_NH3_CLOUD, ATURAN_NH3_ICE,
        ATURAN_NH4SH, ATURAN_THERMALMASSFLUX };
    static const int THZ[POST_NTHZ] = { ATURAN_V, ATURAN_W, ATURAN_MASSFLUX_H2S,         // BC_Uran.cpp:61-71
        ATURAN_MASSFLUX_NH3, ATURAN_MASSFLUX_NH4SH, ATURAN_FLUXLIM_NH4SH, ATURAN_DIFFLUX_H2S,
        ATURAN_DIFFLUX_NH3, ATURAN_DIFFLUX_NH4SH };
    static const int SP[POST_NSP] = { ATURAN_H2O, ATURAN_H2O_CLOUD, ATURAN_H2O_ICE,      // BC_Uran.h:83-89
        ATURAN_H2S, ATURAN_H2S_CLOUD, ATURAN_H2S_ICE, ATURAN_NH3, ATURAN_NH3_CLOUD, ATURAN_NH3_ICE,
        ATURAN_CH4, ATURAN_CH4_CLOUD, ATURAN_CH4_ICE, ATURAN_NH4SH };
    PostArgs<S> a;
    a.g = g;
    for(int n = 0; n < POST_NRAD; n++) a.rad[n] = fld(RAD[n]);
    for(int n = 0; n < POST_NTHX; n++) a.thx[n] = fld(THX[n]);
    for(int n = 0; n < POST_NTHZ; n++) a.thz[n] = fld(THZ[n]);
    for(int n = 0; n < POST_NSP; n++) a.sp[n] = fld(SP[n]);
    a.u = fld(ATURAN_U); a.v = fld(ATURAN_V); a.w = fld(ATURAN_W);
    a.tlo = ctx->tlo;
    a.radius_form = pp->radius_form; a.bottom_form = pp->bottom_form; a.pole_form = pp->pole_form;
    a.lid_u = pp->lid_u; a.top_taper = pp->top_taper; a.lid_vw = pp->lid_vw;
    a.positive = pp->radius_positive; a.phi_periodic = pp->phi_periodic;
    PostPlan pl;
    pl.damp_t_horiz = pp->damp_t_horiz; pl.damp_t_vert = pp->damp_t_vert; pl.vel_shapiro = pp->vel_shapiro;
    pl.damp_t_j = pp->damp_t_j; pl.species_clamp = pp->species_clamp;
    // the clamp's partial sums borrow the pressure source's scratch (free between calls)
    // one wave: 8 resident blocks of 256 threads on each of 148 SMs, shared by the 13 species
    pl.nb = (int)std::min<size_t>(148 * 8 / POST_NSP, (fs - 2 * POST_NSP) / (2 * POST_NSP));
    pl.part = ctx->scratch;
    pl.out = ctx->scratch + (size_t)2 * POST_NSP * pl.nb;
    int nl;
    {
        Region reg(ctx, ATURAN_K_POST, 0);
        nl = launch_post(a, pl, fld(ATURAN_T), ctx->tlo, ctx->st);
        reg.n = nl;
        CK_LAUNCH("post step");
    }
    if(clamp_added || clamp_cells){
        double h[2 * POST_NSP] = {0.0};
        if(pp->species_clamp){
            CK(cudaMemcpyAsync(h, pl.out, sizeof h, cudaMemcpyDeviceToHost, ctx->st));
            CK(cudaStreamSynchronize(ctx->st));
        }
        for(int n = 0; n < POST_NSP; n++){
            if(clamp_added) clamp_added[n] = h[n];
            if(clamp_cells) clamp_cells[n] = (long)h[POST_NSP + n];
        }
    }
    return ATURAN_OK;
}

// The chemistry on the context's fields (aturan_chemistry).
template <typename S>
int run_chem(aturan_ctx* ctx, const aturan_chem_params* cp, int what, cudaStream_t st = nullptr){
    if(!st) st = ctx->st;
    const Grid& g = ctx->g;
    const size_t fs = g.fstride;
    const aturan_params& p = ctx->p;
    S* X = reinterpret_cast<S*>(ctx->state);
    S* Fo = reinterpret_cast<S*>(ctx->forc);
    S* Ch = reinterpret_cast<S*>(ctx->chem);
    auto fo = [&](int id) -> S* { return Fo + (size_t)(id - ATURAN_NUE) * fs; };
    ChemArgs<S> a;
    a.g = g;
    a.t = X + (size_t)ATURAN_T * fs; a.nh3 = X + (size_t)ATURAN_NH3 * fs;
    a.h2s = X + (size_t)ATURAN_H2S * fs; a.nh4sh = X + (size_t)ATURAN_NH4SH * fs;
    a.tlo = ctx->tlo;
    a.u = X + (size_t)ATURAN_U * fs; a.v = X + (size_t)ATURAN_V * fs; a.w = X + (size_t)ATURAN_W * fs;
    a.ps = reinterpret_cast<const S*>(ctx->pstat);
    a.rho_mix = fo(ATURAN_RHO_MIX); a.tmf = fo(ATURAN_THERMALMASSFLUX);
    a.mf_h2s = fo(ATURAN_MASSFLUX_H2S); a.mf_nh3 = fo(ATURAN_MASSFLUX_NH3); a.mf_nh4sh = fo(ATURAN_MASSFLUX_NH4SH);
    a.fl = fo(ATURAN_FLUXLIM_NH4SH);
    a.df_h2s = Ch; a.df_nh3 = Ch + fs; a.df_nh4sh = Ch + 2 * fs;
    a.tab.rad = ctx->chem_tab; a.tab.rmm = ctx->chem_tab + g.im;
    a.tab.sin = ctx->chem_tab + 2 * g.im; a.tab.cos = ctx->chem_tab + 2 * g.im + g.jm;
    ChemConst& c = a.c;
    c.t_ref = p.t_ref; c.R_mix = p.R_mix; c.r_mix = p.r_mix; c.cp_mix = p.cp_mix;
    c.L_f = 4705.0 * std::log(10.0) * 8314.46 / 51.1114;                    // ChemistryUran.h:132
    c.m_nh3 = cp->m_nh3; c.m_h2s = cp->m_h2s; c.m_nh4sh = cp->m_nh4sh;
    const double nu_mix = p.mue_mix / p.r_mix;                                // ChemistryUran.h:303-309
    c.D_nh3 = nu_mix / p.sc_nh3; c.D_h2s = nu_mix / p.sc_h2s;
    c.DT_nh3 = nu_mix / p.sc_nh3; c.DT_h2s = nu_mix / p.sc_h2s;
    c.D_nh4sh = cp->D_nh4sh; c.DT_nh4sh = cp->DT_nh4sh; c.c_mix = cp->c_mix;
    c.cp_nh3 = cp->cp_nh3; c.cp_h2s = cp->cp_h2s; c.cp_nh4sh = cp->cp_nh4sh;
    c.k_nh3 = cp->k_nh3; c.k_h2s = cp->k_h2s; c.k_nh4sh = cp->k_nh4sh;
    c.dr = p.dr; c.dthe = p.dthe; c.dphi = p.dphi;
    c.dsign = cp->difflux_plus ? 1.0 : -1.0;                                  // ChemistryUran.h:64-65
    c.sinthe_min = p.sinthe_min; c.floor = cp->polar_floor;
    c.per = cp->phi_periodic != 0;
    a.counts = ctx->counters + 4;
    a.scratch = reinterpret_cast<S*>(ctx->ybuf[0]);           // free outside the RK4 step
    Region reg(ctx, ATURAN_K_CHEM, 0, st);
    reg.n = launch_chem(a, what, st);
    CK_LAUNCH("chemistry");
    return ATURAN_OK;
}

// The turbulence closure on the context's fields (aturan_turbulence).
template <typename S>
int run_turb(aturan_ctx* ctx, const aturan_turb_params* tp){
    const Grid& g = ctx->g;
    const size_t fs = g.fstride;
    const aturan_params& p = ctx->p;
    S* X = reinterpret_cast<S*>(ctx->state);
    S* Nc = reinterpret_cast<S*>(ctx->ncopy);
    S* Fo = reinterpret_cast<S*>(ctx->forc);
    S* Ch = reinterpret_cast<S*>(ctx->chem);
    TurbArgs<S> a;
    a.g = g;
    a.tke = X + (size_t)ATURAN_TKE * fs; a.dis = X + (size_t)ATURAN_DIS * fs;
    a.tken = Nc + (size_t)ATURAN_TKE * fs; a.disn = Nc + (size_t)ATURAN_DIS * fs;
    a.nue = Fo + (size_t)(ATURAN_NUE - ATURAN_NUE) * fs;
    a.tks = Fo + (size_t)(ATURAN_TKE_SOURCE - ATURAN_NUE) * fs;
    a.dss = Fo + (size_t)(ATURAN_DIS_SOURCE - ATURAN_NUE) * fs;
    a.prod = Ch + (size_t)(ATURAN_PROD - ATURAN_DIFFLUX_H2S) * fs;
    a.u = X + (size_t)ATURAN_U * fs; a.v = X + (size_t)ATURAN_V * fs; a.w = X + (size_t)ATURAN_W * fs;
    a.rmm = ctx->chem_tab + g.im; a.sin = ctx->chem_tab + 2 * g.im; a.cos = ctx->chem_tab + 2 * g.im + g.jm;
    TurbConst& c = a.c;
    const double L_m = p.L_atm * 1.0e3;                                       // Turbulence.h:266-269
    c.dis_min = 1.0e-10;                                                      // :195
    c.nue_max = tp->nue_max / (p.u_0 * L_m);
    c.k_bg_nd = tp->k_bg / (p.u_0 * p.u_0);                                   // :622-628
    c.nue_air_nd = tp->nue_air / (p.u_0 * L_m);
    c.y_star = 1.0e20 / L_m;                                                  // free_wall_dist(), :147
    c.dr = p.dr; c.dthe = p.dthe; c.dphi = p.dphi;
    c.curv = tp->curv != 0; c.per = tp->phi_periodic != 0;
    Region reg(ctx, ATURAN_K_TURB, 0);
    reg.n = launch_turb(a, ctx->st);
    CK_LAUNCH("turbulence closure");
    return ATURAN_OK;
}

// The precipitation on the context's fields (aturan_precipitation).
template <typename S>
int run_precip(aturan_ctx* ctx, const aturan_precip_params* pp, cudaStream_t st = nullptr){
    if(!st) st = ctx->st;
    const Grid& g = ctx->g;
    const size_t fs = g.fstride;
    const aturan_params& p = ctx->p;
    S* X = reinterpret_cast<S*>(ctx->state);
    S* Fo = reinterpret_cast<S*>(ctx->forc);
    auto fo = [&](int id) -> S* { return Fo + (size_t)(id - ATURAN_NUE) * fs; };
    PrecipArgs<S> a;
    a.g = g;
    a.t = X + (size_t)ATURAN_T * fs;
    a.tlo = ctx->tlo;
    a.ps = reinterpret_cast<const S*>(ctx->pstat);
    a.rho = fo(ATURAN_RHO_MIX);
    a.Q = fo(ATURAN_Q_PRECIP);
    // the reference's species order H2O, NH3, CH4, H2S (Precipitation.h:214-262, cUranusModel.h:280-297)
    const int vap[4] = { ATURAN_H2O, ATURAN_NH3, ATURAN_CH4, ATURAN_H2S };
    const int src[4] = { ATURAN_S_PRECIP_H2O, ATURAN_S_PRECIP_NH3, ATURAN_S_PRECIP_CH4, ATURAN_S_PRECIP_H2S };
    const int gas[4] = { 0, 2, 3, 1 };                           // the params' order is H2O, H2S, NH3, CH4
    for(int n = 0; n < 4; n++){
        for(int c = 0; c < 3; c++){
            a.sp[n][c] = X + (size_t)(vap[n] + c) * fs;
            a.ss[n][c] = fo(src[n] + c);
        }
        const aturan_gas& G = p.gas[gas[n]];
        a.gas[n] = PrecipGas{ G.C, G.L0, 1e-3 * G.R, G.del_alf, G.del_bet, G.ep, G.lv, G.ls - G.lv, G.t_0, G.t_00 };
    }
    a.dz = ctx->dz_tab;
    a.rs = pp->rate_scale;
    a.nd = (p.L_atm * 1.0e3) / p.u_0;                                         // Precipitation.h:420
    a.r_mix = p.r_mix; a.t_ref = p.t_ref;
    a.coupling = pp->coupling != 0; a.h2s = pp->h2s != 0; a.local_rho = p.local_rho != 0;
    Region reg(ctx, ATURAN_K_PRECIP, 0, st);
    reg.n = launch_precip(a, st);
    CK_LAUNCH("precipitation");
    return ATURAN_OK;
}

// The moist convective adjustment on the context's fields (aturan_mca).
template <typename S>
int run_mca(aturan_ctx* ctx){
    const Grid& g = ctx->g;
    const aturan_params& p = ctx->p;
    if(mca_warp_bytes(g.im) > MCA_SMEM_MAX) return fail(ctx, ATURAN_E_UNSUPPORTED, "column too deep for the shared memory");
    int nl = 0;
    if(!ctx->mca_H_ready){
        // the cp table's running integral, formed once; ready only once its kernel has launched
        if(!ctx->mca_H && cudaMalloc((void**)&ctx->mca_H, CP_TABLE_N * sizeof(double)) != cudaSuccess){
            cudaGetLastError(); ctx->mca_H = nullptr; return fail(ctx, ATURAN_E_NOMEM, "mca: cp integral");
        }
        launch_mca_H(ctx->cp_tab64, ctx->mca_H, ctx->st);
        CK_LAUNCH("moist convective adjustment: cp integral");
        ctx->mca_H_ready = true;
        nl++;
    }
    McaArgs<S> a;
    a.g = g;
    McaConst& c = a.c;
    const int order[MCA_NG] = { 0, 2, 1, 3 };                  // H2O, NH3, H2S, CH4 from the params' H2O, H2S, NH3, CH4
    const int fv[MCA_NG] = { ATURAN_H2O, ATURAN_NH3, ATURAN_H2S, ATURAN_CH4 };
    S* X = reinterpret_cast<S*>(ctx->state);
    const size_t fs = g.fstride;
    for(int n = 0; n < MCA_NG; n++){
        const aturan_gas& s = p.gas[order[n]];
        c.G[n] = McaGas{ s.ep, s.lv, s.ls, s.t_0, s.C, s.L0, s.R, s.del_alf, s.del_bet, s.C_i, s.L0_i, s.del_alf_i, s.del_bet_i };
        for(int q = 0; q < 3; q++) a.sp[n][q] = X + (size_t)(fv[n] + q) * fs;
    }
    c.L_tr = p.nh4sh_sync ? 4705.0 * std::log(10.0) * 8314.46 / 51.1114 : 0.0;   // ChemistryUran.h:132
    c.t_ref = p.t_ref; c.grav = p.g; c.cp_mix = p.cp_mix; c.r_mix = p.r_mix; c.cp_h2 = p.cp_h2;
    c.r_h2 = p.r_h2; c.r_he = p.r_he; c.r_ch4 = p.r_ch4; c.cp_he = p.cp_he; c.cp_ch4 = p.cp_ch4;
    c.hz = (float)(p.L_atm / (g.im - 1));                      // cUranusModel.h:1205-1208
    c.cp_dyn = p.cp_dyn; c.cp_mode = p.cp_h2_mode; c.cp_gas = p.cp_gas; c.local_rho = p.local_rho;
    c.cp_tab = ctx->cp_tab64; c.H_tab = ctx->mca_H;
    a.t = X + (size_t)ATURAN_T * fs;
    a.tlo = ctx->tlo;
    a.nh4sh = X + (size_t)ATURAN_NH4SH * fs;
    a.ps = reinterpret_cast<const S*>(ctx->pstat);
    a.rho = reinterpret_cast<const S*>(ctx->forc) + (size_t)(ATURAN_RHO_MIX - ATURAN_NUE) * fs;
    Region reg(ctx, ATURAN_K_MCA, 0);
    const int n = launch_mca(a, ctx->st);
    if(n < 0) return fail(ctx, ATURAN_E_UNSUPPORTED, "mca: the column's shared memory");
    reg.n = nl + n;
    CK_LAUNCH("moist convective adjustment");
    return ATURAN_OK;
}

extern "C" {

int aturan_params_default(aturan_params* p){
    if(!p) return ATURAN_E_INVALID;
    std::memset(p, 0, sizeof(*p));
    p->abi_version = ATURAN_ABI_VERSION;
    p->im = 41; p->jm = 181; p->km = 361;
    p->precision = ATURAN_FP64;
    p->turb_active = 1; p->coriolis_full = 1; p->cp_h2_mode = 2; p->cp_gas = 1; p->cp_dyn = 1;
    p->press_consistent = 1; p->press_incr = 1; p->rigid_lid = 1;
    p->satadj_conserve = 1; p->satadj_newton = 1; p->satadj_evap = 1; p->satadj_ice_entry = 0;
    p->satadj_bergeron = 2; p->satadj_freeze = 1; p->satadj_dry_exit = 1; p->local_rho = 1;
    p->nh4sh_sync = 1; p->exact_reductions = 1;
    const double pi180 = 180.0 / M_PI;                        // cUranusModel.cpp:340-351
    p->r0 = 1.0; p->dr = 0.025; p->the0 = 0.0; p->dthe = 1.0 / pi180; p->phi0 = 0.0; p->dphi = 1.0 / pi180;
    p->dt = 0.001; p->metric_R_km = 25362.0; p->sinthe_min = 0.4;
    p->L_atm = 225.0; p->u_0 = 100.0; p->t_ref = 76.4; p->g = 8.69; p->omega = 0.000101;
    p->re = 1000.0; p->pr = 0.69; p->Coriolis = 1.0; p->centrifugal = 1.0; p->buoyancy = 1.0;
    p->chemical_reaction = 1.0; p->R_ref = 3.61491; p->p_ref = 1.0;
    p->r_mix = 0x1.d296ea433d4a6p+1; p->R_mix = 0x1.31fad52a5899ap+11;
    p->cp_mix = 0x1.0f59f37b7f291p+13; p->mue_mix = 0x1.5e6b31135aa58p-17;
    p->r_h2 = 0x1.e0c778070069fp+0; p->r_he = 0x1.2eb67afaed4c3p-2; p->r_ch4 = 0x1.a6e858fcad66bp-2;
    p->cp_h2 = 14.32e3; p->cp_he = 5.19e3; p->cp_ch4 = 2.232e3;
    p->sc_ch4 = 0.99; p->sc_h2o = 0.61; p->sc_h2s = 0.94; p->sc_nh3 = 0.61; p->sc_nh4sh = 0.7;
    p->alpha_sponge = 10.0; p->r_p_nh4sh = 1.0e-5; p->rho_cond_nh4sh = 1170.0;
    p->turb_coupling = 1.0; p->precip_coupling = 1.0; p->tmf_scale = 0.0; p->cent_mom = 0.0;
    p->pbaro_follow = 64.0; p->t_min_K = 7.5; p->t_max_K = 2000.0; p->p_dyn_cap = 0.2;
    p->satadj_stop_tol = 1.0e-3;
    const double G[4][14] = {
        {273.15, 210.15, 8.1253, 2.5009e6, 2.8339e6, 25.096, 3148.2, 461.52, 0.0, -8.7e-3, 28.418, 3567.3, 0.0, -8.7e-3},
        {187.65, 140.0, 14.5192, 5.5e5, 7.45e5, 17.064, 747.0, 243.96, 0.0, -2.9e-3, 17.064, 747.0, 0.0, -2.9e-3},
        {195.5, 140.0, 7.6752, 1.3720e6, 1.8320e6, 27.863, 2016.0, 488.21, -0.888, 0.0, 34.948, 2692.5, -0.888, 0.0},
        {90.69, 67.36, 7.6752, 5.11e5, 5.11e5, 1.627, 553.1, 518.28, 1.002, -4.1e-3, 1.627, 553.1, 1.002, -4.1e-3}};
    for(int n = 0; n < 4; n++) std::memcpy(&p->gas[n], G[n], sizeof(G[n]));
    return ATURAN_OK;
}

const char* aturan_last_error(const aturan_ctx* ctx){
    return ctx ? ctx->err.c_str() : aturan::static_last_error();
}

int aturan_ctx_create(const aturan_params* p, aturan_ctx** out){
    if(!p || !out) return ATURAN_E_INVALID;
    *out = nullptr;
    std::string why;
    int rc = validate(p, why);
    if(rc){ std::fprintf(stderr, "aturan_ctx_create: %s\n", why.c_str()); return rc; }
    int ndev = 0;
    if(cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0){
        cudaGetLastError();
        std::fprintf(stderr, "aturan_ctx_create: no CUDA device\n");
        return ATURAN_E_CUDA;
    }
    aturan_ctx* ctx = new (std::nothrow) aturan_ctx();
    if(!ctx) return ATURAN_E_NOMEM;
    ctx->p = *p;
    cudaGetDevice(&ctx->device);
    ctx->mixed = p->precision == ATURAN_MIXED;
    ctx->esz = ctx->mixed ? sizeof(float) : sizeof(double);
    Grid& g = ctx->g;
    g.im = p->im; g.jm = p->jm; g.km = p->km;
    g.kp = (int)round_up(p->km, 32);
    g.fstride = (size_t)g.im * g.jm * g.kp;
    ctx->nblk = 32;
    const size_t fs = g.fstride, e = ctx->esz;
    const size_t nij = (size_t)g.im * g.jm;
    const size_t sgeo = ctx->mixed ? sizeof(GeoIJ<float>) : sizeof(GeoIJ<double>);
    size_t bytes = 0;
    auto add = [&](size_t n){ bytes += round_up(n, 256); };
    add(19 * fs * e); add(19 * fs * e); add(19 * fs * e); add(19 * fs * e); add(19 * fs * e);
    add(22 * fs * e); add(6 * fs * e); add(4 * fs * e); add(fs * e);
    for(int n = 0; n < 7; n++) add(fs * 8);                   // pdyn phydro pbaro pb0 pbf scratch stage64
    add(g.im * 8); add(2 * (size_t)g.im * ctx->nblk * 8);
    // the exact level means (FP64 with exact_reductions): terms, chunk sums, binades, units
    const bool bx_on = !ctx->mixed && p->exact_reductions;
    const size_t ncell = (size_t)g.jm * g.km;
    ctx->bx.nbx = (int)((ncell + BX_CH - 1) / BX_CH);
    const size_t nbx_all = (size_t)g.im * ctx->bx.nbx;
    if(bx_on){ add(2 * g.im * ncell * 8); add(3 * nbx_all * 8); add(2 * nbx_all * 4); add(4 * nbx_all * 8); }
    add(g.jm * 8); add(g.im * 8); add(g.jm * 8); add(CP_TABLE_N * 8);
    add((size_t)(2 * g.im + 2 * g.jm) * 8); add((size_t)g.im * 8);
    add(nij * sgeo); add(CP_TABLE_N * e); add(nij * sizeof(GSW)); add(nij * sizeof(RBW)); add(64);
    const int sJ = g.jm - 2, sN = g.km - 1, sNM = sN / 2;
    ctx->sor_nblk = ((sN + 31) / 32) * sJ;
    ctx->sor_pm = std::max(1, std::min(4, (200 * 1024 / (8 * sJ) - 4) / 5));
    for(int n = 0; n < 4; n++) add((size_t)(sNM + 1) * sN * 8);        // ct, st, ctT, stT
    add((size_t)sJ * sN * 8); add((size_t)SOR_KSPLIT * (sNM + 1) * sJ * 8); add((size_t)SOR_KSPLIT * (sNM + 1) * sJ * 8);
    add((size_t)(2 * ctx->sor_nblk + 2) * 8); add((size_t)SOR_KSPLIT * sJ * sN * 8);     // partials (+ the shift); q
    for(int n = 0; n < 6; n++) add((size_t)(sNM + 1) * sJ * 8);        // mode factorisations (Lc, Lc^T)
    for(int n = 0; n < 6; n++) add(nij * 8);                           // line factorisations (Lc, Lc^T)
    add(fs * 4); add(fs * 4);
    if(ctx->mixed) add(2 * fs * 4);                                    // the temperature pair's low parts
    ctx->mem_bytes = bytes;
    // the stage kernels address every buffer of the allocation by 32-bit element offsets
    if(bytes / e >= (size_t)INT32_MAX){
        std::fprintf(stderr, "aturan_ctx_create: grid too large (%zu elements of context memory, limit 2^31)\n", bytes / e);
        delete ctx; return ATURAN_E_UNSUPPORTED;
    }
    int prio_lo = 0, prio_hi = 0;                         // least and most urgent
    if(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi) != cudaSuccess){ cudaGetLastError(); prio_lo = prio_hi = 0; }
    if(cudaStreamCreateWithPriority(&ctx->st, cudaStreamNonBlocking, prio_hi) != cudaSuccess){
        delete ctx; return ATURAN_E_CUDA;
    }
    if(cudaStreamCreateWithPriority(&ctx->st2, cudaStreamNonBlocking, prio_lo) != cudaSuccess){
        cudaStreamDestroy(ctx->st); delete ctx; return ATURAN_E_CUDA;
    }
    {
        cudaEvent_t* evs[6] = {&ctx->ev_fork, &ctx->ev_join, &ctx->ev_xcopy[0], &ctx->ev_xcopy[1],
                               &ctx->ev_xpack[0], &ctx->ev_xpack[1]};
        for(cudaEvent_t* e : evs){
            if(cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess){
                cudaGetLastError();
                aturan_ctx_destroy(ctx); return ATURAN_E_CUDA;
            }
        }
    }
    if(cudaMalloc((void**)&ctx->mem, bytes) != cudaSuccess){
        cudaGetLastError();
        aturan_ctx_destroy(ctx); return ATURAN_E_NOMEM;
    }
    char* cur = ctx->mem;
    ctx->state = carve<char>(cur, 19 * fs * e);
    ctx->ncopy = carve<char>(cur, 19 * fs * e);
    ctx->ybuf[0] = carve<char>(cur, 19 * fs * e);
    ctx->ybuf[1] = carve<char>(cur, 19 * fs * e);
    ctx->acc = carve<char>(cur, 19 * fs * e);
    ctx->forc = carve<char>(cur, 22 * fs * e);
    ctx->proj = carve<char>(cur, 6 * fs * e);
    ctx->chem = carve<char>(cur, 4 * fs * e);
    ctx->pstat = carve<char>(cur, fs * e);
    ctx->pdyn = carve<double>(cur, fs); ctx->phydro = carve<double>(cur, fs);
    ctx->pbaro = carve<double>(cur, fs); ctx->pb0 = carve<double>(cur, fs); ctx->pbf = carve<double>(cur, fs);
    ctx->scratch = carve<double>(cur, fs); ctx->stage64 = carve<double>(cur, fs);
    ctx->ref_level = carve<double>(cur, g.im);
    ctx->part_sum = carve<double>(cur, 2 * (size_t)g.im * ctx->nblk);
    ctx->part_w = ctx->part_sum + (size_t)g.im * ctx->nblk;
    if(bx_on){
        ctx->bx.terms = carve<double>(cur, 2 * g.im * ncell);
        ctx->bx.bpart = carve<double>(cur, 3 * nbx_all);
        ctx->bx.bexp = carve<int>(cur, 2 * nbx_all);
        ctx->bx.bunits = carve<long long>(cur, 4 * nbx_all);
    }
    ctx->wsin = carve<double>(cur, g.jm); ctx->rm_i = carve<double>(cur, g.im); ctx->cor_j = carve<double>(cur, g.jm);
    ctx->cp_tab64 = carve<double>(cur, CP_TABLE_N);
    ctx->chem_tab = carve<double>(cur, 2 * (size_t)g.im + 2 * (size_t)g.jm);
    ctx->dz_tab = carve<double>(cur, g.im);
    ctx->geo = carve<char>(cur, nij * sgeo);
    ctx->cp_tab = carve<char>(cur, CP_TABLE_N * e);
    ctx->gsw = carve<GSW>(cur, nij); ctx->rbw = carve<RBW>(cur, nij);
    ctx->counters = carve<unsigned long long>(cur, 8);
    ctx->sor_ct = carve<double>(cur, (size_t)(sNM + 1) * sN); ctx->sor_st = carve<double>(cur, (size_t)(sNM + 1) * sN);
    ctx->sor_ctT = carve<double>(cur, (size_t)(sNM + 1) * sN); ctx->sor_stT = carve<double>(cur, (size_t)(sNM + 1) * sN);
    ctx->sor_colR = carve<double>(cur, (size_t)sJ * sN);
    ctx->sor_Ac = carve<double>(cur, (size_t)SOR_KSPLIT * (sNM + 1) * sJ);
    ctx->sor_As = carve<double>(cur, (size_t)SOR_KSPLIT * (sNM + 1) * sJ);
    ctx->sor_part = carve<double>(cur, (size_t)2 * ctx->sor_nblk + 2);
    ctx->sor_q = carve<double>(cur, (size_t)SOR_KSPLIT * sJ * sN);
    ctx->mlu_a = carve<double>(cur, (size_t)(sNM + 1) * sJ); ctx->mlu_cf = carve<double>(cur, (size_t)(sNM + 1) * sJ);
    ctx->mlu_idn = carve<double>(cur, (size_t)(sNM + 1) * sJ);
    ctx->llu_a = carve<double>(cur, nij); ctx->llu_cf = carve<double>(cur, nij); ctx->llu_idn = carve<double>(cur, nij);
    ctx->mluT_a = carve<double>(cur, (size_t)(sNM + 1) * sJ); ctx->mluT_cf = carve<double>(cur, (size_t)(sNM + 1) * sJ);
    ctx->mluT_idn = carve<double>(cur, (size_t)(sNM + 1) * sJ);
    ctx->lluT_a = carve<double>(cur, nij); ctx->lluT_cf = carve<double>(cur, nij); ctx->lluT_idn = carve<double>(cur, nij);
    ctx->r32 = carve<float>(cur, fs); ctx->e32 = carve<float>(cur, fs);
    ctx->tlo = ctx->mixed ? carve<float>(cur, 2 * fs) : nullptr;
    ctx->host_part.resize(2 * ctx->sor_nblk);

    // zero everything once: padding columns and unused planes read as 0, never as garbage
    if(cudaMemsetAsync(ctx->mem, 0, bytes, ctx->st) != cudaSuccess){ aturan_ctx_destroy(ctx); return ATURAN_E_CUDA; }

    // ---- host tables ----
    std::vector<double> rad, the;
    coords(*p, rad, the);
    std::vector<double> wsin(g.jm), rm_i(g.im), cor_j(g.jm), cp64(CP_TABLE_N);
    const double scale_Cor = (p->coriolis_full ? p->L_atm * 1.0e3 : p->L_atm) / p->u_0;
    for(int j = 0; j < g.jm; j++){
        wsin[j] = std::sin(the[j]);                                             // RungeKutta_Uran_Turb.cpp:25
        cor_j[j] = p->Coriolis * scale_Cor * 2.0 * p->omega * std::abs(std::sin(the[j]));   // :132-133
    }
    for(int i = 0; i < g.im; i++) rm_i[i] = metric_radius(*p, rad[i]);
    const int mode = p->cp_h2_mode > 0 ? p->cp_h2_mode : 2;
    for(int n = 0; n < CP_TABLE_N; n++) cp64[n] = cpR_exact(5.0 + n * 0.5, mode) * 8.314462618 / 2.01588e-3;

    std::vector<GeoIJ<double>> geo(nij);
    std::vector<GSW> gsw(nij);
    std::vector<RBW> rbw(nij);
    const double inv_dr2 = 1.0 / (p->dr * p->dr), inv_dthe2 = 1.0 / (p->dthe * p->dthe), inv_dphi2 = 1.0 / (p->dphi * p->dphi);
    std::vector<double> st_uran(g.jm), st_shared(g.jm);
    for(int j = 0; j < g.jm; j++){                     // PressureSolverUran.h:42-47, PressureSolver.h:156-162
        st_uran[j] = std::sin(the[j]);
        if(st_uran[j] < p->sinthe_min) st_uran[j] = p->sinthe_min;
        st_shared[j] = st_uran[j];
        if(st_shared[j] == 0.0) st_shared[j] = 1.0e-5;
    }
    const int im = g.im;
    for(int i = 0; i < g.im; i++){
        double frac_sp = (double)(i - (im - 1) * 3 / 4) / (double)((im - 1) / 4);   // RHS_Uran_Turb.cpp:594-595
        frac_sp = stdmax(0.0, frac_sp);
        const double sponge = p->alpha_sponge * frac_sp * frac_sp;
        for(int j = 0; j < g.jm; j++){
            GeoIJ<double>& G = geo[(size_t)i * g.jm + j];
            // RungeKutta_Uran_Turb.cpp:192-197, 266-277
            const double rm = metric_radius(*p, rad[i]);
            const double rm2 = rm * rm;
            const double sinthe = stdmax(p->sinthe_min, std::abs(std::sin(the[j])));
            const double sinthe2 = sinthe * sinthe;
            const double costhe = std::cos(the[j]);
            G.cotanthe = costhe / sinthe;
            G.inv_rm = 1.0 / rm;
            G.inv_rm2 = 1.0 / rm2;
            G.inv_rmsinthe = 1.0 / (rm * sinthe);
            G.inv_rm2sinthe = G.inv_rm2 / sinthe;
            G.inv_rm2sinthe2 = G.inv_rm2 / sinthe2;
            G.costhe_inv_rm2sinthe = costhe * G.inv_rm2sinthe;
            G.costhe = costhe;
            G.v_metric = (1.0 + costhe / sinthe2) * G.inv_rm2;                         // RHS_Uran_Turb.cpp:331
            G.two_inv_rm = 2.0 * G.inv_rm;                                              // :330
            G.sinthe_bf = std::sqrt(stdmax(0.0, 1.0 - costhe * costhe));               // :224
            G.cent_rad = p->omega * p->omega * rm * G.sinthe_bf * G.sinthe_bf;          // :276
            G.cent_the = p->omega * p->omega * rm * G.sinthe_bf * costhe;               // :277
            G.sponge = sponge;

            // PressureSolverUran weights (:151-157, :180-190)
            const double rmc = p->press_consistent ? rm : rad[i];
            GSW& W = gsw[(size_t)i * g.jm + j];
            {
                const double s = st_uran[j];
                const double inv_rm = 1.0 / rmc;
                const double inv_rmsinthe = 1.0 / (rmc * s);
                const double inv_rm2 = inv_rm * inv_rm;
                const double inv_rm2sinthe2 = inv_rm2 / (s * s);
                W.n1 = 1.0 / (p->dr * p->dr); W.n2 = inv_rm2 / (p->dthe * p->dthe);
                W.n3 = inv_rm2sinthe2 / (p->dphi * p->dphi);
                W.denom = 2.0 * (W.n1 + W.n2 + W.n3);
                W.inv_rm = inv_rm; W.inv_rmsinthe = inv_rmsinthe;
                const double rm2c = rmc * rmc;
                const double inv_rm2b = 1.0 / rm2c;
                const double inv_rm2sinthe2b = inv_rm2b / (s * s);
                const double denom = 2.0 * inv_dr2 + 2.0 * inv_rm2b * inv_dthe2 + 2.0 * inv_rm2sinthe2b * inv_dphi2;
                W.inv_denom = 1.0 / denom;
                W.num1 = inv_dr2; W.num2 = inv_rm2b * inv_dthe2; W.num3 = inv_rm2sinthe2b * inv_dphi2;
            }
            // shared solver weights (PressureSolver.h:326-353, 484)
            RBW& R = rbw[(size_t)i * g.jm + j];
            {
                const double s = st_shared[j];
                const double inv_rm2 = 1.0 / rm2;
                const double inv_rm2sinthe2 = inv_rm2 / (s * s);
                const double exp_2_rm = 1.0 * 1.0;
                R.num1 = exp_2_rm * inv_dr2; R.num2 = inv_rm2 * inv_dthe2; R.num3 = inv_rm2sinthe2 * inv_dphi2;
                R.den = 2.0 * R.num1 + 2.0 * R.num2 + 2.0 * R.num3;
                R.inv_rm = 1.0 / rm; R.inv_rmsinthe = 1.0 / (rm * s);
                R.src_max = R.den * p->p_dyn_cap;
            }
        }
    }
    ctx->k64 = make_rhs_const<double>(*p);
    ctx->k32 = make_rhs_const<float>(*p);
    HydroConst& h = ctx->hc;                             // RungeKutta_Uran_Turb.cpp:76-99
    h.g = p->g; h.rR = p->r_mix * p->R_mix; h.t_ref = p->t_ref;
    const double nd_rel = p->g * (p->L_atm * 1.0e3) / (p->u_0 * p->u_0);
    h.m_nd_rel_b = -nd_rel * 1.0 * p->buoyancy;
    h.dr = p->dr; h.follow_tau = p->pbaro_follow; h.follow_on = p->pbaro_follow > 0.0;
    SatConst& sc = ctx->sc;
    for(int n = 0; n < 4; n++){
        const aturan_gas& G = p->gas[n];
        GasConst& K = sc.gas[n];
        K.t_0 = G.t_0; K.t_00 = G.t_00; K.ep = G.ep; K.lv = G.lv; K.ls = G.ls;
        K.C = G.C; K.L0 = G.L0; K.den = 1e-3 * G.R; K.del_alf = G.del_alf; K.del_bet = G.del_bet;
        K.inv_den = 1.0 / K.den;
        K.C_i = G.C_i; K.L0_i = G.L0_i; K.del_alf_i = G.del_alf_i; K.del_bet_i = G.del_bet_i;
        K.t_range_inv = 1.0 / (G.t_0 - G.t_00);
        K.Lf = G.ls - G.lv;
        K.freeze_on = p->satadj_freeze && p->satadj_conserve && G.t_00 > 0.0 && G.t_00 < G.t_0;
    }
    sc.cp_mix = p->cp_mix; sc.t_ref = p->t_ref; sc.r_mix = p->r_mix;
    sc.stop_tol = p->satadj_stop_tol > 0.0 ? p->satadj_stop_tol : 1.0e-3;
    sc.entry_tol = p->satadj_entry_tol == 0.0 ? 1.0e-3 : (p->satadj_entry_tol < 0.0 ? 0.0 : p->satadj_entry_tol);
    sc.conserve = p->satadj_conserve; sc.newton = p->satadj_newton; sc.evap = p->satadj_evap;
    sc.ice_entry = p->satadj_ice_entry; sc.bergeron = p->satadj_bergeron; sc.dry_exit = p->satadj_dry_exit;
    sc.local_rho = p->local_rho;
    PressConst& pc = ctx->pc;
    pc.inv_2dr = 1.0 / (2.0 * p->dr); pc.inv_2dthe = 1.0 / (2.0 * p->dthe); pc.inv_2dphi = 1.0 / (2.0 * p->dphi);
    pc.two_dr = 2.0 * p->dr; pc.two_dthe = 2.0 * p->dthe; pc.two_dphi = 2.0 * p->dphi;
    pc.src_scale = p->press_consistent ? (p->r_mix * p->u_0 * p->u_0) / 1.0e5 : 1.0;
    pc.press_incr = p->press_incr;

    // RB_SOR tables: Fourier bases with the exact (m k mod N) reduction (PressureSolver.h:614-617),
    // eigenvalues of the phi ring, the shared solver's floored sine of the interior rows, and
    // A2y = sum_i y_i / rm_i^2 with the folded operator's left null vector y.
    std::vector<double> sct((size_t)(sNM + 1) * sN), sst((size_t)(sNM + 1) * sN);
    std::vector<double> sctT((size_t)(sNM + 1) * sN), sstT((size_t)(sNM + 1) * sN);
    std::vector<double> ma((size_t)(sNM + 1) * sJ), mcf((size_t)(sNM + 1) * sJ), midn((size_t)(sNM + 1) * sJ);
    std::vector<double> maT(ma.size()), mcfT(ma.size()), midnT(ma.size());
    // LU of a tridiagonal (sub A, diagonal B, super C) without pivoting: forward y_q = (d_q -
    // A_q y_{q-1}) idn_q, back x_q = y_q - cf_q x_{q+1}; and the transpose's (sub and super swap
    // and shift by one row).
    auto factor = [](const std::vector<double>& A, const std::vector<double>& B, const std::vector<double>& Cc,
                     double* fa, double* fc, double* fi, size_t stride){
        const int n = (int)B.size();
        for(int q = 0; q < n; q++){
            const double dn = (q == 0) ? B[0] : B[q] - A[q] * fc[(q - 1) * stride];
            fa[q * stride] = (q == 0) ? 0.0 : A[q]; fi[q * stride] = 1.0 / dn; fc[q * stride] = Cc[q] * fi[q * stride];
        }
    };
    auto transpose3 = [](const std::vector<double>& A, const std::vector<double>& Cc,
                         std::vector<double>& AT, std::vector<double>& CT){
        const int n = (int)A.size();
        for(int q = 0; q < n; q++){
            AT[q] = (q == 0) ? 0.0 : Cc[q - 1];
            CT[q] = (q == n - 1) ? 0.0 : A[q + 1];
        }
    };
    for(int m = 0; m <= sNM; m++){
        for(int k = 0; k < sN; k++){
            const double a = 2.0 * M_PI * (double)((long)m * k % sN) / sN;
            sct[(size_t)m * sN + k] = std::cos(a); sst[(size_t)m * sN + k] = std::sin(a);
            sctT[(size_t)k * (sNM + 1) + m] = std::cos(a); sstT[(size_t)k * (sNM + 1) + m] = std::sin(a);
        }
        // theta tridiagonal of mode m, ends folded (q0 = c43 q1 - c13 q2), factored once
        const double sl = std::sin(M_PI * m / sN);
        const double lam = 4.0 * sl * sl * inv_dphi2;
        const double e = inv_dthe2;
        std::vector<double> A(sJ), B(sJ), Cc(sJ);
        for(int q = 0; q < sJ; q++){
            const double s_ = st_shared[q + 1];
            A[q] = e; Cc[q] = e; B[q] = -2.0 * e - lam / (s_ * s_);
        }
        A[0] = 0.0;       B[0] += C43 * e;      Cc[0] -= C13 * e;
        Cc[sJ - 1] = 0.0; B[sJ - 1] += C43 * e; A[sJ - 1] -= C13 * e;
        std::vector<double> AT(sJ), BT(B), CT(sJ);
        transpose3(A, Cc, AT, CT);
        if(m == 0){ B[0] = 1.0; Cc[0] = 0.0; BT[0] = 1.0; CT[0] = 0.0; }   // pin q at the first row
        factor(A, B, Cc, &ma[(size_t)m * sJ], &mcf[(size_t)m * sJ], &midn[(size_t)m * sJ], 1);
        factor(AT, BT, CT, &maT[(size_t)m * sJ], &mcfT[(size_t)m * sJ], &midnT[(size_t)m * sJ], 1);
    }
    // radial-line tridiagonal of every (i,j) column of the folded operator, and of its transpose,
    // factored once (row q of column j at index (q+1)*jm + j)
    std::vector<double> la(nij, 0.0), lcf(nij, 0.0), lidn(nij, 0.0);
    std::vector<double> laT(nij, 0.0), lcfT(nij, 0.0), lidnT(nij, 0.0);
    for(int j = 1; j < g.jm - 1; j++){
        const int n = g.im - 2;
        std::vector<double> A(n), B(n), Cc(n);
        for(int q = 0; q < n; q++){
            const RBW& R = rbw[(size_t)(q + 1) * g.jm + j];
            double d = R.den;
            if(j == 1) d -= C43 * R.num2;
            if(j == g.jm - 2) d -= C43 * R.num2;
            A[q] = -R.num1; B[q] = d; Cc[q] = -R.num1;
        }
        B[0] += A[0] * C43; Cc[0] -= A[0] * C13; A[0] = 0.0;
        B[n - 1] += Cc[n - 1] * C43; A[n - 1] -= Cc[n - 1] * C13; Cc[n - 1] = 0.0;
        std::vector<double> AT(n), CT(n);
        transpose3(A, Cc, AT, CT);
        const size_t f0 = (size_t)g.jm + j;
        factor(A, B, Cc, &la[f0], &lcf[f0], &lidn[f0], g.jm);
        factor(AT, B, CT, &laT[f0], &lcfT[f0], &lidnT[f0], g.jm);
    }
    double A2y = 0.0;
    for(int i = 1; i < g.im - 1; i++){
        const double rm = metric_radius(*p, rad[i]);
        A2y += ((i == 1 || i == g.im - 2) ? 1.5 : 1.0) / (rm * rm);
    }
    ctx->sorc.J = sJ; ctx->sorc.N = sN; ctx->sorc.NM = sNM; ctx->sorc.inv_dthe2 = inv_dthe2; ctx->sorc.A2y = A2y;
    {
        const size_t tri = (size_t)8 * sJ * (5 * ctx->sor_pm + 4);   // the tridiagonal kernel's shared memory
        if(tri > 48 * 1024 && tri <= 227 * 1024 &&
           cudaFuncSetAttribute(sor_tridiag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tri) != cudaSuccess){
            cudaGetLastError();
            aturan_ctx_destroy(ctx);
            return ATURAN_E_CUDA;
        }
    }

    auto up = [&](void* dst, const void* src, size_t n) -> int {
        return cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, ctx->st) == cudaSuccess ? 0 : 1;
    };
    int bad = 0;
    bad |= up(ctx->wsin, wsin.data(), g.jm * 8);
    bad |= up(ctx->rm_i, rm_i.data(), g.im * 8);
    bad |= up(ctx->cor_j, cor_j.data(), g.jm * 8);
    bad |= up(ctx->cp_tab64, cp64.data(), CP_TABLE_N * 8);
    std::vector<double> chem_tab(2 * (size_t)g.im + 2 * (size_t)g.jm);
    for(int i = 0; i < g.im; i++){ chem_tab[i] = rad[i]; chem_tab[g.im + i] = rm_i[i]; }
    for(int j = 0; j < g.jm; j++){ chem_tab[2 * g.im + j] = std::sin(the[j]); chem_tab[2 * g.im + g.jm + j] = std::cos(the[j]); }
    bad |= up(ctx->chem_tab, chem_tab.data(), chem_tab.size() * 8);
    // cUranusModel.h:1199-1210 and :372-375: heights i * h in float, h = L_atm / (im-1) rounded
    // to float, the thickness as the float difference in metres (0 for the lid level)
    std::vector<double> dz_tab(g.im, 0.0);
    {
        const float h = (float)(p->L_atm / (g.im - 1));
        for(int i = 0; i + 1 < g.im; i++){
            const float hi = (float)(i + 1) * h, lo = (float)i * h;
            dz_tab[i] = (double)(hi - lo) * 1.0e3;
        }
    }
    bad |= up(ctx->dz_tab, dz_tab.data(), dz_tab.size() * 8);
    bad |= up(ctx->gsw, gsw.data(), nij * sizeof(GSW));
    bad |= up(ctx->rbw, rbw.data(), nij * sizeof(RBW));
    bad |= up(ctx->sor_ct, sct.data(), sct.size() * 8);
    bad |= up(ctx->sor_st, sst.data(), sst.size() * 8);
    bad |= up(ctx->sor_ctT, sctT.data(), sctT.size() * 8);
    bad |= up(ctx->sor_stT, sstT.data(), sstT.size() * 8);
    bad |= up(ctx->mlu_a, ma.data(), ma.size() * 8);
    bad |= up(ctx->mlu_cf, mcf.data(), mcf.size() * 8);
    bad |= up(ctx->mlu_idn, midn.data(), midn.size() * 8);
    bad |= up(ctx->llu_a, la.data(), nij * 8);
    bad |= up(ctx->llu_cf, lcf.data(), nij * 8);
    bad |= up(ctx->llu_idn, lidn.data(), nij * 8);
    bad |= up(ctx->mluT_a, maT.data(), maT.size() * 8);
    bad |= up(ctx->mluT_cf, mcfT.data(), mcfT.size() * 8);
    bad |= up(ctx->mluT_idn, midnT.data(), midnT.size() * 8);
    bad |= up(ctx->lluT_a, laT.data(), nij * 8);
    bad |= up(ctx->lluT_cf, lcfT.data(), nij * 8);
    bad |= up(ctx->lluT_idn, lidnT.data(), nij * 8);
    std::vector<GeoIJ<float>> geo32;
    std::vector<float> cp32;
    if(ctx->mixed){
        geo32.resize(nij);
        for(size_t n = 0; n < nij; n++){
            const double* s = reinterpret_cast<const double*>(&geo[n]);
            float* d = reinterpret_cast<float*>(&geo32[n]);
            for(size_t q = 0; q < sizeof(GeoIJ<double>) / sizeof(double); q++) d[q] = (float)s[q];
        }
        cp32.resize(CP_TABLE_N);
        for(int n = 0; n < CP_TABLE_N; n++) cp32[n] = (float)cp64[n];
        bad |= up(ctx->geo, geo32.data(), nij * sizeof(GeoIJ<float>));
        bad |= up(ctx->cp_tab, cp32.data(), CP_TABLE_N * sizeof(float));
    } else {
        bad |= up(ctx->geo, geo.data(), nij * sizeof(GeoIJ<double>));
        bad |= up(ctx->cp_tab, cp64.data(), CP_TABLE_N * 8);
    }
    if(bad || cudaStreamSynchronize(ctx->st) != cudaSuccess){
        cudaGetLastError();
        aturan_ctx_destroy(ctx);
        return ATURAN_E_CUDA;
    }
    *out = ctx;
    return ATURAN_OK;
}

int aturan_ctx_destroy(aturan_ctx* ctx){
    if(!ctx) return ATURAN_E_INVALID;
    if(ctx->st) cudaStreamSynchronize(ctx->st);
    if(ctx->st2) cudaStreamSynchronize(ctx->st2);
    if(ctx->gs_exec) cudaGraphExecDestroy(ctx->gs_exec);
    if(ctx->tape) cudaFree(ctx->tape);
    if(ctx->heat) cudaFree(ctx->heat);
    if(ctx->mca_H) cudaFree(ctx->mca_H);
    for(auto& e : ctx->evs){ cudaEventDestroy(e.a); cudaEventDestroy(e.b); }
    if(ctx->mem) cudaFree(ctx->mem);
    if(ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    if(ctx->ev_join) cudaEventDestroy(ctx->ev_join);
    for(int b = 0; b < 2; b++){
        if(ctx->ev_xcopy[b]) cudaEventDestroy(ctx->ev_xcopy[b]);
        if(ctx->ev_xpack[b]) cudaEventDestroy(ctx->ev_xpack[b]);
    }
    if(ctx->st2) cudaStreamDestroy(ctx->st2);
    if(ctx->st) cudaStreamDestroy(ctx->st);
    delete ctx;
    return ATURAN_OK;
}

void* aturan_stream(aturan_ctx* ctx){ return ctx ? (void*)ctx->st : nullptr; }

static int xfer(aturan_ctx* ctx, int field, void* other, bool up, bool other_is_device){
    if(!ctx || !other) return ATURAN_E_INVALID;
    if(field < 0 || field >= ATURAN_NFIELDS) return fail(ctx, ATURAN_E_INVALID, "field id out of range");
    bool is64;
    void* dev = field_ptr(ctx, field, &is64);
    const Grid& g = ctx->g;
    const size_t rows = (size_t)g.im * g.jm;
    // One contiguous copy of the caller's [im][jm][km] array into (out of) the staging field, and a
    // kernel that changes the layout to the padded rows (and the type, for FP32 fields): one large
    // DMA instead of im*jm row-sized ones. A device-side caller buffer is read (written) directly.
    const size_t n = rows * g.km;
    if(up){
        const double* src_c = reinterpret_cast<const double*>(other);
        if(!other_is_device){
            CK(cudaMemcpyAsync(ctx->stage64, other, n * 8, cudaMemcpyHostToDevice, ctx->st));
            src_c = ctx->stage64;
        }
        float* lo = t_lo_of(ctx, field);
        if(is64)    launch_pack_in_f64(src_c, reinterpret_cast<double*>(dev), g.km, g.kp, rows, ctx->st);
        else if(lo) launch_pack_in_pair(src_c, reinterpret_cast<float*>(dev), lo, g.km, g.kp, rows, ctx->st);
        else        launch_pack_in_f32(src_c, reinterpret_cast<float*>(dev), g.km, g.kp, rows, ctx->st);
        CK_LAUNCH("layout in");
        if(!other_is_device) CK(cudaStreamSynchronize(ctx->st));
    } else {
        double* tgt = other_is_device ? reinterpret_cast<double*>(other) : ctx->stage64;
        const float* lo = t_lo_of(ctx, field);
        if(is64)    launch_pack_out_f64(reinterpret_cast<const double*>(dev), tgt, g.km, g.kp, rows, ctx->st);
        else if(lo) launch_pack_out_pair(reinterpret_cast<const float*>(dev), lo, tgt, g.km, g.kp, rows, ctx->st);
        else        launch_pack_out_f32(reinterpret_cast<const float*>(dev), tgt, g.km, g.kp, rows, ctx->st);
        CK_LAUNCH("layout out");
        if(!other_is_device) CK(cudaMemcpyAsync(other, ctx->stage64, n * 8, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
    }
    return ATURAN_OK;
}

// Several fields in one call. With host buffers the DMA copies run on the side stream and the
// layout kernels on the main one, through two staging fields (stage64 and scratch, both free
// between calls) used in turn: field q's copy overlaps field q-1's layout kernel, and the call
// waits once, at the end, instead of once per field. Device buffers need no staging: the layout
// kernels run back to back on the main stream.
static int xfer_many(aturan_ctx* ctx, int n, const int* fields, void* const* ptrs, bool up, bool on_device){
    if(!ctx || n < 0 || (n > 0 && (!fields || !ptrs))) return ATURAN_E_INVALID;
    for(int q = 0; q < n; q++){
        if(fields[q] < 0 || fields[q] >= ATURAN_NFIELDS) return fail(ctx, ATURAN_E_INVALID, "field id out of range");
        if(!ptrs[q]) return fail(ctx, ATURAN_E_INVALID, "null buffer");
    }
    const Grid& g = ctx->g;
    const size_t rows = (size_t)g.im * g.jm, nval = rows * g.km;
    auto pack = [&](int field, const double* src, double* tgt) -> int {
        bool is64;
        void* dev = field_ptr(ctx, field, &is64);
        float* lo = t_lo_of(ctx, field);
        if(src){
            if(is64)    launch_pack_in_f64(src, reinterpret_cast<double*>(dev), g.km, g.kp, rows, ctx->st);
            else if(lo) launch_pack_in_pair(src, reinterpret_cast<float*>(dev), lo, g.km, g.kp, rows, ctx->st);
            else        launch_pack_in_f32(src, reinterpret_cast<float*>(dev), g.km, g.kp, rows, ctx->st);
        } else {
            if(is64)    launch_pack_out_f64(reinterpret_cast<const double*>(dev), tgt, g.km, g.kp, rows, ctx->st);
            else if(lo) launch_pack_out_pair(reinterpret_cast<const float*>(dev), lo, tgt, g.km, g.kp, rows, ctx->st);
            else        launch_pack_out_f32(reinterpret_cast<const float*>(dev), tgt, g.km, g.kp, rows, ctx->st);
        }
        CK_LAUNCH(src ? "layout in" : "layout out");
        return ATURAN_OK;
    };
    if(on_device){
        for(int q = 0; q < n; q++){
            const int rc = up ? pack(fields[q], reinterpret_cast<const double*>(ptrs[q]), nullptr)
                              : pack(fields[q], nullptr, reinterpret_cast<double*>(ptrs[q]));
            if(rc) return rc;
        }
        if(!up) CK(cudaStreamSynchronize(ctx->st));
        return ATURAN_OK;
    }
    double* buf[2] = {ctx->stage64, ctx->scratch};
    // the staging fields are free only once the work already queued on the main stream is done
    CK(cudaEventRecord(ctx->ev_fork, ctx->st));
    CK(cudaStreamWaitEvent(ctx->st2, ctx->ev_fork, 0));
    for(int q = 0; q < n; q++){
        const int b = q & 1;
        if(up){
            if(q >= 2) CK(cudaStreamWaitEvent(ctx->st2, ctx->ev_xpack[b], 0));     // field q-2's layout has read buf[b]
            CK(cudaMemcpyAsync(buf[b], ptrs[q], nval * 8, cudaMemcpyHostToDevice, ctx->st2));
            CK(cudaEventRecord(ctx->ev_xcopy[b], ctx->st2));
            CK(cudaStreamWaitEvent(ctx->st, ctx->ev_xcopy[b], 0));
            const int rc = pack(fields[q], buf[b], nullptr); if(rc) return rc;
            CK(cudaEventRecord(ctx->ev_xpack[b], ctx->st));
        } else {
            if(q >= 2) CK(cudaStreamWaitEvent(ctx->st, ctx->ev_xcopy[b], 0));      // field q-2's copy has read buf[b]
            const int rc = pack(fields[q], nullptr, buf[b]); if(rc) return rc;
            CK(cudaEventRecord(ctx->ev_xpack[b], ctx->st));
            CK(cudaStreamWaitEvent(ctx->st2, ctx->ev_xpack[b], 0));
            CK(cudaMemcpyAsync(ptrs[q], buf[b], nval * 8, cudaMemcpyDeviceToHost, ctx->st2));
            CK(cudaEventRecord(ctx->ev_xcopy[b], ctx->st2));
        }
    }
    CK(cudaEventRecord(ctx->ev_join, ctx->st2));
    CK(cudaStreamWaitEvent(ctx->st, ctx->ev_join, 0));
    CK(cudaStreamSynchronize(ctx->st));
    return ATURAN_OK;
}

int aturan_upload(aturan_ctx* ctx, int field, const double* host){ return xfer(ctx, field, (void*)host, true, false); }
int aturan_download(aturan_ctx* ctx, int field, double* host){ return xfer(ctx, field, host, false, false); }
int aturan_upload_many(aturan_ctx* ctx, int n, const int* fields, const double* const* src, int on_device){
    return xfer_many(ctx, n, fields, const_cast<void* const*>(reinterpret_cast<const void* const*>(src)), true, on_device != 0);
}
int aturan_download_many(aturan_ctx* ctx, int n, const int* fields, double* const* dst, int on_device){
    return xfer_many(ctx, n, fields, reinterpret_cast<void* const*>(dst), false, on_device != 0);
}
int aturan_upload_device(aturan_ctx* ctx, int field, const double* dev){ return xfer(ctx, field, (void*)dev, true, true); }
int aturan_download_device(aturan_ctx* ctx, int field, double* dev){ return xfer(ctx, field, dev, false, true); }

int aturan_download_buoy_ref(aturan_ctx* ctx, double* host){
    if(!ctx || !host) return ATURAN_E_INVALID;
    CK(cudaMemcpyAsync(host, ctx->ref_level, ctx->g.im * 8, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return ATURAN_OK;
}

int aturan_rk4_step(aturan_ctx* ctx){
    if(!ctx) return ATURAN_E_INVALID;
    return ctx->mixed ? run_rk4<float, float>(ctx, ctx->k32) : run_rk4<double, double>(ctx, ctx->k64);
}

int aturan_tape(aturan_ctx* ctx, int on){
    if(!ctx) return ATURAN_E_INVALID;
    if(!on){
        if(ctx->tape){ CK(cudaStreamSynchronize(ctx->st)); cudaFree(ctx->tape); }
        ctx->tape = nullptr;
        ctx->tape_valid = false;
        ctx->tape_p_valid = false;
        return ATURAN_OK;
    }
    if(on != 1 && on != 2) return fail(ctx, ATURAN_E_INVALID, "aturan_tape: on is 0, 1 (dry) or 2 (moist)");
    if(ctx->mixed) return fail(ctx, ATURAN_E_UNSUPPORTED, "the RK4 adjoint needs an FP64 context");
    const int want = on == 2 ? ADJ_NF_MOIST : ADJ_NF;
    if(ctx->tape && ctx->tape_nf == want) return ATURAN_OK;
    if(ctx->tape){ CK(cudaStreamSynchronize(ctx->st)); cudaFree(ctx->tape); ctx->tape = nullptr; }
    const Grid& g = ctx->g;
    const size_t fs = g.fstride;
    const int NT = want;
    const size_t nslot = NT == ADJ_NF ? ADJ_SLOTS : ADJ_SLOTS_MOIST;
    // stage inputs 4 x NT, T output, p_dyn, pressure source, slots, ybar NT, kbar NT, g0 NT, phbar,
    // rbar, pdbar, aux adjoint 3, heating accumulator, the moist tape's adjustment input NT; level
    // means + sums
    const size_t nf = 4 * NT + 3 + nslot + 3 * NT + 3 + 3 + 1 + (NT == ADJ_NF ? 0 : NT);
    const size_t bytes = (nf * fs + 3 * (size_t)g.im) * sizeof(double);
    void* mem = nullptr;
    if(cudaMalloc(&mem, bytes) != cudaSuccess){ cudaGetLastError(); return fail(ctx, ATURAN_E_NOMEM, "tape allocation"); }
    CK(cudaMemsetAsync(mem, 0, bytes, ctx->st));      // slots stay zero outside the interior
    double* cur = reinterpret_cast<double*>(mem);
    auto take = [&](size_t n){ double* r = cur; cur += n; return r; };
    ctx->tape = reinterpret_cast<double*>(mem);
    ctx->tape_nf = NT;
    ctx->tX = take(4 * NT * fs);
    ctx->tTout = take(fs);
    ctx->tPd = take(fs);
    ctx->tSrc = take(fs);
    ctx->aslot = take(nslot * fs);
    ctx->aybar = take(NT * fs);
    ctx->akbar = take(NT * fs);
    ctx->ag0 = take(NT * fs);
    ctx->aphbar = take(fs);
    ctx->arbar = take(fs);
    ctx->apdbar = take(fs);
    ctx->aaux = take(3 * fs);
    ctx->ahacc = take(fs);
    ctx->tPre = NT == ADJ_NF ? nullptr : take(NT * fs);
    ctx->tref = take(g.im);
    ctx->alev = take(2 * g.im);
    ctx->tape_valid = false;
    ctx->tape_p_valid = false;
    ctx->tape_sat_pending = false;
    ctx->tape_sat_valid = false;
    return ATURAN_OK;
}

int aturan_rk4_adjoint(aturan_ctx* ctx, const double* const* ybar, double* const* xbar){
    return aturan_rk4_adjoint_ex(ctx, ybar, nullptr, xbar, nullptr, nullptr);
}

}  // extern "C"

namespace {

// The reverse of the taped step over its nf fields (ADJ_NF: t, u, v, w; ADJ_NF_MOIST: and the
// twelve condensable species, then the saturation adjustment's implicit adjoint when the taped
// step ran one).
int rk4_adjoint_impl(aturan_ctx* ctx, int nf, const double* const* ybar, const double* const* auxbar,
                     double* const* xbar, double* pbar, double* heatbar){
    if(!ctx || !ybar || !xbar) return ATURAN_E_INVALID;
    if(auxbar) for(int q = 0; q < 3; q++) if(!auxbar[q]) return fail(ctx, ATURAN_E_INVALID, "null aux adjoint pointer");
    for(int q = 0; q < nf; q++) if(!ybar[q] || !xbar[q]) return fail(ctx, ATURAN_E_INVALID, "null adjoint pointer");
    if(!ctx->tape || !ctx->tape_valid) return fail(ctx, ATURAN_E_INVALID, "no taped RK4 step (aturan_tape, then aturan_rk4_step)");
    if(ctx->tape_nf != nf)
        return fail(ctx, ATURAN_E_INVALID, nf == ADJ_NF ? "the tape is moist: use aturan_moist_adjoint"
                                                        : "the tape is dry: switch it on with aturan_tape(ctx, 2)");
    const Grid g = ctx->g;
    const size_t fs = g.fstride, rows = (size_t)g.im * g.jm;
    const double dt = ctx->p.dt;
    Region reg(ctx, ATURAN_K_ADJOINT, 0);
    long nl = 0;
    for(int q = 0; q < nf; q++)                        // the caller's ybar' into the padded layout
        CK(cudaMemcpy2DAsync(ctx->ag0 + q * fs, g.kp * 8, ybar[q], g.km * 8, g.km * 8, rows,
                             cudaMemcpyDeviceToDevice, ctx->st));
    const RhsConst<double>& K = ctx->k64;
    const double t_min = K.t_min, t_max = K.t_max;
    const dim3 gc((g.km + 127) / 128, g.jm, g.im);
    adj_init_kernel<<<gc, 128, 0, ctx->st>>>(g, ctx->ag0, ctx->tTout, t_min, t_max, dt / 6.0 * 1.0,
                                             ctx->ag0, ctx->aybar, ctx->akbar, ctx->aphbar, ctx->apdbar, nf);
    CK_LAUNCH("adjoint init"); nl++;
    if(auxbar)                                         // the aux adjoint into the padded layout
        for(int q = 0; q < 3; q++)
            CK(cudaMemcpy2DAsync(ctx->aaux + q * fs, g.kp * 8, auxbar[q], g.km * 8, g.km * 8, rows,
                                 cudaMemcpyDeviceToDevice, ctx->st));
    AdjArgs a;
    a.g = g;
    a.X0 = ctx->tX;
    a.kbar = ctx->akbar;
    a.pdyn = ctx->tPd;                                  // p_dyn as the taped step read it
    a.forc = reinterpret_cast<const double*>(ctx->forc);
    a.geo = reinterpret_cast<const GeoIJ<double>*>(ctx->geo);
    a.cp_tab = reinterpret_cast<const double*>(ctx->cp_tab);
    a.k = K;
    a.slot = ctx->aslot;
    a.hacc = heatbar ? ctx->ahacc : nullptr;
    if(heatbar) CK(cudaMemsetAsync(ctx->ahacc, 0, fs * 8, ctx->st));
    const dim3 gs((g.km - 1 + 31) / 32, (g.jm - 2 + 3) / 4, g.im - 2);
    const dim3 gg((g.km - 1 + 127) / 128, g.jm, g.im);
    for(int stage = 3; stage >= 0; stage--){
        a.X = ctx->tX + (size_t)stage * nf * fs;
        a.auxbar = (stage == 3 && auxbar) ? ctx->aaux : nullptr;   // aux is stage 3's output
        adj_local_kernel<<<gs, dim3(32, 4), 0, ctx->st>>>(a);
        nl++;
        if(nf == ADJ_NF_MOIST){ adj_species_local_kernel<<<gs, dim3(32, 4), 0, ctx->st>>>(a); nl++; }
        const int prev = stage - 1;
        const double w_prev = prev >= 0 ? dt / 6.0 * ((prev == 0 || prev == 3) ? 1.0 : 2.0) : 0.0;
        const double c_prev = prev >= 0 ? ((prev == 0 || prev == 1) ? 0.5 * dt : (prev == 2 ? dt : 0.0)) : 0.0;
        adj_gather_kernel<<<gg, 128, 0, ctx->st>>>(g, ctx->aslot, ctx->aybar, ctx->aphbar, ctx->apdbar, ctx->ag0,
                                                  ctx->akbar, w_prev, c_prev, prev >= 0 ? 1 : 0, nf);
        CK_LAUNCH("adjoint stage"); nl++;
    }
    const double* t0 = ctx->tX;
    adj_hydro_kernel<<<(g.jm * g.km + 255) / 256, 256, 0, ctx->st>>>(
        g, t0, reinterpret_cast<const double*>(ctx->pstat), t0 + 2 * fs, t0 + 3 * fs, ctx->tref, ctx->rm_i, ctx->cor_j,
        ctx->aphbar, ctx->aybar, ctx->arbar, ctx->hc);
    adj_level_sum_kernel<<<g.im, 256, 0, ctx->st>>>(g, t0, reinterpret_cast<const double*>(ctx->pstat), ctx->wsin,
                                                   ctx->arbar, ctx->hc, ctx->alev);
    adj_level_apply_kernel<<<gc, 128, 0, ctx->st>>>(g, t0, reinterpret_cast<const double*>(ctx->pstat), ctx->wsin,
                                                    ctx->alev, ctx->hc, ctx->aybar);
    CK_LAUNCH("adjoint hydrostatic"); nl += 3;
    if(nf == ADJ_NF_MOIST && ctx->tape_sat_valid){     // the step's adjustment, before its RK4
        adj_satadj_kernel<<<gc, 128, 0, ctx->st>>>(g, ctx->tPre, ctx->tX, reinterpret_cast<const double*>(ctx->pstat),
                                                   reinterpret_cast<const double*>(ctx->forc) + (size_t)(ATURAN_RHO_MIX - ATURAN_NUE) * fs,
                                                   ctx->sc, ctx->aybar);
        CK_LAUNCH("adjoint saturation adjustment"); nl++;
    }
    reg.n = nl;
    for(int q = 0; q < nf; q++)
        CK(cudaMemcpy2DAsync(xbar[q], g.km * 8, ctx->aybar + q * fs, g.kp * 8, g.km * 8, rows,
                             cudaMemcpyDeviceToDevice, ctx->st));
    if(pbar)
        CK(cudaMemcpy2DAsync(pbar, g.km * 8, ctx->apdbar, g.kp * 8, g.km * 8, rows, cudaMemcpyDeviceToDevice, ctx->st));
    if(heatbar){
        adj_heat_reduce_kernel<<<(g.jm * g.km + 255) / 256, 256, 0, ctx->st>>>(g, ctx->ahacc, K.heat_scale, heatbar);
        CK_LAUNCH("heating adjoint");
    }
    CK(cudaStreamSynchronize(ctx->st));
    return ATURAN_OK;
}

}  // namespace

extern "C" {

int aturan_rk4_adjoint_ex(aturan_ctx* ctx, const double* const* ybar, const double* const* auxbar,
                          double* const* xbar, double* pbar, double* heatbar){
    return rk4_adjoint_impl(ctx, ADJ_NF, ybar, auxbar, xbar, pbar, heatbar);
}

int aturan_moist_adjoint(aturan_ctx* ctx, const double* const* ybar, const double* const* auxbar,
                         double* const* xbar, double* pbar, double* heatbar){
    return rk4_adjoint_impl(ctx, ADJ_NF_MOIST, ybar, auxbar, xbar, pbar, heatbar);
}

int aturan_set_heating(aturan_ctx* ctx, const double* H, int on_device){
    if(!ctx) return ATURAN_E_INVALID;
    const Grid& g = ctx->g;
    if(!H){
        if(ctx->heat){ CK(cudaStreamSynchronize(ctx->st)); cudaFree(ctx->heat); ctx->heat = nullptr; }
        return ATURAN_OK;
    }
    if(!ctx->heat){
        void* m = nullptr;
        if(cudaMalloc(&m, (size_t)g.jm * g.km * 8) != cudaSuccess){ cudaGetLastError(); return fail(ctx, ATURAN_E_NOMEM, "heating field"); }
        ctx->heat = reinterpret_cast<double*>(m);
    }
    CK(cudaMemcpyAsync(ctx->heat, H, (size_t)g.jm * g.km * 8, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return ATURAN_OK;
}

int aturan_pressure_adjoint(aturan_ctx* ctx, int kind, double omega, int max_sweeps, double tol,
                            const double* pbar, double* const* auxbar, int* sweeps_done, double* resid){
    if(!ctx || !pbar || !auxbar) return ATURAN_E_INVALID;
    for(int q = 0; q < 3; q++) if(!auxbar[q]) return fail(ctx, ATURAN_E_INVALID, "null aux adjoint pointer");
    if(sweeps_done) *sweeps_done = 0;
    if(resid) *resid = 0.0;
    if(kind != ATURAN_PRESS_RB_SOR && kind != ATURAN_PRESS_RB_LINE)
        return fail(ctx, ATURAN_E_INVALID, "the pressure adjoint is that of ATURAN_PRESS_RB_SOR / RB_LINE");
    if(!ctx->tape || !ctx->tape_p_valid)
        return fail(ctx, ATURAN_E_INVALID, "no taped pressure solve (aturan_tape, then aturan_pressure)");
    const bool line = kind == ATURAN_PRESS_RB_LINE;
    int rc = sor_check_sizes(ctx, omega, line); if(rc) return rc;
    if(max_sweeps < 1) max_sweeps = 1;
    const Grid g = ctx->g;
    const size_t fs = g.fstride, rows = (size_t)g.im * g.jm;
    long nl = 0;
    Region reg(ctx, ATURAN_K_ADJOINT, 0);
    double* B = ctx->akbar;                 // work fields: p_dyn's adjoint, the transposed solution,
    double* lam = ctx->akbar + fs;          // the source's adjoint
    double* sbar = ctx->akbar + 2 * fs;
    CK(cudaMemsetAsync(B, 0, 3 * fs * 8, ctx->st));
    CK(cudaMemcpy2DAsync(B, g.kp * 8, pbar, g.km * 8, g.km * 8, rows, cudaMemcpyDeviceToDevice, ctx->st));
    // the boundary passes' adjoint, in reverse order
    adj_pbc_p_kernel<<<(g.im * g.jm + 255) / 256, 256, 0, ctx->st>>>(g, B);
    adj_pbc_t_kernel<<<dim3((g.km + 127) / 128, g.im), 128, 0, ctx->st>>>(g, B);
    adj_pbc_r_kernel<<<dim3((g.km + 127) / 128, g.jm), 128, 0, ctx->st>>>(g, B);
    sor_compat(ctx, B, true);               // zero-mean (it is, up to rounding, when p_dyn enters by differences)
    CK_LAUNCH("pressure adjoint: boundary passes");
    nl += 6;
    int s = 0;
    double r = 0.0;
    const int status = solve_fp64<true>(ctx, lam, B, omega, max_sweeps, tol, line, &s, &r, nl);
    if(status < 0) return status;
    const int ny = ((g.jm - 2) * (g.km - 1) + 255) / 256;
    sor_ysum_kernel<<<ny, 256, 0, ctx->st>>>(g, lam, ctx->sor_part, 1);
    sor_shift_finish_kernel<<<1, 256, 0, ctx->st>>>(ctx->sor_part, ny, ctx->sor_part + 2 * ny);
    const double n_int = (double)(g.im - 2) * (g.jm - 2) * (g.km - 1);
    const double sum_w = (double)(g.im - 1) * (g.jm - 1) * (g.km - 1);   // sum of y_i y_j over the interior
    adj_compat_mask_kernel<<<dim3((g.km - 1 + 127) / 128, g.jm - 2, g.im - 2), 128, 0, ctx->st>>>(
        g, lam, ctx->sor_part + 2 * ny, n_int / sum_w, ctx->tSrc, ctx->rbw, sbar);
    double* aub = ctx->ag0;
    adj_div_kernel<<<dim3((g.km + 127) / 128, g.jm, g.im), 128, 0, ctx->st>>>(
        g, sbar, ctx->rbw, ctx->pc, ctx->p.rigid_lid, aub, aub + fs, aub + 2 * fs);
    CK_LAUNCH("pressure adjoint: source");
    nl += 4;
    for(int q = 0; q < 3; q++)
        CK(cudaMemcpy2DAsync(auxbar[q], g.km * 8, aub + q * fs, g.kp * 8, g.km * 8, rows,
                             cudaMemcpyDeviceToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    reg.n = nl;
    if(sweeps_done) *sweeps_done = s;
    if(resid) *resid = r;
    return status;
}

int aturan_satadj(aturan_ctx* ctx, int gas_mask, long* n_adjusted, long* n_noconv){
    if(!ctx) return ATURAN_E_INVALID;
    if(gas_mask & ~0xF) return fail(ctx, ATURAN_E_INVALID, "gas_mask has bits above 3");
    const bool count = n_adjusted || n_noconv;
    if(count) CK(cudaMemsetAsync(ctx->counters, 0, 2 * sizeof(unsigned long long), ctx->st));
    int rc = ctx->mixed ? run_satadj<float>(ctx, gas_mask, count, ctx->st)
                         : run_satadj<double>(ctx, gas_mask, count, ctx->st);
    if(rc) return rc;
    if(count){
        unsigned long long h[2];
        CK(cudaMemcpyAsync(h, ctx->counters, sizeof h, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        if(n_adjusted) *n_adjusted = (long)h[0];
        if(n_noconv) *n_noconv = (long)h[1];
    }
    return ATURAN_OK;
}

static int sync_ncopies(aturan_ctx* ctx, cudaStream_t st){
    const size_t fs = ctx->g.fstride, e = ctx->esz;
    char* s = (char*)ctx->state; char* n = (char*)ctx->ncopy;
    Region reg(ctx, ATURAN_K_COPY, 0, st);
    CK(cudaMemcpyAsync(n + ATURAN_CH4 * fs * e, s + ATURAN_CH4 * fs * e, 12 * fs * e, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(n, s, fs * e, cudaMemcpyDeviceToDevice, st));
    if(ctx->p.nh4sh_sync)
        CK(cudaMemcpyAsync(n + ATURAN_NH4SH * fs * e, s + ATURAN_NH4SH * fs * e, fs * e, cudaMemcpyDeviceToDevice, st));
    if(ctx->tlo) CK(cudaMemcpyAsync(ctx->tlo + fs, ctx->tlo, fs * 4, cudaMemcpyDeviceToDevice, st));
    return ATURAN_OK;
}

int aturan_sync_ncopies(aturan_ctx* ctx){
    if(!ctx) return ATURAN_E_INVALID;
    return sync_ncopies(ctx, ctx->st);
}

int aturan_restore_ncopies(aturan_ctx* ctx, double coeff){
    if(!ctx) return ATURAN_E_INVALID;
    const size_t fs = ctx->g.fstride, e = ctx->esz;
    Region reg(ctx, ATURAN_K_COPY, coeff == 1.0 ? 0 : 1);
    if(coeff == 1.0){                                     // 1.0 * x == x: a copy
        CK(cudaMemcpyAsync(ctx->ncopy, ctx->state, 19 * fs * e, cudaMemcpyDeviceToDevice, ctx->st));
        if(ctx->tlo) CK(cudaMemcpyAsync(ctx->tlo + fs, ctx->tlo, fs * 4, cudaMemcpyDeviceToDevice, ctx->st));
    } else {
        if(ctx->mixed){
            launch_scale_copy_f32(reinterpret_cast<const float*>(ctx->state), reinterpret_cast<float*>(ctx->ncopy), 19 * fs, coeff, ctx->st);
            // tn = coeff * (hi + lo) in FP64, split again
            launch_scale_copy_pair(reinterpret_cast<const float*>(ctx->state), ctx->tlo,
                                   reinterpret_cast<float*>(ctx->ncopy), ctx->tlo + fs, fs, coeff, ctx->st);
        }
        else launch_scale_copy_f64(reinterpret_cast<const double*>(ctx->state), reinterpret_cast<double*>(ctx->ncopy), 19 * fs, coeff, ctx->st);
        CK_LAUNCH("restore n-copies");
    }
    return ATURAN_OK;
}

int aturan_pressure(aturan_ctx* ctx, int kind, double omega, int max_sweeps, double tol,
                    int* sweeps_done, double* resid){
    if(!ctx) return ATURAN_E_INVALID;
    if(sweeps_done) *sweeps_done = 0;
    if(resid) *resid = 0.0;
    ctx->last_sweeps = 0;
    ctx->last_resid = 0.0;
    int rc, s = 0;
    double r = 0.0;
    switch(kind){
    case ATURAN_PRESS_GS_LEX:
        rc = ctx->mixed ? run_gs<float>(ctx) : run_gs<double>(ctx);
        if(!rc) s = 1;
        break;
    case ATURAN_PRESS_RB_SHARED:
        rc = ctx->mixed ? run_rb<float>(ctx, max_sweeps, 1.0) : run_rb<double>(ctx, max_sweeps, 1.0);
        if(!rc) s = max_sweeps < 1 ? 1 : max_sweeps;
        break;
    case ATURAN_PRESS_RB_SOR:
    case ATURAN_PRESS_RB_LINE:
        rc = ctx->mixed ? run_sor<float>(ctx, omega, max_sweeps, tol, kind == ATURAN_PRESS_RB_LINE, &s, &r)
                        : run_sor<double>(ctx, omega, max_sweeps, tol, kind == ATURAN_PRESS_RB_LINE, &s, &r);
        break;
    default:
        return fail(ctx, ATURAN_E_INVALID, "unknown pressure kind");
    }
    if(rc >= 0){
        ctx->last_sweeps = s;
        ctx->last_resid = r;
        if(sweeps_done) *sweeps_done = s;
        if(resid) *resid = r;
    }
    return rc;
}

int aturan_pressure_last(aturan_ctx* ctx, int* sweeps_done, double* resid){
    if(!ctx) return ATURAN_E_INVALID;
    if(sweeps_done) *sweeps_done = ctx->last_sweeps;
    if(resid) *resid = ctx->last_resid;
    return ATURAN_OK;
}

int aturan_pressure_solve(aturan_ctx* ctx, int kind, int transposed, double omega, int max_sweeps, double tol,
                          const double* b, double* x, int* sweeps_done, double* resid){
    if(!ctx || !b || !x) return ATURAN_E_INVALID;
    if(sweeps_done) *sweeps_done = 0;
    if(resid) *resid = 0.0;
    if(kind != ATURAN_PRESS_RB_SOR && kind != ATURAN_PRESS_RB_LINE)
        return fail(ctx, ATURAN_E_INVALID, "aturan_pressure_solve takes ATURAN_PRESS_RB_SOR or ATURAN_PRESS_RB_LINE");
    const bool line = kind == ATURAN_PRESS_RB_LINE;
    int rc = sor_check_sizes(ctx, omega, line); if(rc) return rc;
    if(max_sweeps < 1) max_sweeps = 1;
    const Grid g = ctx->g;
    const size_t rows = (size_t)g.im * g.jm;
    long nl = 0;
    Region reg(ctx, ATURAN_K_RB, 0);
    // working copies in the padded layout: the right-hand side in scratch, the iterate in stage64
    CK(cudaMemcpy2DAsync(ctx->scratch, g.kp * 8, b, g.km * 8, g.km * 8, rows, cudaMemcpyDeviceToDevice, ctx->st));
    CK(cudaMemcpy2DAsync(ctx->stage64, g.kp * 8, x, g.km * 8, g.km * 8, rows, cudaMemcpyDeviceToDevice, ctx->st));
    sor_compat(ctx, ctx->scratch, transposed != 0);
    CK_LAUNCH("solve right-hand side");
    nl += 3;
    int s = 0;
    double r = 0.0;
    double* X = ctx->stage64;
    const double* B = ctx->scratch;
    const int status = ctx->mixed
        ? (transposed ? solve_mixed<true>(ctx, X, B, omega, max_sweeps, tol, line, &s, &r, nl)
                      : solve_mixed<false>(ctx, X, B, omega, max_sweeps, tol, line, &s, &r, nl))
        : (transposed ? solve_fp64<true>(ctx, X, B, omega, max_sweeps, tol, line, &s, &r, nl)
                      : solve_fp64<false>(ctx, X, B, omega, max_sweeps, tol, line, &s, &r, nl));
    if(status < 0) return status;
    CK(cudaMemcpy2DAsync(x, g.km * 8, ctx->stage64, g.kp * 8, g.km * 8, rows, cudaMemcpyDeviceToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    reg.n = nl;
    if(sweeps_done) *sweeps_done = s;
    if(resid) *resid = r;
    return status;
}

// The reference's order is pressure, saturation adjustment, n-copy sync, RK4. The pressure solve
// reads and writes p_dyn and the projection fields only; the adjustment and the sync (fused into
// the adjustment's launch here) read t, p_stat, rho_mix, the species and NH4SH and write t, the
// species and their n-copies only; RK4's prelude
// (level means, hydrostatic integral) reads t, p_stat, v, w and writes the level means, p_hydro and
// p_bfollow only. So the solve on one side and adjustment, sync and prelude on the other are
// disjoint, and they run side by side with the same results as in order: the latter (one large
// FP64-bound launch, two small launches) on the low-priority side stream, the solve (a
// chain of small launches and residual reads) on the main stream, whose blocks the scheduler
// places first. The RK4 stages wait for both.
int aturan_step(aturan_ctx* ctx, int press_kind, double omega, int max_sweeps, double tol){
    if(!ctx) return ATURAN_E_INVALID;
    CK(cudaEventRecord(ctx->ev_fork, ctx->st));
    CK(cudaStreamWaitEvent(ctx->st2, ctx->ev_fork, 0));
    int rc2 = ctx->mixed ? run_satadj<float>(ctx, 0xF, false, ctx->st2, true)
                         : run_satadj<double>(ctx, 0xF, false, ctx->st2, true);
    if(!rc2) rc2 = ctx->mixed ? rk4_prelude<float>(ctx, ctx->st2) : rk4_prelude<double>(ctx, ctx->st2);
    CK(cudaEventRecord(ctx->ev_join, ctx->st2));
    const int rc = rc2 ? rc2 : aturan_pressure(ctx, press_kind, omega, max_sweeps, tol, nullptr, nullptr);
    CK(cudaStreamWaitEvent(ctx->st, ctx->ev_join, 0));
    if(rc < 0 || rc2) return rc < 0 ? rc : rc2;
    rc2 = ctx->mixed ? run_rk4<float, float>(ctx, ctx->k32, true) : run_rk4<double, double>(ctx, ctx->k64, true);
    if(rc2) return rc2;
    return rc;
}

// ---- the passes after RK4 (cUranusModel.cpp:1218-1248) ----
int aturan_post_params_default(aturan_post_params* pp){
    if(!pp) return ATURAN_E_INVALID;
    std::memset(pp, 0, sizeof *pp);
    pp->abi_version = ATURAN_ABI_VERSION;
    pp->damp_t_j = 0;              // cUranusModel.cpp:1216-1217, !geo_balance() with GEO_BALANCE's default 1
    pp->radius_form = 0;           // cUranusModel.h:406
    pp->bottom_form = 0;           // cUranusModel.h:409
    pp->pole_form = 0;             // cUranusModel.h:405
    pp->lid_u = 1;                 // BC_LID_U defaults to BC_RIGID_LID, cUranusModel.h:403
    pp->top_taper = 0;             // cUranusModel.h:404
    pp->lid_vw = 2;                // BC_Uran.h:155, with geo_balance()
    pp->radius_positive = 1;       // BC_Uran.h:92
    pp->phi_periodic = 1;          // cUranusModel.h:412
    pp->species_clamp = 1;         // BC_Uran.h:111
    pp->damp_t_horiz = 1.0;        // cUranusModel.cpp:1214-1215
    pp->damp_t_vert = 0.0;         // cUranusModel.cpp:1204-1205
    pp->vel_shapiro = 0.0;         // cUranusModel.cpp:1229-1230, with geo_balance()
    return ATURAN_OK;
}

int aturan_mca(aturan_ctx* ctx){
    if(!ctx) return ATURAN_E_INVALID;
    return ctx->mixed ? run_mca<float>(ctx) : run_mca<double>(ctx);
}

int aturan_chem_params_default(aturan_chem_params* cp){
    if(!cp) return ATURAN_E_INVALID;
    std::memset(cp, 0, sizeof(*cp));
    cp->abi_version = ATURAN_ABI_VERSION;
    cp->nh4sh_eq = 1; cp->difflux_plus = 1; cp->difflux_laplacian = 1; cp->phi_periodic = 1;
    cp->m_nh3 = 17.03052; cp->m_h2s = 34.08088; cp->m_nh4sh = 51.1114;       // cUranusModel.h:997-999
    // ThermalPropertiesUran's sum of the species' molar densities c_x = r_x / m_x
    cp->c_mix = 0x1.12b14645f7a58p+0;
    cp->D_nh4sh = 1.45e-9; cp->DT_nh4sh = 1.45e-9;                           // cUranusModel.h:1135-1140
    cp->cp_nh3 = 2.19e3; cp->cp_h2s = 2.24e3; cp->cp_nh4sh = 2.00e3;         // :1085-1087
    cp->k_nh3 = 0.02102; cp->k_h2s = 0.013; cp->k_nh4sh = 0.02102;          // :1076-1078
    cp->polar_floor = 0.4;                                                   // ATPhys.h:104-107
    return ATURAN_OK;
}

int aturan_chemistry(aturan_ctx* ctx, const aturan_chem_params* cp, int what, long* n_formed, long* n_decomposed){
    if(!ctx || !cp) return ATURAN_E_INVALID;
    if(cp->abi_version != ATURAN_ABI_VERSION) return fail(ctx, ATURAN_E_INVALID, "abi_version mismatch");
    if(what & ~(ATURAN_CHEM_NH4SH_EQ | ATURAN_CHEM_FORCING)) return fail(ctx, ATURAN_E_INVALID, "unknown chemistry part");
    if(cp->nh4sh_eq != 1) return fail(ctx, ATURAN_E_UNSUPPORTED, "only the NH4SH equilibrium form (nh4sh_eq = 1) is implemented");
    if(cp->difflux_laplacian != 1) return fail(ctx, ATURAN_E_UNSUPPORTED, "only difflux_laplacian = 1 is implemented");
    const bool count = (what & ATURAN_CHEM_NH4SH_EQ) && (n_formed || n_decomposed);
    if(count) CK(cudaMemsetAsync(ctx->counters + 4, 0, 2 * sizeof(unsigned long long), ctx->st));
    const int rc = ctx->mixed ? run_chem<float>(ctx, cp, what) : run_chem<double>(ctx, cp, what);
    if(rc) return rc;
    if(n_formed) *n_formed = 0;
    if(n_decomposed) *n_decomposed = 0;
    if(count){
        unsigned long long h[2];
        CK(cudaMemcpyAsync(h, ctx->counters + 4, sizeof h, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        if(n_formed) *n_formed = (long)h[0];
        if(n_decomposed) *n_decomposed = (long)h[1];
    }
    return ATURAN_OK;
}

int aturan_iter_params_default(aturan_iter_params* ip){
    if(!ip) return ATURAN_E_INVALID;
    std::memset(ip, 0, sizeof(*ip));
    ip->abi_version = ATURAN_ABI_VERSION;
    ip->press_kind = ATURAN_PRESS_GS_LEX; ip->max_sweeps = 1;   // PressureSolverUran (cUranusModel.cpp:970-972)
    ip->chemistry = 1; ip->precipitation = 1;                    // NH4SH_EQ, ATURAN_PRECIP (:105-108)
    ip->turbulence = 1; ip->mca_stride = 1;                      // turb_active (:482), ATURAN_MCA (:131-134)
    ip->omega = 1.0; ip->tol = 0.0;
    ip->damp_p_horiz = 0.0;                                      // :979-980 with GEO_BALANCE
    aturan_post_params_default(&ip->post);
    aturan_chem_params_default(&ip->chem);
    aturan_turb_params_default(&ip->turb);
    aturan_precip_params_default(&ip->precip);
    return ATURAN_OK;
}

int aturan_iteration(aturan_ctx* ctx, const aturan_iter_params* ip, int iter_n){
    if(!ctx || !ip) return ATURAN_E_INVALID;
    if(ip->abi_version != ATURAN_ABI_VERSION || ip->post.abi_version != ATURAN_ABI_VERSION ||
       ip->chem.abi_version != ATURAN_ABI_VERSION || ip->turb.abi_version != ATURAN_ABI_VERSION ||
       ip->precip.abi_version != ATURAN_ABI_VERSION) return fail(ctx, ATURAN_E_INVALID, "abi_version mismatch");
    if(iter_n < 1) return fail(ctx, ATURAN_E_INVALID, "iter_n counts from 1");
    // every knob checked before the first launch
    if(ip->chemistry && (ip->chem.nh4sh_eq != 1 || ip->chem.difflux_laplacian != 1))
        return fail(ctx, ATURAN_E_UNSUPPORTED, "chemistry: only nh4sh_eq = 1 and difflux_laplacian = 1 are implemented");
    if(ip->turbulence && (ip->turb.model != 2 || ip->turb.turb_free != 1 || ip->turb.clamp_pass != 1 ||
                          ip->turb.buoy != 0 || ip->turb.abl_taper != 0))
        return fail(ctx, ATURAN_E_UNSUPPORTED, "turbulence: only the default knobs are implemented");
    const bool mca = ip->mca_stride > 0 && iter_n % ip->mca_stride == 0;
    if(ip->mca_stride > 0 && mca_warp_bytes(ctx->g.im) > MCA_SMEM_MAX)
        return fail(ctx, ATURAN_E_UNSUPPORTED, "moist convective adjustment: column too deep for the shared memory");
    int rc;
    if(iter_n % 2 == 0){
        // the saturation adjustment and what follows it up to the chemistry forcing touch no field
        // of the pressure solve and its filter: they run on the second stream beside it
        CK(cudaEventRecord(ctx->ev_fork, ctx->st));
        CK(cudaStreamWaitEvent(ctx->st2, ctx->ev_fork, 0));
        int rc2 = ctx->mixed ? run_satadj<float>(ctx, 0xF, false, ctx->st2) : run_satadj<double>(ctx, 0xF, false, ctx->st2);
        if(!rc2 && ip->chemistry)
            rc2 = ctx->mixed ? run_chem<float>(ctx, &ip->chem, ATURAN_CHEM_NH4SH_EQ, ctx->st2)
                             : run_chem<double>(ctx, &ip->chem, ATURAN_CHEM_NH4SH_EQ, ctx->st2);
        if(!rc2 && ip->precipitation)
            rc2 = ctx->mixed ? run_precip<float>(ctx, &ip->precip, ctx->st2) : run_precip<double>(ctx, &ip->precip, ctx->st2);
        if(!rc2) rc2 = sync_ncopies(ctx, ctx->st2);
        if(!rc2 && ip->chemistry)
            rc2 = ctx->mixed ? run_chem<float>(ctx, &ip->chem, ATURAN_CHEM_FORCING, ctx->st2)
                             : run_chem<double>(ctx, &ip->chem, ATURAN_CHEM_FORCING, ctx->st2);
        if(!rc2) rc2 = ctx->mixed ? rk4_prelude<float>(ctx, ctx->st2) : rk4_prelude<double>(ctx, ctx->st2);
        CK(cudaEventRecord(ctx->ev_join, ctx->st2));
        rc = rc2 ? rc2 : aturan_pressure(ctx, ip->press_kind, ip->omega, ip->max_sweeps, ip->tol, nullptr, nullptr);
        if(rc >= 0 && !rc2){
            // cUranusModel.cpp:974-986, the p_dyn filter (FP64 in both precisions)
            Region reg(ctx, ATURAN_K_POST, 0);
            const int per = ip->post.phi_periodic;
            if(ip->damp_p_horiz == 1.0) reg.n += launch_filter_f64(ctx->g, ctx->pdyn, true, true, true, 1.0, per, ctx->st);
            else {
                if(ip->damp_p_horiz != 0.0) reg.n += launch_filter_f64(ctx->g, ctx->pdyn, false, true, true, ip->damp_p_horiz, per, ctx->st);
                reg.n += launch_filter_f64(ctx->g, ctx->pdyn, true, false, false, 1.0, per, ctx->st);
            }
            CK_LAUNCH("p_dyn filter");
        }
        CK(cudaStreamWaitEvent(ctx->st, ctx->ev_join, 0));
        if(rc < 0 || rc2) return rc < 0 ? rc : rc2;
        rc2 = ctx->mixed ? run_rk4<float, float>(ctx, ctx->k32, true) : run_rk4<double, double>(ctx, ctx->k64, true);
        if(rc2) return rc2;
    } else {
        rc = aturan_rk4_step(ctx);
        if(rc) return rc;
    }
    int r = ctx->mixed ? run_post<float>(ctx, &ip->post, nullptr, nullptr) : run_post<double>(ctx, &ip->post, nullptr, nullptr);
    if(r) return r;
    r = aturan_restore_ncopies(ctx, 1.0);                      // cUranusModel.cpp:1264
    if(r) return r;
    if(ip->turbulence){
        r = ctx->mixed ? run_turb<float>(ctx, &ip->turb) : run_turb<double>(ctx, &ip->turb);
        if(r) return r;
    }
    if(mca){
        r = aturan_mca(ctx);
        if(r) return r;
    }
    return rc;
}

int aturan_turb_params_default(aturan_turb_params* tp){
    if(!tp) return ATURAN_E_INVALID;
    std::memset(tp, 0, sizeof(*tp));
    tp->abi_version = ATURAN_ABI_VERSION;
    tp->model = 2;                                   // k_omega_SST (the configured turb_model)
    tp->turb_free = 1; tp->clamp_pass = 1; tp->curv = 1;
    tp->buoy = 0;                                    // cUranusModel.h:411
    tp->abl_taper = 0; tp->phi_periodic = 1;
    tp->nue_max = 1.0e5; tp->k_bg = 1.0;             // Turbulence.h:123-126, :156-159
    tp->nue_air = 1.8e-5;                            // the constructor's nue_gas
    return ATURAN_OK;
}

int aturan_turbulence(aturan_ctx* ctx, const aturan_turb_params* tp){
    if(!ctx || !tp) return ATURAN_E_INVALID;
    if(tp->abi_version != ATURAN_ABI_VERSION) return fail(ctx, ATURAN_E_INVALID, "abi_version mismatch");
    if(tp->model != 2) return fail(ctx, ATURAN_E_UNSUPPORTED, "only the k-omega SST closure (model 2) is implemented");
    if(tp->turb_free != 1 || tp->clamp_pass != 1 || tp->buoy != 0 || tp->abl_taper != 0)
        return fail(ctx, ATURAN_E_UNSUPPORTED, "only turb_free = 1, clamp_pass = 1, buoy = 0, abl_taper = 0 are implemented");
    if(ctx->g.im < 3 || ctx->g.jm < 3) return fail(ctx, ATURAN_E_INVALID, "grid too small");
    return ctx->mixed ? run_turb<float>(ctx, tp) : run_turb<double>(ctx, tp);
}

int aturan_precip_params_default(aturan_precip_params* pp){
    if(!pp) return ATURAN_E_INVALID;
    std::memset(pp, 0, sizeof(*pp));
    pp->abi_version = ATURAN_ABI_VERSION;
    pp->coupling = 1; pp->h2s = 1;                   // Precipitation.h:164-167, cUranusModel.h:276-279
    pp->rate_scale = 0.00071;                        // cUranusModel.h:610
    return ATURAN_OK;
}

int aturan_precipitation(aturan_ctx* ctx, const aturan_precip_params* pp){
    if(!ctx || !pp) return ATURAN_E_INVALID;
    if(pp->abi_version != ATURAN_ABI_VERSION) return fail(ctx, ATURAN_E_INVALID, "abi_version mismatch");
    return ctx->mixed ? run_precip<float>(ctx, pp) : run_precip<double>(ctx, pp);
}

int aturan_post_step(aturan_ctx* ctx, const aturan_post_params* pp, double* clamp_added, long* clamp_cells){
    if(!ctx || !pp) return ATURAN_E_INVALID;
    if(pp->abi_version != ATURAN_ABI_VERSION) return ATURAN_E_INVALID;
    return ctx->mixed ? run_post<float>(ctx, pp, clamp_added, clamp_cells) : run_post<double>(ctx, pp, clamp_added, clamp_cells);
}

int aturan_profile(aturan_ctx* ctx, int enable){
    if(!ctx) return ATURAN_E_INVALID;
    CK(cudaStreamSynchronize(ctx->st));
    for(long& l : ctx->launches) l = 0;
    ctx->ev_used = 0;
    ctx->prof_timing = enable ? 1 : 0;
    return ATURAN_OK;
}

int aturan_profile_read(aturan_ctx* ctx, double* ms, long* launches, int nkinds){
    if(!ctx || nkinds < 0) return ATURAN_E_INVALID;
    CK(cudaStreamSynchronize(ctx->st));
    const int n = nkinds < ATURAN_K_NKINDS ? nkinds : ATURAN_K_NKINDS;
    if(launches) for(int q = 0; q < n; q++) launches[q] = ctx->launches[q];
    if(ms){
        for(int q = 0; q < n; q++) ms[q] = 0.0;
        for(size_t u = 0; u < ctx->ev_used; u++){
            float t = 0.f;
            CK(cudaEventElapsedTime(&t, ctx->evs[u].a, ctx->evs[u].b));
            if(ctx->evs[u].kind < n) ms[ctx->evs[u].kind] += t;
        }
    }
    return ATURAN_OK;
}

int aturan_sync(aturan_ctx* ctx){
    if(!ctx) return ATURAN_E_INVALID;
    CK(cudaStreamSynchronize(ctx->st));
    return ATURAN_OK;
}

}  // extern "C"
