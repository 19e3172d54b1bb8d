// The precipitation microphysics (planet/Precipitation.h, Precipitation<cUranusModel>::run,
// :192-277, and its column solver, :280-446) for H2O, NH3, CH4 and then H2S
// (cUranusModel.h:280-297), no land cells.
//
// Each (j, k) column walks the levels top down (the scheme is a downward sweep: each level's
// collection and phase-change terms read the fluxes the level above produced). Four adjacent lanes
// take the four species of one column, each with its rain / snow / graupel fluxes in registers, so
// a warp runs 8 adjacent columns and a block of 128 threads 32, with no barrier: per level the
// lane of H2O gathers the other three species' latent heating by shuffles and writes Q_precip once,
// summed in the reference's order (H2O, NH3, CH4, H2S), and each lane writes its species' three
// S_precip_* (or, with the coupling off, its condensate fields in place); the lid row and every S
// field the call does not fill are written with the zeros the reference's first pass puts there,
// so nothing is launched besides this kernel. The fluxes themselves, the NH4SH settling flux and
// the surface maps are diagnostics and are not stored. The 8 lanes of one species take 8 adjacent
// k, so every load and store of a level covers whole 32-byte sectors; the work is per-cell FP64
// arithmetic with an exp and a log per species and level (two pow where rain falls) on ~16 values
// read and ~13 written.
#pragma once
#include "common.cuh"

namespace aturan {

struct PrecipGas {
    double C, L0, den, del_alf, del_bet;   // liquid saturation set, den = 1e-3 R
    double ep, lv, Lf, t_frz, t_low;
};

template <typename S>
struct PrecipArgs {
    Grid g;
    const S *t, *ps, *rho;
    const float* tlo;                    // the mixed form's temperature pair, else null
    S* Q;
    S* sp[4][3];                         // vapour, cloud, ice of H2O, NH3, CH4, H2S
    S* ss[4][3];                         // S_precip_<gas>, _cloud, _ice
    PrecipGas gas[4];
    const double* dz;                    // layer thickness [m] per level (the float layer heights)
    double rs, nd, r_mix, t_ref;
    int coupling, h2s, local_rho;
};

__device__ __forceinline__ double pr_max(double a, double b){ return (a < b) ? b : a; }   // std::max
__device__ __forceinline__ double pr_min(double a, double b){ return (b < a) ? b : a; }   // std::min

// Lane 4c + n of a warp: species n of the warp's column c (k = 8 * warp + c of the block's 32).
template <typename S>
__global__ void __launch_bounds__(128) precip_kernel(const __grid_constant__ PrecipArgs<S> a){
    const Grid& g = a.g;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, n = lane & 3;
    const int k = blockIdx.x * 32 + (threadIdx.x >> 5) * 8 + (lane >> 2), j = blockIdx.y;
    const bool kin = k < g.km;
    const size_t pl = (size_t)g.jm * g.kp;
    const size_t o = gidx(g, 0, j, kin ? k : 0);
    // Precipitation.h:89-131 and :286-302
    const double c_c_au = 2.0e-8, c_i_au = 5.0e-8, q_c_crit = 5.0e-4, c_ac = 1.0e-7, c_rim = 1.0e-8;
    const double z_csg = 2.5e-8, a_ev = 2.76e-3, c_melt_K = 0.2, c_frz_K = 0.2, P_ref = 1.0e-4;
    const double v_fall = 2.0, P_max_flux = 1.0e-4, dep_frac = 1.0, ratio_cap = 5.0;
    const double rs = a.rs;
    const bool on = n < 3 || a.h2s;
    const PrecipGas& s = a.gas[n];
    S* const fv = a.sp[n][0];
    S* const fc = a.sp[n][1];
    S* const fi = a.sp[n][2];
    S* const sv = a.ss[n][0];
    S* const sc = a.ss[n][1];
    S* const si = a.ss[n][2];
    double Pr = 0.0, Ps = 0.0, Pg = 0.0;
    if(kin){   // the lid row: zeroed by the first pass, never reached by the sweep
        const size_t q = o + (size_t)(g.im - 1) * pl;
        if(n == 0) a.Q[q] = (S)0.0;
        sv[q] = (S)0.0; sc[q] = (S)0.0; si[q] = (S)0.0;
    }
    // A level's inputs are loaded one level ahead, before the level above's stores (they are other
    // cells; in program order after those stores the loads would wait for them, as the compiler
    // must assume they may alias).
    struct LevelIn { double t, p, r; S v, c, ic; };
    auto load_level = [&](int i) -> LevelIn {
        LevelIn L;
        const size_t q = o + (size_t)i * pl;
        L.t = t_ld(a.t, a.tlo, q);
        L.p = (double)a.ps[q];
        L.r = a.local_rho ? (double)a.rho[q] : 0.0;
        L.v = fv[q]; L.c = fc[q]; L.ic = fi[q];
        return L;
    };
    LevelIn nxt{};
    if(kin && g.im >= 2) nxt = load_level(g.im - 2);
    for(int i = g.im - 2; i >= 0; i--){
        const size_t q = o + (size_t)i * pl;
        const LevelIn cur = nxt;
        if(kin && i > 0) nxt = load_level(i - 1);
        const double dz = pr_max(0.0, a.dz[i]);
        double term = 0.0;
        bool added = false;
        if(kin){
            if(!on || dz <= 0.0){                             // dz <= 0: the fluxes pass through
                sv[q] = (S)0.0; sc[q] = (S)0.0; si[q] = (S)0.0;
            } else {
                const double T = cur.t * a.t_ref;
                const double p_u = cur.p;
                double rho = a.r_mix;                          // rho_at, cUranusModel.h:526-531
                if(a.local_rho){ const double r = cur.r; rho = (r > 0.0 && isfinite(r)) ? r : a.r_mix; }
                const double q_v = pr_max(0.0, (double)cur.v);
                const double q_c = pr_max(0.0, (double)cur.c);
                const double q_i = pr_max(0.0, (double)cur.ic);
                const double E_r = exp(s.C + (-s.L0 / T + s.del_alf * log(T) + s.del_bet * T) / s.den);   // ATPhys.h:49-52
                const double q_sat = (p_u > E_r) ? rho * s.ep * E_r / p_u : q_v;
                const double F_r_in = Pr, F_s_in = Ps, F_g_in = Pg;
                const double Rain = pr_min(ratio_cap, F_r_in / P_ref);
                const double Snow = pr_min(ratio_cap, F_s_in / P_ref);
                const double Graupel = pr_min(ratio_cap, F_g_in / P_ref);
                const double Rain_79 = (Rain > 0.0) ? pow(Rain, 7.0 / 9.0) : 0.0;
                const double Rain_49 = (Rain > 0.0) ? pow(Rain, 4.0 / 9.0) : 0.0;
                const bool warm = (T >= s.t_frz);
                const double S_c_au = (warm && q_c > q_c_crit) ? (rs * c_c_au) * (q_c - q_c_crit) : 0.0;
                const double S_i_au = (!warm && T >= s.t_low) ? (rs * c_i_au) * q_i : 0.0;
                const double S_ac = warm ? (rs * c_ac) * q_c * Rain_79 : 0.0;
                const double S_s_rim = !warm ? (rs * c_rim) * q_c * Snow : 0.0;
                const double S_g_rim = !warm ? (rs * c_rim) * q_c * Graupel : 0.0;
                const double S_csg = (!warm && q_c > q_c_crit) ? (rs * z_csg) * q_c * Snow : 0.0;
                const double f_melt = warm ? pr_min(1.0, c_melt_K * (T - s.t_frz)) : 0.0;
                const double f_frz = warm ? 0.0 : pr_min(1.0, c_frz_K * (s.t_frz - T));
                const double F_s_melt = f_melt * F_s_in;
                const double F_g_melt = f_melt * F_g_in;
                const double F_r_frz = f_frz * F_r_in;
                const double F_r_avail = pr_max(0.0, F_r_in - F_r_frz + F_s_melt + F_g_melt + (S_c_au + S_ac) * dz);
                const double S_ev_raw = (warm && Rain > 0.0 && q_v < q_sat) ? a_ev * (q_sat - q_v) * Rain_49 : 0.0;
                const double F_ev_sat = pr_max(0.0, q_sat - q_v) * v_fall;
                const double F_ev = pr_min(pr_min(S_ev_raw * dz, F_r_avail), F_ev_sat);
                const double S_ev = F_ev / dz;
                term = s.Lf * (S_s_rim + S_g_rim + S_csg)
                     + s.Lf * (F_r_frz - F_s_melt - F_g_melt) / dz
                     - s.lv * F_ev / dz;
                added = true;
                const double tau = dz / v_fall;
                const double d_c = pr_min(dep_frac * q_c, (S_c_au + S_ac + S_s_rim + S_g_rim + S_csg) * tau);
                const double d_i = pr_min(dep_frac * q_i, S_i_au * tau);
                if(a.coupling){
                    sc[q] = (S)(-pr_max(0.0, d_c) / tau * a.nd);
                    si[q] = (S)(-pr_max(0.0, d_i) / tau * a.nd);
                    sv[q] = (S)(+S_ev * a.nd);
                } else {
                    fc[q] = (S)(q_c - pr_max(0.0, d_c));
                    fi[q] = (S)(q_i - pr_max(0.0, d_i));
                    fv[q] = (S)(q_v + S_ev * tau);
                    sv[q] = (S)0.0; sc[q] = (S)0.0; si[q] = (S)0.0;
                }
                const double F_r = F_r_in - F_r_frz + F_s_melt + F_g_melt - F_ev + (S_c_au + S_ac) * dz;
                const double F_s = F_s_in - F_s_melt + (S_i_au + S_s_rim - S_csg) * dz;
                const double F_g = F_g_in - F_g_melt + F_r_frz + (S_g_rim + S_csg) * dz;
                Pr = pr_min(P_max_flux, pr_max(0.0, F_r));
                Ps = pr_min(P_max_flux, pr_max(0.0, F_s));
                Pg = pr_min(P_max_flux, pr_max(0.0, F_g));
            }
        }
        // Q_precip zeroed by the first pass, then each species' += in the reference's order
        const double t1 = __shfl_down_sync(FULL, term, 1), t2 = __shfl_down_sync(FULL, term, 2), t3 = __shfl_down_sync(FULL, term, 3);
        const unsigned on_mask = __ballot_sync(FULL, added);
        if(n == 0 && kin){
            double Qc = 0.0;
            if(added) Qc += term;
            if(on_mask & (1u << (lane + 1))) Qc += t1;
            if(on_mask & (1u << (lane + 2))) Qc += t2;
            if(on_mask & (1u << (lane + 3))) Qc += t3;
            a.Q[q] = (S)Qc;
        }
    }
}

}  // namespace aturan
