// Mixed-phase saturation adjustment (Tao et al. 1988) of up to four condensables, fused per cell.
//
// Reference: planet/SaturationAdjustment.h:255-746 (the shared routine the model selects,
// SaturationAdjustmentUran.cpp:208-239), called for H2O, H2S, NH3, CH4 in that order
// (cUranusModel.cpp:998-1027). Every cell is independent and each call ends with a clamp of its
// own three fields, so running the four gases back to back inside one thread, temperature
// carried in a register, gives the same result as four sweeps over the grid while reading
// t, p_stat and rho_mix once and writing t once.
//
// The arithmetic is FP64 whatever the storage type S (the Clausius-Clapeyron Newton iteration
// is the part of the step the mixed-precision form keeps in FP64). Every iteration is capped at
// the reference's 15 passes; nothing here can spin.
#pragma once
#include "common.cuh"

namespace aturan {

struct GasConst {
    double t_0, t_00, ep, lv, ls;
    double C, L0, den, del_alf, del_bet;        // den = 1e-3 * R (ATPhys.h:52)
    double inv_den;                             // 1 / den (the mixed form's fast vapour pressure)
    double C_i, L0_i, del_alf_i, del_bet_i;
    double t_range_inv, Lf;
    int freeze_on;
};

struct SatConst {
    GasConst gas[4];
    double cp_mix, t_ref, r_mix;
    double stop_tol;                // the stopping test (:551): the reference's 1e-3 by default
    double entry_tol;               // the entry test (:446): the reference's 1e-3 by default
    int conserve, newton, evap, ice_entry, bergeron, dry_exit, local_rho;
};

// ATPhys.h:49-53
__device__ __forceinline__ double svp(double T, double C, double L0, double den, double a, double b){
    return exp(C + (-L0 / T + a * log(T) + b * T) / den);
}

template <typename S>
struct SatArgs {
    Grid g;
    S* t; const S* ps; const S* rho_mix;
    S* spec[4][3];          // (vapour, cloud, ice) per gas in the loop's order
    SatConst k;
    int gas_mask;
    unsigned long long* counters;   // [0] adjusted, [1] not converged (summed over gases)
    // n-copy sync fused into the adjustment (aturan_step): when sync != 0, t, the twelve species and
    // (sync == 2) NH4SH are also written to their start-of-step copies, nc_off elements from the
    // fields, the values the adjustment leaves -- what the copy after it would write.
    long long nc_off;
    int sync;
    S* nh4sh;
    // the mixed form's temperature pair (common.cuh): the low parts of t and of its n-copy; null in
    // an FP64 context
    float* tlo;
    float* tnlo;
};

// The saturation vapour density rho ep svp(T) / p of the liquid (ice = false) or ice set.
// FP64 path (exact): the reference's expression and operand order, bit for bit. Mixed path
// (FAST): the same FP64 mathematics with the divisions folded into per-cell and per-gas
// reciprocals and log(T), 1/T shared by the liquid and ice sets at one T -- a few ulps
// different, which the mixed form allows, and about a third fewer FP64 divisions and logs.
struct SatT { double T, lg, inv; };
__device__ __forceinline__ SatT sat_t(double T){ SatT r; r.T = T; r.lg = log(T); r.inv = 1.0 / T; return r; }

// SatT at T + dT from SatT at T (mixed form): with x = dT / T, log(T + dT) = log T + log1p(x) and
// 1 / (T + dT) = (1 / T) / (1 + x), both by their Taylor series through x^7 (truncation below
// |x|^8 / 8, i.e. below 1e-20 of the result for |x| <= 2e-3); a full log and division above that.
// Used for the Newton pass's finite difference (dT = 0.1, T >= 50 K) and for a pass's own T
// when it lies within 0.2 % of the last full evaluation.
__device__ __forceinline__ SatT sat_t_next(const SatT& s, double dT){
    const double x = dT * s.inv;
    if(!(fabs(x) <= 2.0e-3)) return sat_t(s.T + dT);
    SatT r;
    r.T = s.T + dT;
    const double l1p = x * (1.0 + x * (-0.5 + x * (1.0 / 3.0 + x * (-0.25 + x * (0.2 + x * (-1.0 / 6.0 + x * (1.0 / 7.0)))))));
    const double rcp = 1.0 + x * (-1.0 + x * (1.0 + x * (-1.0 + x * (1.0 + x * (-1.0 + x * (1.0 - x))))));
    r.lg = s.lg + l1p;
    r.inv = s.inv * rcp;
    return r;
}

template <bool FAST>
__device__ __forceinline__ double qsat(const GasConst& G, bool ice, double rho_c, double ep, double p_u,
                                       double rep, double T, const SatT& st){
    const double C = ice ? G.C_i : G.C, L0 = ice ? G.L0_i : G.L0;
    const double al = ice ? G.del_alf_i : G.del_alf, be = ice ? G.del_bet_i : G.del_bet;
    if constexpr(FAST) return rep * exp(C + (-L0 * st.inv + al * st.lg + be * st.T) * G.inv_den);
    else return rho_c * ep * svp(T, C, L0, G.den, al, be) / p_u;
}

// NT threads per block, 1024 / NT resident blocks per SM (64 registers, a few spilled): the kernel
// is bound by dependent FP64 exp/log chains, so more warps in flight beat the spill traffic
// (measured: 6 % faster than half as many).
template <typename S, int NT>
__global__ void __launch_bounds__(NT, 1024 / NT) satadj_kernel(const SatArgs<S> a){
    constexpr bool FAST = sizeof(S) == 4;            // the mixed form
    const Grid& g = a.g;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int i = blockIdx.z;
    unsigned n_adj = 0, n_nc = 0;
    if(k < g.km){
        const size_t q = gidx(g, i, j, k);
        const SatConst& K = a.k;
        double tt = t_ld(a.t, a.tlo, q);
        const double p_u = (double)__ldg(a.ps + q);
        double rho_c = K.r_mix;                               // rho_at, cUranusModel.h:526-531
        if(K.local_rho){ const double r_ = (double)__ldg(a.rho_mix + q); rho_c = (r_ > 0.0 && isfinite(r_)) ? r_ : K.r_mix; }
        const double cp_mix = K.cp_mix, t_ref = K.t_ref;
        // latent heat to temperature: x / (cp_mix rho_c), a multiplication in the mixed form
        const double inv_hc = FAST ? 1.0 / (cp_mix * rho_c) : 0.0;
        auto per_hc = [&](double x) -> double {
            if constexpr(FAST) return x * inv_hc; else return x / (cp_mix * rho_c);
        };
        // log T and 1/T at the entry temperature, shared by the gases while none changes T (mixed form)
        SatT st_entry; st_entry.T = -1.0;
        for(int gi = 0; gi < 4; gi++){
            if(!(a.gas_mask & (1 << gi))){
                if(a.sync){ S* f[3] = {a.spec[gi][0], a.spec[gi][1], a.spec[gi][2]};
                            for(int n = 0; n < 3; n++) f[n][q + a.nc_off] = f[n][q]; }
                continue;
            }
            const GasConst& G = K.gas[gi];
            S* cP = a.spec[gi][0]; S* clP = a.spec[gi][1]; S* iP = a.spec[gi][2];
            double c = (double)cP[q], cloud = (double)clP[q], ice = (double)iP[q];
            double t_u = tt * t_ref;
            // :358 skip cells without a usable state
            if((t_u > 0.0) && (p_u > 0.0)){
                const double t_0 = G.t_0, t_00 = G.t_00, Lf = G.Lf;
                if(t_u > t_0){                                        // :365-385
                    if(K.conserve){
                        if(ice > 0.0){
                            double dm = ice;
                            if(Lf > 0.0){
                                const double hc = cp_mix * rho_c;
                                const double cap = hc * (t_u - t_0) / Lf;
                                if(dm > cap) dm = cap;
                                t_u -= Lf * dm / hc;
                                tt = t_u / t_ref;
                            }
                            ice -= dm;
                            cloud += dm;
                        }
                    } else {
                        ice = 0.0;
                    }
                }
                if(G.freeze_on && t_u < t_00 && cloud > 0.0){         // :388-399
                    double dm = cloud;
                    if(Lf > 0.0){
                        const double hc = cp_mix * rho_c;
                        const double cap = hc * (t_00 - t_u) / Lf;
                        if(dm > cap) dm = cap;
                        t_u += Lf * dm / hc;
                        tt = t_u / t_ref;
                    }
                    cloud -= dm;
                    ice += dm;
                }
                if(c < 0.0) c = 0.0;                                  // :400-402
                if(cloud < 0.0) cloud = 0.0;
                if(ice < 0.0) ice = 0.0;

                const double ep = G.ep, lv = G.lv, ls = G.ls, tri = G.t_range_inv;
                const double rep = FAST ? rho_c * ep / p_u : 0.0;
                SatT st0;
                if constexpr(FAST){
                    if(t_u != st_entry.T) st_entry = sat_t(t_u);
                    st0 = st_entry;
                }
                const double q_Rain_0 = qsat<FAST>(G, false, rho_c, ep, p_u, rep, t_u, st0);
                bool go = q_Rain_0 > 0.0;                             // :422
                if(go){
                    double q_entry = q_Rain_0;
                    if(K.ice_entry && cloud <= 0.0 && ice <= 0.0){
                        const double cnd0 = t_u <= t_00 ? 0.0 : (t_u >= t_0 ? 1.0 : (t_u - t_00) * tri);
                        if(cnd0 < 1.0)
                            q_entry = cnd0 * q_Rain_0 + (1.0 - cnd0) * qsat<FAST>(G, true, rho_c, ep, p_u, rep, t_u, st0);
                    }
                    if(K.bergeron >= 2 && cloud <= 0.0 && ice <= 0.0 && t_u < t_0)
                        q_entry = qsat<FAST>(G, true, rho_c, ep, p_u, rep, t_u, st0);
                    if(c <= q_entry){                                 // :436-448
                        const double q_c0 = cloud, q_i0 = ice;
                        if(!K.evap || !K.conserve || (q_c0 <= 0.0 && q_i0 <= 0.0)) go = false;
                        else {
                            const double q_Ice_0 = qsat<FAST>(G, true, rho_c, ep, p_u, rep, t_u, st0);
                            double q_t0;
                            if(q_c0 > 0.0 && q_i0 > 0.0) q_t0 = (q_c0 * q_Rain_0 + q_i0 * q_Ice_0) / (q_c0 + q_i0);
                            else if(q_i0 <= 0.0)         q_t0 = q_Rain_0;
                            else                         q_t0 = q_Ice_0;
                            if(fabs(c - q_t0) <= K.entry_tol * q_t0) go = false;
                        }
                    }
                }
                if(go){
                    // ---- :450-590, at most 15 passes ----
                    double q_v_b = c, q_c_b = cloud, q_i_b = ice;
                    double T = t_u, q_v_hyp = q_v_b;
                    SatT st_full = st0;                 // the last full log / reciprocal (mixed form)
                    bool found = false, dry = false;
                    double q_rain_now = q_Rain_0;
                    for(int itr = 1; itr <= 15; itr++){
                        double CND = (T - t_00) * tri;
                        double DEP = (t_0 - T) * tri;
                        if(T <= t_00){ CND = 0.0; DEP = 1.0; }
                        if(T >= t_0) { CND = 1.0; DEP = 0.0; }
                        const bool berg = K.bergeron != 0 && T < t_0 && q_v_b <= q_rain_now
                                        && (q_i_b > 0.0 || (K.bergeron >= 2 && q_c_b <= 0.0));
                        if(berg){
                            CND = 0.0; DEP = 1.0;
                            if(q_c_b > 0.0){
                                T -= per_hc(lv * q_c_b);
                                q_v_b += q_c_b;
                                q_c_b = 0.0;
                            }
                        }
                        double d_q_v = q_v_hyp - q_v_b;
                        double d_q_c = -d_q_v * CND;
                        double d_q_i = -d_q_v * DEP;
                        if(K.conserve){
                            if(d_q_v < -q_v_b){ d_q_v = -q_v_b; d_q_c = -d_q_v * CND; d_q_i = -d_q_v * DEP; }
                            if(q_c_b + d_q_c < 0.0){ const double ex = -(q_c_b + d_q_c); d_q_c = -q_c_b; d_q_i -= ex; }
                            if(q_i_b + d_q_i < 0.0){ const double ex = -(q_i_b + d_q_i); d_q_i = -q_i_b; d_q_c -= ex;
                                                     if(q_c_b + d_q_c < 0.0) d_q_c = -q_c_b; }
                            d_q_v = -(d_q_c + d_q_i);
                        }
                        T     += per_hc(lv * d_q_c + ls * d_q_i);
                        q_v_b += d_q_v;
                        q_c_b += d_q_c;
                        q_i_b += d_q_i;
                        if(q_v_b < 0.0) q_v_b = 0.0;
                        if(q_c_b < 0.0) q_c_b = 0.0;
                        if(q_i_b < 0.0) q_i_b = 0.0;

                        // Which saturation pressures the closure below reads (1 liquid, 2 ice, 3 both):
                        // the one it does not read is not computed (same values where read).
                        auto need = [&](double Tx) -> int {
                            if(q_c_b > 0.0 && q_i_b > 0.0) return 3;
                            if(K.bergeron >= 2 && q_c_b <= 0.0 && q_i_b <= 0.0 && Tx < t_0) return 2;
                            if(K.ice_entry && q_c_b <= 0.0 && q_i_b <= 0.0) return 3;
                            return (q_i_b == 0.0) ? 1 : 2;
                        };
                        SatT stT;
                        if constexpr(FAST){
                            const double dT0 = T - st_full.T;      // exact: T and st_full.T are close
                            if(fabs(dT0) * st_full.inv <= 2.0e-3) stT = sat_t_next(st_full, dT0);
                            else { stT = sat_t(T); st_full = stT; }
                        }
                        const double q_Rain = qsat<FAST>(G, false, rho_c, ep, p_u, rep, T, stT);
                        const double q_Ice  = (need(T) & 2) ? qsat<FAST>(G, true, rho_c, ep, p_u, rep, T, stT) : 0.0;
                        q_rain_now = q_Rain;
                        if(q_c_b > 0.0 && q_i_b > 0.0)
                            q_v_hyp = (q_c_b * q_Rain + q_i_b * q_Ice) / (q_c_b + q_i_b);
                        else if(K.bergeron >= 2 && q_c_b <= 0.0 && q_i_b <= 0.0 && T < t_0) q_v_hyp = q_Ice;
                        else if(K.ice_entry && q_c_b <= 0.0 && q_i_b <= 0.0){
                            const double cn = T <= t_00 ? 0.0 : (T >= t_0 ? 1.0 : (T - t_00) * tri);
                            q_v_hyp = cn * q_Rain + (1.0 - cn) * q_Ice; }
                        else if(q_i_b == 0.0) q_v_hyp = q_Rain;
                        else                  q_v_hyp = q_Ice;

                        if(T >= t_0){
                            if(K.conserve){
                                if(q_i_b > 0.0){
                                    double dm = q_i_b;
                                    if(Lf > 0.0){
                                        const double hc = cp_mix * rho_c;
                                        const double cap = hc * (T - t_0) / Lf;
                                        if(dm > cap) dm = cap;
                                        T -= Lf * dm / hc;
                                    }
                                    q_i_b -= dm;
                                    q_c_b += dm;
                                }
                            } else {
                                q_i_b = 0.0;
                            }
                        }
                        const double q_diff = fabs(q_v_b - q_v_hyp) / (q_v_hyp + 1e-20);
                        if(q_diff <= K.stop_tol){ found = true; break; }
                        if(K.dry_exit && K.conserve && q_c_b <= 0.0 && q_i_b <= 0.0 && q_v_b < q_v_hyp){ dry = true; break; }
                        if(K.newton){
                            const double dT = 0.1;
                            const int nd = need(T);
                            SatT stD;
                            if constexpr(FAST) stD = (T == stT.T) ? sat_t_next(stT, dT) : sat_t(T + dT);
                            const double q_Rain_d = (nd & 1) ? qsat<FAST>(G, false, rho_c, ep, p_u, rep, T + dT, stD) : 0.0;
                            const double q_Ice_d  = (nd & 2) ? qsat<FAST>(G, true, rho_c, ep, p_u, rep, T + dT, stD) : 0.0;
                            double q_hyp_d;
                            if(q_c_b > 0.0 && q_i_b > 0.0)
                                q_hyp_d = (q_c_b * q_Rain_d + q_i_b * q_Ice_d) / (q_c_b + q_i_b);
                            else if(K.bergeron >= 2 && q_c_b <= 0.0 && q_i_b <= 0.0 && T < t_0) q_hyp_d = q_Ice_d;
                            else if(K.ice_entry && q_c_b <= 0.0 && q_i_b <= 0.0){
                                const double cn = T <= t_00 ? 0.0 : (T >= t_0 ? 1.0 : (T - t_00) * tri);
                                q_hyp_d = cn * q_Rain_d + (1.0 - cn) * q_Ice_d; }
                            else if(q_i_b == 0.0) q_hyp_d = q_Rain_d;
                            else                  q_hyp_d = q_Ice_d;
                            double CNDn = (T - t_00) * tri;
                            if(T <= t_00) CNDn = 0.0;
                            if(T >= t_0)  CNDn = 1.0;
                            if(berg)      CNDn = 0.0;
                            double Gf;
                            if constexpr(FAST) Gf = (lv * CNDn + ls * (1.0 - CNDn)) * inv_hc * (q_hyp_d - q_v_hyp) * (1.0 / dT);
                            else Gf = (lv * CNDn + ls * (1.0 - CNDn)) / (cp_mix * rho_c) * (q_hyp_d - q_v_hyp) / dT;
                            const double Gp = (Gf < 0.0) ? 0.0 : Gf;          // std::max(G, 0.0)
                            double wn = 1.0 / (1.0 + Gp);
                            if(wn < 0.05) wn = 0.05;
                            q_v_hyp = q_v_b + wn * (q_v_hyp - q_v_b);
                        } else {
                            q_v_hyp = 0.5 * (q_v_hyp + q_v_b);
                        }
                    }
                    n_adj++;
                    if(!found && !dry) n_nc++;
                    c = q_v_b; cloud = q_c_b; ice = q_i_b;
                    tt = T / t_ref;
                }
            }
            // final clamp of this gas's fields over every cell (:673-685)
            if(c <= 0.0) c = 0.0;
            if(cloud <= 0.0) cloud = 0.0;
            if(ice <= 0.0) ice = 0.0;
            cP[q] = (S)c; clP[q] = (S)cloud; iP[q] = (S)ice;
            if(a.sync){ cP[q + a.nc_off] = (S)c; clP[q + a.nc_off] = (S)cloud; iP[q + a.nc_off] = (S)ice; }
        }
        t_st(a.t, a.tlo, q, tt);
        if(a.sync){
            t_st(a.t + a.nc_off, a.tnlo, q, tt);
            if(a.sync == 2) a.nh4sh[q + a.nc_off] = a.nh4sh[q];
        }
    }
    // per-block counter reduction: integer adds, order-independent. Without counters (uniform
    // over the block) each warp leaves as soon as its cells are done.
    if(!a.counters) return;
    __shared__ unsigned s_adj, s_nc;
    if(threadIdx.x == 0){ s_adj = 0; s_nc = 0; }
    __syncthreads();
    if(n_adj) atomicAdd(&s_adj, n_adj);
    if(n_nc) atomicAdd(&s_nc, n_nc);
    __syncthreads();
    if(threadIdx.x == 0 && a.counters){
        if(s_adj) atomicAdd(a.counters + 0, (unsigned long long)s_adj);
        if(s_nc) atomicAdd(a.counters + 1, (unsigned long long)s_nc);
    }
}

}  // namespace aturan
