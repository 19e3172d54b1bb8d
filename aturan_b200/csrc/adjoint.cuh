// Hand-written adjoint of one RK4 step of the dry dynamics (t, u, v, w), FP64.
//
// Forward (rk4.cuh, RungeKutta_Uran_Turb.cpp:18-403): level means ref(T), p_hydro = H(T, v, w, ref),
// then four stages k_s = RHS(X_s, p_hydro) with X_0 = y, X_{s+1} = y + c_s k_s on the interior
// (boundary rows of every X_s are y's), and y' = y + dt/6 sum_s w_s k_s, T' clamped. The inputs y
// are the state and its start-of-step copies together; p_dyn, p_stat, the forcing and every
// other field are held fixed (the tendencies of t, u, v, w do not read the scalars).
//
// Reverse: with g = ybar' masked by the clamp, ybar = g, kbar_3 = dt/6 w_3 g, and for s = 3..0
//   Xbar_s = J_s^T kbar_s (+ p_hydro part), ybar += Xbar_s, kbar_{s-1} = dt/6 w_{s-1} g + c_{s-1} Xbar_s,
// then the hydrostatic integral's and the level means' adjoints add into ybar (T, v, w).
//
// J_s^T is a scatter of every interior cell's local partial derivatives onto its 7-point stencil.
// It runs as gather, without atomics and in a fixed order: adj_local_kernel writes, per cell and
// per field, the seven contributions the cell sends to its stencil points (ADJ_SLOTS arrays), and
// adj_gather_kernel sums, per cell, the seven it receives from the cells whose stencils contain it.
// The partial derivatives are those of the forward's formulas (RHS_Uran_Turb.cpp:92-788), derived
// term by term; cp(T) is the piecewise-linear table, differentiated within its interval (a kink
// convention: the derivative of the interval the value falls in).
#pragma once
#include "common.cuh"
#include "rk4.cuh"
#include "satadj.cuh"

namespace aturan {

constexpr int ADJ_NF = 4;                          // t, u, v, w (state fields 0..3)
constexpr int ADJ_SLOT_PH = 7 * ADJ_NF;            // p_hydro tp, tm, pe, pw
constexpr int ADJ_SLOT_PD = ADJ_SLOT_PH + 4;       // p_dyn rp, rm, tp, tm, pe, pw
constexpr int ADJ_SLOTS = ADJ_SLOT_PD + 6;         // per field rp, rm, tp, tm, pe, pw, c; then p_hydro, p_dyn
// The moist form: the twelve condensable species (state fields 4..15, ATURAN_CH4 .. ATURAN_NH3_ICE)
// join the dry four, their seven slots each after the dry layout.
constexpr int ADJ_NF_MOIST = 16;
constexpr int ADJ_NSP = ADJ_NF_MOIST - ADJ_NF;
constexpr int ADJ_SLOTS_MOIST = ADJ_SLOTS + 7 * ADJ_NSP;
__host__ __device__ constexpr size_t adj_slot_base(int q){
    return q < ADJ_NF ? (size_t)q * 7 : (size_t)ADJ_SLOTS + (size_t)(q - ADJ_NF) * 7;
}

struct AdjArgs {
    Grid g;
    const double* X;            // stage input, field q (0..3) at X + q * fstride
    const double* X0;           // the step's input (boundary rows of every stage input)
    const double* kbar;         // adjoint of the stage's tendencies, field q at kbar + q * fstride
    const double* auxbar;       // stage 3 only, else null: adjoint of aux_u, aux_v, aux_w (the tendencies
                                // of u, v, w without the p_dyn gradient, RHS_Uran_Turb.cpp:1020-1022)
    const double* pdyn;
    const double* forc;         // forcing group (nue at offset 0)
    const GeoIJ<double>* geo;
    const double* cp_tab;
    RhsConst<double> k;
    double* slot;               // ADJ_SLOTS fields
    double* hacc;               // null, or the T tendencies' adjoint summed over the stages (heating)
};

// cp_lapse (rk4.cuh) and its derivative in T (K), the table's slope inside its 0.5 K interval.
__device__ __forceinline__ void cp_lapse_d(const RhsConst<double>& k, const double* tab, double T,
                                           double* cp, double* dcp){
    double ch, dch;
    if(k.cp_mode <= 0){ ch = k.cp_h2_const; dch = 0.0; }
    else {
        const double Tc = T < 5.0 ? 5.0 : T;
        const double x = ((Tc > 1500.0 ? 1500.0 : Tc) - 5.0) / 0.5;
        int i = (int)x; if(i > CP_TABLE_N - 2) i = CP_TABLE_N - 2;
        const double f = x - (double)i;
        const double a = __ldg(tab + i), b = __ldg(tab + i + 1);
        ch = a + f * (b - a);
        dch = (T > 5.0 && T < 1500.0) ? (b - a) / 0.5 : 0.0;
    }
    if(k.cp_gas){ *cp = (k.cp_rh2 * ch + k.cp_he_term + k.cp_ch4_term) / k.cp_rsum; *dcp = k.cp_rh2 * dch / k.cp_rsum; }
    else        { *cp = k.cp_mix + k.cp_rh2 * (ch - k.cp_h2_const);               *dcp = k.cp_rh2 * dch; }
}

// Adjoints of one field's six differences -> the seven stencil values it was formed from.
struct G6 { double d1r, d2r, d1t, d2t, d1p, d2p; };

__device__ __forceinline__ void put7(double* slot, size_t fs, size_t o, int field, const G6& g, double dc,
                                     const RhsConst<double>& k){
    double* S = slot + (size_t)field * 7 * fs + o;
    S[0 * fs] =  g.d1r * k.inv_2dr   + g.d2r * k.inv_dr2;      // to (i+1)
    S[1 * fs] = -g.d1r * k.inv_2dr   + g.d2r * k.inv_dr2;      // to (i-1)
    S[2 * fs] =  g.d1t * k.inv_2dthe + g.d2t * k.inv_dthe2;    // to (j+1)
    S[3 * fs] = -g.d1t * k.inv_2dthe + g.d2t * k.inv_dthe2;    // to (j-1)
    S[4 * fs] =  g.d1p * k.inv_2dphi + g.d2p * k.inv_dphi2;    // to (k+1)
    S[5 * fs] = -g.d1p * k.inv_2dphi + g.d2p * k.inv_dphi2;    // to (k-1)
    S[6 * fs] = dc - 2.0 * (g.d2r * k.inv_dr2 + g.d2t * k.inv_dthe2 + g.d2p * k.inv_dphi2);
}

// Per interior cell: the local partial derivatives of rhs_t, rhs_u, rhs_v, rhs_w times the
// tendencies' adjoints, as the contributions to each stencil point (RHS_Uran_Turb.cpp:92-788).
__global__ void __launch_bounds__(128) adj_local_kernel(const AdjArgs a){
    const Grid& g = a.g;
    const int k = blockIdx.x * 32 + threadIdx.x;
    const int j = 1 + blockIdx.y * 4 + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if(k > g.km - 2 || j > g.jm - 2 || i > g.im - 2) return;
    const RhsConst<double>& K = a.k;
    const GeoIJ<double> geo = a.geo[i * g.jm + j];
    Nbr<double> nb;
    nb.fs  = g.fstride;
    nb.o   = gidx(g, i, j, k);
    nb.oim = nb.o - (size_t)g.jm * g.kp; nb.oip = nb.o + (size_t)g.jm * g.kp;
    nb.ojm = nb.o - g.kp;                nb.ojp = nb.o + g.kp;
    nb.okw = nb.o - k + phi_wrap(k - 1, g.km);
    nb.oke = nb.o - k + phi_wrap(k + 1, g.km);
    nb.X   = a.X;
    nb.xim = (i == 1) ? a.X0 : a.X;
    nb.xip = (i == g.im - 2) ? a.X0 : a.X;
    nb.xjm = (j == 1) ? a.X0 : a.X;
    nb.xjp = (j == g.jm - 2) ? a.X0 : a.X;
    const size_t o = nb.o, fs = g.fstride;

    const D6<double> T = diff6(K, load7<double, double>(nb, 0));
    const D6<double> U = diff6(K, load7<double, double>(nb, 1));
    const D6<double> V = diff6(K, load7<double, double>(nb, 2));
    const D6<double> W = diff6(K, load7<double, double>(nb, 3));
    const double* P = a.pdyn;
    const double dpdr   = (ld(P + nb.oip) - ld(P + nb.oim)) * K.inv_2dr;
    const double dpdthe = (ld(P + nb.ojp) - ld(P + nb.ojm)) * K.inv_2dthe;
    const double dpdphi = (ld(P + nb.oke) - ld(P + nb.okw)) * K.inv_2dphi;
    const double nue_c = ld(a.forc + o);
    const double nue_t = (K.turb_coupling != 0.0 && isfinite(nue_c)) ? K.turb_coupling * cmax(0.0, nue_c) : 0.0;
    const double nue_t_s = nue_t / 0.9;
    const double at = a.kbar[0 * fs + o];
    if(a.hacc) a.hacc[o] += at;                 // rhs_t += heat_scale H(j,k) (aturan_set_heating)
    const double au0 = a.kbar[1 * fs + o], av0 = a.kbar[2 * fs + o], aw0 = a.kbar[3 * fs + o];
    // aux = the tendency without the p_dyn gradient: its adjoint joins the tendency's in every
    // partial except those in p_dyn
    const double au = au0 + (a.auxbar ? a.auxbar[0 * fs + o] : 0.0);
    const double av = av0 + (a.auxbar ? a.auxbar[1 * fs + o] : 0.0);
    const double aw = aw0 + (a.auxbar ? a.auxbar[2 * fs + o] : 0.0);

    const double u = U.c, v = V.c, w = W.c;
    const double inv_rm = geo.inv_rm, inv_rm2 = geo.inv_rm2, inv_rs = geo.inv_rmsinthe;
    const double inv_rm2s = geo.inv_rm2sinthe, inv_rm2s2 = geo.inv_rm2sinthe2, cir = geo.costhe_inv_rm2sinthe;
    const double costhe = geo.costhe, cot = geo.cotanthe, tir = geo.two_inv_rm;
    const double D = 1.0 / K.re_eff + nue_t, Dt = 1.0 / K.re_pr + nue_t_s;

    // pressure work and its cp(T) factor
    double cpf = 1.0, dcpf = 0.0;
    if(K.cp_dyn && T.c > 0.0){
        double cp, dcp;
        cp_lapse_d(K, a.cp_tab, T.c * K.t_ref, &cp, &dcp);
        cpf = K.cp_mix / cp;
        dcpf = -K.cp_mix / (cp * cp) * dcp * K.t_ref;
    }
    const double P0 = K.ce_sp * (u * dpdr + v * inv_rm * dpdthe + w * inv_rs * dpdphi);

    // direct (centre) partials of the four tendencies
    const double du = au * (-U.d1r + 2.0 * inv_rm2 * D - geo.sponge)
                    + av * (-V.d1r - v * inv_rm)
                    + aw * (-W.d1r - w * inv_rm - K.cor_sc * K.p2om * geo.sinthe_bf)
                    + at * (K.ce_sp * dpdr * cpf - T.d1r);
    const double dv = au * (-inv_rm * U.d1t)
                    + av * (-inv_rm * V.d1t - u * inv_rm - geo.v_metric * D)
                    + aw * (-inv_rm * W.d1t - w * cot * inv_rm - K.cor_sc * K.p2om * costhe)
                    + at * (K.ce_sp * inv_rm * dpdthe * cpf - inv_rm * T.d1t);
    const double dw = au * (-inv_rs * U.d1p - K.cor_rad_f * K.m2om * geo.sinthe_bf)
                    + av * (-inv_rs * V.d1p + 2.0 * w * cot * inv_rm - K.cor_sc * K.m2om * costhe)
                    + aw * (-inv_rs * W.d1p - (u + v * cot) * inv_rm - geo.v_metric * D)
                    + at * (K.ce_sp * inv_rs * dpdphi * cpf - inv_rs * T.d1p);
    const double dT = at * P0 * dcpf;

    G6 gT, gU, gV, gW;
    gT.d1r = at * (-u + tir * Dt);            gT.d2r = at * Dt;
    gT.d1t = at * (-v * inv_rm + cir * Dt);   gT.d2t = at * inv_rm2 * Dt;
    gT.d1p = at * (-w * inv_rs);              gT.d2p = at * inv_rm2s2 * Dt;

    gU.d1r = au * (-u + 4.0 * inv_rm * D);    gU.d2r = au * D;
    gU.d1t = au * (-v * inv_rm + cir * D) + av * (2.0 * inv_rm2 * D);
    gU.d2t = au * inv_rm2 * D;
    gU.d1p = au * (-w * inv_rs) + aw * (2.0 * inv_rm2s * D);
    gU.d2p = au * inv_rm2s2 * D;

    gV.d1r = av * (-u + tir * D);             gV.d2r = av * D;
    gV.d1t = av * (-v * inv_rm + cir * D);    gV.d2t = av * inv_rm2 * D;
    gV.d1p = av * (-w * inv_rs) + aw * (2.0 * costhe * inv_rm2s2 * D);
    gV.d2p = av * inv_rm2s2 * D;

    gW.d1r = aw * (-u + tir * D);             gW.d2r = aw * D;
    gW.d1t = aw * (-v * inv_rm + cir * D);    gW.d2t = aw * inv_rm2 * D;
    gW.d1p = aw * (-w * inv_rs) - av * (2.0 * costhe * inv_rm2s2 * D);
    gW.d2p = aw * inv_rm2s2 * D;

    put7(a.slot, fs, o, 0, gT, dT, K);
    put7(a.slot, fs, o, 1, gU, du, K);
    put7(a.slot, fs, o, 2, gV, dv, K);
    put7(a.slot, fs, o, 3, gW, dw, K);
    // p_hydro: rhs_v -= (ph[j+1] - ph[j-1]) inv_2dthe inv_rm, rhs_w -= (ph[k+1] - ph[k-1]) inv_2dphi inv_rs
    double* S = a.slot + (size_t)ADJ_SLOT_PH * fs + o;
    S[0 * fs] = -av * K.inv_2dthe * inv_rm;   // to (j+1)
    S[1 * fs] =  av * K.inv_2dthe * inv_rm;   // to (j-1)
    S[2 * fs] = -aw * K.inv_2dphi * inv_rs;   // to (k+1)
    S[3 * fs] =  aw * K.inv_2dphi * inv_rs;   // to (k-1)
    // p_dyn: rhs_u -= dpdr scale_p, rhs_v -= dpdthe scale_p inv_rm, rhs_w -= dpdphi scale_p inv_rs,
    // rhs_t += ce_sp (u dpdr + v inv_rm dpdthe + w inv_rs dpdphi) cpf (aux carries none of it)
    const double gdr = -K.scale_p * au0 + K.ce_sp * u * cpf * at;
    const double gdt = -K.scale_p * inv_rm * av0 + K.ce_sp * v * inv_rm * cpf * at;
    const double gdp = -K.scale_p * inv_rs * aw0 + K.ce_sp * w * inv_rs * cpf * at;
    double* Q = a.slot + (size_t)ADJ_SLOT_PD * fs + o;
    Q[0 * fs] =  gdr * K.inv_2dr;             // to (i+1)
    Q[1 * fs] = -gdr * K.inv_2dr;             // to (i-1)
    Q[2 * fs] =  gdt * K.inv_2dthe;           // to (j+1)
    Q[3 * fs] = -gdt * K.inv_2dthe;           // to (j-1)
    Q[4 * fs] =  gdp * K.inv_2dphi;           // to (k+1)
    Q[5 * fs] = -gdp * K.inv_2dphi;           // to (k-1)
}

// The twelve condensable species' tendencies (RHS_Uran_Turb.cpp:790-850, scalar_rhs in rk4.cuh):
// rhs_q = -(u d1r + v/r d1t + w/(r sin) d1p)(q) + D_q lap(q) + forcing, D_q = 1/(Sc_g Re) + nue_t/0.9,
// the forcing (precipitation sources, mass fluxes) held fixed. Per interior cell and species: the
// seven stencil contributions into the species' slots, and the transport's partials in u, v, w
// added to the centre slots of u, v, w that adj_local_kernel wrote (same cell, same thread, the
// next launch on the stream). a.X, a.X0, a.kbar hold ADJ_NF_MOIST fields.
__global__ void __launch_bounds__(128) adj_species_local_kernel(const AdjArgs a){
    const Grid& g = a.g;
    const int k = blockIdx.x * 32 + threadIdx.x;
    const int j = 1 + blockIdx.y * 4 + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if(k > g.km - 2 || j > g.jm - 2 || i > g.im - 2) return;
    const RhsConst<double>& K = a.k;
    const GeoIJ<double> geo = a.geo[i * g.jm + j];
    Nbr<double> nb;
    nb.fs  = g.fstride;
    nb.o   = gidx(g, i, j, k);
    nb.oim = nb.o - (size_t)g.jm * g.kp; nb.oip = nb.o + (size_t)g.jm * g.kp;
    nb.ojm = nb.o - g.kp;                nb.ojp = nb.o + g.kp;
    nb.okw = nb.o - k + phi_wrap(k - 1, g.km);
    nb.oke = nb.o - k + phi_wrap(k + 1, g.km);
    nb.X   = a.X;
    nb.xim = (i == 1) ? a.X0 : a.X;
    nb.xip = (i == g.im - 2) ? a.X0 : a.X;
    nb.xjm = (j == 1) ? a.X0 : a.X;
    nb.xjp = (j == g.jm - 2) ? a.X0 : a.X;
    const size_t o = nb.o, fs = g.fstride;
    const double u = a.X[1 * fs + o], v = a.X[2 * fs + o], w = a.X[3 * fs + o];
    const double nue_c = ld(a.forc + o);
    const double nue_t = (K.turb_coupling != 0.0 && isfinite(nue_c)) ? K.turb_coupling * cmax(0.0, nue_c) : 0.0;
    const double nue_t_s = nue_t / 0.9;
    const double inv_rm = geo.inv_rm, inv_rm2 = geo.inv_rm2, inv_rs = geo.inv_rmsinthe;
    const double inv_rm2s2 = geo.inv_rm2sinthe2, cir = geo.costhe_inv_rm2sinthe, tir = geo.two_inv_rm;
    double du = 0.0, dv = 0.0, dw = 0.0;
    for(int n = 0; n < ADJ_NSP; n++){
        const int q = ADJ_NF + n;
        const D6<double> Q = diff6(K, load7<double, double>(nb, q));
        const double aq = a.kbar[(size_t)q * fs + o];
        const double Dq = K.inv_sc_re[n / 3] + nue_t_s;
        G6 gq;
        gq.d1r = aq * (-u + tir * Dq);           gq.d2r = aq * Dq;
        gq.d1t = aq * (-v * inv_rm + cir * Dq);  gq.d2t = aq * inv_rm2 * Dq;
        gq.d1p = aq * (-w * inv_rs);             gq.d2p = aq * inv_rm2s2 * Dq;
        put7(a.slot + (size_t)ADJ_SLOTS * fs, fs, o, n, gq, 0.0, K);
        du -= aq * Q.d1r;
        dv -= aq * inv_rm * Q.d1t;
        dw -= aq * inv_rs * Q.d1p;
    }
    a.slot[(1 * 7 + 6) * fs + o] += du;
    a.slot[(2 * 7 + 6) * fs + o] += dv;
    a.slot[(3 * 7 + 6) * fs + o] += dw;
}

// ---- the saturation adjustment's implicit adjoint ----
// Per cell the forward (satadj_kernel, SaturationAdjustment.h:255-746) runs the four gases in the
// loop's order H2O, H2S, NH3, CH4, the temperature carried from one to the next. For one gas every
// step it takes -- the entry melt (:365-385) and freeze (:388-399), the Newton passes with their
// Bergeron conversion and in-pass melt (:450-590) -- moves mass between vapour q_v, cloud q_c and
// ice q_i and heat by the latent heats (L_f = L_s - L_v), so the total W = q_v + q_c + q_i and the
// moist enthalpy E = h T - L_v q_c - L_s q_i (h = cp_mix rho) are invariant. The converged state
// is the root of the closure q_v = H(T, q_c, q_i) on that invariant set, with the phases present
// at convergence frozen (the branch of the forward):
//   ice only      q_v = q_I(T), q_i = W - q_v              h dT = dE + L_s dW - L_s q_I'(T) dT
//   liquid only   q_v = q_R(T), q_c = W - q_v              (L_v, q_R likewise)
//   both          H = r q_R + (1 - r) q_I with the condensate split r = q_c / (q_c + q_i) frozen,
//                 L = r L_v + (1 - r) L_s
//   none          q_v = W, T = E / h (everything evaporated)
// so dT = (dE + L dW) / (h + L H'(T)) and the rest follows; this is the derivative of the exact
// root, which the forward approaches to its 1e-3 stopping test. A gas the forward leaves alone
// (no adjustment needed) contributes the derivative of its entry melt / freeze, each linear on its
// frozen branch (full, or capped at the phase temperature), and of the entry clamps.
// The temperature entering each gas is reconstructed from the invariants: the gas's entry state
// (the taped input, then each earlier gas's own entry and result) gives E, and its result gives
// T = (E + L_v q_c + L_s q_i) / h. The entry logic deciding whether a gas adjusts is the forward's
// FP64 path restated.
struct SatEntry {
    bool skip, go, cneg, clneg, ineg;
    int melt, freeze;            // 0 none, 1 whole amount, 2 capped at the phase temperature,
                                 // 3 mass only (L_f <= 0), 4 ice dropped (no conservation: melt only)
    double t_u, c, cloud, ice;   // after the entry steps and clamps
};

__device__ __forceinline__ double sat_q_d(const GasConst& G, bool ice, double rho_c, double p_u, double T, double* dq){
    const double C = ice ? G.C_i : G.C, L0 = ice ? G.L0_i : G.L0;
    const double al = ice ? G.del_alf_i : G.del_alf, be = ice ? G.del_bet_i : G.del_bet;
    const double q = rho_c * G.ep * svp(T, C, L0, G.den, al, be) / p_u;
    if(dq) *dq = q * (L0 / (T * T) + al / T + be) / G.den;
    return q;
}

// :358-448 on the FP64 path: the entry steps and the decision to adjust.
__device__ SatEntry sat_entry(const SatConst& K, const GasConst& G, double rho_c, double p_u, double t_u,
                              double c, double cloud, double ice){
    SatEntry e;
    e.skip = !((t_u > 0.0) && (p_u > 0.0));
    e.go = false; e.melt = 0; e.freeze = 0; e.cneg = e.clneg = e.ineg = false;
    e.t_u = t_u; e.c = c; e.cloud = cloud; e.ice = ice;
    if(e.skip) return e;
    const double t_0 = G.t_0, t_00 = G.t_00, Lf = G.Lf, hc = K.cp_mix * rho_c;
    if(t_u > t_0){
        if(K.conserve){
            if(ice > 0.0){
                double dm = ice;
                if(Lf > 0.0){
                    const double cap = hc * (t_u - t_0) / Lf;
                    e.melt = 1;
                    if(dm > cap){ dm = cap; e.melt = 2; }
                    t_u -= Lf * dm / hc;
                } else e.melt = 3;
                ice -= dm;
                cloud += dm;
            }
        } else { e.melt = 4; ice = 0.0; }
    }
    if(G.freeze_on && t_u < t_00 && cloud > 0.0){
        double dm = cloud;
        if(Lf > 0.0){
            const double cap = hc * (t_00 - t_u) / Lf;
            e.freeze = 1;
            if(dm > cap){ dm = cap; e.freeze = 2; }
            t_u += Lf * dm / hc;
        } else e.freeze = 3;
        cloud -= dm;
        ice += dm;
    }
    if(c < 0.0){ c = 0.0; e.cneg = true; }
    if(cloud < 0.0){ cloud = 0.0; e.clneg = true; }
    if(ice < 0.0){ ice = 0.0; e.ineg = true; }
    e.t_u = t_u; e.c = c; e.cloud = cloud; e.ice = ice;
    const double q_Rain_0 = sat_q_d(G, false, rho_c, p_u, t_u, nullptr);
    bool go = q_Rain_0 > 0.0;
    if(go){
        double q_entry = q_Rain_0;
        if(K.ice_entry && cloud <= 0.0 && ice <= 0.0){
            const double cnd0 = t_u <= t_00 ? 0.0 : (t_u >= t_0 ? 1.0 : (t_u - t_00) * G.t_range_inv);
            if(cnd0 < 1.0) q_entry = cnd0 * q_Rain_0 + (1.0 - cnd0) * sat_q_d(G, true, rho_c, p_u, t_u, nullptr);
        }
        if(K.bergeron >= 2 && cloud <= 0.0 && ice <= 0.0 && t_u < t_0) q_entry = sat_q_d(G, true, rho_c, p_u, t_u, nullptr);
        if(c <= q_entry){
            if(!K.evap || !K.conserve || (cloud <= 0.0 && ice <= 0.0)) go = false;
            else {
                const double q_Ice_0 = sat_q_d(G, true, rho_c, p_u, t_u, nullptr);
                double q_t0;
                if(cloud > 0.0 && ice > 0.0) q_t0 = (cloud * q_Rain_0 + ice * q_Ice_0) / (cloud + ice);
                else if(ice <= 0.0)          q_t0 = q_Rain_0;
                else                         q_t0 = q_Ice_0;
                if(fabs(c - q_t0) <= K.entry_tol * q_t0) go = false;
            }
        }
    }
    e.go = go;
    return e;
}

// The entry steps' adjoint: cotangents of (t_u, c, cloud, ice) after them -> before them.
__device__ void sat_entry_adj(const GasConst& G, double hc, const SatEntry& e, double& Tb, double& cb, double& clb, double& ib){
    const double Lf = G.Lf;
    if(e.cneg) cb = 0.0;
    if(e.clneg) clb = 0.0;
    if(e.ineg) ib = 0.0;
    if(e.freeze == 1){ clb = Tb * Lf / hc + ib; }
    else if(e.freeze == 2){ Tb = (clb - ib) * hc / Lf; }
    else if(e.freeze == 3){ clb = ib; }
    if(e.melt == 1){ ib = -Tb * Lf / hc + clb; }
    else if(e.melt == 2){ Tb = (clb - ib) * hc / Lf; }
    else if(e.melt == 3){ ib = clb; }
    else if(e.melt == 4){ ib = 0.0; }
}

// One cell: ybar (fields 0..15 of the step's RK4 input, i.e. after the adjustment) -> the same
// before it. pre: the taped state before the adjustment; post: after it (ADJ_NF_MOIST fields each).
__global__ void __launch_bounds__(128) adj_satadj_kernel(Grid g, const double* pre, const double* post, const double* ps,
                                                         const double* rho_mix, SatConst K, double* ybar){
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, i = blockIdx.z;
    if(k >= g.km) return;
    const size_t fs = g.fstride, q = gidx(g, i, j, k);
    const double p_u = ps[q];
    double rho_c = K.r_mix;                               // rho_at, cUranusModel.h:526-531
    if(K.local_rho){ const double r_ = rho_mix[q]; rho_c = (r_ > 0.0 && isfinite(r_)) ? r_ : K.r_mix; }
    const double hc = K.cp_mix * rho_c, t_ref = K.t_ref;
    const int base[4] = {ATURAN_H2O, ATURAN_H2S, ATURAN_NH3, ATURAN_CH4};
    // forward replay: each gas's entry record and the temperature after it
    SatEntry ent[4];
    double Tout[4];
    double T = pre[q] * t_ref;
    for(int gi = 0; gi < 4; gi++){
        const GasConst& G = K.gas[gi];
        const size_t f = (size_t)base[gi] * fs + q;
        ent[gi] = sat_entry(K, G, rho_c, p_u, T, pre[f], pre[f + fs], pre[f + 2 * fs]);
        const SatEntry& e = ent[gi];
        if(e.skip){ Tout[gi] = T; continue; }
        if(e.go){
            const double E = hc * e.t_u - G.lv * e.cloud - G.ls * e.ice;
            T = (E + G.lv * post[f + fs] + G.ls * post[f + 2 * fs]) / hc;
        } else T = e.t_u;
        Tout[gi] = T;
    }
    // reverse
    double Tb = ybar[q] / t_ref;
    for(int gi = 3; gi >= 0; gi--){
        const GasConst& G = K.gas[gi];
        const size_t f = (size_t)base[gi] * fs + q;
        const SatEntry& e = ent[gi];
        if(e.skip) continue;
        double cb = ybar[f], clb = ybar[f + fs], ib = ybar[f + 2 * fs];
        if(e.go){
            const double qc = post[f + fs], qi = post[f + 2 * fs], Tp = Tout[gi];
            double Eb, Wb;
            if(qc > 0.0 && qi > 0.0){
                const double r = qc / (qc + qi), L = r * G.lv + (1.0 - r) * G.ls;
                double dR, dI;
                sat_q_d(G, false, rho_c, p_u, Tp, &dR);
                sat_q_d(G, true, rho_c, p_u, Tp, &dI);
                const double dH = r * dR + (1.0 - r) * dI, Cb = r * clb + (1.0 - r) * ib;
                const double a = (Tb + (cb - Cb) * dH) / (hc + L * dH);
                Eb = a; Wb = a * L + Cb;
            } else if(qi > 0.0){
                double dI;
                sat_q_d(G, true, rho_c, p_u, Tp, &dI);
                const double a = (Tb + (cb - ib) * dI) / (hc + G.ls * dI);
                Eb = a; Wb = a * G.ls + ib;
            } else if(qc > 0.0){
                double dR;
                sat_q_d(G, false, rho_c, p_u, Tp, &dR);
                const double a = (Tb + (cb - clb) * dR) / (hc + G.lv * dR);
                Eb = a; Wb = a * G.lv + clb;
            } else {
                Eb = Tb / hc; Wb = cb;
            }
            Tb = Eb * hc; cb = Wb; clb = Wb - G.lv * Eb; ib = Wb - G.ls * Eb;
        }
        sat_entry_adj(G, hc, e, Tb, cb, clb, ib);
        ybar[f] = cb; ybar[f + fs] = clb; ybar[f + 2 * fs] = ib;
    }
    ybar[q] = Tb * t_ref;
}

// Per cell (every row, every meridian; the seam copy k = km-1 is read by no stencil and receives
// nothing): the sum of what the cells whose stencils contain it sent, in a fixed order. Adds the
// result into ybar and phbar; for s > 0 also forms the previous stage's kbar on the interior.
__global__ void __launch_bounds__(128) adj_gather_kernel(Grid g, const double* slot, double* ybar, double* phbar,
                                                         double* pdbar, const double* g0, double* kbar, double w_prev,
                                                         double c_prev, int has_prev, int nf){
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int i = blockIdx.z;
    if(k >= g.km - 1) return;
    const size_t fs = g.fstride, si = (size_t)g.jm * g.kp, sj = g.kp;
    const size_t o = gidx(g, i, j, k);
    const size_t okw = o - k + phi_wrap(k - 1, g.km), oke = o - k + phi_wrap(k + 1, g.km);
    const bool interior = i >= 1 && i <= g.im - 2 && j >= 1 && j <= g.jm - 2;
    for(int q = 0; q < nf; q++){
        const double* S = slot + adj_slot_base(q) * fs;
        double x = S[6 * fs + o];
        if(i >= 1)        x += S[0 * fs + o - si];
        if(i <= g.im - 2) x += S[1 * fs + o + si];
        if(j >= 1)        x += S[2 * fs + o - sj];
        if(j <= g.jm - 2) x += S[3 * fs + o + sj];
        x += S[4 * fs + okw];
        x += S[5 * fs + oke];
        ybar[q * fs + o] += x;
        if(has_prev && interior) kbar[q * fs + o] = w_prev * g0[q * fs + o] + c_prev * x;
    }
    const double* S = slot + (size_t)ADJ_SLOT_PH * fs;
    double h = 0.0;
    if(j >= 1)        h += S[0 * fs + o - sj];
    if(j <= g.jm - 2) h += S[1 * fs + o + sj];
    h += S[2 * fs + okw];
    h += S[3 * fs + oke];
    phbar[o] += h;
    const double* Q = slot + (size_t)ADJ_SLOT_PD * fs;
    double pd = 0.0;
    if(i >= 1)        pd += Q[0 * fs + o - si];
    if(i <= g.im - 2) pd += Q[1 * fs + o + si];
    if(j >= 1)        pd += Q[2 * fs + o - sj];
    if(j <= g.jm - 2) pd += Q[3 * fs + o + sj];
    pd += Q[4 * fs + okw];
    pd += Q[5 * fs + oke];
    pdbar[o] += pd;
}

// The final update's adjoint: g = ybar' (times 0 where T' was clamped), ybar = g, kbar_3 =
// dt/6 w_3 g on the interior. ybar_in is the caller's adjoint of the step's output.
__global__ void adj_init_kernel(Grid g, const double* ybar_in, const double* t_out, double t_min, double t_max,
                                double w3, double* g0, double* ybar, double* kbar, double* phbar, double* pdbar, int nf){
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int i = blockIdx.z;
    if(k >= g.km) return;
    const size_t fs = g.fstride;
    const size_t o = gidx(g, i, j, k);
    const bool interior = i >= 1 && i <= g.im - 2 && j >= 1 && j <= g.jm - 2 && k <= g.km - 2;
    for(int q = 0; q < nf; q++){
        double v = ybar_in[q * fs + o];
        if(q == 0 && interior && !(t_out[o] > t_min && t_out[o] < t_max)) v = 0.0;
        g0[q * fs + o] = interior ? v : 0.0;
        ybar[q * fs + o] = v;
        kbar[q * fs + o] = interior ? w3 * v : 0.0;
    }
    phbar[o] = 0.0;
    pdbar[o] = 0.0;
}

// Hydrostatic integral's adjoint, per column (RungeKutta_Uran_Turb.cpp:62-177): p_hydro(i) =
// sum_{n=1..i} (F(n-1) + F(n)) dr / 2 + const, F = cB buoy + met (cB = 1 - 1/follow_tau when the
// follow filter advances, else 1). Fbar(m) = dr/2 (S(m+1) + [m >= 1] S(m)), S the suffix sums of
// phbar. Adds the met part into vbar, wbar and the local buoy part into Tbar; leaves, per cell,
// the contribution to its level mean's adjoint in rbar.
__global__ void __launch_bounds__(256) adj_hydro_kernel(Grid g, const double* t, const double* ps, const double* v,
                                                        const double* w, const double* ref, const double* rm_i,
                                                        const double* cor_j, const double* phbar, double* ybar,
                                                        double* rbar, HydroConst h){
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if(c >= g.jm * g.km) return;
    const int j = c / g.km, k = c - j * g.km;
    const size_t fs = g.fstride;
    const double cB = h.follow_on ? 1.0 - 1.0 / h.follow_tau : 1.0;
    const double cor = cor_j[j];
    double S_next = 0.0;                           // S(m+1)
    for(int m = g.im - 1; m >= 0; m--){
        const size_t o = gidx(g, m, j, k);
        const double Sm = S_next + phbar[o];
        const double Fb = 0.5 * h.dr * (S_next + (m >= 1 ? Sm : 0.0));
        S_next = Sm;
        const double vv = v[o], ww = w[o];
        ybar[2 * fs + o] += Fb * 2.0 * vv / rm_i[m];
        ybar[3 * fs + o] += Fb * (2.0 * ww / rm_i[m] + cor);
        const double T = t[o];
        double rb = 0.0;
        if(T > 0.0){
            const double b = h.g * ps[o] / (h.rR * T * h.t_ref);
            const double f = h.m_nd_rel_b * (b - ref[m]) / ref[m];
            if(isfinite(f)){
                const double FbB = cB * Fb;
                ybar[o] += FbB * h.m_nd_rel_b / ref[m] * (-b / T);
                rb = FbB * (-h.m_nd_rel_b * b / (ref[m] * ref[m]));
            }
        }
        rbar[o] = rb;
    }
}

// Level mean's adjoint (RungeKutta_Uran_Turb.cpp:18-37): per level, Rbar = sum rbar and the
// weight sum W over the valid cells, in a fixed tree order; then per valid cell
// Tbar += Rbar / W * wsin_j * db/dT, db/dT = -b / T.
__global__ void __launch_bounds__(256) adj_level_sum_kernel(Grid g, const double* t, const double* ps,
                                                            const double* wsin, const double* rbar,
                                                            HydroConst h, double* lev){
    const int m = blockIdx.x;
    double s = 0.0, ws = 0.0;
    for(int c = threadIdx.x; c < g.jm * g.km; c += blockDim.x){
        const int j = c / g.km, k = c - j * g.km;
        const size_t o = gidx(g, m, j, k);
        const double T = t[o];
        if(!(T > 0.0)) continue;
        const double b = h.g * ps[o] / (h.rR * T * h.t_ref);
        if(!isfinite(b)) continue;
        s += rbar[o];
        ws += wsin[j];
    }
    __shared__ double ss[256], sw[256];
    ss[threadIdx.x] = s; sw[threadIdx.x] = ws;
    __syncthreads();
    for(int st = 128; st > 0; st >>= 1){
        if(threadIdx.x < st){ ss[threadIdx.x] += ss[threadIdx.x + st]; sw[threadIdx.x] += sw[threadIdx.x + st]; }
        __syncthreads();
    }
    if(threadIdx.x == 0){ lev[2 * m] = ss[0]; lev[2 * m + 1] = sw[0]; }
}

__global__ void adj_level_apply_kernel(Grid g, const double* t, const double* ps, const double* wsin,
                                       const double* lev, HydroConst h, double* ybar){
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int m = blockIdx.z;
    if(k >= g.km) return;
    const size_t o = gidx(g, m, j, k);
    const double T = t[o];
    if(!(T > 0.0) || !(lev[2 * m + 1] > 0.0)) return;
    const double b = h.g * ps[o] / (h.rR * T * h.t_ref);
    if(!isfinite(b)) return;
    ybar[o] += lev[2 * m] / lev[2 * m + 1] * wsin[j] * (-b / T);
}

// The heating field's adjoint: heat_scale times the T tendencies' adjoint summed over the stages and
// the interior levels, per (j,k); 0 on the polar rows and the seam column, which no stage reads.
__global__ void adj_heat_reduce_kernel(Grid g, const double* hacc, double scale, double* out){
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if(c >= g.jm * g.km) return;
    const int j = c / g.km, k = c - j * g.km;
    double s = 0.0;
    if(j >= 1 && j <= g.jm - 2 && k <= g.km - 2)
        for(int i = 1; i < g.im - 1; i++) s += hacc[gidx(g, i, j, k)];
    out[c] = scale * s;
}

// ---- The pressure step's adjoint (RB_SOR / RB_LINE path): p_dyn = F(solve(compat(clamp(div aux))))
// with F the boundary passes. Reverse: F^T, the transposed solve, compat^T, the clamp mask, div^T. ----

// F^T in reverse order of launch_pdyn_bcs: seam copy, theta folds (every level), radial folds.
__global__ void adj_pbc_p_kernel(Grid g, double* B){
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if(c >= g.im * g.jm) return;
    const int i = c / g.jm, j = c - i * g.jm;
    B[gidx(g, i, j, 0)] += B[gidx(g, i, j, g.km - 1)];
    B[gidx(g, i, j, g.km - 1)] = 0.0;
}
__global__ void adj_pbc_t_kernel(Grid g, double* B){
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if(k >= g.km) return;
    const double b0 = B[gidx(g, i, 0, k)], bn = B[gidx(g, i, g.jm - 1, k)];
    B[gidx(g, i, 0, k)] = 0.0; B[gidx(g, i, g.jm - 1, k)] = 0.0;
    B[gidx(g, i, 1, k)] += C43 * b0;        B[gidx(g, i, 2, k)] -= C13 * b0;
    B[gidx(g, i, g.jm - 2, k)] += C43 * bn; B[gidx(g, i, g.jm - 3, k)] -= C13 * bn;
}
__global__ void adj_pbc_r_kernel(Grid g, double* B){
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if(k >= g.km) return;
    const double b0 = B[gidx(g, 0, j, k)], bn = B[gidx(g, g.im - 1, j, k)];
    B[gidx(g, 0, j, k)] = 0.0; B[gidx(g, g.im - 1, j, k)] = 0.0;
    B[gidx(g, 1, j, k)] += C43 * b0;        B[gidx(g, 2, j, k)] -= C13 * b0;
    B[gidx(g, g.im - 2, j, k)] += C43 * bn; B[gidx(g, g.im - 3, j, k)] -= C13 * bn;
}

// compat^T: the forward subtracts the constant (sum w src) / (sum w) from the interior source
// (w = y_i y_j), so its transpose maps lam to lam - w (sum lam) / (sum w); `mean` holds
// sum lam / n_interior and ratio = n_interior / sum w. Then the clamp mask from the forward's
// clamped source.
__global__ void adj_compat_mask_kernel(Grid g, const double* lam, const double* mean, double ratio,
                                       const double* src_fwd, const RBW* w, double* sbar){
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    const int i = 1 + blockIdx.z;
    if(k > g.km - 2) return;
    const size_t o = gidx(g, i, j, k);
    const double wy = ywt(i, 1, g.im - 2) * ywt(j, 1, g.jm - 2);
    const double v = lam[o] - wy * ratio * (*mean);
    const double s = src_fwd[o];
    const bool free_ = fabs(s) < w[i * g.jm + j].src_max;   // not clamped (clamped values sit at the bound)
    sbar[o] = free_ ? v : 0.0;
}

// div^T (rb_src_kernel): src(i,j,k) = (au[i+1] - au[i-1]) inv_2dr + (av[j+1] - av[j-1]) inv_2dthe inv_rm
// + (aw[k+1] - aw[k-1]) inv_2dphi inv_rmsinthe, with au = 0 on the radial boundary rows (rigid lid)
// or cubically extrapolated from the interior, and av = 0 on the polar rows (Pressure_Uran.cpp:30-146).
__global__ void adj_div_kernel(Grid g, const double* sbar, const RBW* w, PressConst c, int rigid_lid,
                               double* aub, double* avb, double* awb){
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int i = blockIdx.z;
    if(k >= g.km) return;
    const size_t o = gidx(g, i, j, k);
    const bool inner = i >= 1 && i <= g.im - 2 && j >= 1 && j <= g.jm - 2 && k <= g.km - 2;
    double u = 0.0, v = 0.0, ww = 0.0;
    if(inner){
        const size_t si = (size_t)g.jm * g.kp, sj = g.kp;
        if(i - 1 >= 1)        u += sbar[o - si] * c.inv_2dr;
        if(i + 1 <= g.im - 2) u -= sbar[o + si] * c.inv_2dr;
        if(!rigid_lid){       // au[0] = au[3] - 3 au[2] + 3 au[1], au[im-1] likewise (reads of the rows 1, im-2)
            const double b0 = -sbar[gidx(g, 1, j, k)] * c.inv_2dr;        // adjoint of au[0]
            const double bn =  sbar[gidx(g, g.im - 2, j, k)] * c.inv_2dr; // adjoint of au[im-1]
            if(i == 1) u += 3.0 * b0;
            if(i == 2) u -= 3.0 * b0;
            if(i == 3) u += b0;
            if(i == g.im - 2) u += 3.0 * bn;
            if(i == g.im - 3) u -= 3.0 * bn;
            if(i == g.im - 4) u += bn;
        }
        if(j - 1 >= 1)        v += sbar[o - sj] * c.inv_2dthe * w[i * g.jm + j - 1].inv_rm;
        if(j + 1 <= g.jm - 2) v -= sbar[o + sj] * c.inv_2dthe * w[i * g.jm + j + 1].inv_rm;
        const int kw = phi_wrap(k - 1, g.km), ke = phi_wrap(k + 1, g.km);
        ww = (sbar[o - k + kw] - sbar[o - k + ke]) * c.inv_2dphi * w[i * g.jm + j].inv_rmsinthe;
    }
    aub[o] = u; avb[o] = v; awb[o] = ww;
}

}  // namespace aturan
