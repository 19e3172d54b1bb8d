// RK4 step of the dynamical core: buoyancy reference level, hydrostatic column integral and the
// four fused RHS + stage-update passes.
//
// Reference: planet/RungeKutta_Uran_Turb.cpp:18-404 and planet/RHS_Uran_Turb.cpp:20-1023.
//
// The reference runs each stage as two barrier-separated passes over all interior cells (pass A
// evaluates RHSUran into 19 rhs_* arrays, pass B folds them into acc_* and writes the next stage
// input). Here one kernel per stage does both for its cell: it reads the stage input X_s with a
// 7-point stencil, forms the tendencies in registers and immediately writes acc and X_{s+1} to
// a SEPARATE buffer (ping-pong), so no thread ever reads a value another thread of the same
// launch writes. That removes the 19 rhs_* round trips through HBM. Stage 3 writes the new
// state y_{n+1} in place of the state and the projection fields rhs_u/v/w, aux_u/v/w.
//
// Boundary rows (i = 0, im-1; j = 0, jm-1) are never integrated; the reference's stage inputs
// keep the state's values there, so a neighbour on a boundary row is read from the state.
//
// Templates: S is the storage type of the state (double / float), C the arithmetic type. The
// FP64 instantiation is compiled without FMA contraction and keeps the reference's operand order
// in every expression, so it reproduces the CPU's IEEE results.
#pragma once
#include <climits>
#include "common.cuh"

namespace aturan {

template <typename S, typename C>
struct StageArgs {
    Grid g;
    const S* X;        // stage input: prognostic field q at X + q * fstride
    const S* St;       // the state (read for boundary neighbours)
    const S* Nc;       // start-of-step copies
    S* acc;            // RK4 accumulator
    S* Y;              // stage < 3: next stage input; stage 3: the state (y_{n+1})
    const double* pdyn;      // FP64 always: p_dyn and p_hydro enter as differences
    const double* phydro;
    const S* forc;     // forcing group: field (id - ATURAN_NUE) at forc + m * fstride
    S* proj;           // rhs_u, rhs_v, rhs_w, aux_u, aux_v, aux_w (stage 3 only)
    const GeoIJ<C>* geo;
    const C* cp_tab;
    const double* heat;      // [jm][km] heating rate in K/s (aturan_set_heating), or null: no such term
    RhsConst<C> k;
    C c_in, wgt;
    int stage;
    // the mixed form's temperature pair (common.cuh): the low parts of t (written by stage 3) and of
    // tn (read by stage 3); null in an FP64 context
    float* tlo;
    const float* tnlo;
};

template <typename S>
__device__ __forceinline__ S ld(const S* p){ return __ldg(p); }

template <typename C>
__device__ __forceinline__ C cmax(C a, C b){ return (a < b) ? b : a; }   // std::max
// x / d: the reference's division in the FP64 form; in the mixed form x times the reciprocal of
// the constant d formed once on the host (one rounding more, inside the form's tolerance, where an
// FP32 division costs about ten instructions).
template <typename C>
__device__ __forceinline__ C qdiv(C x, C d, C inv_d){
    if constexpr(sizeof(C) == 4) return x * inv_d; else return x / d;
}
template <typename C>
__device__ __forceinline__ C cclamp(C v, C lo, C hi){ return v < lo ? lo : (v > hi ? hi : v); }

// CpH2.h:77-84 and 122-134 (gas form): cp(T) from the equilibrium-H2 table.
template <typename C>
__device__ __forceinline__ C cp_lapse(const RhsConst<C>& k, const C* tab, C T){
    C ch;
    if(k.cp_mode <= 0) ch = k.cp_h2_const;
    else {
        const C Tc = T < C(5.0) ? C(5.0) : T;
        const C x = ((Tc > C(1500.0) ? C(1500.0) : Tc) - C(5.0)) / C(0.5);
        int i = (int)x; if(i > CP_TABLE_N - 2) i = CP_TABLE_N - 2;
        const C f = x - (C)i;
        const C a = __ldg(tab + i), b = __ldg(tab + i + 1);
        ch = a + f * (b - a);
    }
    if(k.cp_gas) return qdiv(k.cp_rh2 * ch + k.cp_he_term + k.cp_ch4_term, k.cp_rsum, k.inv_cp_rsum);
    return k.cp_mix + k.cp_rh2 * (ch - k.cp_h2_const);   // cp_rh2 holds r_h2 / r_mix here
}

template <typename C>
struct D6 { C c, d1r, d2r, d1t, d2t, d1p, d2p; };

// The seven stencil values of one field at one cell, as loaded.
template <typename C>
struct R7 { C c, rp, rm, tp, tm, pe, pw; };

// Neighbour addressing of one cell: offsets and, per direction, the array a neighbour is read
// from (the stage input, or the state on a boundary row).
template <typename S>
struct Nbr {
    size_t o, oim, oip, ojm, ojp, okw, oke, fs;
    const S *X, *xim, *xip, *xjm, *xjp;
};

template <typename S, typename C>
__device__ __forceinline__ R7<C> load7(const Nbr<S>& n, int q){
    const size_t f = (size_t)q * n.fs;
    R7<C> r;
    r.c  = (C)ld(n.X + f + n.o);
    r.rp = (C)ld(n.xip + f + n.oip); r.rm = (C)ld(n.xim + f + n.oim);
    r.tp = (C)ld(n.xjp + f + n.ojp); r.tm = (C)ld(n.xjm + f + n.ojm);
    r.pe = (C)ld(n.X + f + n.oke);   r.pw = (C)ld(n.X + f + n.okw);
    return r;
}

// The forward stage's addressing of one cell: offsets in elements from the stage input X -- of the
// cell and its six stencil neighbours (a neighbour on a boundary row lies in the state St, reached
// through the same base), of a field (fs), and of the accumulator, n-copy, forcing and stage-output
// buffers (d*). Every buffer the stage touches is carved from the context's one allocation, which
// the host keeps below 2^31 elements, so 32-bit offsets reach all of it: an address is one 32-bit
// add and one wide multiply-add, and a thread holds 12 registers of addressing instead of seven
// 64-bit offsets and five pointers (10 % faster stage in FP32: more resident blocks).
struct Cell { int o, oim, oip, ojm, ojp, okw, oke, fs, dacc, dnc, dforc, dY; };

// keast: the offset in k of the east neighbour (1 for one cell, 2 for a pair's second cell).
template <typename S, typename C>
__device__ __forceinline__ Cell make_cell(const StageArgs<S, C>& a, int i, int j, int k, int keast){
    const Grid& g = a.g;
    const int dSt = (int)(a.St - a.X);
    const int JK = g.jm * g.kp;
    Cell c;
    c.fs  = (int)g.fstride;
    c.o   = (int)gidx(g, i, j, k);
    c.oim = c.o - JK + (i == 1 ? dSt : 0);       c.oip = c.o + JK + (i == g.im - 2 ? dSt : 0);
    c.ojm = c.o - g.kp + (j == 1 ? dSt : 0);     c.ojp = c.o + g.kp + (j == g.jm - 2 ? dSt : 0);
    c.okw = c.o - k + phi_wrap(k - 1, g.km);     c.oke = c.o - k + phi_wrap(k + keast, g.km);
    c.dacc = (int)(a.acc - a.X); c.dnc = (int)(a.Nc - a.X); c.dforc = (int)(a.forc - a.X); c.dY = (int)(a.Y - a.X);
    return c;
}

template <typename S, typename C>
__device__ __forceinline__ R7<C> load7c(const S* X, const Cell& c, int q){
    const int f = q * c.fs;
    R7<C> r;
    r.c  = (C)ld(X + (f + c.o));
    r.rp = (C)ld(X + (f + c.oip)); r.rm = (C)ld(X + (f + c.oim));
    r.tp = (C)ld(X + (f + c.ojp)); r.tm = (C)ld(X + (f + c.ojm));
    r.pe = (C)ld(X + (f + c.oke)); r.pw = (C)ld(X + (f + c.okw));
    return r;
}

// RHS_Uran_Turb.cpp:93-176: central first and second differences of one field.
template <typename C>
__device__ __forceinline__ D6<C> diff6(const RhsConst<C>& k, const R7<C>& v){
    D6<C> d;
    const C c = v.c;
    d.c   = c;
    d.d1r = (v.rp - v.rm) * k.inv_2dr;
    d.d2r = (v.rp - C(2.0) * c + v.rm) * k.inv_dr2;
    d.d1t = (v.tp - v.tm) * k.inv_2dthe;
    d.d2t = (v.tp - C(2.0) * c + v.tm) * k.inv_dthe2;
    d.d1p = (v.pe - v.pw) * k.inv_2dphi;
    d.d2p = (v.pe - C(2.0) * c + v.pw) * k.inv_dphi2;
    return d;
}

// The accumulator (stages 1-3) and the start-of-step copy of one field at one cell.
template <typename C>
struct AccNc { C acc, nc; };

template <typename S, typename C>
__device__ __forceinline__ AccNc<C> load_acc_nc(const StageArgs<S, C>& a, const S* X, const Cell& c, int q){
    const int off = q * c.fs + c.o;
    AccNc<C> v;
    v.acc = (a.stage == 0) ? C(0.0) : (C)X[c.dacc + off];
    v.nc = (C)ld(X + (c.dnc + off));
    return v;
}

// acc and next-stage / final update of one prognostic field (RungeKutta_Uran_Turb.cpp:291-403).
// kind: 0 plain, 1 temperature (final clamp), 2 k* (clamp), 3 dis* (floor).
template <typename S, typename C>
__device__ __forceinline__ void stage_update(const StageArgs<S, C>& a, S* W, const Cell& c, int q, C r, int kind,
                                             const AccNc<C>& an){
    const int off = q * c.fs + c.o;
    C accv;
    if(a.stage == 0) accv = a.wgt * r;
    else accv = an.acc + a.wgt * r;
    const C yn = an.nc;
    if(a.stage < 3){
        W[c.dacc + off] = (S)accv;
        C y = yn + a.c_in * r;
        if(kind == 2) y = cclamp(y, C(0.0), a.k.tke_max);
        else if(kind == 3) y = cmax(y, a.k.dis_min);
        W[c.dY + off] = (S)y;
    } else {
        if constexpr(sizeof(S) == 4){
            if(kind == 1 && a.tlo){           // the temperature pair: y_n + dt acc / 6 in FP64
                const double inc = (double)qdiv(a.k.dt * accv, C(6.0), C(1.0 / 6.0));
                const double y = cclamp((double)yn + (double)a.tnlo[c.o] + inc, (double)a.k.t_min, (double)a.k.t_max);
                const S h = (S)y;
                W[c.dY + off] = h;
                a.tlo[c.o] = (float)(y - (double)h);
                return;
            }
        }
        C y = yn + qdiv(a.k.dt * accv, C(6.0), C(1.0 / 6.0));
        if(kind == 1) y = cclamp(y, a.k.t_min, a.k.t_max);
        else if(kind == 2) y = cclamp(cmax(y, C(0.0)), C(0.0), a.k.tke_max);
        else if(kind == 3) y = cmax(y, a.k.dis_min);
        W[c.dY + off] = (S)y;
    }
}

// Everything one scalar field's tendency reads at one cell: its stencil, accumulator, n-copy and
// up to three forcing values.
template <typename C>
struct ScalarIn { R7<C> v; AccNc<C> an; C f1, f2, f3; };

// Scalar field n of the stage's second part: 0..11 the condensables (ATURAN_CH4 + n), 12 NH4SH,
// 13 k*, 14 dis*.
constexpr int N_SCALARS = 15;
__host__ __device__ constexpr int scalar_field(int n){
    return n < 12 ? ATURAN_CH4 + n : (n == 12 ? ATURAN_NH4SH : (n == 13 ? ATURAN_TKE : ATURAN_DIS));
}


// Tendency of scalar field n from its loaded inputs (:790-913, :989-1018).
template <typename C>
__device__ __forceinline__ C scalar_rhs(const RhsConst<C>& K, const ScalarIn<C>& in, int n, const GeoIJ<C>& geo,
                                        C u_ijk, C v_ijk, C w_ijk, C v_invrm, C w_invrs, C nue_c, C nue_t_s){
    const int q = scalar_field(n);
    const D6<C> Q = diff6(K, in.v);
    if(n < 12){
        // ---- the twelve condensables (:790-850) ----
        const C transport = u_ijk * Q.d1r + v_invrm * Q.d1t + w_invrs * Q.d1p;
        const C diffusion = Q.d2r + Q.d1r * geo.two_inv_rm + Q.d2t * geo.inv_rm2
            + Q.d1t * geo.costhe_inv_rm2sinthe + Q.d2p * geo.inv_rm2sinthe2;
        C r = - transport + qdiv(diffusion, K.sc_re[n / 3], K.inv_sc_re[n / 3]) + diffusion * nue_t_s;
        if(q == ATURAN_H2S || q == ATURAN_NH3) r = r + K.chemical_reaction * in.f2;
        r = r + K.precip_coupling * in.f1;
        return r;
    } else if(n == 12){
        // ---- NH4SH: flux limiter, chemistry and Stokes settling (:852-913) ----
        const C transport = u_ijk * Q.d1r + v_invrm * Q.d1t + w_invrs * Q.d1p;
        const C diffusion = Q.d2r + Q.d1r * geo.two_inv_rm + Q.d2t * geo.inv_rm2
            + Q.d1t * geo.costhe_inv_rm2sinthe + Q.d2p * geo.inv_rm2sinthe2;
        const C v_stokes = qdiv(K.stokes_a * (K.rho_cond_nh4sh - in.f3) * K.g, K.mue_mix, K.inv_mue_mix);
        return - transport + in.f1
               + qdiv(diffusion, K.sc_re[4], K.inv_sc_re[4]) + diffusion * nue_t_s
               + K.chemical_reaction * in.f2
               + qdiv(v_stokes, K.u_0, K.inv_u_0) * Q.d1r;
    } else {
        // ---- k* and dis* (:989-1018) ----
        const C transport = u_ijk * Q.d1r + v_ijk * Q.d1t * geo.inv_rm + w_ijk * Q.d1p * geo.inv_rmsinthe;
        const C diffusion = Q.d2r + Q.d1r * C(2.0) * geo.inv_rm + Q.d2t * geo.inv_rm2
            + Q.d1t * geo.costhe_inv_rm2sinthe + Q.d2p * geo.inv_rm2sinthe2;
        const C sig = n == 13 ? C(0.85) : C(0.5);
        return - transport + diffusion * (K.inv_re + qdiv(nue_c, sig, n == 13 ? C(1.0 / 0.85) : C(2.0))) + in.f1;
    }
}
__host__ __device__ constexpr int scalar_kind(int n){ return n < 13 ? 0 : (n == 13 ? 2 : 3); }


// Everything the momentum and temperature tendencies of one cell read: the stencils of u, v, w,
// t, the p_dyn and p_hydro neighbours (FP64), the accumulators and n-copies, two forcing values.
template <typename C>
struct MomIn {
    R7<C> rU, rV, rW, rT;
    double p_ip, p_im, p_jp, p_jm, p_ke, p_kw, ph_jp, ph_jm, ph_ke, ph_kw;
    AccNc<C> anU, anV, anW, anT;
    C f_tmf, f_qp;
};

template <typename S, typename C>
__device__ __forceinline__ void load_momentum(MomIn<C>& in, const StageArgs<S, C>& a, const S* X, const Cell& c,
                                              const RhsConst<C>& K){
    const double* P = a.pdyn;                   // FP64, no boundary substitution: offsets from the cell
    const double* PH = a.phydro;
    const int JK = a.g.jm * a.g.kp, kp = a.g.kp;
    in.p_ip = ld(P + (c.o + JK)); in.p_im = ld(P + (c.o - JK)); in.p_jp = ld(P + (c.o + kp)); in.p_jm = ld(P + (c.o - kp));
    in.p_ke = ld(P + c.oke); in.p_kw = ld(P + c.okw);
    in.ph_jp = ld(PH + (c.o + kp)); in.ph_jm = ld(PH + (c.o - kp)); in.ph_ke = ld(PH + c.oke); in.ph_kw = ld(PH + c.okw);
    in.rU = load7c<S, C>(X, c, ATURAN_U); in.rV = load7c<S, C>(X, c, ATURAN_V); in.rW = load7c<S, C>(X, c, ATURAN_W);
    in.rT = load7c<S, C>(X, c, ATURAN_T);
    in.anU = load_acc_nc(a, X, c, ATURAN_U); in.anV = load_acc_nc(a, X, c, ATURAN_V);
    in.anW = load_acc_nc(a, X, c, ATURAN_W); in.anT = load_acc_nc(a, X, c, ATURAN_T);
    const S* F = X + (c.dforc + c.o);
    in.f_tmf = (K.tmf != C(0.0)) ? (C)ld(F + (ATURAN_THERMALMASSFLUX - ATURAN_NUE) * c.fs) : C(0.0);
    in.f_qp = (K.precip_coupling != C(0.0)) ? (C)ld(F + (ATURAN_Q_PRECIP - ATURAN_NUE) * c.fs) : C(0.0);
}

// The tendencies of u, v, w and t of one cell (RHS_Uran_Turb.cpp:117-175, :208-331, :382-391,
// :528-557, :717-788) and the pressure-gradient terms aux needs (:1020-1022). j, k locate the
// heating field's value.
template <typename S, typename C>
__device__ __forceinline__ void momentum_rhs(const StageArgs<S, C>& a, const MomIn<C>& in, const GeoIJ<C>& geo,
                                             C nue_t, C nue_t_s, int j, int k, C& rhs_u, C& rhs_v, C& rhs_w,
                                             C& rhs_t, C& dpdr_term, C& dpdthe_term, C& dpdphi_term){
    const RhsConst<C>& K = a.k;
    const C inv_rm = geo.inv_rm, inv_rm2 = geo.inv_rm2, inv_rmsinthe = geo.inv_rmsinthe;
    const C inv_rm2sinthe = geo.inv_rm2sinthe, inv_rm2sinthe2 = geo.inv_rm2sinthe2;
    const C costhe_inv_rm2sinthe = geo.costhe_inv_rm2sinthe, costhe = geo.costhe;
    const C cotanthe = geo.cotanthe, two_inv_rm = geo.two_inv_rm;
    // pressure gradients (:117, :146, :175), FP64 differences
    const C dpdr   = (C)((in.p_ip - in.p_im) * (double)K.inv_2dr);
    const C dpdthe = (C)((in.p_jp - in.p_jm) * (double)K.inv_2dthe);
    const C dpdphi = (C)((in.p_ke - in.p_kw) * (double)K.inv_2dphi);

    const D6<C> U = diff6(K, in.rU), V = diff6(K, in.rV), W = diff6(K, in.rW);
    const C u_ijk = U.c, v_ijk = V.c, w_ijk = W.c;
    const C v_invrm = v_ijk * inv_rm;
    const C w_invrs = w_ijk * inv_rmsinthe;
    // ---- momentum ----
    {
        const C sinthe_bf = geo.sinthe_bf;
        const C Coriolis_rad = K.m2om * sinthe_bf * w_ijk;
        const C Coriolis_the = K.m2om * costhe * w_ijk;
        const C Coriolis_phi = K.p2om * (costhe * v_ijk + sinthe_bf * u_ijk);
        const C transport_u = u_ijk * U.d1r + v_invrm * U.d1t + w_invrs * U.d1p
            - C(0.0) * (v_ijk * v_ijk + w_ijk * w_ijk) * inv_rm;
        const C transport_v = u_ijk * V.d1r + v_invrm * V.d1t + w_invrs * V.d1p
            + (u_ijk * v_ijk - w_ijk * w_ijk * cotanthe) * inv_rm;
        const C transport_w = u_ijk * W.d1r + v_invrm * W.d1t + w_invrs * W.d1p
            + (w_ijk * u_ijk + v_ijk * w_ijk * cotanthe) * inv_rm;
        const C v_metric = geo.v_metric;
        const C diffusion_u = U.d2r + C(2.0) * u_ijk * inv_rm2 + U.d2t * inv_rm2
            + C(4.0) * U.d1r * inv_rm + U.d1t * costhe_inv_rm2sinthe
            + U.d2p * inv_rm2sinthe2;
        const C diffusion_v = V.d2r + V.d1r * two_inv_rm + V.d2t * inv_rm2
            + V.d1t * costhe_inv_rm2sinthe - v_metric * v_ijk
            + V.d2p * inv_rm2sinthe2
            + C(2.0) * U.d1t * inv_rm2
            - W.d1p * C(2.0) * costhe * inv_rm2sinthe2;
        const C diffusion_w = W.d2r + W.d1r * two_inv_rm + W.d2t * inv_rm2
            + W.d1t * costhe_inv_rm2sinthe - v_metric * w_ijk
            + W.d2p * inv_rm2sinthe2
            + C(2.0) * U.d1p * inv_rm2sinthe
            + V.d1p * C(2.0) * costhe * inv_rm2sinthe2;
        dpdr_term   = dpdr   * K.scale_p;
        dpdthe_term = dpdthe * K.scale_p * inv_rm;
        dpdphi_term = dpdphi * K.scale_p * inv_rmsinthe;
        const C dphdthe_term = (C)((in.ph_jp - in.ph_jm) * (double)K.inv_2dthe) * inv_rm;
        const C dphdphi_term = (C)((in.ph_ke - in.ph_kw) * (double)K.inv_2dphi) * inv_rmsinthe;
        const C re_eff = K.re_eff;
        rhs_u = - dpdr_term + C(0.0) - transport_u + qdiv(diffusion_u, re_eff, K.inv_re_eff) + diffusion_u * nue_t
                - K.cor_rad_f * Coriolis_rad
                + K.cen_f * geo.cent_rad
                - geo.sponge * u_ijk;
        rhs_v = - dpdthe_term - dphdthe_term - transport_v + qdiv(diffusion_v, re_eff, K.inv_re_eff) + diffusion_v * nue_t
                - K.cor_sc * Coriolis_the
                + K.cen_f * geo.cent_the;
        rhs_w = - dpdphi_term - dphdphi_term - transport_w + qdiv(diffusion_w, re_eff, K.inv_re_eff) + diffusion_w * nue_t
                - K.cor_sc * Coriolis_phi;
    }
    // ---- temperature ----
    {
        const D6<C> T = diff6(K, in.rT);
        C pressure_t = K.ce_sp * (u_ijk * dpdr + v_invrm * dpdthe + w_invrs * dpdphi);
        if(K.cp_dyn && T.c > C(0.0)) pressure_t *= K.cp_mix / cp_lapse(K, a.cp_tab, T.c * K.t_ref);
        const C transport_t = u_ijk * T.d1r + v_invrm * T.d1t + w_invrs * T.d1p;
        const C diffusion_t = T.d2r + T.d1r * two_inv_rm + T.d2t * inv_rm2
            + T.d1t * costhe_inv_rm2sinthe + T.d2p * inv_rm2sinthe2;
        const C tmf = (K.tmf != C(0.0)) ? K.tmf * in.f_tmf : C(0.0);
        C precip_t = C(0.0);
        if(K.precip_coupling != C(0.0)){
            precip_t = qdiv(K.precip_coupling * in.f_qp * K.precip_L, K.precip_den, K.inv_precip_den);
            if(!isfinite(precip_t)) precip_t = C(0.0);
            else if(precip_t >  C(0.5)) precip_t =  C(0.5);
            else if(precip_t < -C(0.5)) precip_t = -C(0.5);
        }
        rhs_t = + pressure_t - transport_t + qdiv(diffusion_t, K.re_pr, K.inv_re_pr) + diffusion_t * nue_t_s
                - tmf + C(0.0) + precip_t;
        if(a.heat) rhs_t = rhs_t + K.heat_scale * (C)a.heat[(size_t)j * a.g.km + k];   // not in the reference
    }
}

// ---- two cells per thread along k (the scalar launch's vectorised form) ----
// Cells k0 and k0 + 1 (k0 even; km - 1 is even, so a pair never straddles the seam): the centre,
// r and theta neighbours come as one 8-byte (FP32) or 16-byte (FP64) load each, the k neighbours
// of the pair are the pair's own values plus one load on each side; accumulator, n-copy, forcing
// and the stores are vector accesses too. Half the memory instructions and address arithmetic
// per cell of the one-cell form, the same arithmetic per cell.
template <typename S> struct Pair;
template <> struct Pair<float>  { using T = float2; };
template <> struct Pair<double> { using T = double2; };

template <typename S, typename C>
__device__ __forceinline__ void ld2(const S* p, C& x, C& y){
    const typename Pair<S>::T v = __ldg(reinterpret_cast<const typename Pair<S>::T*>(p));
    x = (C)v.x; y = (C)v.y;
}
template <typename S, typename C>
__device__ __forceinline__ void ld2_rw(const S* p, C& x, C& y){      // memory this launch also writes
    const typename Pair<S>::T v = *reinterpret_cast<const typename Pair<S>::T*>(p);
    x = (C)v.x; y = (C)v.y;
}
template <typename S, typename C>
__device__ __forceinline__ void st2(S* p, C x, C y){
    typename Pair<S>::T v; v.x = (S)x; v.y = (S)y;
    *reinterpret_cast<typename Pair<S>::T*>(p) = v;
}

template <typename C>
struct ScalarIn2 { ScalarIn<C> c0, c1; };

template <typename S, typename C>
__device__ __forceinline__ void load_scalar2(ScalarIn2<C>& in, const StageArgs<S, C>& a, const S* X, const Cell& c, int n){
    const int q = scalar_field(n);
    const int f = q * c.fs;
    ScalarIn<C>& A = in.c0;
    ScalarIn<C>& B = in.c1;
    ld2<S, C>(X + (f + c.o), A.v.c, B.v.c);
    ld2<S, C>(X + (f + c.oip), A.v.rp, B.v.rp);
    ld2<S, C>(X + (f + c.oim), A.v.rm, B.v.rm);
    ld2<S, C>(X + (f + c.ojp), A.v.tp, B.v.tp);
    ld2<S, C>(X + (f + c.ojm), A.v.tm, B.v.tm);
    A.v.pw = (C)ld(X + (f + c.okw));            // k0 - 1
    B.v.pe = (C)ld(X + (f + c.oke));            // k0 + 2
    A.v.pe = B.v.c;
    B.v.pw = A.v.c;
    if(a.stage == 0){ A.an.acc = C(0.0); B.an.acc = C(0.0); }
    else ld2_rw<S, C>(X + (c.dacc + f + c.o), A.an.acc, B.an.acc);
    ld2<S, C>(X + (c.dnc + f + c.o), A.an.nc, B.an.nc);
    const S* F = X + (c.dforc + c.o);
    const int fs = c.fs;
    A.f2 = B.f2 = C(0.0); A.f3 = B.f3 = C(0.0);
    if(n < 12){
        ld2<S, C>(F + (ATURAN_S_PRECIP_CH4 + n - ATURAN_NUE) * fs, A.f1, B.f1);
        if(q == ATURAN_H2S) ld2<S, C>(F + (ATURAN_MASSFLUX_H2S - ATURAN_NUE) * fs, A.f2, B.f2);
        if(q == ATURAN_NH3) ld2<S, C>(F + (ATURAN_MASSFLUX_NH3 - ATURAN_NUE) * fs, A.f2, B.f2);
    } else if(n == 12){
        ld2<S, C>(F + (ATURAN_FLUXLIM_NH4SH - ATURAN_NUE) * fs, A.f1, B.f1);
        ld2<S, C>(F + (ATURAN_MASSFLUX_NH4SH - ATURAN_NUE) * fs, A.f2, B.f2);
        ld2<S, C>(F + (ATURAN_RHO_MIX - ATURAN_NUE) * fs, A.f3, B.f3);
    } else {
        ld2<S, C>(F + ((n == 13 ? ATURAN_TKE_SOURCE : ATURAN_DIS_SOURCE) - ATURAN_NUE) * fs, A.f1, B.f1);
    }
}

// stage_update for the pair, with vector stores.
template <typename S, typename C>
__device__ __forceinline__ void stage_update2(const StageArgs<S, C>& a, S* W, const Cell& c, int q, C r0, C r1, int kind,
                                              const AccNc<C>& n0, const AccNc<C>& n1){
    const int off = q * c.fs + c.o;
    C acc0, acc1;
    if(a.stage == 0){ acc0 = a.wgt * r0; acc1 = a.wgt * r1; }
    else { acc0 = n0.acc + a.wgt * r0; acc1 = n1.acc + a.wgt * r1; }
    C y0, y1;
    if(a.stage < 3){
        st2<S, C>(W + (c.dacc + off), acc0, acc1);
        y0 = n0.nc + a.c_in * r0; y1 = n1.nc + a.c_in * r1;
        if(kind == 2){ y0 = cclamp(y0, C(0.0), a.k.tke_max); y1 = cclamp(y1, C(0.0), a.k.tke_max); }
        else if(kind == 3){ y0 = cmax(y0, a.k.dis_min); y1 = cmax(y1, a.k.dis_min); }
    } else {
        if constexpr(sizeof(S) == 4){
            if(kind == 1 && a.tlo){           // the temperature pair: y_n + dt acc / 6 in FP64
                const float2 ln = *reinterpret_cast<const float2*>(a.tnlo + c.o);
                const double tmin = (double)a.k.t_min, tmax = (double)a.k.t_max;
                const double z0 = cclamp((double)n0.nc + (double)ln.x + (double)qdiv(a.k.dt * acc0, C(6.0), C(1.0 / 6.0)), tmin, tmax);
                const double z1 = cclamp((double)n1.nc + (double)ln.y + (double)qdiv(a.k.dt * acc1, C(6.0), C(1.0 / 6.0)), tmin, tmax);
                const S h0 = (S)z0, h1 = (S)z1;
                st2<S, C>(W + (c.dY + off), (C)h0, (C)h1);
                *reinterpret_cast<float2*>(a.tlo + c.o) = make_float2((float)(z0 - (double)h0), (float)(z1 - (double)h1));
                return;
            }
        }
        y0 = n0.nc + qdiv(a.k.dt * acc0, C(6.0), C(1.0 / 6.0)); y1 = n1.nc + qdiv(a.k.dt * acc1, C(6.0), C(1.0 / 6.0));
        if(kind == 1){ y0 = cclamp(y0, a.k.t_min, a.k.t_max); y1 = cclamp(y1, a.k.t_min, a.k.t_max); }
        else if(kind == 2){ y0 = cclamp(cmax(y0, C(0.0)), C(0.0), a.k.tke_max); y1 = cclamp(cmax(y1, C(0.0)), C(0.0), a.k.tke_max); }
        else if(kind == 3){ y0 = cmax(y0, a.k.dis_min); y1 = cmax(y1, a.k.dis_min); }
    }
    st2<S, C>(W + (c.dY + off), y0, y1);
}

// The scalar part of a stage (the fifteen scalar fields), two cells per thread; the same
// arithmetic per cell, in the same order, as rk_stage_kernel<..., 2, ...>.
template <typename S, typename C, int PD, int MINB>
__global__ void __launch_bounds__(128, MINB) rk_scalar_pair_kernel(const StageArgs<S, C> a){
    const Grid& g = a.g;
    const int k = 2 * (blockIdx.x * 32 + threadIdx.x);
    const int j = 1 + blockIdx.y * 4 + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if(k > g.km - 2 || j > g.jm - 2 || i > g.im - 2) return;
    const RhsConst<C>& K = a.k;
    const GeoIJ<C> geo = a.geo[i * g.jm + j];
    const S* X = a.X;
    S* W = const_cast<S*>(a.X);                  // acc and Y, reached through the same base
    const Cell c = make_cell(a, i, j, k, 2);
    C nue0, nue1, u0, u1, v0, v1, w0, w1;
    ld2<S, C>(X + (c.dforc + c.o), nue0, nue1);                 // ATURAN_NUE, the forcing group's first
    ld2<S, C>(X + (ATURAN_U * c.fs + c.o), u0, u1);
    ld2<S, C>(X + (ATURAN_V * c.fs + c.o), v0, v1);
    ld2<S, C>(X + (ATURAN_W * c.fs + c.o), w0, w1);
    auto nts = [&](C nue_c) -> C {
        const C nue_t = (K.turb_coupling != C(0.0) && isfinite(nue_c)) ? K.turb_coupling * cmax(C(0.0), nue_c) : C(0.0);
        return qdiv(nue_t, C(0.9), C(1.0 / 0.9));
    };
    const C nts0 = nts(nue0), nts1 = nts(nue1);
    const C vr0 = v0 * geo.inv_rm, vr1 = v1 * geo.inv_rm;
    const C wr0 = w0 * geo.inv_rmsinthe, wr1 = w1 * geo.inv_rmsinthe;
    const int nfield = K.turb_active ? N_SCALARS : N_SCALARS - 2;
    ScalarIn2<C> ring[PD + 1];
#pragma unroll
    for(int n = 0; n < PD; n++) if(n < nfield) load_scalar2(ring[n], a, X, c, n);
#pragma unroll
    for(int n = 0; n < N_SCALARS; n++){
        if(n + PD < nfield) load_scalar2(ring[(n + PD) % (PD + 1)], a, X, c, n + PD);
        if(n < nfield){
            const ScalarIn2<C>& in = ring[n % (PD + 1)];
            const C r0 = scalar_rhs(K, in.c0, n, geo, u0, v0, w0, vr0, wr0, nue0, nts0);
            const C r1 = scalar_rhs(K, in.c1, n, geo, u1, v1, w1, vr1, wr1, nue1, nts1);
            stage_update2(a, W, c, scalar_field(n), r0, r1, scalar_kind(n), in.c0.an, in.c1.an);
        }
    }
}

// ---- the scalar part with its loads staged through shared memory by cp.async ----
// The same cells, arithmetic and order as rk_scalar_pair_kernel; only the way the inputs arrive
// differs. Each thread copies the inputs of its own pair for the next D fields into a ring of D
// shared-memory slots with asynchronous copies (cp.async, L1-allocating, so the neighbours other
// threads fetch are L1 hits), and waits for the oldest group only when it computes that field.
// The loads in flight no longer hold registers, so the ring can be deeper than the register ring
// of the plain kernel at more resident warps. A thread reads back only what it copied itself, and
// refills a slot only after the stores that consumed it, so no barrier is needed.
template <typename S>
struct AsyncSlot {                       // one field's inputs for the 128 threads of a block
    typename Pair<S>::T c[128], rp[128], rm[128], tp[128], tm[128], acc[128], nc[128], f1[128], f2[128], f3[128];
    S pw[128], pe[128];
};

template <int N>
__device__ __forceinline__ void cp_async_n(void* smem, const void* gmem){
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" :: "r"(sa), "l"(gmem), "n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_commit(){ asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait(){ asm volatile("cp.async.wait_group %0;\n" :: "n"(N) : "memory"); }

template <typename S, typename C>
__device__ __forceinline__ void issue_scalar2(AsyncSlot<S>& sl, int t, const StageArgs<S, C>& a, const S* X, const Cell& c, int n){
    constexpr int V = (int)sizeof(typename Pair<S>::T);
    const int q = scalar_field(n);
    const int f = q * c.fs;
    cp_async_n<V>(&sl.c[t], X + (f + c.o));
    cp_async_n<V>(&sl.rp[t], X + (f + c.oip));
    cp_async_n<V>(&sl.rm[t], X + (f + c.oim));
    cp_async_n<V>(&sl.tp[t], X + (f + c.ojp));
    cp_async_n<V>(&sl.tm[t], X + (f + c.ojm));
    cp_async_n<(int)sizeof(S)>(&sl.pw[t], X + (f + c.okw));
    cp_async_n<(int)sizeof(S)>(&sl.pe[t], X + (f + c.oke));
    if(a.stage != 0) cp_async_n<V>(&sl.acc[t], X + (c.dacc + f + c.o));
    cp_async_n<V>(&sl.nc[t], X + (c.dnc + f + c.o));
    const S* F = X + (c.dforc + c.o);
    const int fs = c.fs;
    if(n < 12){
        cp_async_n<V>(&sl.f1[t], F + (ATURAN_S_PRECIP_CH4 + n - ATURAN_NUE) * fs);
        if(q == ATURAN_H2S) cp_async_n<V>(&sl.f2[t], F + (ATURAN_MASSFLUX_H2S - ATURAN_NUE) * fs);
        if(q == ATURAN_NH3) cp_async_n<V>(&sl.f2[t], F + (ATURAN_MASSFLUX_NH3 - ATURAN_NUE) * fs);
    } else if(n == 12){
        cp_async_n<V>(&sl.f1[t], F + (ATURAN_FLUXLIM_NH4SH - ATURAN_NUE) * fs);
        cp_async_n<V>(&sl.f2[t], F + (ATURAN_MASSFLUX_NH4SH - ATURAN_NUE) * fs);
        cp_async_n<V>(&sl.f3[t], F + (ATURAN_RHO_MIX - ATURAN_NUE) * fs);
    } else {
        cp_async_n<V>(&sl.f1[t], F + ((n == 13 ? ATURAN_TKE_SOURCE : ATURAN_DIS_SOURCE) - ATURAN_NUE) * fs);
    }
}

// The slot read back into the register form load_scalar2 produces.
template <typename S, typename C>
__device__ __forceinline__ void take_scalar2(ScalarIn2<C>& in, const AsyncSlot<S>& sl, int t, const StageArgs<S, C>& a, int n){
    const int q = scalar_field(n);
    ScalarIn<C>& A = in.c0;
    ScalarIn<C>& B = in.c1;
    auto get = [&](const typename Pair<S>::T& v, C& x, C& y){ x = (C)v.x; y = (C)v.y; };
    get(sl.c[t], A.v.c, B.v.c);
    get(sl.rp[t], A.v.rp, B.v.rp);
    get(sl.rm[t], A.v.rm, B.v.rm);
    get(sl.tp[t], A.v.tp, B.v.tp);
    get(sl.tm[t], A.v.tm, B.v.tm);
    A.v.pw = (C)sl.pw[t];
    B.v.pe = (C)sl.pe[t];
    A.v.pe = B.v.c;
    B.v.pw = A.v.c;
    if(a.stage == 0){ A.an.acc = C(0.0); B.an.acc = C(0.0); }
    else get(sl.acc[t], A.an.acc, B.an.acc);
    get(sl.nc[t], A.an.nc, B.an.nc);
    A.f2 = B.f2 = C(0.0); A.f3 = B.f3 = C(0.0);
    get(sl.f1[t], A.f1, B.f1);
    if(n == 12 || q == ATURAN_H2S || q == ATURAN_NH3) get(sl.f2[t], A.f2, B.f2);
    if(n == 12) get(sl.f3[t], A.f3, B.f3);
}

template <typename S, typename C, int D, int MINB>
__global__ void __launch_bounds__(128, MINB) rk_scalar_async_kernel(const StageArgs<S, C> a){
    extern __shared__ __align__(16) unsigned char ring_raw[];
    AsyncSlot<S>* ring = reinterpret_cast<AsyncSlot<S>*>(ring_raw);
    const Grid& g = a.g;
    const int t = threadIdx.y * 32 + threadIdx.x;
    const int k = 2 * (blockIdx.x * 32 + threadIdx.x);
    const int j = 1 + blockIdx.y * 4 + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if(k > g.km - 2 || j > g.jm - 2 || i > g.im - 2) return;
    const RhsConst<C>& K = a.k;
    const S* X = a.X;
    S* W = const_cast<S*>(a.X);
    const Cell c = make_cell(a, i, j, k, 2);
    const int nfield = K.turb_active ? N_SCALARS : N_SCALARS - 2;
#pragma unroll
    for(int n = 0; n < D; n++){
        if(n < nfield) issue_scalar2(ring[n], t, a, X, c, n);
        cp_async_commit();
    }
    const GeoIJ<C> geo = a.geo[i * g.jm + j];
    C nue0, nue1, u0, u1, v0, v1, w0, w1;
    ld2<S, C>(X + (c.dforc + c.o), nue0, nue1);
    ld2<S, C>(X + (ATURAN_U * c.fs + c.o), u0, u1);
    ld2<S, C>(X + (ATURAN_V * c.fs + c.o), v0, v1);
    ld2<S, C>(X + (ATURAN_W * c.fs + c.o), w0, w1);
    auto nts = [&](C nue_c) -> C {
        const C nue_t = (K.turb_coupling != C(0.0) && isfinite(nue_c)) ? K.turb_coupling * cmax(C(0.0), nue_c) : C(0.0);
        return qdiv(nue_t, C(0.9), C(1.0 / 0.9));
    };
    const C nts0 = nts(nue0), nts1 = nts(nue1);
    const C vr0 = v0 * geo.inv_rm, vr1 = v1 * geo.inv_rm;
    const C wr0 = w0 * geo.inv_rmsinthe, wr1 = w1 * geo.inv_rmsinthe;
#pragma unroll
    for(int n = 0; n < N_SCALARS; n++){
        cp_async_wait<D - 1>();                      // field n's group has landed
        if(n < nfield){
            ScalarIn2<C> in;
            take_scalar2(in, ring[n % D], t, a, n);
            const C r0 = scalar_rhs(K, in.c0, n, geo, u0, v0, w0, vr0, wr0, nue0, nts0);
            const C r1 = scalar_rhs(K, in.c1, n, geo, u1, v1, w1, vr1, wr1, nue1, nts1);
            stage_update2(a, W, c, scalar_field(n), r0, r1, scalar_kind(n), in.c0.an, in.c1.an);
        }
        if(n + D < nfield) issue_scalar2(ring[n % D], t, a, X, c, n + D);   // after the stores that used the slot
        cp_async_commit();
    }
    cp_async_wait<0>();
}

// The first launch of a stage: fused RHS evaluation and stage update of momentum and temperature
// (u, v, w, t and, at the last stage, the projection fields) of one cell. The second launch
// (rk_scalar_pair_kernel / rk_scalar_async_kernel) takes the fifteen scalar fields: the two read
// disjoint stencil fields and write disjoint accumulator / stage-output fields, so they run as two
// launches of one stage with half the live registers each.
//
// The kernel is bound by the latency of its loads, so it keeps many loads in flight per thread:
// a store to acc or Y could alias any later load as far as the compiler knows, so all ~50 loads
// of the cell are issued before its first store. MINB is the launch bound on resident blocks per SM.
template <typename S, typename C, int MINB>
__global__ void __launch_bounds__(128, MINB) rk_stage_kernel(const StageArgs<S, C> a){
    const Grid& g = a.g;
    const int k = blockIdx.x * 32 + threadIdx.x;
    const int j = 1 + blockIdx.y * 4 + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if(k > g.km - 2 || j > g.jm - 2 || i > g.im - 2) return;
    const RhsConst<C>& K = a.k;
    const GeoIJ<C> geo = a.geo[i * g.jm + j];
    const S* X = a.X;
    S* W = const_cast<S*>(a.X);
    const Cell c = make_cell(a, i, j, k, 1);

    const C nue_c = (C)ld(X + (c.dforc + c.o));                 // ATURAN_NUE, the forcing group's first
    const C nue_t = (K.turb_coupling != C(0.0) && isfinite(nue_c)) ? K.turb_coupling * cmax(C(0.0), nue_c) : C(0.0);
    const C nue_t_s = qdiv(nue_t, C(0.9), C(1.0 / 0.9));

    MomIn<C> in;
    load_momentum(in, a, X, c, K);
    C rhs_u, rhs_v, rhs_w, rhs_t, dpdr_term, dpdthe_term, dpdphi_term;
    momentum_rhs(a, in, geo, nue_t, nue_t_s, j, k, rhs_u, rhs_v, rhs_w, rhs_t, dpdr_term, dpdthe_term, dpdphi_term);
    stage_update(a, W, c, ATURAN_U, rhs_u, 0, in.anU);
    stage_update(a, W, c, ATURAN_V, rhs_v, 0, in.anV);
    stage_update(a, W, c, ATURAN_W, rhs_w, 0, in.anW);
    if(a.stage == 3){
        S* Pj = a.proj + c.o;
        const int fs = c.fs;
        Pj[0 * fs] = (S)rhs_u;
        Pj[1 * fs] = (S)rhs_v;
        Pj[2 * fs] = (S)rhs_w;
        Pj[3 * fs] = (S)(rhs_u + dpdr_term);
        Pj[4 * fs] = (S)(rhs_v + dpdthe_term);
        Pj[5 * fs] = (S)(rhs_w + dpdphi_term);
    }
    stage_update(a, W, c, ATURAN_T, rhs_t, 1, in.anT);
}

// The seven stencil values of one field at the pair k0, k0 + 1 (as load_scalar2 forms them).
template <typename S, typename C>
__device__ __forceinline__ void load7c2(const S* X, const Cell& c, int q, R7<C>& A, R7<C>& B){
    const int f = q * c.fs;
    ld2<S, C>(X + (f + c.o), A.c, B.c);
    ld2<S, C>(X + (f + c.oip), A.rp, B.rp);
    ld2<S, C>(X + (f + c.oim), A.rm, B.rm);
    ld2<S, C>(X + (f + c.ojp), A.tp, B.tp);
    ld2<S, C>(X + (f + c.ojm), A.tm, B.tm);
    A.pw = (C)ld(X + (f + c.okw));
    B.pe = (C)ld(X + (f + c.oke));
    A.pe = B.c;
    B.pw = A.c;
}

template <typename S, typename C>
__device__ __forceinline__ void load_acc_nc2(const StageArgs<S, C>& a, const S* X, const Cell& c, int q, AccNc<C>& A, AccNc<C>& B){
    const int off = q * c.fs + c.o;
    if(a.stage == 0){ A.acc = C(0.0); B.acc = C(0.0); }
    else ld2_rw<S, C>(X + (c.dacc + off), A.acc, B.acc);
    ld2<S, C>(X + (c.dnc + off), A.nc, B.nc);
}

// load_momentum for the pair: the same values, by 8-byte (FP32) or 16-byte (FP64 / pressure) loads
// where the two cells' values are adjacent.
template <typename S, typename C>
__device__ __forceinline__ void load_momentum2(MomIn<C>& A, MomIn<C>& B, const StageArgs<S, C>& a, const S* X,
                                               const Cell& c, const RhsConst<C>& K){
    const double* P = a.pdyn;
    const double* PH = a.phydro;
    const int JK = a.g.jm * a.g.kp, kp = a.g.kp;
    auto ldd2 = [](const double* p, double& x, double& y){
        const double2 v = __ldg(reinterpret_cast<const double2*>(p)); x = v.x; y = v.y;
    };
    ldd2(P + (c.o + JK), A.p_ip, B.p_ip); ldd2(P + (c.o - JK), A.p_im, B.p_im);
    ldd2(P + (c.o + kp), A.p_jp, B.p_jp); ldd2(P + (c.o - kp), A.p_jm, B.p_jm);
    ldd2(P + c.o, B.p_kw, A.p_ke);                      // p(k0) is k0 + 1's west, p(k0 + 1) k0's east
    A.p_kw = ld(P + c.okw); B.p_ke = ld(P + c.oke);
    ldd2(PH + (c.o + kp), A.ph_jp, B.ph_jp); ldd2(PH + (c.o - kp), A.ph_jm, B.ph_jm);
    ldd2(PH + c.o, B.ph_kw, A.ph_ke);
    A.ph_kw = ld(PH + c.okw); B.ph_ke = ld(PH + c.oke);
    load7c2<S, C>(X, c, ATURAN_U, A.rU, B.rU); load7c2<S, C>(X, c, ATURAN_V, A.rV, B.rV);
    load7c2<S, C>(X, c, ATURAN_W, A.rW, B.rW); load7c2<S, C>(X, c, ATURAN_T, A.rT, B.rT);
    load_acc_nc2(a, X, c, ATURAN_U, A.anU, B.anU); load_acc_nc2(a, X, c, ATURAN_V, A.anV, B.anV);
    load_acc_nc2(a, X, c, ATURAN_W, A.anW, B.anW); load_acc_nc2(a, X, c, ATURAN_T, A.anT, B.anT);
    const S* F = X + (c.dforc + c.o);
    if(K.tmf != C(0.0)) ld2<S, C>(F + (ATURAN_THERMALMASSFLUX - ATURAN_NUE) * c.fs, A.f_tmf, B.f_tmf);
    else A.f_tmf = B.f_tmf = C(0.0);
    if(K.precip_coupling != C(0.0)) ld2<S, C>(F + (ATURAN_Q_PRECIP - ATURAN_NUE) * c.fs, A.f_qp, B.f_qp);
    else A.f_qp = B.f_qp = C(0.0);
}

// rk_stage_kernel with two cells per thread along k (k0 even; km - 1 is even, so a pair never
// straddles the seam): the same arithmetic per cell, in the same order, with about half the load
// and store instructions and address arithmetic per cell. Grid as the scalar launch's.
template <typename S, typename C, int MINB>
__global__ void __launch_bounds__(128, MINB) rk_stage_pair_kernel(const StageArgs<S, C> a){
    const Grid& g = a.g;
    const int k = 2 * (blockIdx.x * 32 + threadIdx.x);
    const int j = 1 + blockIdx.y * 4 + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if(k > g.km - 2 || j > g.jm - 2 || i > g.im - 2) return;
    const RhsConst<C>& K = a.k;
    const GeoIJ<C> geo = a.geo[i * g.jm + j];
    const S* X = a.X;
    S* W = const_cast<S*>(a.X);
    const Cell c = make_cell(a, i, j, k, 2);

    C nue0, nue1;
    ld2<S, C>(X + (c.dforc + c.o), nue0, nue1);                 // ATURAN_NUE, the forcing group's first
    auto nts = [&](C nue_c) -> C {
        return (K.turb_coupling != C(0.0) && isfinite(nue_c)) ? K.turb_coupling * cmax(C(0.0), nue_c) : C(0.0);
    };
    const C nue_t0 = nts(nue0), nue_t1 = nts(nue1);
    const C nue_t_s0 = qdiv(nue_t0, C(0.9), C(1.0 / 0.9)), nue_t_s1 = qdiv(nue_t1, C(0.9), C(1.0 / 0.9));

    MomIn<C> A, B;
    load_momentum2(A, B, a, X, c, K);
    C ru0, rv0, rw0, rt0, pr0, pt0, pp0, ru1, rv1, rw1, rt1, pr1, pt1, pp1;
    momentum_rhs(a, A, geo, nue_t0, nue_t_s0, j, k, ru0, rv0, rw0, rt0, pr0, pt0, pp0);
    momentum_rhs(a, B, geo, nue_t1, nue_t_s1, j, k + 1, ru1, rv1, rw1, rt1, pr1, pt1, pp1);
    stage_update2(a, W, c, ATURAN_U, ru0, ru1, 0, A.anU, B.anU);
    stage_update2(a, W, c, ATURAN_V, rv0, rv1, 0, A.anV, B.anV);
    stage_update2(a, W, c, ATURAN_W, rw0, rw1, 0, A.anW, B.anW);
    if(a.stage == 3){
        S* Pj = a.proj + c.o;
        const int fs = c.fs;
        st2<S, C>(Pj + 0 * fs, ru0, ru1);
        st2<S, C>(Pj + 1 * fs, rv0, rv1);
        st2<S, C>(Pj + 2 * fs, rw0, rw1);
        st2<S, C>(Pj + 3 * fs, ru0 + pr0, ru1 + pr1);
        st2<S, C>(Pj + 4 * fs, rv0 + pt0, rv1 + pt1);
        st2<S, C>(Pj + 5 * fs, rw0 + pp0, rw1 + pp1);
    }
    stage_update2(a, W, c, ATURAN_T, rt0, rt1, 1, A.anT, B.anT);
}

// ---- RungeKutta_Uran_Turb.cpp:18-37: per level, sin(theta)-weighted mean of g p / (r R T t_ref)
// over every cell with T > 0 and a finite value. Fast form: each block reduces a contiguous
// chunk of one level in a fixed tree order into partials[level][block]; a second kernel adds a
// level's partials in block order. Deterministic run to run; the order differs from the
// reference's serial j, k sum, which moves the mean by about an ulp. ----
template <typename S>
__global__ void __launch_bounds__(256) buoy_partial_kernel(Grid g, const S* t, const S* ps, const double* wsin,
                                                           HydroConst h, double* part_sum, double* part_w, int nblk){
    const int lev = blockIdx.y;
    const int ncell = g.jm * g.km;
    double s = 0.0, w = 0.0;
    for(int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += nblk * blockDim.x){
        const int j = c / g.km, k = c - j * g.km;
        const size_t o = gidx(g, lev, j, k);
        const double T = (double)__ldg(t + o);
        if(!(T > 0.0)) continue;
        const double b = h.g * (double)__ldg(ps + o) / (h.rR * T * h.t_ref);
        if(!isfinite(b)) continue;
        const double wg = wsin[j];
        s += wg * b;
        w += wg;
    }
    __shared__ double ss[256], sw[256];
    ss[threadIdx.x] = s; sw[threadIdx.x] = w;
    __syncthreads();
    for(int st = 128; st > 0; st >>= 1){
        if(threadIdx.x < st){ ss[threadIdx.x] += ss[threadIdx.x + st]; sw[threadIdx.x] += sw[threadIdx.x + st]; }
        __syncthreads();
    }
    if(threadIdx.x == 0){ part_sum[lev * nblk + blockIdx.x] = ss[0]; part_w[lev * nblk + blockIdx.x] = sw[0]; }
}

static __global__ void buoy_finish_kernel(int im, int nblk, const double* part_sum, const double* part_w, double* ref){
    const int lev = blockIdx.x * blockDim.x + threadIdx.x;
    if(lev >= im) return;
    double s = 0.0, w = 0.0;
    for(int b = 0; b < nblk; b++){ s += part_sum[lev * nblk + b]; w += part_w[lev * nblk + b]; }
    ref[lev] = (w > 0.0) ? s / w : 0.0;
}

// Exact form: the reference's serial j-then-k running sums, bit-equal to the reference, computed
// in parallel. The terms are w b >= 0 (w the sin(theta) weight, 0 for a skipped cell), so the
// running sum s never decreases. While s stays in one binade [2^e, 2^(e+1)) every representable
// value there is an integer multiple of u = 2^(e-52), and fl(s + x) = s + u round(x / u) with
// ties to the even multiple -- integer arithmetic, exact, in which only the ties depend on s (on
// the parity of s / u). So a chunk of BX_CH terms whose running sum provably stays in one binade
// acts on s as "add I_p units", p the parity of s / u at the chunk's start, and the chunk's two
// integers I_0, I_1 can be formed independently of every other chunk.
//   pass 1 (buoy_terms_kernel, one block per chunk): the terms, into a scratch array, and each
//     chunk's sum in any order (an approximate prefix is all pass 2 needs of them);
//   pass 2 (buoy_predict_kernel, one block per level): the approximate prefix of the chunk sums
//     predicts the binade each chunk's running sum stays in, if one;
//   pass 3 (buoy_units_kernel, one block per chunk): (I_0, I_1) of every predicted chunk, by an
//     ordered tree over its terms' own actions;
//   pass 4 (buoy_serial_pass_kernel, one warp per level): the chunks in order, each applied in O(1)
//     when s lies in the predicted binade and the result stays below its top, and term by term
//     otherwise (the first chunks, where s is small, and the ~9 where s crosses a power of two).
// Every O(1) step is checked exactly, so the prediction only decides speed. A level with a
// negative term (not monotone) runs all its chunks term by term.
// Both sums (w b and w) go this way; the mean is s / w as in the reference.
constexpr int BX_CH = 256;

template <typename S>
__global__ void __launch_bounds__(BX_CH) buoy_terms_kernel(Grid g, const S* t, const S* ps, const double* wsin,
                                                          HydroConst h, double* terms, double* bpart, int nbx){
    const int lev = blockIdx.y;
    const int ncell = g.jm * g.km;
    const int c = blockIdx.x * BX_CH + threadIdx.x;
    double bv = 0.0, wv = 0.0;                         // wv = 0 marks a skipped cell
    if(c < ncell){
        const int j = c / g.km, k = c - j * g.km;
        const size_t o = gidx(g, lev, j, k);
        const double T = (double)__ldg(t + o);
        if(T > 0.0){
            const double b = h.g * (double)__ldg(ps + o) / (h.rR * T * h.t_ref);
            if(isfinite(b)){ const double wg = wsin[j]; bv = wg * b; wv = wg; }
        }
        double* xb = terms + (size_t)lev * 2 * ncell;
        xb[c] = bv; xb[ncell + c] = wv;
    }
    __shared__ double sb[BX_CH], sw[BX_CH];
    __shared__ int neg;
    if(threadIdx.x == 0) neg = 0;
    sb[threadIdx.x] = bv; sw[threadIdx.x] = wv;
    __syncthreads();
    if(bv < 0.0) neg = 1;
    for(int st = BX_CH / 2; st > 0; st >>= 1){
        if(threadIdx.x < st){ sb[threadIdx.x] += sb[threadIdx.x + st]; sw[threadIdx.x] += sw[threadIdx.x + st]; }
        __syncthreads();
    }
    if(threadIdx.x == 0){
        double* q = bpart + 3 * ((size_t)lev * nbx + blockIdx.x);
        q[0] = sb[0]; q[1] = sw[0]; q[2] = neg ? 1.0 : 0.0;
    }
}

// pass 2: the approximate prefix of the chunk sums (a block scan over tiles of 256 chunks) and the
// predicted binade of each chunk's running sum (INT_MIN: not predicted to stay in one binade, or
// the level has a negative term), one block per level.
static __global__ void __launch_bounds__(256) buoy_predict_kernel(int nbx, const double* bpart, int* bexp){
    const int lev = blockIdx.x;
    const double* bp = bpart + 3 * (size_t)lev * nbx;
    int* E = bexp + 2 * (size_t)lev * nbx;
    __shared__ double scb[256], scw[256];
    __shared__ int negl;
    if(threadIdx.x == 0) negl = 0;
    __syncthreads();
    for(int b = threadIdx.x; b < nbx; b += 256) if(bp[3 * b + 2] != 0.0) negl = 1;
    __syncthreads();
    double carry_b = 0.0, carry_w = 0.0;
    for(int b0 = 0; b0 < nbx; b0 += 256){
        const int b = b0 + threadIdx.x;
        const double vb = (b < nbx) ? bp[3 * b] : 0.0, vw = (b < nbx) ? bp[3 * b + 1] : 0.0;
        scb[threadIdx.x] = vb; scw[threadIdx.x] = vw;
        __syncthreads();
        for(int off = 1; off < 256; off <<= 1){
            const double tb = threadIdx.x >= off ? scb[threadIdx.x - off] : 0.0;
            const double tw = threadIdx.x >= off ? scw[threadIdx.x - off] : 0.0;
            __syncthreads();
            scb[threadIdx.x] += tb; scw[threadIdx.x] += tw;
            __syncthreads();
        }
        if(b < nbx){
            const double pb_end = carry_b + scb[threadIdx.x], pw_end = carry_w + scw[threadIdx.x];
            const double eb_lo = (pb_end - vb) * (1.0 - 1e-9), eb_hi = pb_end * (1.0 + 1e-9);
            const double ew_lo = (pw_end - vw) * (1.0 - 1e-9), ew_hi = pw_end * (1.0 + 1e-9);
            // binades whose unit and scale are normal powers of two: -970 <= e <= 1000
            auto pred = [&](double lo, double hi) -> int {
                if(negl || !(lo > 0.0)) return INT_MIN;
                const int e = ilogb(lo);
                return (e == ilogb(hi) && e >= -970 && e <= 1000) ? e : INT_MIN;
            };
            E[2 * b] = pred(eb_lo, eb_hi); E[2 * b + 1] = pred(ew_lo, ew_hi);
        }
        carry_b += scb[255]; carry_w += scw[255];
        __syncthreads();
    }
}

// 2^n as a double for normal n (-1022 <= n <= 1023): the exponent field alone; x * pow2(n) is then
// exact for x and the product normal.
__device__ __forceinline__ double pow2(int n){ return __longlong_as_double((long long)(1023 + n) << 52); }

// A term's action on the units of a running sum in binade e, for an even (r.x) and odd (r.y)
// parity of s / u at the term: round(x / u) with ties to the even total.
__device__ __forceinline__ longlong2 term_units(double x, int e){
    const double q = x * pow2(52 - e);                 // exact: a power-of-two scaling, q < 2^53
    const double m = floor(q);
    const double f = q - m;                            // exact
    const long long mi = (long long)m;
    longlong2 r;
    if(f < 0.5)      { r.x = r.y = mi; }
    else if(f > 0.5) { r.x = r.y = mi + 1; }
    else             { r.x = mi + (mi & 1); r.y = mi + ((1 + mi) & 1); }      // the tie: to even
    return r;
}
// A then B, as actions on (parity -> units): C(p) = A(p) + B((p + A(p)) mod 2).
__device__ __forceinline__ longlong2 units_then(longlong2 A, longlong2 B){
    longlong2 C;
    C.x = A.x + ((A.x & 1) ? B.y : B.x);
    C.y = A.y + (((1 + A.y) & 1) ? B.y : B.x);
    return C;
}

// pass 3: each chunk's action (units for an even and an odd start) in its predicted binade, by an
// ordered tree over its terms, one block per chunk; the same for the weights.
static __global__ void __launch_bounds__(BX_CH) buoy_units_kernel(Grid g, int nbx, const double* terms, const int* bexp,
                                                                  long long* bunits){
    const int lev = blockIdx.y, b = blockIdx.x;
    const int ncell = g.jm * g.km;
    const int c = b * BX_CH + threadIdx.x;
    const int* E = bexp + 2 * ((size_t)lev * nbx + b);
    const double* xb = terms + (size_t)lev * 2 * ncell;
    __shared__ longlong2 ub[BX_CH], uw[BX_CH];
    const int eb = E[0], ew = E[1];
    const longlong2 zero = make_longlong2(0, 0);
    ub[threadIdx.x] = (eb != INT_MIN && c < ncell) ? term_units(xb[c], eb) : zero;
    uw[threadIdx.x] = (ew != INT_MIN && c < ncell) ? term_units(xb[ncell + c], ew) : zero;
    __syncthreads();
    for(int st = 1; st < BX_CH; st <<= 1){               // ordered: (t, t + st) into t
        if((threadIdx.x & (2 * st - 1)) == 0){
            ub[threadIdx.x] = units_then(ub[threadIdx.x], ub[threadIdx.x + st]);
            uw[threadIdx.x] = units_then(uw[threadIdx.x], uw[threadIdx.x + st]);
        }
        __syncthreads();
    }
    if(threadIdx.x == 0){
        long long* U = bunits + 4 * ((size_t)lev * nbx + b);
        U[0] = ub[0].x; U[1] = ub[0].y; U[2] = uw[0].x; U[3] = uw[0].y;
    }
}

// pass 4: the chunks in order, one warp per level. Lane 0 applies a chunk in O(1) when s lies in
// its predicted binade and the result stays below the binade's top; otherwise the warp stages the
// chunk's terms in shared memory and lane 0 adds them one by one. Between O(1) chunks of one binade
// the running sum stays an integer count of units (si), so the dependent chain is one integer add.
struct RunSum {
    double s;        // the running sum, when !in_units
    long long si;    // s / 2^(e-52), when in_units
    int e;
    bool in_units;
};
__device__ __forceinline__ void run_to_double(RunSum& r){
    if(r.in_units){ r.s = (double)r.si * pow2(r.e - 52); r.in_units = false; }    // exact
}
__device__ __forceinline__ bool chunk_fast(RunSum& r, int e, const long long* I){
    if(e == INT_MIN){ run_to_double(r); return false; }
    if(!(r.in_units && r.e == e)){
        run_to_double(r);
        const double lo = pow2(e);
        if(!(r.s >= lo && r.s < 2.0 * lo)) return false;
        r.si = (long long)(r.s * pow2(52 - e));        // exact integer
        r.e = e;
        r.in_units = true;
    }
    const long long ni = r.si + I[r.si & 1];
    if(ni >= (1LL << 53)){ run_to_double(r); return false; }
    r.si = ni;
    return true;
}

static __global__ void __launch_bounds__(32) buoy_serial_pass_kernel(Grid g, int nbx, const double* terms, const int* bexp,
                                                                     const long long* bunits, double* ref){
    constexpr int TILE = 256;                          // chunks whose binades and units are staged at once
    const int lev = blockIdx.x, lane = threadIdx.x;
    const int ncell = g.jm * g.km;
    const double* xs[2] = {terms + (size_t)lev * 2 * ncell, terms + (size_t)lev * 2 * ncell + ncell};
    const int* E = bexp + 2 * (size_t)lev * nbx;
    const long long* U = bunits + 4 * (size_t)lev * nbx;
    __shared__ int se[2 * TILE];
    __shared__ long long su[4 * TILE];
    // the terms of chunks taken term by term, [chunk parity][chain]: a chunk predicted to need it
    // is copied in (cp.async) while the chunk before it is applied
    __shared__ double stg[2][2][BX_CH];
    RunSum rs{0.0, 0, 0, false}, rw{0.0, 0, 0, false};   // lane 0's
    for(int b0 = 0; b0 < nbx; b0 += TILE){
        const int nt = min(TILE, nbx - b0);
        for(int q = lane; q < 2 * nt; q += 32) se[q] = E[2 * b0 + q];
        for(int q = lane; q < 4 * nt; q += 32) su[q] = U[4 * (size_t)b0 + q];
        __syncwarp();
        int staged = 0;                                // chains whose chunk bt is copied in: bit c
        for(int bt = 0; bt < nt; bt++){
            const int b = b0 + bt;
            const int n = min(BX_CH, ncell - b * BX_CH);
            // copy in the next chunk's terms for each chain predicted to take it term by term
            int next = 0;
            if(bt + 1 < nt){
                const int b1 = b + 1, n1 = min(BX_CH, ncell - b1 * BX_CH);
                for(int c = 0; c < 2; c++){
                    if(se[2 * (bt + 1) + c] != INT_MIN) continue;
                    next |= 1 << c;
                    const double* x = xs[c] + (size_t)b1 * BX_CH;
                    for(int q = lane; q < n1; q += 32) cp_async_n<8>(&stg[b1 & 1][c][q], x + q);
                }
            }
            cp_async_commit();                         // one group per chunk, possibly empty
            int ok = 0;
            if(lane == 0){                             // the two chains' O(1) steps side by side
                const bool okb = chunk_fast(rs, se[2 * bt], su + 4 * bt);
                const bool okw = chunk_fast(rw, se[2 * bt + 1], su + 4 * bt + 2);
                ok = (okb ? 1 : 0) | (okw ? 2 : 0);
            }
            ok = __shfl_sync(0xffffffffu, ok, 0);
            // the chains that failed their O(1) step, term by term (RunSum in double form); the
            // two chains are named, not selected through a reference, so they stay in registers
            auto by_terms = [&](RunSum& r, int c){
                if(!(staged & (1 << c))){               // not predicted: copy now
                    const double* x = xs[c] + (size_t)b * BX_CH;
                    for(int q = lane; q < n; q += 32) stg[b & 1][c][q] = x[q];
                }
                __syncwarp();
                if(lane == 0){
                    const double* t = stg[b & 1][c];
                    double acc = r.s;
#pragma unroll 8
                    for(int q = 0; q < n; q++) acc += t[q];
                    r.s = acc;
                }
                __syncwarp();
            };
            if((ok & 3) != 3) cp_async_wait<1>();     // chunk b's copies (all but the newest group)
            if(!(ok & 1)) by_terms(rs, 0);
            if(!(ok & 2)) by_terms(rw, 1);
            staged = next;
        }
        cp_async_wait<0>();
        __syncwarp();
    }
    if(lane == 0){
        run_to_double(rs); run_to_double(rw);
        ref[lev] = (rw.s > 0.0) ? rs.s / rw.s : 0.0;
    }
}

// ---- RungeKutta_Uran_Turb.cpp:62-177: per column (j, k) -- every column, the seam copy and the
// pole rows included -- the trapezoid integral from the base of the buoyancy anomaly and the
// metric + radial Coriolis force, plus p_baro minus what p_bfollow has taken up of B(t) - B0.
//
// A block owns 32 consecutive columns and walks up i in chunks of HYD_CH levels, in three
// phases per chunk: (1) all 256 threads form the per-cell integrands (the divisions, the loads of
// t, p_stat, v, w) for the chunk's cells into shared memory; (2) one warp, one lane per column,
// runs the two running sums up the chunk in the reference's order (only the dependent adds are
// serial) and leaves the prefix at each level in place; (3) all threads read p_baro, p_b0,
// p_bfollow and write p_bfollow and p_hydro for the chunk. The arithmetic per cell and the
// summation order are the reference's, so the FP64 form stays bit-equal to it. ----
constexpr int HYD_CH = 48;          // levels per chunk (41 levels: one chunk)

// ROWS threads per column in phases 1 and 3 (HYD_CH / ROWS levels each); MINB resident blocks.
template <typename S, int ROWS, int MINB>
__global__ void __launch_bounds__(32 * ROWS, MINB) hydro_kernel(Grid g, const S* __restrict__ t, const S* __restrict__ ps,
                                                    const S* __restrict__ v, const S* __restrict__ w,
                                                    const double* __restrict__ ref, const double* __restrict__ rm_i,
                                                    const double* __restrict__ cor_j, const double* __restrict__ pbaro,
                                                    const double* __restrict__ pb0, double* __restrict__ pbf,
                                                    double* __restrict__ ph, HydroConst h, int advance){
    constexpr int HYD_PER = HYD_CH / ROWS;
    static_assert(HYD_CH % ROWS == 0, "a chunk splits evenly over the rows");
    __shared__ double sm[HYD_CH][32], sb[HYD_CH][32];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int c = blockIdx.x * 32 + tx;
    const bool col = c < g.jm * g.km;
    const int j = col ? c / g.km : 0, k = col ? c - j * g.km : 0;
    const double cor_ = cor_j[j];
    auto buoy = [&](int i, double T, double p) -> double {
        if(!(T > 0.0)) return 0.0;
        const double b = h.g * p / (h.rR * T * h.t_ref) - ref[i];
        const double f = h.m_nd_rel_b * b / ref[i];
        return isfinite(f) ? f : 0.0;
    };
    // running state of the serial lane (phase 2), carried across chunks
    double Pm = 0.0, Pb = 0.0, m_prev = 0.0, b_prev = 0.0;
    for(int i0 = 0; i0 < g.im; i0 += HYD_CH){
        const int n = min(HYD_CH, g.im - i0);
        // phase 1: integrands; every load of the thread's levels first
        if(col){
            S tv[HYD_PER], pv[HYD_PER], vv[HYD_PER], wv[HYD_PER];
#pragma unroll
            for(int q = 0; q < HYD_PER; q++){
                const int r = ty + q * ROWS;
                if(r < n){
                    const size_t o = gidx(g, i0 + r, j, k);
                    tv[q] = __ldg(t + o); pv[q] = __ldg(ps + o); vv[q] = __ldg(v + o); wv[q] = __ldg(w + o);
                }
            }
#pragma unroll
            for(int q = 0; q < HYD_PER; q++){
                const int r = ty + q * ROWS;
                if(r < n){
                    const int i = i0 + r;
                    const double V = (double)vv[q], W = (double)wv[q];
                    if(h.follow_on){
                        sm[r][tx] = (V * V + W * W) / rm_i[i] + cor_ * W;
                        sb[r][tx] = buoy(i, (double)tv[q], (double)pv[q]);
                    } else {
                        // ATURAN_PBARO_FOLLOW=0: f_(i) = buoy(i) + (v^2 + w^2) / rm + cor_ w, :134-161
                        sm[r][tx] = buoy(i, (double)tv[q], (double)pv[q]) + (V * V + W * W) / rm_i[i] + cor_ * W;
                    }
                }
            }
        }
        __syncthreads();
        // phase 2: the running sums, in order, replaced in place by the prefix at each level
        if(ty == 0 && col){
            if(h.follow_on){
                for(int r = 0; r < n; r++){
                    const double m_i = sm[r][tx], b_i = sb[r][tx];
                    if(i0 + r > 0){
                        Pm += 0.5 * (m_prev + m_i) * h.dr;
                        Pb += 0.5 * (b_prev + b_i) * h.dr;
                    }
                    m_prev = m_i; b_prev = b_i;
                    sm[r][tx] = Pm; sb[r][tx] = Pb;
                }
            } else {
                for(int r = 0; r < n; r++){
                    const double f_i = sm[r][tx];
                    if(i0 + r > 0) Pm = Pm + 0.5 * (m_prev + f_i) * h.dr;
                    m_prev = f_i;
                    sm[r][tx] = Pm;
                }
            }
        }
        __syncthreads();
        // phase 3: p_bfollow and p_hydro, loads first
        if(col){
            double bfv[HYD_PER], b0v[HYD_PER], pbv[HYD_PER];
#pragma unroll
            for(int q = 0; q < HYD_PER; q++){
                const int r = ty + q * ROWS;
                if(r < n){
                    const size_t o = gidx(g, i0 + r, j, k);
                    pbv[q] = pbaro[o];
                    if(h.follow_on){ bfv[q] = pbf[o]; if(advance) b0v[q] = pb0[o]; }
                }
            }
#pragma unroll
            for(int q = 0; q < HYD_PER; q++){
                const int r = ty + q * ROWS;
                if(r < n){
                    const size_t o = gidx(g, i0 + r, j, k);
                    if(h.follow_on){
                        const double pm = sm[r][tx], pb = sb[r][tx];
                        double bf = bfv[q];
                        if(advance){ bf += (pb - b0v[q] - bf) / h.follow_tau; pbf[o] = bf; }
                        ph[o] = pm + pb + pbv[q] - bf;
                    } else {
                        ph[o] = sm[r][tx] + pbv[q];
                    }
                }
            }
        }
        __syncthreads();
    }
}

}  // namespace aturan
