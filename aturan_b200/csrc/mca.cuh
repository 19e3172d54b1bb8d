// The moist convective adjustment (planet/ConvectiveAdjustment.h:402-849,
// MoistConvectiveAdjustment<cUranusModel>::run) with the reference's default knobs: Ledoux test
// with condensate loading, relaxation 1, no latitude smoothing (cUranusModel.h:572), at most 64
// sweeps, no phase split (SATADJ_BERGERON = 2), interior levels only (cUranusModel.h:566); the gas
// list H2O, NH3, H2S (its liquid set for both phases), CH4 and the NH4SH tracer of
// cUranusModel.cpp:1276-1290.
//
// Every (j, k) column is independent: one thread per column, FP64, the column's state (at most
// MCA_MAXI levels) in the thread's local memory. Every loop is bounded: 60 regula-falsi steps,
// 30 Newton steps of the enthalpy inverse, 64 sweeps, and a segment grows by one level per step
// within the column.
#pragma once
#include "common.cuh"

namespace aturan {

constexpr int MCA_MAXI = 64, MCA_NG = 4;
constexpr double CP_T_LO_D = 5.0, CP_T_HI_D = 1500.0, CP_DT_D = 0.5;   // CpH2.h:13

struct McaGas { double ep, lv, ls, t_0, C, L0, R, del_alf, del_bet, C_i, L0_i, del_alf_i, del_bet_i; };

struct McaArgs {
    Grid g;
    McaGas G[MCA_NG];                // H2O, NH3, H2S, CH4
    double L_tr, t_ref, grav, cp_mix, r_mix, cp_h2, r_h2, r_he, r_ch4, cp_he, cp_ch4;
    float hz;                        // level spacing [km] as the model stores it (float)
    int cp_dyn, cp_mode, cp_gas, local_rho;
    const double *cp_tab, *H_tab;    // H2 cp table and its running integral (CpH2.h:66-75)
    double* t;
    double* sp[MCA_NG][3];           // vapour, cloud, ice
    double* nh4sh;
    const double *ps, *rho;
};

__device__ __forceinline__ double mca_mx(double a, double b){ return (a < b) ? b : a; }   // std::max

// CpH2.h:88-101, 122-157
static __device__ double mca_cp_h2(const McaArgs& A, double T){
    if(A.cp_mode <= 0) return A.cp_h2;
    const double Tc = T < CP_T_LO_D ? CP_T_LO_D : T;
    const double x = ((Tc > CP_T_HI_D ? CP_T_HI_D : Tc) - CP_T_LO_D) / CP_DT_D;
    int i = (int)x; if(i > CP_TABLE_N - 2) i = CP_TABLE_N - 2;
    const double f = x - i;
    return A.cp_tab[i] + f * (A.cp_tab[i + 1] - A.cp_tab[i]);
}
static __device__ double mca_enth_h2(const McaArgs& A, double T){
    if(A.cp_mode <= 0) return A.cp_h2 * T;
    const int n = CP_TABLE_N;
    if(T <= CP_T_LO_D) return A.cp_tab[0] * T;
    if(T >= CP_T_HI_D) return A.H_tab[n - 1] + A.cp_tab[n - 1] * (T - CP_T_HI_D);
    const double x = (T - CP_T_LO_D) / CP_DT_D;
    int i = (int)x; if(i > n - 2) i = n - 2;
    const double f = x - i;
    return A.H_tab[i] + CP_DT_D * f * (A.cp_tab[i] + 0.5 * f * (A.cp_tab[i + 1] - A.cp_tab[i]));
}
static __device__ double mca_cp(const McaArgs& A, double T){
    if(!A.cp_dyn) return A.cp_mix;
    const double ch = mca_cp_h2(A, T);
    if(A.cp_gas) return (A.r_h2 * ch + A.r_he * A.cp_he + A.r_ch4 * A.cp_ch4) / (A.r_h2 + A.r_he + A.r_ch4);
    return A.cp_mix + (A.r_h2 / A.r_mix) * (ch - A.cp_h2);
}
static __device__ double mca_enth(const McaArgs& A, double T){
    if(!A.cp_dyn) return A.cp_mix * T;
    const double hh = mca_enth_h2(A, T);
    if(A.cp_gas) return (A.r_h2 * hh + (A.r_he * A.cp_he + A.r_ch4 * A.cp_ch4) * T) / (A.r_h2 + A.r_he + A.r_ch4);
    return (A.cp_mix - (A.r_h2 / A.r_mix) * A.cp_h2) * T + (A.r_h2 / A.r_mix) * hh;
}
static __device__ double mca_enth_inv(const McaArgs& A, double h, double T0){
    if(!A.cp_dyn) return h / A.cp_mix;
    double T = (T0 > 0.0) ? T0 : h / A.cp_mix;
    for(int it = 0; it < 30; it++){
        const double f = mca_enth(A, T) - h, c = mca_cp(A, T);
        const double dT = f / c;
        T -= dT; if(T < 1.0) T = 1.0;
        if(fabs(dT) < 1.0e-10 * T) break;
    }
    return T;
}

// ATPhys.h:49-53 (the saturation pressure) and ConvectiveAdjustment.h:437-453 without the phase split
__device__ __forceinline__ double mca_qsat(const McaGas& s, double T, double pr){
    const double E = (T >= s.t_0) ? exp(s.C + (-s.L0 / T + s.del_alf * log(T) + s.del_bet * T) / (1e-3 * s.R))
                                  : exp(s.C_i + (-s.L0_i / T + s.del_alf_i * log(T) + s.del_bet_i * T) / (1e-3 * s.R));
    const double q = s.ep * E / pr;
    return isfinite(q) ? q : 0.0;
}
__device__ __forceinline__ double mca_lat(const McaGas& s, double T){ return T >= s.t_0 ? s.lv : s.ls; }

static __device__ double mca_fof(const McaArgs& A, double TT, double hL, const double* qt, double pr, double z){
    double f = mca_enth(A, TT) + A.grav * z - hL;
    for(int g = 0; g < MCA_NG; g++) f -= mca_lat(A.G[g], TT) * mca_mx(0.0, qt[g] - mca_qsat(A.G[g], TT, pr));
    return f;
}

// :455-488, the equilibrium of (hL, qt) at (p, z): Illinois regula falsi on the energy balance
static __device__ bool mca_equil(const McaArgs& A, double hL, const double* qt, double pr, double z, double& T, double* cond){
    const double cp = A.cp_mix, tol_T = 1.0e-10;
    const double T_lo = A.cp_dyn ? mca_enth_inv(A, hL - A.grav * z, 0.0) : (hL - A.grav * z) / cp;
    if(!(T_lo > 0.0) || !(pr > 0.0)) return false;
    bool any = false;
    for(int g = 0; g < MCA_NG; g++) if(qt[g] > mca_qsat(A.G[g], T_lo, pr)){ any = true; break; }
    if(!any){ T = T_lo; for(int g = 0; g < MCA_NG; g++) cond[g] = 0.0; return true; }
    double span = 0.0;
    for(int g = 0; g < MCA_NG; g++) span += mca_mx(A.G[g].lv, A.G[g].ls) * mca_mx(0.0, qt[g]);
    double a = T_lo, b = A.cp_dyn ? mca_enth_inv(A, mca_enth(A, T_lo) + span, T_lo) + 1.0e-9 : T_lo + span / cp + 1.0e-9;
    double fa = mca_fof(A, a, hL, qt, pr, z), fb = mca_fof(A, b, hL, qt, pr, z);
    int side = 0;
    for(int it = 0; it < 60 && b - a > tol_T; it++){
        double c = (fb - fa != 0.0) ? b - fb * (b - a) / (fb - fa) : 0.5 * (a + b);
        if(!(c > a && c < b)) c = 0.5 * (a + b);
        const double fc = mca_fof(A, c, hL, qt, pr, z);
        if(fc < 0.0){ a = c; fa = fc; if(side == -1) fb *= 0.5; side = -1; }
        else        { b = c; fb = fc; if(side == +1) fa *= 0.5; side = +1; }
        if(fabs(fc) <= cp * tol_T){ a = b = c; break; }
    }
    T = b;
    for(int g = 0; g < MCA_NG; g++) cond[g] = mca_mx(0.0, qt[g] - mca_qsat(A.G[g], T, pr));
    return true;
}

// One column's state (levels i0..i1 used).
struct McaCol {
    double T[MCA_MAXI], p[MCA_MAXI], z[MCA_MAXI], rho[MCA_MAXI], w[MCA_MAXI], hL[MCA_MAXI], qr[MCA_MAXI], Teq[MCA_MAXI];
    double qt[MCA_MAXI * MCA_NG], qv[MCA_MAXI * MCA_NG], qc[MCA_MAXI * MCA_NG], qi[MCA_MAXI * MCA_NG], ceq[MCA_MAXI * MCA_NG];
    bool touched[MCA_MAXI], eq_ok[MCA_MAXI], cen_u[MCA_MAXI], cen_m[MCA_MAXI];
};

__device__ __forceinline__ double mca_trE(const McaArgs& A, const McaCol& C, int i){ double e = 0.0; e += A.L_tr * C.qr[i]; return e; }

// :613-624, Ledoux virtual temperature with condensate loading; NH4SH is a condensed tracer
static __device__ double mca_tv(const McaArgs& A, const McaCol& C, double TT, const double* v_, const double* cnd, int i_tr){
    double f = 1.0;
    for(int g = 0; g < MCA_NG; g++){ f += v_[g] * (1.0 / A.G[g].ep - 1.0); f -= cnd[g]; }
    f -= C.qr[i_tr];
    return TT * f;
}

// :627-644
static __device__ bool mca_unstable(const McaArgs& A, McaCol& C, int a, int b, bool* held, bool* moist){
    const double tol_K = 1.0e-7;
    double Tp, pc[MCA_NG], pv[MCA_NG], ec[MCA_NG], ev[MCA_NG];
    if(!mca_equil(A, C.hL[a] + mca_trE(A, C, a), &C.qt[a * MCA_NG], C.p[b], C.z[b], Tp, pc)) return false;
    if(!C.eq_ok[b]){
        if(!mca_equil(A, C.hL[b] + mca_trE(A, C, b), &C.qt[b * MCA_NG], C.p[b], C.z[b], C.Teq[b], &C.ceq[b * MCA_NG])) return false;
        C.eq_ok[b] = true;
    }
    const double Tb = C.Teq[b];
    for(int g = 0; g < MCA_NG; g++) ec[g] = C.ceq[b * MCA_NG + g];
    bool wet = false;
    for(int g = 0; g < MCA_NG; g++){ pv[g] = C.qt[a * MCA_NG + g] - pc[g]; if(pc[g] > 0.0) wet = true; ev[g] = C.qt[b * MCA_NG + g] - ec[g]; }
    const double dTv = mca_tv(A, C, Tp, pv, pc, a) - mca_tv(A, C, Tb, ev, ec, b);
    if(held) *held = (Tp - Tb > tol_K) && !(dTv > tol_K);
    if(moist) *moist = wet;
    return dTv > tol_K;
}

// :645-661, cell q to equilibrium from hL / qt
static __device__ bool mca_settle(const McaArgs& A, McaCol& C, int q){
    double TT, pc[MCA_NG];
    if(!mca_equil(A, C.hL[q] + mca_trE(A, C, q), &C.qt[q * MCA_NG], C.p[q], C.z[q], TT, pc)) return false;
    C.T[q] = TT;
    C.Teq[q] = TT; C.eq_ok[q] = true;
    for(int g = 0; g < MCA_NG; g++){
        const int x = q * MCA_NG + g;
        C.ceq[x] = pc[g];
        C.qv[x] = C.qt[x] - pc[g];
        if(TT >= A.G[g].t_0){ C.qc[x] = pc[g]; C.qi[x] = 0.0; } else { C.qi[x] = pc[g]; C.qc[x] = 0.0; }
    }
    C.touched[q] = true;
    return true;
}

// One thread per (j, k) column, k over all km stored meridians as the reference loops.
static __global__ void __launch_bounds__(64) mca_kernel(const McaArgs A){
    const Grid& g = A.g;
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if(k >= g.km) return;
    const int im = g.im, i0 = 1, i1 = im - 2;
    if(i1 - i0 < 1) return;
    McaCol C;
    bool ok = true;
    for(int i = i0; i <= i1 && ok; i++){
        const size_t o = gidx(g, i, j, k);
        C.T[i] = A.t[o] * A.t_ref;
        C.p[i] = A.ps[o];
        C.z[i] = (double)((float)i * A.hz) * 1.0e3;
        double rr = A.r_mix;                                // rho_at, cUranusModel.h:526-531
        if(A.local_rho){ const double r_ = A.rho[o]; rr = (r_ > 0.0 && isfinite(r_)) ? r_ : A.r_mix; }
        C.rho[i] = rr;
        if(!(C.T[i] > 0.0) || !(C.p[i] > 0.0) || !(C.rho[i] > 0.0) || !isfinite(C.T[i] + C.p[i] + C.rho[i])) ok = false;
    }
    if(!ok) return;
    for(int i = i0; i <= i1 && ok; i++){
        const size_t o = gidx(g, i, j, k);
        const double lo = (i > i0) ? 0.5 * (C.z[i - 1] + C.z[i]) : C.z[i0];
        const double hi = (i < i1) ? 0.5 * (C.z[i] + C.z[i + 1]) : C.z[i1];
        C.w[i] = C.rho[i] * (hi - lo);
        if(!(C.w[i] > 0.0)) ok = false;
        double h = mca_enth(A, C.T[i]) + A.grav * C.z[i];
        for(int q = 0; q < MCA_NG; q++){
            const int x = i * MCA_NG + q;
            C.qv[x] = mca_mx(0.0, A.sp[q][0][o]) / C.rho[i];
            C.qc[x] = mca_mx(0.0, A.sp[q][1][o]) / C.rho[i];
            C.qi[x] = mca_mx(0.0, A.sp[q][2][o]) / C.rho[i];
            C.qt[x] = C.qv[x] + C.qc[x] + C.qi[x];
            h -= A.G[q].lv * C.qc[x] + A.G[q].ls * C.qi[x];
        }
        C.qr[i] = A.nh4sh[o] / C.rho[i];
        h -= A.L_tr * C.qr[i];
        C.hL[i] = h;
    }
    if(!ok) return;
    for(int i = 0; i < im; i++){ C.touched[i] = false; C.eq_ok[i] = false; }
    for(int i = i0; i < i1; i++){
        bool held = false, moist = false;
        C.cen_u[i] = mca_unstable(A, C, i, i + 1, &held, &moist);
        C.cen_m[i] = moist;
    }
    int passes = 0;
    bool changed = true, fail = false;
    long layers = 0;
    while(changed && passes < 64 && !fail){
        changed = false; passes++;
        int i = i0;
        while(i < i1 && !fail){
            bool moist = false, uns;
            if(passes == 1 && !C.touched[i] && !C.touched[i + 1]){ uns = C.cen_u[i]; moist = C.cen_m[i]; }
            else uns = mca_unstable(A, C, i, i + 1, nullptr, &moist);
            if(!uns){ i++; continue; }
            int a = i, b = i + 1;
            for(;;){
                double sw = 0.0, sh = 0.0, sq[MCA_NG] = {0.0, 0.0, 0.0, 0.0}, sr = 0.0;
                for(int q = a; q <= b; q++){
                    sw += C.w[q]; sh += C.w[q] * C.hL[q];
                    for(int s = 0; s < MCA_NG; s++) sq[s] += C.w[q] * C.qt[q * MCA_NG + s];
                    sr += C.w[q] * C.qr[q];
                }
                for(int q = a; q <= b; q++){
                    C.hL[q] = sh / sw;
                    for(int s = 0; s < MCA_NG; s++) C.qt[q * MCA_NG + s] = sq[s] / sw;
                    C.qr[q] = sr / sw;
                    if(!mca_settle(A, C, q)){ fail = true; break; }
                }
                if(fail) break;
                bool ext = false;
                if(a > i0 && mca_unstable(A, C, a - 1, a, nullptr, nullptr)){ a--; ext = true; }
                if(b < i1 && mca_unstable(A, C, b, b + 1, nullptr, nullptr)){ b++; ext = true; }
                if(!ext) break;
            }
            layers += b - a + 1;
            changed = true;
            i = b;
        }
    }
    if(fail || layers == 0) return;                        // nothing written: the column keeps its state
    for(int q = i0; q <= i1; q++){
        if(!C.touched[q]) continue;
        const size_t o = gidx(g, q, j, k);
        A.t[o] = C.T[q] / A.t_ref;
        for(int s = 0; s < MCA_NG; s++){
            const int x = q * MCA_NG + s;
            A.sp[s][0][o] = C.qv[x] * C.rho[q];
            A.sp[s][1][o] = C.qc[x] * C.rho[q];
            A.sp[s][2][o] = C.qi[x] * C.rho[q];
        }
        A.nh4sh[o] = C.qr[q] * C.rho[q];
    }
}

// CpH2.h:66-75: the running integral of the cp table, in the table's order (one thread).
static __global__ void mca_H_kernel(const double* cp, double* H){
    if(threadIdx.x != 0 || blockIdx.x != 0) return;
    H[0] = cp[0] * CP_T_LO_D;
    for(int i = 1; i < CP_TABLE_N; i++) H[i] = H[i - 1] + 0.5 * CP_DT_D * (cp[i] + cp[i - 1]);
}

}  // namespace aturan
