// The chemistry of the iteration loop in its equilibrium form (planet/ChemistryUran.h,
// FluxLimiter.h): the NH4SH equilibrium (EquilibriumNH4SH("loop"), cUranusModel.cpp:1034) and the
// chemistry forcing (DiffMassFluxUran, ChemMassRateUran, FluxLimiterNH4SH and the 1-2-1 filters
// between them, cUranusModel.cpp:1074-1087).
//
// The equilibrium is cell-local: one thread per cell brackets the cell's K_p(T) condition and
// bisects it as the reference does, evaluating K_p only at the midpoints near the root that a
// Newton estimate locates (nh4sh_bisect: the reference's midpoints and result). The forcing
// is two 7-point stencil passes over the interior (the diffusive tendencies and the thermal mass
// flux; then the mass rates and the Superbee limiter) with the filters between and after them;
// every pass streams a few planes of the state and is bound by HBM; each filter is one fused pass
// over the three axes (post.cuh, post_filter3_kernel) and a copy back. Arithmetic is FP64 on the
// stored values (FP32 storage in the mixed form is widened, computed in FP64 and rounded back), in
// the reference's operand order; the per-level and per-latitude factors (radius, metric radius,
// sin and cos of the colatitude) come from a host table made with the host's libm, so the FP64
// forcing equals the CPU's bit for bit.
#pragma once
#include "common.cuh"

namespace aturan {

struct ChemConst {
    double t_ref, R_mix, r_mix, cp_mix, L_f;          // equilibrium
    double m_nh3, m_h2s, m_nh4sh;
    double D_nh3, D_h2s, DT_nh3, DT_h2s, D_nh4sh, DT_nh4sh, c_mix;
    double cp_nh3, cp_h2s, cp_nh4sh, k_nh3, k_h2s, k_nh4sh;
    double dr, dthe, dphi, dsign;
    double sinthe_min, floor;                         // the model's polar metric floor; ATPhys's divisor floor
    int per;                                          // the periodic phi seam
};

// Host table made with the host's libm: radius, metric radius (im each), sin and cos of the
// colatitude (jm each).
struct ChemTab {
    const double *rad, *rmm, *sin, *cos;
};

template <typename S>
struct ChemArgs {
    Grid g;
    S *t, *nh3, *h2s, *nh4sh;
    float* tlo;                                       // the mixed form's temperature pair, else null
    const S *u, *v, *w, *ps;
    S *rho_mix, *tmf, *mf_h2s, *mf_nh3, *mf_nh4sh, *fl, *df_h2s, *df_nh3, *df_nh4sh;
    ChemTab tab;
    ChemConst c;
    unsigned long long* counts;                       // [formed, decomposed]
    S* scratch;                                       // one field the fused filters write before the copy back
};

__device__ __forceinline__ double chem_max(double a, double b){ return (a < b) ? b : a; }   // std::max
__device__ __forceinline__ double chem_min(double a, double b){ return (b < a) ? b : a; }   // std::min

// ChemistryUran.h:144 and :154-156: K_p(T) [Pa^2] (Lewis 1969) and the cell's equilibrium condition
// f(x) = (a - x)(b - x)(R* T)^2 - K_p(T), T = T0 + heat x, as the reference evaluates it; and f
// with its derivative in x for the Newton estimate of the root (K_p by exp10 there).
__device__ __forceinline__ double nh4sh_kp(double T){
    const double atm = 101325.0;
    return pow(10.0, 14.82 - 4705.0 / T) * atm * atm;
}
__device__ __forceinline__ double nh4sh_f(double x, double T0, double heat, double a, double b){
    const double T = T0 + heat * x, RT = 8314.46 * T;
    return (a - x) * (b - x) * RT * RT - nh4sh_kp(T);
}
__device__ __forceinline__ double nh4sh_df(double x, double T0, double heat, double a, double b, double& f){
    const double R = 8314.46, T = T0 + heat * x, RT = R * T;
    const double P = (a - x) * (b - x), K = exp10(14.82 - 4705.0 / T) * 101325.0 * 101325.0;
    f = P * RT * RT - K;
    return (2.0 * x - a - b) * RT * RT + P * 2.0 * R * RT * heat - K * 2.302585092994046 * 4705.0 / (T * T) * heat;
}

// The reference's bisection of f on [lo, hi] (f(lo) > 0 >= f(hi); ChemistryUran.h:163-168), with
// the same midpoints and the same result, evaluating f only where its sign is in question. f is
// decreasing on the bracket (the formation heat moves T by millikelvin, against (a-x)(b-x) going
// from ab to 0), so at a midpoint farther than `band` from the root r its sign is that of r - xm;
// r comes from safeguarded Newton (a step that leaves the bracket is replaced by its midpoint),
// and f itself is evaluated, as the reference does, at the ~4 midpoints inside the band instead
// of at all ~50. The final bracket is checked with f at both ends; a bracket that does not hold
// (no single root, or Newton astray) is bisected again with f at every midpoint.
__device__ __forceinline__ void nh4sh_bisect(double& lo, double& hi, double stop, double T0, double heat,
                                             double a, double b, double x0){
    const double lo0 = lo, hi0 = hi;
    // Newton estimate of the root
    double r = (x0 > lo && x0 < hi) ? x0 : 0.5 * (lo + hi);
    {
        double l = lo, h = hi;
        for(int it = 0; it < 60; it++){
            double f;
            const double d = nh4sh_df(r, T0, heat, a, b, f);
            if(f > 0.0) l = r; else h = r;
            double rn = (d != 0.0 && isfinite(d)) ? r - f / d : 0.5 * (l + h);
            if(!(rn > l && rn < h)) rn = 0.5 * (l + h);
            const bool done = fabs(rn - r) <= 1.0e-3 * stop || h - l <= 1.0e-3 * stop;
            r = rn;
            if(done) break;
        }
    }
    // Newton leaves r within 1e-3 stop of the root; the computed sign of f is unreliable only within
    // rounding of it (relative ~1e-16 of the bracket, stop being 1e-15 of it), so 8 stop is ample
    const double band = 8.0 * stop;
    // whether the sign of f at each end was evaluated (the initial ends' signs are the caller's
    // tests: f(lo) > 0, and f(hi) <= 0 at x = 0 or x = min(a, b), where f = -K_p) or inferred
    bool lo_ev = true, hi_ev = true;
    for(int it = 0; it < 80; it++){
        const double xm = 0.5 * (lo + hi);
        bool pos, ev = false;
        if(xm < r - band) pos = true;
        else if(xm > r + band) pos = false;
        else { pos = nh4sh_f(xm, T0, heat, a, b) > 0.0; ev = true; }
        if(pos){ lo = xm; lo_ev = ev; } else { hi = xm; hi_ev = ev; }
        if(hi - lo <= stop) break;
    }
    // the final bracket holds if f changes sign over it: only the inferred ends are evaluated
    if(hi > lo && (lo_ev || nh4sh_f(lo, T0, heat, a, b) > 0.0) && (hi_ev || !(nh4sh_f(hi, T0, heat, a, b) > 0.0))) return;
    if(!(hi > lo)) return;
    lo = lo0; hi = hi0;                                       // the plain bisection
    for(int it = 0; it < 80; it++){
        const double xm = 0.5 * (lo + hi);
        if(nh4sh_f(xm, T0, heat, a, b) > 0.0) lo = xm; else hi = xm;
        if(hi - lo <= stop) break;
    }
}

// ChemistryUran.h:140-177 per cell, :210-275 over every cell; counts formed / decomposed cells.
template <typename S>
__global__ void __launch_bounds__(128) nh4sh_eq_kernel(ChemArgs<S> a){
    const Grid& g = a.g;
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, i = blockIdx.z;
    int formed = 0, decomposed = 0;
    if(k < g.km){
        const ChemConst& c = a.c;
        const size_t q = gidx(g, i, j, k);
        const double T0 = t_ld(a.t, a.tlo, q) * c.t_ref;
        if(T0 > 0.0){
            double rho = (double)a.ps[q] * 1e5 / (c.R_mix * T0);
            if(!(rho > 0.0) || !isfinite(rho)) rho = c.r_mix;
            const double n3 = (double)a.nh3[q], hs = (double)a.h2s[q], ns = (double)a.nh4sh[q];
            const double A = chem_max(0.0, n3) / c.m_nh3;
            const double B = chem_max(0.0, hs) / c.m_h2s;
            const double Sx = chem_max(0.0, ns) / c.m_nh4sh;
            const double heat = c.L_f * c.m_nh4sh / (c.cp_mix * rho);
            const double f0 = nh4sh_f(0.0, T0, heat, A, B);
            double lo = 0.0, hi = 0.0, x0 = 0.0;
            bool go = true;
            if(f0 > 0.0){
                lo = 0.0; hi = chem_min(A, B);
                // the fixed-T root (ChemistryUran.h:199-208's cancellation-free form) starts Newton
                const double RT = 8314.46 * T0;
                const double K = nh4sh_kp(T0) / (RT * RT), d = A - B;
                x0 = (A * B > K) ? 2.0 * (A * B - K) / ((A + B) + sqrt(d * d + 4.0 * K)) : 0.0;
            } else if(Sx > 0.0){
                if(nh4sh_f(-Sx, T0, heat, A, B) <= 0.0){ lo = hi = -Sx; }
                else { lo = -Sx; hi = 0.0; x0 = -0.5 * Sx; }
            } else go = false;
            if(go){
                if(hi > lo) nh4sh_bisect(lo, hi, 1.0e-15 * chem_max(A, chem_max(B, Sx)), T0, heat, A, B, x0);
                const double x = (f0 > 0.0) ? lo : hi;
                if(x != 0.0){
                    a.nh3[q] = (S)chem_max(0.0, n3 - c.m_nh3 * x);
                    a.h2s[q] = (S)chem_max(0.0, hs - c.m_h2s * x);
                    a.nh4sh[q] = (S)chem_max(0.0, ns + c.m_nh4sh * x);
                    const double dT = heat * x;
                    t_st(a.t, a.tlo, q, (T0 + dT) / c.t_ref);
                    if(x > 0.0) formed = 1; else decomposed = 1;
                }
            }
        }
    }
    // counts: a warp sum, one atomic per warp
    formed = __reduce_add_sync(0xffffffffu, formed);
    decomposed = __reduce_add_sync(0xffffffffu, decomposed);
    if((threadIdx.x & 31) == 0 && (formed | decomposed)){
        if(formed) atomicAdd(a.counts, (unsigned long long)formed);
        if(decomposed) atomicAdd(a.counts + 1, (unsigned long long)decomposed);
    }
}

// The phi neighbours' offsets k-1 and k+1 of k in a row: round the ring of km-1 meridians with the
// periodic seam, else the plain neighbours (k runs over 1..km-2 then).
__device__ __forceinline__ void chem_kn(int k, int km, int per, int& dkw, int& dke){
    dkw = per ? k - phi_wrap(k - 1, km) : 1;
    dke = per ? phi_wrap(k + 1, km) - k : 1;
}

// The seven values of x around a cell, in FP64: centre, r, theta and phi neighbours.
struct Chem7 { double c, ip, im, jp, jm, kp, km; };
template <typename S>
__device__ __forceinline__ Chem7 chem_ld7(const S* x, size_t q, size_t pl, size_t kp, int dkw, int dke){
    Chem7 v;
    v.c = (double)x[q];
    v.ip = (double)x[q + pl]; v.im = (double)x[q - pl];
    v.jp = (double)x[q + kp]; v.jm = (double)x[q - kp];
    v.kp = (double)x[q + dke]; v.km = (double)x[q - dkw];
    return v;
}
// ChemistryUran.h:601-686 without SeaMount cells: the central first differences at the cell
__device__ __forceinline__ void chem_d1v(const Chem7& x, const ChemConst& c, double& dr_, double& dt_, double& dp_){
    dr_ = (x.ip - x.im) / (2.0 * c.dr);
    dt_ = (x.jp - x.jm) / (2.0 * c.dthe);
    dp_ = (x.kp - x.km) / (2.0 * c.dphi);
}
// ChemistryUran.h:576-598 (exp_rm = 1: coord_stretching is false)
__device__ __forceinline__ double chem_lapv(const Chem7& x, double rm, double rmsinthe, double costhe, const ChemConst& c){
    const double exp_rm = 1.0, exp_2_rm = exp_rm * exp_rm;
    const double v = x.c;
    const double d2cdr2 = (x.ip - 2.0 * v + x.im) / (c.dr * c.dr) * exp_2_rm;
    const double d2cdthe2 = (x.jp - 2.0 * v + x.jm) / (c.dthe * c.dthe);
    const double d2cdphi2 = (x.kp - 2.0 * v + x.km) / (c.dphi * c.dphi);
    const double dcdr = (x.ip - x.im) / (2.0 * c.dr) * exp_rm;
    const double dcdthe = (x.jp - x.jm) / (2.0 * c.dthe);
    return d2cdr2 + 2.0 / rm * dcdr + d2cdthe2 / (rm * rm) + costhe / (rm * rmsinthe) * dcdthe
         + d2cdphi2 / (rmsinthe * rmsinthe);
}

// rho_mix on every cell (ChemistryUran.h:312-320); on the interior the thermal mass flux and the
// diffusive tendencies difflux_x = D_x lap(c_x) (passes 1 and 2, ChemistryUran.h:322-419, with
// j_* formed at the cell where pass 2 reads them). Every load of a cell comes before its first
// store (a store could alias a later load as far as the compiler knows).
template <typename S>
__global__ void __launch_bounds__(128) chem_diff_kernel(ChemArgs<S> a){
    const Grid& g = a.g;
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, i = blockIdx.z;
    if(k >= g.km) return;
    const ChemConst& c = a.c;
    const size_t q = gidx(g, i, j, k);
    const double t0 = t_ld(a.t, a.tlo, q);
    const double rho = (double)a.ps[q] * 1e5 / (c.R_mix * t0 * c.t_ref);
    const int k_first = c.per ? 0 : 1;
    if(i < 1 || i > g.im - 2 || j < 1 || j > g.jm - 2 || k < k_first || k > g.km - 2){
        a.rho_mix[q] = (S)rho;
        return;
    }
    const size_t pl = (size_t)g.jm * g.kp, kp = (size_t)g.kp;
    int dkw, dke;
    chem_kn(k, g.km, c.per, dkw, dke);
    Chem7 T;
    if(a.tlo){
        T.c = t0;
        T.ip = t_ld(a.t, a.tlo, q + pl); T.im = t_ld(a.t, a.tlo, q - pl);
        T.jp = t_ld(a.t, a.tlo, q + kp); T.jm = t_ld(a.t, a.tlo, q - kp);
        T.kp = t_ld(a.t, a.tlo, q + dke); T.km = t_ld(a.t, a.tlo, q - dkw);
    } else T = chem_ld7(a.t, q, pl, kp, dkw, dke);
    const Chem7 H = chem_ld7(a.h2s, q, pl, kp, dkw, dke);
    const Chem7 N = chem_ld7(a.nh3, q, pl, kp, dkw, dke);
    const Chem7 X = chem_ld7(a.nh4sh, q, pl, kp, dkw, dke);
    // pass 1's metric: the raw radius and max(sinthe_min, |sin|)
    const double rm = a.tab.rad[i];
    const double rmsinthe = rm * chem_max(c.sinthe_min, fabs(a.tab.sin[j]));
    double dtdr, dtdthe, dtdphi;
    chem_d1v(T, c, dtdr, dtdthe, dtdphi);
    double hr, ht, hp, nr, nt, np, sr, stt, sp;
    chem_d1v(H, c, hr, ht, hp);
    chem_d1v(N, c, nr, nt, np);
    chem_d1v(X, c, sr, stt, sp);
    const double jT_nh3 = c.DT_nh3 / t0 * dtdr;
    const double jT_h2s = c.DT_h2s / t0 * dtdr;
    const double jT_nh4sh = c.DT_nh4sh / t0 * dtdr;
    const double d_nh3 = nr + fabs(nt) / rm + np / rmsinthe;
    const double d_h2s = hr + fabs(ht) / rm + hp / rmsinthe;
    const double d_nh4sh = sr + fabs(stt) / rm + sp / rmsinthe;
    const double j_nh3 = c.c_mix / c.r_mix * (c.m_nh3 * c.D_nh3 * d_nh3 - jT_nh3);
    const double j_h2s = c.c_mix / c.r_mix * (c.m_h2s * c.D_h2s * d_h2s - jT_h2s);
    const double j_nh4sh = c.c_mix / c.r_mix * (c.m_nh4sh * c.D_nh4sh * d_nh4sh - jT_nh4sh);
    const double w0 = 0.0;                            // w_nh3, w_h2s, w_nh4sh in the equilibrium form
    const double tmf = (j_nh3 * c.cp_nh3 + j_h2s * c.cp_h2s + j_nh4sh * c.cp_nh4sh)
                       * (dtdr + fabs(dtdthe) / rm + dtdphi / rmsinthe)
                       + t0 * (w0 * c.k_nh3 + w0 * c.k_h2s + w0 * c.k_nh4sh);
    // the Laplacian's metric: the metric radius and max(sin, floor)
    const double rml = a.tab.rmm[i];
    const double rmsl = rml * chem_max(a.tab.sin[j], c.floor);
    const double cl = a.tab.cos[j];
    const double dfh = c.D_h2s * chem_lapv(H, rml, rmsl, cl, c);
    const double dfn = c.D_nh3 * chem_lapv(N, rml, rmsl, cl, c);
    const double dfx = c.D_nh4sh * chem_lapv(X, rml, rmsl, cl, c);
    a.rho_mix[q] = (S)rho;
    a.tmf[q] = (S)tmf;
    a.df_h2s[q] = (S)dfh;
    a.df_nh3[q] = (S)dfn;
    a.df_nh4sh[q] = (S)dfx;
}

// FluxLimiter.h:68-70
__device__ __forceinline__ double chem_superbee(double r){
    return chem_max(0.0, chem_max(chem_min(2.0 * r, 1.0), chem_min(r, 2.0)));
}

// On the interior: massflux_x = w_x + sign difflux_x with w_x = 0 (ChemistryUran.h:38-110) and
// the Superbee correction fluxlim_nh4sh (FluxLimiter.h:89-186).
template <typename S>
__global__ void __launch_bounds__(128) chem_limit_kernel(ChemArgs<S> a){
    const Grid& g = a.g;
    const ChemConst& c = a.c;
    const int k_first = c.per ? 0 : 1;
    const int k = k_first + blockIdx.x * blockDim.x + threadIdx.x, j = 1 + blockIdx.y, i = 1 + blockIdx.z;
    if(k > g.km - 2) return;
    const size_t o = gidx(g, i, j, k), pl = (size_t)g.jm * g.kp, kp = (size_t)g.kp;
    // every load of the cell before its first store (a store could alias a later load as far as
    // the compiler knows); the far upwind values loaded whether or not the flow's sign reads them
    const double dh = (double)a.df_h2s[o], dn = (double)a.df_nh3[o], dx = (double)a.df_nh4sh[o];
    const S* x = a.nh4sh;
    int dkw, dke;
    chem_kn(k, g.km, c.per, dkw, dke);
    const double q = (double)x[o], q_rp = (double)x[o + pl], q_rm = (double)x[o - pl];
    const double q_tp = (double)x[o + kp], q_tm = (double)x[o - kp];
    const double q_pp = (double)x[o + dke], q_pm = (double)x[o - dkw];
    const double uu = (double)a.u[o], vv = (double)a.v[o], ww = (double)a.w[o];
    const double x_r2 = (i + 2 < g.im) ? (double)x[o + 2 * pl] : q_rp;
    const double x_t2 = (j + 2 < g.jm) ? (double)x[o + 2 * kp] : (C43 * q_tp - C13 * q);
    const double x_p2 = c.per ? (double)x[o - k + phi_wrap(k + 2, g.km)] : ((k + 2 < g.km) ? (double)x[o + 2] : q_pp);
    const double rm = a.tab.rmm[i];
    const double sinthe = chem_max(c.floor, fabs(a.tab.sin[j]));
    const double inv_rm = 1.0 / rm, inv_rmsinthe = 1.0 / (rm * sinthe);
    const double eps = 1.0e-12;
    double corr = 0.0;
    {
        const double df = q_rp - q, db = q - q_rm;
        const double denom = df + (df >= 0.0 ? eps : -eps);
        const double r = (uu >= 0.0) ? db / denom : (x_r2 - q_rp) / denom;
        corr += (1.0 - chem_superbee(r)) * fabs(uu) * (df - db) / (2.0 * c.dr);
    }
    {
        const double df = q_tp - q, db = q - q_tm;
        const double denom = df + (df >= 0.0 ? eps : -eps);
        const double r = (vv >= 0.0) ? db / denom : (x_t2 - q_tp) / denom;
        corr += (1.0 - chem_superbee(r)) * fabs(vv) * inv_rm * (df - db) / (2.0 * c.dthe);
    }
    {
        const double df = q_pp - q, db = q - q_pm;
        const double denom = df + (df >= 0.0 ? eps : -eps);
        const double r = (ww >= 0.0) ? db / denom : (x_p2 - q_pp) / denom;
        corr += (1.0 - chem_superbee(r)) * fabs(ww) * inv_rmsinthe * (df - db) / (2.0 * c.dphi);
    }
    a.mf_h2s[o] = (S)(0.0 + c.dsign * dh);
    a.mf_nh3[o] = (S)(0.0 + c.dsign * dn);
    a.mf_nh4sh[o] = (S)(0.0 + c.dsign * dx);
    a.fl[o] = (S)corr;
}

}  // namespace aturan
