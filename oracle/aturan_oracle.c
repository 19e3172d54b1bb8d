/*
 * CPU ORACLE for the aturan_b200 hot path — TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.
 * See aturan_oracle.h for what it is, who may call it and how its parity is pinned.
 *
 * Each function restates one reference routine; the citation in front of it names the
 * reference file and lines it follows, by the file's path within the reference project. The
 * expressions keep the reference's operand order (including its association order) because the
 * point of this file is bit equality with the compiled reference; the knobs are the resolved
 * values carried in aturan_params instead of the reference's environment reads.
 */
#include "aturan_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846   /* the value glibc math.h gives M_PI */
#endif
#define IDX(i, j, k) (((size_t)(i) * jm + (j)) * km + (k))
#define NPROG ATURAN_NPROG

static const double C43 = 4.0 / 3.0, C13 = 1.0 / 3.0;   /* cUranusModel.h:866 */

/* std::max(a, b) of <algorithm>: (a < b) ? b : a, NaN handling included. */
static double stdmax(double a, double b){ return (a < b) ? b : a; }

void oracle_set_threads(int n){
#ifdef _OPENMP
    if(n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* lib/Array_1D.cpp:50-60 (Coordinates: a running sum, not i*dz) with the model's r0 = 1,
 * dr = 0.025, the0 = 0, dthe = 1 deg (cUranusModel.cpp:336-372). */
void oracle_coords(const aturan_params* p, double* rad_z, double* the_z){
    rad_z[0] = p->r0;
    for(int l = 1; l < p->im; l++) rad_z[l] = rad_z[l-1] + p->dr;
    the_z[0] = p->the0;
    for(int l = 1; l < p->jm; l++) the_z[l] = the_z[l-1] + p->dthe;
}

/* cUranusModel.h:641-647 */
static double metric_radius(const aturan_params* p, double rm){
    const double R_km = p->metric_R_km;
    if(!(R_km > 0.0)) return rm;
    return rm + (R_km / p->L_atm - 1.0);
}

/* ---- cp(T) of the gas, CpH2.h:43-134 ---- */
#define CP_R_GAS 8.314462618
#define CP_M_H2  2.01588e-3
#define CP_TH_R  87.57
#define CP_TH_V  6332.0
#define CP_T_LO  5.0
#define CP_T_HI  1500.0
#define CP_DT    0.5

/* CpH2.h:43-64 */
static void cp_moments(double T, int J0, double wgt, double* Z, double* E1, double* E2){
    for(int J = J0; J < 60; J += 2){
        const double e = CP_TH_R * J * (J + 1.0), b = wgt * (2.0 * J + 1.0) * exp(-e / T);
        *Z += b; *E1 += b * e; *E2 += b * e * e;
    }
}
static double cp_crot(double T, double Z, double E1, double E2){
    const double m1 = E1 / Z, m2 = E2 / Z;
    return (m2 - m1 * m1) / (T * T);
}
static double cpR_exact(double T, int mode){
    double c;
    if(mode == 1){
        double Zp = 0, Ep = 0, Fp = 0, Zo = 0, Eo = 0, Fo = 0;
        cp_moments(T, 0, 1.0, &Zp, &Ep, &Fp); cp_moments(T, 1, 1.0, &Zo, &Eo, &Fo);
        c = 0.25 * cp_crot(T, Zp, Ep, Fp) + 0.75 * cp_crot(T, Zo, Eo, Fo);
    } else {
        double Z = 0, E1 = 0, E2 = 0;
        cp_moments(T, 0, 1.0, &Z, &E1, &E2); cp_moments(T, 1, 3.0, &Z, &E1, &E2);
        c = cp_crot(T, Z, E1, E2);
    }
    const double x = CP_TH_V / T, cv = (x < 700.0) ? x * x * exp(x) / ((exp(x) - 1.0) * (exp(x) - 1.0)) : 0.0;
    return 2.5 + c + cv;
}

static double* g_cp_table[3];   /* per mode, built once (CpH2.h:66-75) */
static int g_cp_n;

static const double* cp_table(int mode){
    if(g_cp_table[mode]) return g_cp_table[mode];
    const int n = (int)((CP_T_HI - CP_T_LO) / CP_DT) + 1;
    double* t = (double*)malloc(sizeof(double) * n);
    for(int i = 0; i < n; i++) t[i] = cpR_exact(CP_T_LO + i * CP_DT, mode) * CP_R_GAS / CP_M_H2;
    g_cp_n = n;
    g_cp_table[mode] = t;
    return t;
}

/* CpH2.h:77-84 */
static double cp_h2_of(const aturan_params* p, double T){
    if(p->cp_h2_mode <= 0) return p->cp_h2;
    const double* t = cp_table(p->cp_h2_mode);
    const int n = g_cp_n;
    const double Tc = T < CP_T_LO ? CP_T_LO : T;
    const double x = ((Tc > CP_T_HI ? CP_T_HI : Tc) - CP_T_LO) / CP_DT;
    int i = (int)x; if(i > n - 2) i = n - 2;
    const double fr = x - i;
    return t[i] + fr * (t[i+1] - t[i]);
}

/* CpH2.h:122-134 (Lapse::cp with dyn_on) */
double oracle_cp_lapse(const aturan_params* p, double T){
    if(!p->cp_dyn) return p->cp_mix;
    const double ch = cp_h2_of(p, T);
    if(p->cp_gas) return (p->r_h2 * ch + p->r_he * p->cp_he + p->r_ch4 * p->cp_ch4) / (p->r_h2 + p->r_he + p->r_ch4);
    return p->cp_mix + (p->r_h2 / p->r_mix) * (ch - p->cp_h2);
}

/* ATPhys.h:135-139 with the periodic seam on (the only supported setting). */
static int phi_wrap(int kk, int km){
    const int n = km - 1;
    return kk < 0 ? kk + n : (kk >= n ? kk - n : kk);
}

/* ATPhys.h:49-53 */
static double svp(double T_K, double C, double L0, double R, double del_alf, double del_bet){
    return exp(C + (-L0 / T_K + del_alf * log(T_K) + del_bet * T_K) / (1e-3 * R));
}

static double coriolis_scale(const aturan_params* p){   /* cUranusModel.h:1498 */
    return (p->coriolis_full ? p->L_atm * 1.0e3 : p->L_atm) / p->u_0;
}

/* ---- RungeKutta_Uran_Turb.cpp:18-37, computeBuoyancyRefLevel ---- */
int oracle_buoy_ref(const aturan_params* p, double* const* f, double* ref){
    const int im = p->im, jm = p->jm, km = p->km;
    const double* t = f[ATURAN_T];
    const double* ps = f[ATURAN_P_STAT];
    double* rad = (double*)malloc(sizeof(double) * im);
    double* the = (double*)malloc(sizeof(double) * jm);
    oracle_coords(p, rad, the);
    #pragma omp parallel for schedule(static)
    for(int i = 0; i < im; i++){
        double sum = 0.0, wsum = 0.0;
        for(int j = 0; j < jm; j++){
            const double wgt = sin(the[j]);
            for(int k = 0; k < km; k++){
                if(!(t[IDX(i,j,k)] > 0.0)) continue;
                const double b = p->g * ps[IDX(i,j,k)]
                               / (p->r_mix * p->R_mix * t[IDX(i,j,k)] * p->t_ref);
                if(!isfinite(b)) continue;
                sum  += wgt * b;
                wsum += wgt;
            }
        }
        ref[i] = (wsum > 0.0) ? sum / wsum : 0.0;
    }
    free(rad); free(the);
    return 0;
}

/* ---- RungeKutta_Uran_Turb.cpp:62-177, computeHydrostaticPressure, with the default knobs:
 * ATURAN_HYDRO_SPLIT=1, METRIC_SPLIT=1, CORIOLIS_SPLIT=1, BUOY_RHO_LEVEL=1, HYDRO_REF=0,
 * HYDRO_ND_KM=0, BUOY_SCALE=1; p_baro allocated (PDYN_GEO=2), p_b0 already captured. ---- */
int oracle_hydro(const aturan_params* p, double* const* f, const double* ref, int advance){
    const int im = p->im, jm = p->jm, km = p->km;
    const double* t = f[ATURAN_T]; const double* ps = f[ATURAN_P_STAT];
    const double* v = f[ATURAN_V]; const double* w = f[ATURAN_W];
    double* ph = f[ATURAN_P_HYDRO];
    const double* pbaro = f[ATURAN_P_BARO]; const double* pb0 = f[ATURAN_P_B0];
    double* pbf = f[ATURAN_P_BFOLLOW];
    double* rad = (double*)malloc(sizeof(double) * im);
    double* the = (double*)malloc(sizeof(double) * jm);
    oracle_coords(p, rad, the);
    const double nd_rel = p->g * (p->L_atm * 1.0e3) / (p->u_0 * p->u_0);
    const double buoy_scale_local = 1.0;
    const double follow_tau = p->pbaro_follow;
    const int follow_on = follow_tau > 0.0;
    #pragma omp parallel for collapse(2) schedule(static)
    for(int j = 0; j < jm; j++){
        for(int k = 0; k < km; k++){
            const double cor_ = p->Coriolis * coriolis_scale(p) * 2.0 * p->omega * fabs(sin(the[j]));
            #define BUOY(ii) ({ const double T_ = t[IDX(ii,j,k)]; double r_ = 0.0;                    \
                if(T_ > 0.0){                                                                          \
                    const double b_ = p->g * ps[IDX(ii,j,k)] / (p->r_mix * p->R_mix * T_ * p->t_ref)   \
                                    - ref[ii];                                                         \
                    const double f_ = -nd_rel * buoy_scale_local * p->buoyancy * b_ / ref[ii];          \
                    r_ = isfinite(f_) ? f_ : 0.0; }                                                    \
                r_; })
            #define MET0(ii) ((v[IDX(ii,j,k)] * v[IDX(ii,j,k)] + w[IDX(ii,j,k)] * w[IDX(ii,j,k)])     \
                              / metric_radius(p, rad[ii]) + cor_ * w[IDX(ii,j,k)])
            if(follow_on){
                double Pm = 0.0, Pb = 0.0;
                for(int i = 0; i < im; i++){
                    if(i > 0){
                        Pm += 0.5 * (MET0(i-1) + MET0(i)) * p->dr;
                        Pb += 0.5 * (BUOY(i-1) + BUOY(i)) * p->dr;
                    }
                    const size_t q = IDX(i,j,k);
                    if(advance) pbf[q] += (Pb - pb0[q] - pbf[q]) / follow_tau;
                    ph[q] = Pm + Pb + pbaro[q] - pbf[q];
                }
            } else {
                ph[IDX(0,j,k)] = 0.0;
                #define F_(ii) (BUOY(ii) + (v[IDX(ii,j,k)] * v[IDX(ii,j,k)] + w[IDX(ii,j,k)] * w[IDX(ii,j,k)]) \
                                    / metric_radius(p, rad[ii]) + cor_ * w[IDX(ii,j,k)])
                for(int i = 1; i < im; i++){
                    const double fa = F_(i-1);
                    const double fb = F_(i);
                    ph[IDX(i,j,k)] = ph[IDX(i-1,j,k)] + 0.5 * (fa + fb) * p->dr;
                }
                for(int i = 0; i < im; i++) ph[IDX(i,j,k)] += pbaro[IDX(i,j,k)];
                #undef F_
            }
            #undef BUOY
            #undef MET0
        }
    }
    free(rad); free(the);
    return 0;
}

/* ---- cUranusModel.h:1212-1223 CellGeometry, filled as RungeKutta_Uran_Turb.cpp:192-283 ---- */
typedef struct {
    double rm, rm2, sinthe, sinthe2, costhe, cotanthe;
    double inv_rm, inv_rm2, inv_rmsinthe, inv_rm2sinthe, inv_rm2sinthe2, costhe_inv_rm2sinthe;
    double inv_2dr, inv_2dthe, inv_2dphi, inv_dr2, inv_dthe2, inv_dphi2;
} geo_t;

static void geo_fill(const aturan_params* p, const double* rad, const double* the, int i, int j, geo_t* g){
    const double s = fabs(sin(the[j]));
    g->rm      = metric_radius(p, rad[i]);
    g->rm2     = g->rm * g->rm;
    g->sinthe  = stdmax(p->sinthe_min, s);
    g->sinthe2 = g->sinthe * g->sinthe;
    g->costhe  = cos(the[j]);
    g->cotanthe             = g->costhe / g->sinthe;
    g->inv_rm               = 1.0 / g->rm;
    g->inv_rm2              = 1.0 / g->rm2;
    g->inv_rmsinthe         = 1.0 / (g->rm * g->sinthe);
    g->inv_rm2sinthe        = g->inv_rm2 / g->sinthe;
    g->inv_rm2sinthe2       = g->inv_rm2 / g->sinthe2;
    g->costhe_inv_rm2sinthe = g->costhe * g->inv_rm2sinthe;
    g->inv_2dr   = 1.0 / (2.0 * p->dr);
    g->inv_2dthe = 1.0 / (2.0 * p->dthe);
    g->inv_2dphi = 1.0 / (2.0 * p->dphi);
    g->inv_dr2   = 1.0 / (p->dr   * p->dr);
    g->inv_dthe2 = 1.0 / (p->dthe * p->dthe);
    g->inv_dphi2 = 1.0 / (p->dphi * p->dphi);
}

/* Species of the RHS in enum order 4..16 with their Schmidt number, precipitation source and
 * chemistry source (RHS_Uran_Turb.cpp:790-850). */
static const int SP_SPRECIP[12] = {
    ATURAN_S_PRECIP_CH4, ATURAN_S_PRECIP_CH4_CLOUD, ATURAN_S_PRECIP_CH4_ICE,
    ATURAN_S_PRECIP_H2O, ATURAN_S_PRECIP_H2O_CLOUD, ATURAN_S_PRECIP_H2O_ICE,
    ATURAN_S_PRECIP_H2S, ATURAN_S_PRECIP_H2S_CLOUD, ATURAN_S_PRECIP_H2S_ICE,
    ATURAN_S_PRECIP_NH3, ATURAN_S_PRECIP_NH3_CLOUD, ATURAN_S_PRECIP_NH3_ICE };

/* ---- RHS_Uran_Turb.cpp:20-1023, RHSUran(i,j,k,geo), default knobs. out[0..18] = rhs of the
 * prognostic fields in enum order, out[19..21] = aux_u, aux_v, aux_w. ---- */
static void rhs_cell(const aturan_params* p, double* const* f, int i, int j, int k,
                     const geo_t* geo, double* out){
    const int jm = p->jm, km = p->km;
    const double inv_rm = geo->inv_rm, inv_rm2 = geo->inv_rm2, inv_rmsinthe = geo->inv_rmsinthe;
    const double inv_rm2sinthe = geo->inv_rm2sinthe, inv_rm2sinthe2 = geo->inv_rm2sinthe2;
    const double costhe_inv_rm2sinthe = geo->costhe_inv_rm2sinthe;
    const double costhe = geo->costhe, cotanthe = geo->cotanthe, rm = geo->rm;
    const double inv_2dr = geo->inv_2dr, inv_2dthe = geo->inv_2dthe, inv_2dphi = geo->inv_2dphi;
    const double inv_dr2 = geo->inv_dr2, inv_dthe2 = geo->inv_dthe2, inv_dphi2 = geo->inv_dphi2;
    const int kw = phi_wrap(k - 1, km), ke = phi_wrap(k + 1, km);
    const size_t c = IDX(i,j,k);

    /* first and second derivatives of the 19 prognostic fields (:92-176) */
    double d1r[NPROG], d2r[NPROG], d1t[NPROG], d2t[NPROG], d1p[NPROG], d2p[NPROG];
    for(int q = 0; q < NPROG; q++){
        const double* F = f[q];
        d1r[q] = (F[IDX(i+1,j,k)] - F[IDX(i-1,j,k)]) * inv_2dr;
        d2r[q] = (F[IDX(i+1,j,k)] - 2.0*F[c] + F[IDX(i-1,j,k)]) * inv_dr2;
        d1t[q] = (F[IDX(i,j+1,k)] - F[IDX(i,j-1,k)]) * inv_2dthe;
        d2t[q] = (F[IDX(i,j+1,k)] - 2.0*F[c] + F[IDX(i,j-1,k)]) * inv_dthe2;
        d1p[q] = (F[IDX(i,j,ke)] - F[IDX(i,j,kw)]) * inv_2dphi;
        d2p[q] = (F[IDX(i,j,ke)] - 2.0*F[c] + F[IDX(i,j,kw)]) * inv_dphi2;
    }
    const double* P = f[ATURAN_P_DYN];
    const double dpdr   = (P[IDX(i+1,j,k)] - P[IDX(i-1,j,k)]) * inv_2dr;
    const double dpdthe = (P[IDX(i,j+1,k)] - P[IDX(i,j-1,k)]) * inv_2dthe;
    const double dpdphi = (P[IDX(i,j,ke)] - P[IDX(i,j,kw)]) * inv_2dphi;

    const double u_ijk = f[ATURAN_U][c], v_ijk = f[ATURAN_V][c], w_ijk = f[ATURAN_W][c];
    const double omega = p->omega;

    /* Coriolis and centrifugal (:208-278), CORIOLIS_TRUE_SINE=1, no legacy signs */
    const double sinthe_bf = sqrt(stdmax(0.0, 1.0 - costhe * costhe));
    const double Coriolis_rad = -2.0 * omega * sinthe_bf * w_ijk;
    const double Coriolis_the = -2.0 * omega * costhe * w_ijk;
    const double Coriolis_phi = +2.0 * omega * (1.0 * costhe * v_ijk + sinthe_bf * u_ijk);
    const double cent_mom = p->cent_mom;
    const double centrifugal_rad = omega * omega * rm * sinthe_bf * sinthe_bf;
    const double centrifugal_the = omega * omega * rm * sinthe_bf * costhe;

    const double coeff_energy_p = p->u_0 * p->u_0 / (p->cp_mix * p->t_ref);
    const double scale_p   = 1.0e5 / (p->r_mix * p->u_0 * p->u_0);
    const double scale_Cor = coriolis_scale(p);
    const double scale_cen = p->L_atm * p->L_atm / (p->u_0 * p->u_0);

    /* transport (:288-326) */
    const double v_invrm = v_ijk * inv_rm;
    const double w_invrs = w_ijk * inv_rmsinthe;
    double pressure_t = coeff_energy_p * scale_p * (u_ijk * dpdr + v_invrm * dpdthe + w_invrs * dpdphi);
    const double tc = f[ATURAN_T][c];
    if(p->cp_dyn && tc > 0.0) pressure_t *= p->cp_mix / oracle_cp_lapse(p, tc * p->t_ref);
    const double transport_t = u_ijk * d1r[ATURAN_T] + v_invrm * d1t[ATURAN_T] + w_invrs * d1p[ATURAN_T];
    const double metric_on = 0.0, cor_rad_on = 0.0;   /* METRIC_SPLIT = CORIOLIS_SPLIT = 1 */
    const double transport_u = u_ijk * d1r[ATURAN_U] + v_invrm * d1t[ATURAN_U] + w_invrs * d1p[ATURAN_U]
        - metric_on * (v_ijk * v_ijk + w_ijk * w_ijk) * inv_rm;
    const double transport_v = u_ijk * d1r[ATURAN_V] + v_invrm * d1t[ATURAN_V] + w_invrs * d1p[ATURAN_V]
        + (u_ijk * v_ijk - w_ijk * w_ijk * cotanthe) * inv_rm;
    const double transport_w = u_ijk * d1r[ATURAN_W] + v_invrm * d1t[ATURAN_W] + w_invrs * d1p[ATURAN_W]
        + (w_ijk * u_ijk + v_ijk * w_ijk * cotanthe) * inv_rm;

    /* diffusion (:329-379) */
    const double two_inv_rm = 2.0 * inv_rm;
    const double v_metric   = (1.0 + costhe / geo->sinthe2) * inv_rm2;
    const double diffusion_t = d2r[ATURAN_T] + d1r[ATURAN_T] * two_inv_rm + d2t[ATURAN_T] * inv_rm2
        + d1t[ATURAN_T] * costhe_inv_rm2sinthe + d2p[ATURAN_T] * inv_rm2sinthe2;
    const double diffusion_u = d2r[ATURAN_U] + 2.0 * u_ijk * inv_rm2 + d2t[ATURAN_U] * inv_rm2
        + 4.0 * d1r[ATURAN_U] * inv_rm + d1t[ATURAN_U] * costhe_inv_rm2sinthe
        + d2p[ATURAN_U] * inv_rm2sinthe2;
    const double diffusion_v = d2r[ATURAN_V] + d1r[ATURAN_V] * two_inv_rm + d2t[ATURAN_V] * inv_rm2
        + d1t[ATURAN_V] * costhe_inv_rm2sinthe - v_metric * v_ijk
        + d2p[ATURAN_V] * inv_rm2sinthe2
        + 2.0 * d1t[ATURAN_U] * inv_rm2
        - d1p[ATURAN_W] * 2.0 * costhe * inv_rm2sinthe2;
    const double diffusion_w = d2r[ATURAN_W] + d1r[ATURAN_W] * two_inv_rm + d2t[ATURAN_W] * inv_rm2
        + d1t[ATURAN_W] * costhe_inv_rm2sinthe - v_metric * w_ijk
        + d2p[ATURAN_W] * inv_rm2sinthe2
        + 2.0 * d1p[ATURAN_U] * inv_rm2sinthe
        + d1p[ATURAN_V] * 2.0 * costhe * inv_rm2sinthe2;

    const double dpdr_term   = dpdr   * scale_p;
    const double dpdthe_term = dpdthe * scale_p * inv_rm;
    const double dpdphi_term = dpdphi * scale_p * inv_rmsinthe;

    const double re = p->re;
    const double re_eff = re / (1.0 + 2.5 * 0.0);          /* EINSTEIN_VISC = 0 */

    const double nue_c = f[ATURAN_NUE][c];
    const double nue_t = (p->turb_coupling != 0.0 && isfinite(nue_c))
                       ? p->turb_coupling * stdmax(0.0, nue_c) : 0.0;
    const double nue_t_s = nue_t / 0.9;

    const double tmf = p->tmf_scale != 0.0 ? p->tmf_scale * p->chemical_reaction * f[ATURAN_THERMALMASSFLUX][c] : 0.0;
    double precip_t = 0.0;
    if(p->precip_coupling != 0.0 && p->r_mix > 0.0 && p->cp_mix > 0.0){
        precip_t = p->precip_coupling * f[ATURAN_Q_PRECIP][c] * (p->L_atm * 1.0e3) / (p->r_mix * p->cp_mix * p->u_0 * p->t_ref);
        if(!isfinite(precip_t)) precip_t = 0.0;
        else if(precip_t >  0.5) precip_t =  0.5;
        else if(precip_t < -0.5) precip_t = -0.5;
    }
    out[ATURAN_T] = + pressure_t - transport_t + diffusion_t / (re * p->pr) + diffusion_t * nue_t_s
                    - tmf + 0.0 + precip_t;

    /* sponge (:594-595) */
    const int im = p->im;
    double frac_sp = (double)(i - (im - 1) * 3 / 4) / (double)((im - 1) / 4);
    if(frac_sp < 0.0) frac_sp = 0.0;
    const double sponge = p->alpha_sponge * frac_sp * frac_sp;

    /* hydrostatic split (:717-721) */
    const double* PH = f[ATURAN_P_HYDRO];
    const double dphdthe_term = (PH[IDX(i,j+1,k)] - PH[IDX(i,j-1,k)]) * inv_2dthe * inv_rm;
    const double dphdphi_term = (PH[IDX(i,j,ke)] - PH[IDX(i,j,kw)]) * inv_2dphi * inv_rmsinthe;
    const double buoyancy_u = 0.0;

    out[ATURAN_U] = - dpdr_term + buoyancy_u - transport_u + diffusion_u / re_eff + diffusion_u * nue_t
                    - cor_rad_on * p->Coriolis * scale_Cor * Coriolis_rad
                    + 1.0 * p->centrifugal * cent_mom * scale_cen * centrifugal_rad
                    - sponge * u_ijk;
    out[ATURAN_V] = - dpdthe_term - dphdthe_term - transport_v + diffusion_v / re_eff + diffusion_v * nue_t
                    - p->Coriolis * scale_Cor * Coriolis_the
                    + 1.0 * p->centrifugal * cent_mom * scale_cen * centrifugal_the;
    out[ATURAN_W] = - dpdphi_term - dphdphi_term - transport_w + diffusion_w / re_eff + diffusion_w * nue_t
                    - p->Coriolis * scale_Cor * Coriolis_phi;

    /* the twelve condensable species (:790-850) */
    static const int sc_of[12] = {0,0,0, 1,1,1, 2,2,2, 3,3,3};
    const double scs[4] = { p->sc_ch4, p->sc_h2o, p->sc_h2s, p->sc_nh3 };
    for(int s = 0; s < 12; s++){
        const int q = ATURAN_CH4 + s;
        const double transport = u_ijk * d1r[q] + v_invrm * d1t[q] + w_invrs * d1p[q];
        const double diffusion = d2r[q] + d1r[q] * two_inv_rm + d2t[q] * inv_rm2
            + d1t[q] * costhe_inv_rm2sinthe + d2p[q] * inv_rm2sinthe2;
        const double sc = scs[sc_of[s]];
        double r = - transport + diffusion / (sc * re) + diffusion * nue_t_s;
        if(q == ATURAN_H2S) r = r + p->chemical_reaction * f[ATURAN_MASSFLUX_H2S][c];
        if(q == ATURAN_NH3) r = r + p->chemical_reaction * f[ATURAN_MASSFLUX_NH3][c];
        out[q] = r + p->precip_coupling * f[SP_SPRECIP[s]][c];
    }

    /* NH4SH with flux limiter and Stokes settling (:857-913) */
    {
        const int q = ATURAN_NH4SH;
        const double transport = u_ijk * d1r[q] + v_invrm * d1t[q] + w_invrs * d1p[q];
        const double diffusion = d2r[q] + d1r[q] * two_inv_rm + d2t[q] * inv_rm2
            + d1t[q] * costhe_inv_rm2sinthe + d2p[q] * inv_rm2sinthe2;
        const double v_stokes = (2.0 / 9.0) * p->r_p_nh4sh * p->r_p_nh4sh
            * (p->rho_cond_nh4sh - f[ATURAN_RHO_MIX][c]) * p->g / p->mue_mix;
        out[q] = - transport + f[ATURAN_FLUXLIM_NH4SH][c]
                 + diffusion / (p->sc_nh4sh * re) + diffusion * nue_t_s
                 + p->chemical_reaction * f[ATURAN_MASSFLUX_NH4SH][c]
                 + (v_stokes / p->u_0) * d1r[q];
    }

    /* k* and dis* (:989-1018) */
    if(p->turb_active){
        const double sig_k = 0.85, sig_w = 0.5;
        const double nue_here = nue_c;
        const int qt = ATURAN_TKE, qd = ATURAN_DIS;
        const double transport_tke = u_ijk * d1r[qt] + v_ijk * d1t[qt] * inv_rm + w_ijk * d1p[qt] * inv_rmsinthe;
        const double transport_dis = u_ijk * d1r[qd] + v_ijk * d1t[qd] * inv_rm + w_ijk * d1p[qd] * inv_rmsinthe;
        const double diffusion_tke = d2r[qt] + d1r[qt] * 2.0 * inv_rm + d2t[qt] * inv_rm2
            + d1t[qt] * costhe_inv_rm2sinthe + d2p[qt] * inv_rm2sinthe2;
        const double diffusion_dis = d2r[qd] + d1r[qd] * 2.0 * inv_rm + d2t[qd] * inv_rm2
            + d1t[qd] * costhe_inv_rm2sinthe + d2p[qd] * inv_rm2sinthe2;
        out[qt] = - transport_tke + diffusion_tke * (1.0 / re + nue_here / sig_k) + f[ATURAN_TKE_SOURCE][c];
        out[qd] = - transport_dis + diffusion_dis * (1.0 / re + nue_here / sig_w) + f[ATURAN_DIS_SOURCE][c];
    } else {
        out[ATURAN_TKE] = 0.0;
        out[ATURAN_DIS] = 0.0;
    }

    out[19] = out[ATURAN_U] + dpdr_term;   /* aux_u (:1020-1022) */
    out[20] = out[ATURAN_V] + dpdthe_term;
    out[21] = out[ATURAN_W] + dpdphi_term;
}

int oracle_rhs_cell(const aturan_params* p, double* const* f, int i, int j, int k, double* rhs22){
    double rad[256], the[4096];
    if(p->im > 256 || p->jm > 4096) return -1;
    oracle_coords(p, rad, the);
    geo_t g; geo_fill(p, rad, the, i, j, &g);
    rhs_cell(p, f, i, j, k, &g, rhs22);
    return 0;
}

static double clampd(double v, double lo, double hi){ return v < lo ? lo : (v > hi ? hi : v); }


/* ---- RungeKutta_Uran_Turb.cpp:179-404, RungeKuttaUran ---- */
int oracle_rk4(const aturan_params* p, double* const* f, double* ref_out){
    const int im = p->im, jm = p->jm, km = p->km;
    const size_t N = (size_t)im * jm * km;
    double ref[512];
    if(im > 512) return -1;
    oracle_buoy_ref(p, f, ref);
    oracle_hydro(p, f, ref, 1);
    if(ref_out) memcpy(ref_out, ref, sizeof(double) * im);

    double* rad = (double*)malloc(sizeof(double) * im);
    double* the = (double*)malloc(sizeof(double) * jm);
    oracle_coords(p, rad, the);
    double* rhs = (double*)malloc(sizeof(double) * N * NPROG);
    double* acc = (double*)malloc(sizeof(double) * N * NPROG);
    if(!rhs || !acc){ free(rhs); free(acc); free(rad); free(the); return -1; }

    const int turb = p->turb_active;
    const double tke_max_nd = 1000.0 / (p->u_0 * p->u_0);
    const double dis_min_nd = 1.0e-10;
    const double t_min = p->t_min_K / p->t_ref, t_max = p->t_max_K / p->t_ref;
    const double dt = p->dt;

    for(int stage = 0; stage < 4; stage++){
        const double c_in = (stage == 0 || stage == 1) ? 0.5 * dt : (stage == 2 ? dt : 0.0);
        const double wgt  = (stage == 0 || stage == 3) ? 1.0 : 2.0;
        /* pass A */
        #pragma omp parallel for collapse(2) schedule(static)
        for(int i = 1; i < im-1; i++){
            for(int j = 1; j < jm-1; j++){
                geo_t g; geo_fill(p, rad, the, i, j, &g);
                double out[22];
                for(int k = 0; k < km-1; k++){
                    rhs_cell(p, f, i, j, k, &g, out);
                    const size_t c = IDX(i,j,k);
                    for(int q = 0; q < NPROG; q++) rhs[(size_t)q * N + c] = out[q];
                    f[ATURAN_RHS_U][c] = out[ATURAN_U];
                    f[ATURAN_RHS_V][c] = out[ATURAN_V];
                    f[ATURAN_RHS_W][c] = out[ATURAN_W];
                    f[ATURAN_AUX_U][c] = out[19];
                    f[ATURAN_AUX_V][c] = out[20];
                    f[ATURAN_AUX_W][c] = out[21];
                }
            }
        }
        /* pass B */
        #pragma omp parallel for collapse(2) schedule(static)
        for(int i = 1; i < im-1; i++){
            for(int j = 1; j < jm-1; j++){
                for(int k = 0; k < km-1; k++){
                    const size_t c = IDX(i,j,k);
                    const int nq = turb ? NPROG : NPROG - 2;
                    for(int q = 0; q < nq; q++){
                        double* A = acc + (size_t)q * N;
                        const double r = rhs[(size_t)q * N + c];
                        A[c] = (stage == 0) ? wgt * r : A[c] + wgt * r;
                    }
                    if(stage < 3){
                        for(int q = 0; q < NPROG - 2; q++)
                            f[q][c] = f[ATURAN_TN + q][c] + c_in * rhs[(size_t)q * N + c];
                        if(turb){
                            f[ATURAN_TKE][c] = clampd(f[ATURAN_TKEN][c] + c_in * rhs[(size_t)ATURAN_TKE * N + c],
                                                      0.0, tke_max_nd);
                            const double d_ = f[ATURAN_DISN][c] + c_in * rhs[(size_t)ATURAN_DIS * N + c];
                            f[ATURAN_DIS][c] = stdmax(d_, dis_min_nd);
                        }
                    }
                }
            }
        }
    }

    /* the step (:371-403) */
    #pragma omp parallel for collapse(2) schedule(static)
    for(int i = 1; i < im-1; i++){
        for(int j = 1; j < jm-1; j++){
            for(int k = 0; k < km-1; k++){
                const size_t c = IDX(i,j,k);
                f[ATURAN_T][c] = clampd(f[ATURAN_TN][c] + dt * acc[c] / 6.0, t_min, t_max);
                for(int q = 1; q < NPROG - 2; q++)
                    f[q][c] = f[ATURAN_TN + q][c] + dt * acc[(size_t)q * N + c] / 6.0;
                if(turb){
                    double x = f[ATURAN_TKEN][c] + dt * acc[(size_t)ATURAN_TKE * N + c] / 6.0;
                    x = stdmax(x, 0.0);
                    f[ATURAN_TKE][c] = clampd(x, 0.0, tke_max_nd);
                    const double d_ = f[ATURAN_DISN][c] + dt * acc[(size_t)ATURAN_DIS * N + c] / 6.0;
                    f[ATURAN_DIS][c] = stdmax(d_, dis_min_nd);
                }
            }
        }
    }
    free(rhs); free(acc); free(rad); free(the);
    return 0;
}

/* The sin table of both pressure solvers: sin(theta) floored at sinthe_min(), no fabs
 * (PressureSolverUran.h:42-47; PressureSolver.h:156-162 adds the exact-zero guard). */
static void press_sin_table(const aturan_params* p, const double* the, double* s, int shared){
    for(int j = 0; j < p->jm; j++){
        s[j] = sin(the[j]);
        if(s[j] < p->sinthe_min) s[j] = p->sinthe_min;
        if(shared && s[j] == 0.0) s[j] = 1.0e-5;
    }
}

/* p_dyn boundary passes shared by both solvers: r, then theta, then the periodic phi copy
 * (PressureSolverUran.h:213-244; PressureSolver.h:718-746). */
static void p_dyn_bcs(const aturan_params* p, double* P){
    const int im = p->im, jm = p->jm, km = p->km;
    #pragma omp parallel for collapse(2)
    for(int k = 0; k < km; k++) for(int j = 0; j < jm; j++){
        P[IDX(0,j,k)]    = C43 * P[IDX(1,j,k)]    - C13 * P[IDX(2,j,k)];
        P[IDX(im-1,j,k)] = C43 * P[IDX(im-2,j,k)] - C13 * P[IDX(im-3,j,k)];
    }
    #pragma omp parallel for collapse(2)
    for(int k = 0; k < km; k++) for(int i = 0; i < im; i++){
        P[IDX(i,0,k)]    = C43 * P[IDX(i,1,k)]    - C13 * P[IDX(i,2,k)];
        P[IDX(i,jm-1,k)] = C43 * P[IDX(i,jm-2,k)] - C13 * P[IDX(i,jm-3,k)];
    }
    #pragma omp parallel for collapse(2)
    for(int i = 0; i < im; i++) for(int j = 0; j < jm; j++)
        P[IDX(i,j,km-1)] = P[IDX(i,j,0)];
}

/* ---- PressureSolverUran.h:33-250, the default solver: one serial lexicographic sweep ---- */
int oracle_pressure_gs(const aturan_params* p, double* const* f){
    const int im = p->im, jm = p->jm, km = p->km;
    double* rad = (double*)malloc(sizeof(double) * im);
    double* the = (double*)malloc(sizeof(double) * jm);
    double* st  = (double*)malloc(sizeof(double) * jm);
    oracle_coords(p, rad, the);
    press_sin_table(p, the, st, 0);
    const int consistent = p->press_consistent;
    const double src_scale = consistent ? (p->r_mix * p->u_0 * p->u_0) / 1.0e5 : 1.0;
    double* au = f[ATURAN_AUX_U]; double* av = f[ATURAN_AUX_V]; double* aw = f[ATURAN_AUX_W];
    double* P = f[ATURAN_P_DYN];

    /* aux radial BC (:70-81) */
    #pragma omp parallel for collapse(2)
    for(int j = 1; j < jm-1; j++) for(int k = 0; k < km-1; k++){
        au[IDX(0,j,k)]    = C43 * au[IDX(1,j,k)]    - C13 * au[IDX(2,j,k)];
        au[IDX(im-1,j,k)] = C43 * au[IDX(im-2,j,k)] - C13 * au[IDX(im-3,j,k)];
        av[IDX(0,j,k)]    = C43 * av[IDX(1,j,k)]    - C13 * av[IDX(2,j,k)];
        av[IDX(im-1,j,k)] = C43 * av[IDX(im-2,j,k)] - C13 * av[IDX(im-3,j,k)];
        aw[IDX(0,j,k)]    = C43 * aw[IDX(1,j,k)]    - C13 * aw[IDX(2,j,k)];
        aw[IDX(im-1,j,k)] = C43 * aw[IDX(im-2,j,k)] - C13 * aw[IDX(im-3,j,k)];
    }
    const double inv_2dr = 1.0 / (2.0 * p->dr), inv_2dthe = 1.0 / (2.0 * p->dthe), inv_2dphi = 1.0 / (2.0 * p->dphi);
    const double inv_dr2 = 1.0 / (p->dr * p->dr), inv_dthe2 = 1.0 / (p->dthe * p->dthe), inv_dphi2 = 1.0 / (p->dphi * p->dphi);

    /* defect-correction source (:139-175) */
    double* incr = NULL;
    const size_t N = (size_t)im * jm * km;
    if(p->press_incr){
        incr = (double*)calloc(N, sizeof(double));
        const double* ru_u = f[ATURAN_RHS_U]; const double* ru_v = f[ATURAN_RHS_V]; const double* ru_w = f[ATURAN_RHS_W];
        #pragma omp parallel for collapse(2) schedule(static)
        for(int i = 1; i < im-1; i++){
            for(int j = 1; j < jm-1; j++){
                const double rm = consistent ? metric_radius(p, rad[i]) : rad[i];
                const double inv_rm = 1.0 / rm;
                const double inv_rmsinthe = 1.0 / (rm * st[j]);
                const double inv_rm2 = inv_rm * inv_rm;
                const double inv_rm2sinthe2 = inv_rm2 / (st[j] * st[j]);
                const double num1 = 1.0 / (p->dr * p->dr), num2 = inv_rm2 / (p->dthe * p->dthe),
                             num3 = inv_rm2sinthe2 / (p->dphi * p->dphi);
                const double denom = 2.0 * (num1 + num2 + num3);
                for(int k = 0; k < km-1; k++){
                    const int kw = phi_wrap(k-1, km), ke = phi_wrap(k+1, km);
                    #define RU(A, ii, jj, kk) ((ii) == 0 ? C43 * A[IDX(1,jj,kk)] - C13 * A[IDX(2,jj,kk)] : \
                        ((ii) == im-1 ? C43 * A[IDX(im-2,jj,kk)] - C13 * A[IDX(im-3,jj,kk)] : A[IDX(ii,jj,kk)]))
                    const double div_rhs =
                          (RU(ru_u, i+1, j, k) - RU(ru_u, i-1, j, k)) / (2.0 * p->dr)
                        + (RU(ru_v, i, j+1, k) - RU(ru_v, i, j-1, k)) / (2.0 * p->dthe) * inv_rm
                        + (RU(ru_w, i, j, ke)  - RU(ru_w, i, j, kw))  / (2.0 * p->dphi) * inv_rmsinthe;
                    #undef RU
                    const double lc_old =
                          (P[IDX(i+1,j,k)] + P[IDX(i-1,j,k)]) * num1
                        + (P[IDX(i,j+1,k)] + P[IDX(i,j-1,k)]) * num2
                        + (P[IDX(i,j,ke)]  + P[IDX(i,j,kw)])  * num3
                        - denom * P[IDX(i,j,k)];
                    incr[IDX(i,j,k)] = src_scale * div_rhs + lc_old;
                }
            }
        }
    }

    /* the serial sweep (:177-211) */
    for(int i = 1; i < im-1; i++){
        for(int j = 1; j < jm-1; j++){
            const double rm = consistent ? metric_radius(p, rad[i]) : rad[i];
            const double rm2 = rm * rm;
            const double sinthe = st[j];
            const double inv_rm = 1.0 / rm;
            const double inv_rm2 = 1.0 / rm2;
            const double inv_rmsinthe = 1.0 / (rm * sinthe);
            const double inv_rm2sinthe2 = inv_rm2 / (sinthe * sinthe);
            const double denom = 2.0 * inv_dr2 + 2.0 * inv_rm2 * inv_dthe2 + 2.0 * inv_rm2sinthe2 * inv_dphi2;
            const double inv_denom = 1.0 / denom;
            const double num1 = inv_dr2, num2 = inv_rm2 * inv_dthe2, num3 = inv_rm2sinthe2 * inv_dphi2;
            for(int k = 0; k < km-1; k++){
                const int kw = phi_wrap(k-1, km), ke = phi_wrap(k+1, km);
                double src;
                if(incr) src = incr[IDX(i,j,k)];
                else {
                    const double du_dr   = (au[IDX(i+1,j,k)] - au[IDX(i-1,j,k)]) * inv_2dr;
                    const double dv_dthe = (av[IDX(i,j+1,k)] - av[IDX(i,j-1,k)]) * inv_2dthe * inv_rm;
                    const double dw_dphi = (aw[IDX(i,j,ke)] - aw[IDX(i,j,kw)]) * inv_2dphi * inv_rmsinthe;
                    src = src_scale * (du_dr + dv_dthe + dw_dphi);
                }
                P[IDX(i,j,k)] =
                    ((P[IDX(i+1,j,k)] + P[IDX(i-1,j,k)]) * num1
                   + (P[IDX(i,j+1,k)] + P[IDX(i,j-1,k)]) * num2
                   + (P[IDX(i,j,ke)] + P[IDX(i,j,kw)]) * num3
                   - src) * inv_denom;
            }
        }
    }
    p_dyn_bcs(p, P);
    free(incr); free(rad); free(the); free(st);
    return 0;
}

/* ---- Pressure_Uran.cpp:30-146, prepareProjectionBoundaries, periodic phi ---- */
static void prepare_projection_boundaries(const aturan_params* p, double* const* f){
    const int im = p->im, jm = p->jm, km = p->km;
    double* A[6] = { f[ATURAN_AUX_U], f[ATURAN_AUX_V], f[ATURAN_AUX_W],
                     f[ATURAN_RHS_U], f[ATURAN_RHS_V], f[ATURAN_RHS_W] };
    #define CUB0(X, jj, kk) (X[IDX(3,jj,kk)] - 3.0 * X[IDX(2,jj,kk)] + 3.0 * X[IDX(1,jj,kk)])
    #define CUB1(X, jj, kk) (X[IDX(im-4,jj,kk)] - 3.0 * X[IDX(im-3,jj,kk)] + 3.0 * X[IDX(im-2,jj,kk)])
    #pragma omp parallel for
    for(int j = 1; j < jm-1; j++){
        for(int k = 0; k < km-1; k++){
            if(p->rigid_lid){ A[0][IDX(0,j,k)] = 0.0; A[0][IDX(im-1,j,k)] = 0.0; }
            else { A[0][IDX(0,j,k)] = CUB0(A[0], j, k); A[0][IDX(im-1,j,k)] = CUB1(A[0], j, k); }
            for(int q = 1; q < 6; q++){
                A[q][IDX(0,j,k)]    = CUB0(A[q], j, k);
                A[q][IDX(im-1,j,k)] = CUB1(A[q], j, k);
            }
        }
    }
    #undef CUB0
    #undef CUB1
    #define CUBJ0(X, ii, kk) (X[IDX(ii,3,kk)] - 3.0 * X[IDX(ii,2,kk)] + 3.0 * X[IDX(ii,1,kk)])
    #define CUBJ1(X, ii, kk) (X[IDX(ii,jm-4,kk)] - 3.0 * X[IDX(ii,jm-3,kk)] + 3.0 * X[IDX(ii,jm-2,kk)])
    #pragma omp parallel for
    for(int k = 0; k < km-1; k++){
        for(int i = 1; i < im-1; i++){
            A[0][IDX(i,0,k)] = CUBJ0(A[0], i, k);
            A[1][IDX(i,0,k)] = 0.0;
            A[2][IDX(i,0,k)] = 0.0;
            A[0][IDX(i,jm-1,k)] = CUBJ1(A[0], i, k);
            A[1][IDX(i,jm-1,k)] = 0.0;
            A[2][IDX(i,jm-1,k)] = 0.0;
            A[3][IDX(i,0,k)] = CUBJ0(A[3], i, k);
            A[4][IDX(i,0,k)] = 0.0;
            A[5][IDX(i,0,k)] = 0.0;
            A[3][IDX(i,jm-1,k)] = CUBJ1(A[3], i, k);
            A[4][IDX(i,jm-1,k)] = 0.0;
            A[5][IDX(i,jm-1,k)] = 0.0;
        }
    }
    #undef CUBJ0
    #undef CUBJ1
    #pragma omp parallel for
    for(int i = 0; i < im; i++) for(int j = 0; j < jm; j++)
        for(int q = 0; q < 6; q++) A[q][IDX(i,j,km-1)] = A[q][IDX(i,j,0)];
}

/* The shared solver's per-(i,j) weights (PressureSolver.h:326-353). */
typedef struct { double num1, num2, num3, den, inv_rm, inv_rmsinthe; } pweights_t;
static void press_weights(const aturan_params* p, const double* rad, const double* st, int i, int j, pweights_t* w){
    const double rm = metric_radius(p, rad[i]);
    const double rm2 = rm * rm;
    const double exp_rm = 1.0, exp_2_rm = exp_rm * exp_rm;
    const double sinthe2 = st[j] * st[j];
    const double inv_rm2 = 1.0 / rm2;
    const double inv_rm2sinthe2 = inv_rm2 / sinthe2;
    const double inv_dr2 = 1.0 / (p->dr * p->dr), inv_dthe2 = 1.0 / (p->dthe * p->dthe), inv_dphi2 = 1.0 / (p->dphi * p->dphi);
    w->num1 = exp_2_rm * inv_dr2;
    w->num2 = inv_rm2 * inv_dthe2;
    w->num3 = inv_rm2sinthe2 * inv_dphi2;
    w->den  = 2.0 * w->num1 + 2.0 * w->num2 + 2.0 * w->num3;
    w->inv_rm = 1.0 / rm;
    w->inv_rmsinthe = 1.0 / (rm * st[j]);
}

/* The shared solver's source: div(aux) with centred differences, the clamp at den*p_dyn_cap and
 * the non-finite guard (PressureSolver.h:370-487, no obstacle, PRESS_SRC=1, PRESS_INCR=0).
 * Runs prepare_projection_boundaries first, as run() does (:208). */
int oracle_pressure_source(const aturan_params* p, double* const* f, double* src){
    const int im = p->im, jm = p->jm, km = p->km;
    double* rad = (double*)malloc(sizeof(double) * im);
    double* the = (double*)malloc(sizeof(double) * jm);
    double* st  = (double*)malloc(sizeof(double) * jm);
    oracle_coords(p, rad, the);
    press_sin_table(p, the, st, 1);
    prepare_projection_boundaries(p, f);
    const double* au = f[ATURAN_AUX_U]; const double* av = f[ATURAN_AUX_V]; const double* aw = f[ATURAN_AUX_W];
    const double inv_2dr = 1.0 / (2.0 * p->dr), inv_2dthe = 1.0 / (2.0 * p->dthe), inv_2dphi = 1.0 / (2.0 * p->dphi);
    memset(src, 0, sizeof(double) * (size_t)im * jm * km);
    #pragma omp parallel for collapse(2) schedule(static)
    for(int i = 1; i < im-1; i++){
        for(int j = 1; j < jm-1; j++){
            pweights_t w; press_weights(p, rad, st, i, j, &w);
            for(int k = 0; k < km-1; k++){
                const int kw = phi_wrap(k-1, km), ke = phi_wrap(k+1, km);
                const double du_dr   = (au[IDX(i+1,j,k)] - au[IDX(i-1,j,k)]) * inv_2dr;
                const double dv_dthe = (av[IDX(i,j+1,k)] - av[IDX(i,j-1,k)]) * inv_2dthe;
                const double dw_dphi = (aw[IDX(i,j,ke)] - aw[IDX(i,j,kw)]) * inv_2dphi;
                double div_src = du_dr * 1.0 + dv_dthe * w.inv_rm + dw_dphi * w.inv_rmsinthe;
                const double src_max = w.den * p->p_dyn_cap;
                if      (!isfinite(div_src)) div_src = 0.0;
                else if (div_src >  src_max) div_src =  src_max;
                else if (div_src < -src_max) div_src = -src_max;
                src[IDX(i,j,k)] = div_src;
            }
        }
    }
    free(rad); free(the); free(st);
    return 0;
}

/* One red-black colour pass of PressureSolver.h:320-495 at relaxation factor omega (omega = 1
 * is the reference's update p = (acc - src) / den exactly). */
static void rb_colour(const aturan_params* p, const double* rad, const double* st, double* P,
                      const double* src, int colour, double omega){
    const int im = p->im, jm = p->jm, km = p->km;
    #pragma omp parallel for collapse(2) schedule(static)
    for(int i = 1; i < im-1; i++){
        for(int j = 1; j < jm-1; j++){
            pweights_t w; press_weights(p, rad, st, i, j, &w);
            for(int k = 0; k < km-1; k++){
                if(((i + j + k) & 1) != colour) continue;
                const int kw = phi_wrap(k-1, km), ke = phi_wrap(k+1, km);
                const double acc = (P[IDX(i+1,j,k)] + P[IDX(i-1,j,k)]) * w.num1
                                 + (P[IDX(i,j+1,k)] + P[IDX(i,j-1,k)]) * w.num2
                                 + (P[IDX(i,j,ke)] + P[IDX(i,j,kw)]) * w.num3;
                const double pn = (acc - src[IDX(i,j,k)]) / w.den;
                if(omega == 1.0) P[IDX(i,j,k)] = pn;
                else P[IDX(i,j,k)] = P[IDX(i,j,k)] + omega * (pn - P[IDX(i,j,k)]);
            }
        }
    }
}

/* ---- PressureSolver.h:145-766 with ATURAN_PRESS_SWEEPS = sweeps (no line, no barotropic) ---- */
int oracle_pressure_rb(const aturan_params* p, double* const* f, int sweeps){
    const int im = p->im, jm = p->jm, km = p->km;
    double* rad = (double*)malloc(sizeof(double) * im);
    double* the = (double*)malloc(sizeof(double) * jm);
    double* st  = (double*)malloc(sizeof(double) * jm);
    double* src = (double*)malloc(sizeof(double) * (size_t)im * jm * km);
    oracle_coords(p, rad, the);
    press_sin_table(p, the, st, 1);
    oracle_pressure_source(p, f, src);
    if(sweeps < 1) sweeps = 1;
    for(int s = 0; s < sweeps; s++){
        rb_colour(p, rad, st, f[ATURAN_P_DYN], src, 0, 1.0);
        rb_colour(p, rad, st, f[ATURAN_P_DYN], src, 1, 1.0);
        p_dyn_bcs(p, f[ATURAN_P_DYN]);
    }
    free(rad); free(the); free(st); free(src);
    return 0;
}

/* Relative L2 residual ||src - Lc p|| / ||src|| over the interior rows, with Lc the shared
 * solver's compact operator on the current (boundary-folded) p_dyn. */
double oracle_pressure_residual(const aturan_params* p, double* const* f, const double* src){
    const int im = p->im, jm = p->jm, km = p->km;
    double* rad = (double*)malloc(sizeof(double) * im);
    double* the = (double*)malloc(sizeof(double) * jm);
    double* st  = (double*)malloc(sizeof(double) * jm);
    oracle_coords(p, rad, the);
    press_sin_table(p, the, st, 1);
    const double* P = f[ATURAN_P_DYN];
    double rr = 0.0, ss = 0.0;
    #pragma omp parallel for collapse(2) reduction(+:rr,ss) schedule(static)
    for(int i = 1; i < im-1; i++){
        for(int j = 1; j < jm-1; j++){
            pweights_t w; press_weights(p, rad, st, i, j, &w);
            for(int k = 0; k < km-1; k++){
                const int kw = phi_wrap(k-1, km), ke = phi_wrap(k+1, km);
                const double lc = (P[IDX(i+1,j,k)] + P[IDX(i-1,j,k)]) * w.num1
                                + (P[IDX(i,j+1,k)] + P[IDX(i,j-1,k)]) * w.num2
                                + (P[IDX(i,j,ke)] + P[IDX(i,j,kw)]) * w.num3 - w.den * P[IDX(i,j,k)];
                const double r = src[IDX(i,j,k)] - lc;
                rr += r * r; ss += src[IDX(i,j,k)] * src[IDX(i,j,k)];
            }
        }
    }
    free(rad); free(the); free(st);
    return ss > 0.0 ? sqrt(rr / ss) : sqrt(rr);
}

/* Remove the source's component along the all-Neumann operator's left null vector
 * y = a(i) b(j), a = b = (3/2, 1, ..., 1, 3/2) (PressureSolver.h:63-65 states it for theta; the
 * radial fold has the same form), by a constant shift over the interior. */
static void compat_shift(const aturan_params* p, double* src){
    const int im = p->im, jm = p->jm, km = p->km;
    double ys = 0.0, yy = 0.0;
    for(int i = 1; i < im-1; i++) for(int j = 1; j < jm-1; j++){
        const double yi = (i == 1 || i == im-2) ? 1.5 : 1.0, yj = (j == 1 || j == jm-2) ? 1.5 : 1.0;
        for(int k = 0; k < km-1; k++){ ys += yi * yj * src[IDX(i,j,k)]; yy += yi * yj; }
    }
    const double shift = ys / yy;
    for(int i = 1; i < im-1; i++) for(int j = 1; j < jm-1; j++) for(int k = 0; k < km-1; k++)
        src[IDX(i,j,k)] -= shift;
}

int oracle_pressure_source_compat(const aturan_params* p, double* const* f, double* src){
    oracle_pressure_source(p, f, src);
    compat_shift(p, src);
    return 0;
}

/* The shared solver's operator with the 2-point Neumann folds substituted into the rows instead
 * of lagged boundary rows: at i = 1, p[0] = c43 p[1] - c13 p[2] puts c43 num1 on the diagonal
 * and -c13 num1 on p[2]; likewise at i = im-2, j = 1, j = jm-2. Same linear operator on the
 * interior unknowns (hence the same solution), but every row couples only to the other colour,
 * so red-black SOR keeps its consistently-ordered convergence rate. Returns the off-diagonal
 * sum and the diagonal. */
static double folded_acc(const aturan_params* p, const double* P, int i, int j, int k,
                         const pweights_t* w, double* diag){
    const int im = p->im, jm = p->jm, km = p->km;
    const int kw = phi_wrap(k-1, km), ke = phi_wrap(k+1, km);
    double d = w->den;
    const double aim = (i == 1)    ? (d -= C43 * w->num1, -C13 * P[IDX(i+1,j,k)]) : P[IDX(i-1,j,k)];
    const double aip = (i == im-2) ? (d -= C43 * w->num1, -C13 * P[IDX(i-1,j,k)]) : P[IDX(i+1,j,k)];
    const double ajm = (j == 1)    ? (d -= C43 * w->num2, -C13 * P[IDX(i,j+1,k)]) : P[IDX(i,j-1,k)];
    const double ajp = (j == jm-2) ? (d -= C43 * w->num2, -C13 * P[IDX(i,j-1,k)]) : P[IDX(i,j+1,k)];
    *diag = d;
    return (aip + aim) * w->num1 + (ajp + ajm) * w->num2 + (P[IDX(i,j,ke)] + P[IDX(i,j,kw)]) * w->num3;
}

static void rbf_colour(const aturan_params* p, const double* rad, const double* st, double* P,
                       const double* src, int colour, double omega){
    const int im = p->im, jm = p->jm, km = p->km;
    #pragma omp parallel for collapse(2) schedule(static)
    for(int i = 1; i < im-1; i++){
        for(int j = 1; j < jm-1; j++){
            pweights_t w; press_weights(p, rad, st, i, j, &w);
            for(int k = 0; k < km-1; k++){
                if(((i + j + k) & 1) != colour) continue;
                double diag;
                const double acc = folded_acc(p, P, i, j, k, &w, &diag);
                const double pn = (acc - src[IDX(i,j,k)]) / diag;
                P[IDX(i,j,k)] += omega * (pn - P[IDX(i,j,k)]);
            }
        }
    }
}

/* Relative L2 residual of the folded operator (equal to the boundary-row form once the
 * boundary rows are consistent). */
static double folded_residual(const aturan_params* p, const double* rad, const double* st,
                              const double* P, const double* src){
    const int im = p->im, jm = p->jm, km = p->km;
    double rr = 0.0, ss = 0.0;
    #pragma omp parallel for collapse(2) reduction(+:rr,ss) schedule(static)
    for(int i = 1; i < im-1; i++){
        for(int j = 1; j < jm-1; j++){
            pweights_t w; press_weights(p, rad, st, i, j, &w);
            for(int k = 0; k < km-1; k++){
                double diag;
                const double acc = folded_acc(p, P, i, j, k, &w, &diag);
                const double r = src[IDX(i,j,k)] - (acc - diag * P[IDX(i,j,k)]);
                rr += r * r; ss += src[IDX(i,j,k)] * src[IDX(i,j,k)];
            }
        }
    }
    return ss > 0.0 ? sqrt(rr / ss) : sqrt(rr);
}

/* The column-uniform correction: q(j,k) added to every level with
 *   (sum_i y_i / rm_i^2) L2(q) = sum_i y_i (src - Lc p)_i,
 * L2 the horizontal stencil, solved by a DFT over the km-1 meridians and one tridiagonal solve
 * in theta per Fourier mode with the ends folded (the reference's PRESS_BAROTROPIC,
 * PressureSolver.h:572-708, with the folded operator's left null vector as column weights). */
static void column_correction(const aturan_params* p, const double* rad, const double* st,
                              double* P, const double* src){
    const int im = p->im, jm = p->jm, km = p->km;
    const int J = jm - 2, N = km - 1, NM = N / 2;
    double* R  = (double*)calloc((size_t)J * N, sizeof(double));
    double* Ac = (double*)calloc((size_t)(NM + 1) * J, sizeof(double));
    double* As = (double*)calloc((size_t)(NM + 1) * J, sizeof(double));
    double A2y = 0.0;
    for(int i = 1; i < im-1; i++){ const double rm = metric_radius(p, rad[i]); A2y += ((i == 1 || i == im-2) ? 1.5 : 1.0) / (rm * rm); }
    #pragma omp parallel for schedule(static)
    for(int jj = 0; jj < J; jj++){
        const int j = jj + 1;
        for(int k = 0; k < N; k++){
            const int kw = phi_wrap(k-1, km), ke = phi_wrap(k+1, km);
            double acc_r = 0.0;
            (void)kw; (void)ke;
            for(int i = 1; i < im-1; i++){
                pweights_t w; press_weights(p, rad, st, i, j, &w);
                double diag;
                const double accf = folded_acc(p, P, i, j, k, &w, &diag);
                const double lc = accf - diag * P[IDX(i,j,k)];
                acc_r += ((i == 1 || i == im-2) ? 1.5 : 1.0) * (src[IDX(i,j,k)] - lc);
            }
            R[(size_t)jj * N + k] = acc_r;
        }
    }
    const double e = 1.0 / (p->dthe * p->dthe), inv_dphi2 = 1.0 / (p->dphi * p->dphi);
    #pragma omp parallel for schedule(static)
    for(int m = 0; m <= NM; m++){
        double* cp = (double*)malloc(sizeof(double) * J);
        double* dp = (double*)malloc(sizeof(double) * J);
        for(int jj = 0; jj < J; jj++){
            double sc = 0.0, ss = 0.0;
            for(int k = 0; k < N; k++){
                const double a = 2.0 * M_PI * (double)((long)m * k % N) / N;
                const double v = R[(size_t)jj * N + k] / A2y;
                sc += v * cos(a); ss += v * sin(a);
            }
            Ac[(size_t)m * J + jj] = sc; As[(size_t)m * J + jj] = ss;
        }
        const double sl = sin(M_PI * m / N);
        const double lam = 4.0 * sl * sl * inv_dphi2;
        for(int part = 0; part < 2; part++){
            double* d = (part == 0 ? Ac : As) + (size_t)m * J;
            if(part == 1 && (m == 0 || 2 * m == N)){ for(int q = 0; q < J; q++) d[q] = 0.0; continue; }
            if(m == 0){
                double yr = 0.0, ys = 0.0;
                for(int q = 0; q < J; q++){ const double y = (q == 0 || q == J-1) ? 1.5 : 1.0; yr += y * d[q]; ys += y; }
                for(int q = 0; q < J; q++) d[q] -= yr / ys;
            }
            #define TA(q) ((q) == 0 ? 0.0 : ((q) == J-1 ? e - C13 * e : e))
            #define TB(q) (-2.0 * e - lam / (st[(q)+1] * st[(q)+1]) + (((q) == 0 || (q) == J-1) ? C43 * e : 0.0))
            #define TC(q) ((q) == J-1 ? 0.0 : ((q) == 0 ? e - C13 * e : e))
            double b0 = TB(0), c0 = TC(0), d0 = d[0];
            if(m == 0){ b0 = 1.0; c0 = 0.0; d0 = 0.0; }
            cp[0] = c0 / b0; dp[0] = d0 / b0;
            for(int q = 1; q < J; q++){
                const double dn = TB(q) - TA(q) * cp[q-1];
                cp[q] = TC(q) / dn;
                dp[q] = (d[q] - TA(q) * dp[q-1]) / dn;
            }
            #undef TA
            #undef TB
            #undef TC
            d[J-1] = dp[J-1];
            for(int q = J-2; q >= 0; q--) d[q] = dp[q] - cp[q] * d[q+1];
            if(m == 0){
                double yq = 0.0, ys = 0.0;
                for(int q = 0; q < J; q++){ const double y = (q == 0 || q == J-1) ? 1.5 : 1.0; yq += y * d[q]; ys += y; }
                for(int q = 0; q < J; q++) d[q] -= yq / ys;
            }
        }
        free(cp); free(dp);
    }
    #pragma omp parallel for schedule(static)
    for(int jj = 0; jj < J; jj++){
        for(int k = 0; k < N; k++){
            double q = 0.0;
            for(int m = 0; m <= NM; m++){
                const int edge = (m == 0 || 2 * m == N);
                const double a = 2.0 * M_PI * (double)((long)m * k % N) / N;
                q += (edge ? 1.0 : 2.0) * (Ac[(size_t)m * J + jj] * cos(a) + (edge ? 0.0 : As[(size_t)m * J + jj] * sin(a)));
            }
            q /= N;
            for(int i = 1; i < im-1; i++) P[IDX(i, jj + 1, k)] += q;
        }
    }
    free(R); free(Ac); free(As);
}

/* One colour of red-black LINE relaxation of the folded operator: columns (j,k) with
 * (j + k) & 1 == colour are solved exactly in r (Thomas; the radial ends folded into the first and
 * last rows as PressureSolver.h:547-550 does), their horizontal neighbours -- the other colour, or
 * the column itself through the theta fold -- held at their current values, then over-relaxed:
 * p += omega (p_line - p). The reference's PRESS_LINE (:497-570) on the folded operator. */
static void line_colour(const aturan_params* p, const double* rad, const double* st, double* P,
                        const double* src, int colour, double omega){
    const int im = p->im, jm = p->jm, km = p->km;
    const int n = im - 2;
    #pragma omp parallel
    {
        double* aa = (double*)malloc(sizeof(double) * n);
        double* bb = (double*)malloc(sizeof(double) * n);
        double* cc = (double*)malloc(sizeof(double) * n);
        double* dd = (double*)malloc(sizeof(double) * n);
        #pragma omp for collapse(2) schedule(static)
        for(int j = 1; j < jm-1; j++){
            for(int k = 0; k < km-1; k++){
                if(((j + k) & 1) != colour) continue;
                const int kw = phi_wrap(k-1, km), ke = phi_wrap(k+1, km);
                for(int i = 1; i < im-1; i++){
                    pweights_t w; press_weights(p, rad, st, i, j, &w);
                    double d = w.den;
                    double hj;
                    const double ajm = (j == 1)    ? (d -= C43 * w.num2, -C13 * P[IDX(i,j+1,k)]) : P[IDX(i,j-1,k)];
                    const double ajp = (j == jm-2) ? (d -= C43 * w.num2, -C13 * P[IDX(i,j-1,k)]) : P[IDX(i,j+1,k)];
                    hj = (ajp + ajm) * w.num2 + (P[IDX(i,j,ke)] + P[IDX(i,j,kw)]) * w.num3;
                    const int q = i - 1;
                    aa[q] = -w.num1; cc[q] = -w.num1; bb[q] = d;
                    dd[q] = hj - src[IDX(i,j,k)];
                }
                /* radial folds: p0 = c43 p1 - c13 p2 (row 1), p_{im-1} = c43 p_{im-2} - c13 p_{im-3} */
                bb[0] += aa[0] * C43; cc[0] -= aa[0] * C13; aa[0] = 0.0;
                bb[n-1] += cc[n-1] * C43; aa[n-1] -= cc[n-1] * C13; cc[n-1] = 0.0;
                double cprev = cc[0] / bb[0];
                dd[0] = dd[0] / bb[0];
                cc[0] = cprev;
                for(int q = 1; q < n; q++){
                    const double dn = bb[q] - aa[q] * cc[q-1];
                    cc[q] = cc[q] / dn;
                    dd[q] = (dd[q] - aa[q] * dd[q-1]) / dn;
                }
                double x = dd[n-1];
                P[IDX(n, j, k)] += omega * (x - P[IDX(n, j, k)]);
                for(int q = n - 2; q >= 0; q--){
                    x = dd[q] - cc[q] * x;
                    P[IDX(q+1, j, k)] += omega * (x - P[IDX(q+1, j, k)]);
                }
            }
        }
        free(aa); free(bb); free(cc); free(dd);
    }
}

/* Red-black line SOR on the shared solver's equation to a relative residual (no reference oracle:
 * the reference's PRESS_LINE sweeps a fixed count). The column-uniform correction runs before
 * iterations 0, 8, 16, ...: with exact column solves the first correction removes the
 * column-uniform error and later ones do not change the rate. The GPU's RB_LINE runs the same
 * sequence. Returns 0 at tol, 1 at the iteration cap. */
int oracle_pressure_line(const aturan_params* p, double* const* f, double omega, int max_iter,
                         double tol, int* iters_done, double* resid){
    const int im = p->im, jm = p->jm, km = p->km;
    double* rad = (double*)malloc(sizeof(double) * im);
    double* the = (double*)malloc(sizeof(double) * jm);
    double* st  = (double*)malloc(sizeof(double) * jm);
    double* src = (double*)malloc(sizeof(double) * (size_t)im * jm * km);
    oracle_coords(p, rad, the);
    press_sin_table(p, the, st, 1);
    oracle_pressure_source_compat(p, f, src);
    double* P = f[ATURAN_P_DYN];
    int s = 0; double r = folded_residual(p, rad, st, P, src);
    while(s < max_iter && !(r <= tol)){
        if(s % 8 == 0) column_correction(p, rad, st, P, src);
        line_colour(p, rad, st, P, src, 0, omega);
        line_colour(p, rad, st, P, src, 1, omega);
        s++;
        r = folded_residual(p, rad, st, P, src);
    }
    p_dyn_bcs(p, P);
    if(iters_done) *iters_done = s;
    if(resid) *resid = r;
    free(rad); free(the); free(st); free(src);
    return r <= tol ? 0 : 1;
}

/* Red-black SOR on the shared solver's equation to a relative residual, with the column-uniform
 * correction before every block of check_every sweeps (no reference oracle exists for a
 * converged solve: the reference sweeps a fixed count at omega = 1). The GPU's RB_SOR runs the
 * same sequence. Returns 0 when the relative L2 residual reached tol, 1 at the sweep cap. */
int oracle_pressure_sor(const aturan_params* p, double* const* f, double omega, int max_sweeps,
                        double tol, int check_every, int* sweeps_done, double* resid){
    const int im = p->im, jm = p->jm, km = p->km;
    double* rad = (double*)malloc(sizeof(double) * im);
    double* the = (double*)malloc(sizeof(double) * jm);
    double* st  = (double*)malloc(sizeof(double) * jm);
    double* src = (double*)malloc(sizeof(double) * (size_t)im * jm * km);
    oracle_coords(p, rad, the);
    press_sin_table(p, the, st, 1);
    oracle_pressure_source_compat(p, f, src);
    double* P = f[ATURAN_P_DYN];
    if(check_every < 1) check_every = 1;
    int s = 0; double r = folded_residual(p, rad, st, P, src);
    while(s < max_sweeps && !(r <= tol)){
        column_correction(p, rad, st, P, src);
        for(int n = 0; n < check_every && s < max_sweeps; n++, s++){
            rbf_colour(p, rad, st, P, src, 0, omega);
            rbf_colour(p, rad, st, P, src, 1, omega);
        }
        r = folded_residual(p, rad, st, P, src);
    }
    p_dyn_bcs(p, P);
    if(sweeps_done) *sweeps_done = s;
    if(resid) *resid = r;
    free(rad); free(the); free(st); free(src);
    return r <= tol ? 0 : 1;
}

/* ---- The transposed folded operator, for the adjoint of the pressure solve (no reference
 * counterpart: the reference has no adjoint). Lc^T has Lc's sparsity, so red-black point and line
 * relaxation apply unchanged in structure; what changes is where the fold coefficients sit:
 * row (1,j,k) of Lc puts num1 (1 - c13) on (2,j,k) and nothing on (0,j,k), so column (2,j,k) of
 * Lc -- row (2,j,k) of Lc^T -- carries num1 (1 - c13) from (1,j,k); likewise at i = im-2 and in
 * theta at j = 1, jm-2. The left null vector of Lc^T is the constant (Lc's rows sum to zero), so
 * a right-hand side is made compatible by removing its plain mean. The coarse correction swaps
 * the roles of the two radial null vectors: its trial functions are y_i q(j,k) (the radial block
 * of Lc^T annihilates y, as y^T T_r = 0) and its test functions are the plain column sums (the
 * constant annihilates it from the left, as T_r 1 = 0), so sum_i (Lc^T (y q))_i = A2y L2^T q
 * exactly, A2y = sum_i y_i / rm_i^2. ---- */
static double folded_accT(const aturan_params* p, const double* rad, const double* st, const double* L,
                          int i, int j, int k, double* diag){
    const int im = p->im, jm = p->jm, km = p->km;
    const int kw = phi_wrap(k-1, km), ke = phi_wrap(k+1, km);
    pweights_t w; press_weights(p, rad, st, i, j, &w);
    double d = w.den;
    if(i == 1)    d -= C43 * w.num1;
    if(i == im-2) d -= C43 * w.num1;
    if(j == 1)    d -= C43 * w.num2;
    if(j == jm-2) d -= C43 * w.num2;
    *diag = d;
    double acc = (L[IDX(i,j,ke)] + L[IDX(i,j,kw)]) * w.num3;
    pweights_t v;
    if(i - 1 >= 1){ press_weights(p, rad, st, i-1, j, &v); acc += v.num1 * (i - 1 == 1 ? 1.0 - C13 : 1.0) * L[IDX(i-1,j,k)]; }
    if(i + 1 <= im-2){ press_weights(p, rad, st, i+1, j, &v); acc += v.num1 * (i + 1 == im-2 ? 1.0 - C13 : 1.0) * L[IDX(i+1,j,k)]; }
    if(j - 1 >= 1){ press_weights(p, rad, st, i, j-1, &v); acc += v.num2 * (j - 1 == 1 ? 1.0 - C13 : 1.0) * L[IDX(i,j-1,k)]; }
    if(j + 1 <= jm-2){ press_weights(p, rad, st, i, j+1, &v); acc += v.num2 * (j + 1 == jm-2 ? 1.0 - C13 : 1.0) * L[IDX(i,j+1,k)]; }
    return acc;
}

/* out = Lc x (tr = 0) or Lc^T x (tr = 1) on the interior of a [im][jm][km] field. */
int oracle_laplace_apply(const aturan_params* p, const double* x, double* out, int tr){
    const int im = p->im, jm = p->jm, km = p->km;
    double* rad = (double*)malloc(sizeof(double) * im);
    double* the = (double*)malloc(sizeof(double) * jm);
    double* st  = (double*)malloc(sizeof(double) * jm);
    oracle_coords(p, rad, the);
    press_sin_table(p, the, st, 1);
    memset(out, 0, sizeof(double) * (size_t)im * jm * km);
    #pragma omp parallel for collapse(2) schedule(static)
    for(int i = 1; i < im-1; i++) for(int j = 1; j < jm-1; j++){
        pweights_t w; press_weights(p, rad, st, i, j, &w);
        for(int k = 0; k < km-1; k++){
            double diag, acc;
            if(tr) acc = folded_accT(p, rad, st, x, i, j, k, &diag);
            else   acc = folded_acc(p, x, i, j, k, &w, &diag);
            out[IDX(i,j,k)] = acc - diag * x[IDX(i,j,k)];
        }
    }
    free(rad); free(the); free(st);
    return 0;
}

static double residualT(const aturan_params* p, const double* rad, const double* st, const double* L, const double* g){
    const int im = p->im, jm = p->jm, km = p->km;
    double rr = 0.0, ss = 0.0;
    #pragma omp parallel for collapse(2) reduction(+:rr,ss) schedule(static)
    for(int i = 1; i < im-1; i++) for(int j = 1; j < jm-1; j++) for(int k = 0; k < km-1; k++){
        double diag;
        const double acc = folded_accT(p, rad, st, L, i, j, k, &diag);
        const double r = g[IDX(i,j,k)] - (acc - diag * L[IDX(i,j,k)]);
        rr += r * r; ss += g[IDX(i,j,k)] * g[IDX(i,j,k)];
    }
    return ss > 0.0 ? sqrt(rr / ss) : sqrt(rr);
}

static void rbT_colour(const aturan_params* p, const double* rad, const double* st, double* L, const double* g,
                       int colour, double omega){
    const int im = p->im, jm = p->jm, km = p->km;
    #pragma omp parallel for collapse(2) schedule(static)
    for(int i = 1; i < im-1; i++) for(int j = 1; j < jm-1; j++) for(int k = 0; k < km-1; k++){
        if(((i + j + k) & 1) != colour) continue;
        double diag;
        const double acc = folded_accT(p, rad, st, L, i, j, k, &diag);
        const double ln = (acc - g[IDX(i,j,k)]) / diag;
        L[IDX(i,j,k)] += omega * (ln - L[IDX(i,j,k)]);
    }
}

/* Line relaxation of Lc^T: per column the transposed radial tridiagonal (sub-diagonal from the
 * row below's super-diagonal and the other way round), horizontal neighbours from the transposed
 * theta and phi couplings. */
static void lineT_colour(const aturan_params* p, const double* rad, const double* st, double* L, const double* g,
                         int colour, double omega){
    const int im = p->im, jm = p->jm, km = p->km;
    const int n = im - 2;
    #pragma omp parallel
    {
        double* aa = (double*)malloc(sizeof(double) * n);
        double* bb = (double*)malloc(sizeof(double) * n);
        double* cc = (double*)malloc(sizeof(double) * n);
        double* dd = (double*)malloc(sizeof(double) * n);
        #pragma omp for collapse(2) schedule(static)
        for(int j = 1; j < jm-1; j++) for(int k = 0; k < km-1; k++){
            if(((j + k) & 1) != colour) continue;
            const int kw = phi_wrap(k-1, km), ke = phi_wrap(k+1, km);
            for(int i = 1; i < im-1; i++){
                pweights_t w, v; press_weights(p, rad, st, i, j, &w);
                double d = w.den;
                if(i == 1)    d -= C43 * w.num1;
                if(i == im-2) d -= C43 * w.num1;
                if(j == 1)    d -= C43 * w.num2;
                if(j == jm-2) d -= C43 * w.num2;
                double h = (L[IDX(i,j,ke)] + L[IDX(i,j,kw)]) * w.num3;
                if(j - 1 >= 1){ press_weights(p, rad, st, i, j-1, &v); h += v.num2 * (j - 1 == 1 ? 1.0 - C13 : 1.0) * L[IDX(i,j-1,k)]; }
                if(j + 1 <= jm-2){ press_weights(p, rad, st, i, j+1, &v); h += v.num2 * (j + 1 == jm-2 ? 1.0 - C13 : 1.0) * L[IDX(i,j+1,k)]; }
                const int q = i - 1;
                double sub = 0.0, sup = 0.0;
                if(i - 1 >= 1){ press_weights(p, rad, st, i-1, j, &v); sub = -v.num1 * (i - 1 == 1 ? 1.0 - C13 : 1.0); }
                if(i + 1 <= im-2){ press_weights(p, rad, st, i+1, j, &v); sup = -v.num1 * (i + 1 == im-2 ? 1.0 - C13 : 1.0); }
                aa[q] = sub; bb[q] = d; cc[q] = sup;
                dd[q] = h - g[IDX(i,j,k)];
            }
            cc[0] = cc[0] / bb[0];
            dd[0] = dd[0] / bb[0];
            for(int q = 1; q < n; q++){
                const double dn = bb[q] - aa[q] * cc[q-1];
                cc[q] = cc[q] / dn;
                dd[q] = (dd[q] - aa[q] * dd[q-1]) / dn;
            }
            double x = dd[n-1];
            L[IDX(n, j, k)] += omega * (x - L[IDX(n, j, k)]);
            for(int q = n - 2; q >= 0; q--){
                x = dd[q] - cc[q] * x;
                L[IDX(q+1, j, k)] += omega * (x - L[IDX(q+1, j, k)]);
            }
        }
        free(aa); free(bb); free(cc); free(dd);
    }
}

/* The coarse correction of the transposed system: A2y L2^T q = sum_i r_i, then y_i q added to
 * level i; per Fourier mode the transposed theta tridiagonal (the folds' c13 terms move to the
 * neighbouring rows). Mode 0 is singular, left null vector 1 and right null vector y_j: its
 * right-hand side is made zero-sum and q pinned at the first row (which fixes the multiple of y). */
static void column_correction_T(const aturan_params* p, const double* rad, const double* st, double* L, const double* g){
    const int im = p->im, jm = p->jm, km = p->km;
    const int J = jm - 2, N = km - 1, NM = N / 2;
    double* R  = (double*)calloc((size_t)J * N, sizeof(double));
    double* Ac = (double*)calloc((size_t)(NM + 1) * J, sizeof(double));
    double* As = (double*)calloc((size_t)(NM + 1) * J, sizeof(double));
    double A2 = 0.0;
    for(int i = 1; i < im-1; i++){ const double rm = metric_radius(p, rad[i]); A2 += ((i == 1 || i == im-2) ? 1.5 : 1.0) / (rm * rm); }
    #pragma omp parallel for schedule(static)
    for(int jj = 0; jj < J; jj++){
        const int j = jj + 1;
        for(int k = 0; k < N; k++){
            double acc_r = 0.0;
            for(int i = 1; i < im-1; i++){
                double diag;
                const double acc = folded_accT(p, rad, st, L, i, j, k, &diag);
                acc_r += g[IDX(i,j,k)] - (acc - diag * L[IDX(i,j,k)]);
            }
            R[(size_t)jj * N + k] = acc_r;
        }
    }
    const double e = 1.0 / (p->dthe * p->dthe), inv_dphi2 = 1.0 / (p->dphi * p->dphi);
    #pragma omp parallel for schedule(static)
    for(int m = 0; m <= NM; m++){
        double* cp = (double*)malloc(sizeof(double) * J);
        double* dp = (double*)malloc(sizeof(double) * J);
        for(int jj = 0; jj < J; jj++){
            double sc = 0.0, ss = 0.0;
            for(int k = 0; k < N; k++){
                const double a = 2.0 * M_PI * (double)((long)m * k % N) / N;
                const double v = R[(size_t)jj * N + k] / A2;
                sc += v * cos(a); ss += v * sin(a);
            }
            Ac[(size_t)m * J + jj] = sc; As[(size_t)m * J + jj] = ss;
        }
        const double sl = sin(M_PI * m / N);
        const double lam = 4.0 * sl * sl * inv_dphi2;
        for(int part = 0; part < 2; part++){
            double* d = (part == 0 ? Ac : As) + (size_t)m * J;
            if(part == 1 && (m == 0 || 2 * m == N)){ for(int q = 0; q < J; q++) d[q] = 0.0; continue; }
            if(m == 0){
                double sr = 0.0;
                for(int q = 0; q < J; q++) sr += d[q];
                for(int q = 0; q < J; q++) d[q] -= sr / J;
            }
            /* transposed rows: sub(q) = super_fwd(q-1), super(q) = sub_fwd(q+1) */
            #define TA(q) ((q) == 0 ? 0.0 : ((q) == 1 ? e - C13 * e : e))
            #define TB(q) (-2.0 * e - lam / (st[(q)+1] * st[(q)+1]) + (((q) == 0 || (q) == J-1) ? C43 * e : 0.0))
            #define TC(q) ((q) == J-1 ? 0.0 : ((q) == J-2 ? e - C13 * e : e))
            double b0 = TB(0), c0 = TC(0), d0 = d[0];
            if(m == 0){ b0 = 1.0; c0 = 0.0; d0 = 0.0; }
            cp[0] = c0 / b0; dp[0] = d0 / b0;
            for(int q = 1; q < J; q++){
                const double dn = TB(q) - TA(q) * cp[q-1];
                cp[q] = TC(q) / dn;
                dp[q] = (d[q] - TA(q) * dp[q-1]) / dn;
            }
            #undef TA
            #undef TB
            #undef TC
            d[J-1] = dp[J-1];
            for(int q = J-2; q >= 0; q--) d[q] = dp[q] - cp[q] * d[q+1];
        }
        free(cp); free(dp);
    }
    #pragma omp parallel for schedule(static)
    for(int jj = 0; jj < J; jj++){
        for(int k = 0; k < N; k++){
            double q = 0.0;
            for(int m = 0; m <= NM; m++){
                const int edge = (m == 0 || 2 * m == N);
                const double a = 2.0 * M_PI * (double)((long)m * k % N) / N;
                q += (edge ? 1.0 : 2.0) * (Ac[(size_t)m * J + jj] * cos(a) + (edge ? 0.0 : As[(size_t)m * J + jj] * sin(a)));
            }
            q /= N;
            for(int i = 1; i < im-1; i++) L[IDX(i, jj + 1, k)] += ((i == 1 || i == im-2) ? 1.5 : 1.0) * q;
        }
    }
    free(R); free(Ac); free(As);
}

/* Solve Lc x = b (tr = 0) or Lc^T x = b (tr = 1) on the interior to a relative residual, by point
 * (line = 0, check and correction every 16 sweeps) or line (line = 1, check every iteration,
 * correction every 8) red-black SOR from the given x. b is first made compatible (its component
 * along the operator's left null vector removed: y_i y_j for Lc, the constant for Lc^T); the
 * boundary rows of x are not touched. Returns 0 at tol, 1 at the cap. */
int oracle_solve(const aturan_params* p, const double* b_in, double* x, int tr, int line, double omega,
                 int max_iter, double tol, int* iters_done, double* resid){
    const int im = p->im, jm = p->jm, km = p->km;
    const size_t NF = (size_t)im * jm * km;
    double* rad = (double*)malloc(sizeof(double) * im);
    double* the = (double*)malloc(sizeof(double) * jm);
    double* st  = (double*)malloc(sizeof(double) * jm);
    double* b   = (double*)malloc(sizeof(double) * NF);
    oracle_coords(p, rad, the);
    press_sin_table(p, the, st, 1);
    memcpy(b, b_in, sizeof(double) * NF);
    if(!tr) compat_shift(p, b);
    else {
        double sm = 0.0; long nn = 0;
        for(int i = 1; i < im-1; i++) for(int j = 1; j < jm-1; j++) for(int k = 0; k < km-1; k++){ sm += b[IDX(i,j,k)]; nn++; }
        for(int i = 1; i < im-1; i++) for(int j = 1; j < jm-1; j++) for(int k = 0; k < km-1; k++) b[IDX(i,j,k)] -= sm / nn;
    }
    const int check_every = line ? 1 : 16, every = line ? 8 : 16;
    int s = 0;
    double r = tr ? residualT(p, rad, st, x, b) : folded_residual(p, rad, st, x, b);
    while(s < max_iter && !(r <= tol)){
        if(s % every == 0){ if(tr) column_correction_T(p, rad, st, x, b); else column_correction(p, rad, st, x, b); }
        for(int n = 0; n < check_every && s < max_iter; n++, s++){
            for(int colour = 0; colour < 2; colour++){
                if(tr){ if(line) lineT_colour(p, rad, st, x, b, colour, omega); else rbT_colour(p, rad, st, x, b, colour, omega); }
                else  { if(line) line_colour(p, rad, st, x, b, colour, omega);  else rbf_colour(p, rad, st, x, b, colour, omega); }
            }
        }
        r = tr ? residualT(p, rad, st, x, b) : folded_residual(p, rad, st, x, b);
    }
    if(iters_done) *iters_done = s;
    if(resid) *resid = r;
    free(rad); free(the); free(st); free(b);
    return r <= tol ? 0 : 1;
}

/* ---- SaturationAdjustment.h:255-746 for one gas, the non-diagnostic arithmetic ---- */
int oracle_satadj(const aturan_params* p, double* const* f, int gas, long* n_adjusted, long* n_noconv){
    const int im = p->im, jm = p->jm, km = p->km;
    const aturan_gas* G = &p->gas[gas];
    static const int base[4] = { ATURAN_H2O, ATURAN_H2S, ATURAN_NH3, ATURAN_CH4 };
    double* c = f[base[gas]]; double* cloud = f[base[gas] + 1]; double* ice = f[base[gas] + 2];
    double* tt = f[ATURAN_T];
    const double* ps = f[ATURAN_P_STAT];
    const double* rho_mix = f[ATURAN_RHO_MIX];
    const double t_0 = G->t_0, t_00 = G->t_00, ep = G->ep, lv = G->lv, ls = G->ls;
    const double C = G->C, L0 = G->L0, R = G->R, del_alf = G->del_alf, del_bet = G->del_bet;
    const double C_i = G->C_i, L0_i = G->L0_i, del_alf_i = G->del_alf_i, del_bet_i = G->del_bet_i;
    const double t_range_inv = 1.0 / (t_0 - t_00);
    const int conserve = p->satadj_conserve, newton = p->satadj_newton, evap = p->satadj_evap;
    const int ice_entry = p->satadj_ice_entry, bergeron = p->satadj_bergeron;
    const int freeze_on = p->satadj_freeze && conserve && t_00 > 0.0 && t_00 < t_0;
    const int dry_exit = p->satadj_dry_exit;
    const double Lf = ls - lv;
    const double cp_mix = p->cp_mix, t_ref = p->t_ref;
    const int iter_prec_end = 15;
    const double q_diff_min = 1.0e-3;
    /* the stopping test (:551), the reference's 1e-3 unless satadj_stop_tol asks for a tighter one;
       the entry test (:446) keeps 1e-3 */
    const double q_stop = p->satadj_stop_tol > 0.0 ? p->satadj_stop_tol : q_diff_min;
    /* the entry band (:446): 1e-3 unless satadj_entry_tol asks for another (< 0: none) */
    const double q_entry_band = p->satadj_entry_tol == 0.0 ? q_diff_min
                              : (p->satadj_entry_tol < 0.0 ? 0.0 : p->satadj_entry_tol);
    long nadj = 0, nnc = 0;

    #pragma omp parallel for collapse(2) schedule(static) reduction(+:nadj,nnc)
    for(int k = 0; k < km; k++){
        for(int j = 0; j < jm; j++){
            for(int i = 0; i < im; i++){
                const size_t q = IDX(i,j,k);
                double t_u = tt[q] * t_ref;
                const double p_u = ps[q];
                if(!(t_u > 0.0) || !(p_u > 0.0)) continue;
                /* rho_at (cUranusModel.h:526-531) */
                double rho_c = p->r_mix;
                if(p->local_rho){ const double r_ = rho_mix[q]; rho_c = (r_ > 0.0 && isfinite(r_)) ? r_ : p->r_mix; }

                if(t_u > t_0){
                    if(conserve){
                        if(ice[q] > 0.0){
                            double dm = ice[q];
                            if(Lf > 0.0){
                                const double hc  = cp_mix * rho_c;
                                const double cap = hc * (t_u - t_0) / Lf;
                                if(dm > cap) dm = cap;
                                t_u -= Lf * dm / hc;
                                tt[q] = t_u / t_ref;
                            }
                            ice[q]   -= dm;
                            cloud[q] += dm;
                        }
                    } else {
                        ice[q] = 0.0;
                    }
                }
                if(freeze_on && t_u < t_00 && cloud[q] > 0.0){
                    double dm = cloud[q];
                    if(Lf > 0.0){
                        const double hc  = cp_mix * rho_c;
                        const double cap = hc * (t_00 - t_u) / Lf;
                        if(dm > cap) dm = cap;
                        t_u += Lf * dm / hc;
                        tt[q] = t_u / t_ref;
                    }
                    cloud[q] -= dm;
                    ice[q]   += dm;
                }
                if(c[q]     < 0.0) c[q]     = 0.0;
                if(cloud[q] < 0.0) cloud[q] = 0.0;
                if(ice[q]   < 0.0) ice[q]   = 0.0;

                const double E_Rain_0 = svp(t_u, C, L0, R, del_alf, del_bet);
                const double q_Rain_0 = rho_c * ep * E_Rain_0 / p_u;
                if(q_Rain_0 <= 0.0) continue;
                double q_entry = q_Rain_0;
                if(ice_entry && cloud[q] <= 0.0 && ice[q] <= 0.0){
                    const double cnd0 = t_u <= t_00 ? 0.0 : (t_u >= t_0 ? 1.0 : (t_u - t_00) * t_range_inv);
                    if(cnd0 < 1.0)
                        q_entry = cnd0 * q_Rain_0 + (1.0 - cnd0) * rho_c * ep
                                * svp(t_u, C_i, L0_i, R, del_alf_i, del_bet_i) / p_u;
                }
                if(bergeron >= 2 && cloud[q] <= 0.0 && ice[q] <= 0.0 && t_u < t_0)
                    q_entry = rho_c * ep * svp(t_u, C_i, L0_i, R, del_alf_i, del_bet_i) / p_u;
                if(c[q] <= q_entry){
                    const double q_c0 = cloud[q], q_i0 = ice[q];
                    if(!evap || !conserve || (q_c0 <= 0.0 && q_i0 <= 0.0)) continue;
                    const double q_Ice_0 = rho_c * ep * svp(t_u, C_i, L0_i, R, del_alf_i, del_bet_i) / p_u;
                    double q_t0;
                    if(q_c0 > 0.0 && q_i0 > 0.0) q_t0 = (q_c0 * q_Rain_0 + q_i0 * q_Ice_0) / (q_c0 + q_i0);
                    else if(q_i0 <= 0.0)         q_t0 = q_Rain_0;
                    else                         q_t0 = q_Ice_0;
                    if(fabs(c[q] - q_t0) <= q_entry_band * q_t0) continue;
                }

                double q_v_b = c[q], q_c_b = cloud[q], q_i_b = ice[q];
                double T = t_u, q_v_hyp = q_v_b;
                int cell_found = 0, cell_dry = 0;
                double q_rain_now = q_Rain_0;
                for(int itr = 1; itr <= iter_prec_end; itr++){
                    double CND = (T - t_00) * t_range_inv;
                    double DEP = (t_0 - T)  * t_range_inv;
                    if(T <= t_00){ CND = 0.0; DEP = 1.0; }
                    if(T >= t_0) { CND = 1.0; DEP = 0.0; }
                    const int berg = bergeron != 0 && T < t_0 && q_v_b <= q_rain_now
                                   && (q_i_b > 0.0 || (bergeron >= 2 && q_c_b <= 0.0));
                    if(berg){
                        CND = 0.0; DEP = 1.0;
                        if(q_c_b > 0.0){
                            T     -= lv * q_c_b / (cp_mix * rho_c);
                            q_v_b += q_c_b;
                            q_c_b  = 0.0;
                        }
                    }
                    double d_q_v = q_v_hyp - q_v_b;
                    double d_q_c = -d_q_v * CND;
                    double d_q_i = -d_q_v * DEP;
                    if(conserve){
                        if(d_q_v < -q_v_b){ d_q_v = -q_v_b; d_q_c = -d_q_v * CND; d_q_i = -d_q_v * DEP; }
                        if(q_c_b + d_q_c < 0.0){ const double ex = -(q_c_b + d_q_c); d_q_c = -q_c_b; d_q_i -= ex; }
                        if(q_i_b + d_q_i < 0.0){ const double ex = -(q_i_b + d_q_i); d_q_i = -q_i_b; d_q_c -= ex;
                                                 if(q_c_b + d_q_c < 0.0) d_q_c = -q_c_b; }
                        d_q_v = -(d_q_c + d_q_i);
                    }
                    T     += (lv * d_q_c + ls * d_q_i) / (cp_mix * rho_c);
                    q_v_b += d_q_v;
                    q_c_b += d_q_c;
                    q_i_b += d_q_i;
                    if(q_v_b < 0.0) q_v_b = 0.0;
                    if(q_c_b < 0.0) q_c_b = 0.0;
                    if(q_i_b < 0.0) q_i_b = 0.0;

                    const double E_Rain = svp(T, C,   L0,   R, del_alf,   del_bet);
                    const double E_Ice  = svp(T, C_i, L0_i, R, del_alf_i, del_bet_i);
                    const double q_Rain = rho_c * ep * E_Rain / p_u;
                    const double q_Ice  = rho_c * ep * E_Ice  / p_u;
                    q_rain_now = q_Rain;
                    if(q_c_b > 0.0 && q_i_b > 0.0)
                        q_v_hyp = (q_c_b * q_Rain + q_i_b * q_Ice) / (q_c_b + q_i_b);
                    else if(bergeron >= 2 && q_c_b <= 0.0 && q_i_b <= 0.0 && T < t_0) q_v_hyp = q_Ice;
                    else if(ice_entry && q_c_b <= 0.0 && q_i_b <= 0.0){
                        const double cn = T <= t_00 ? 0.0 : (T >= t_0 ? 1.0 : (T - t_00) * t_range_inv);
                        q_v_hyp = cn * q_Rain + (1.0 - cn) * q_Ice; }
                    else if(q_i_b == 0.0) q_v_hyp = q_Rain;
                    else                  q_v_hyp = q_Ice;

                    if(T >= t_0){
                        if(conserve){
                            if(q_i_b > 0.0){
                                double dm = q_i_b;
                                if(Lf > 0.0){
                                    const double hc  = cp_mix * rho_c;
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
                    if(q_diff <= q_stop){ cell_found = 1; break; }
                    if(dry_exit && conserve && q_c_b <= 0.0 && q_i_b <= 0.0 && q_v_b < q_v_hyp){ cell_dry = 1; break; }
                    if(newton){
                        const double dT = 0.1;
                        const double q_Rain_d = rho_c * ep * svp(T + dT, C,   L0,   R, del_alf,   del_bet)   / p_u;
                        const double q_Ice_d  = rho_c * ep * svp(T + dT, C_i, L0_i, R, del_alf_i, del_bet_i) / p_u;
                        double q_hyp_d;
                        if(q_c_b > 0.0 && q_i_b > 0.0)
                            q_hyp_d = (q_c_b * q_Rain_d + q_i_b * q_Ice_d) / (q_c_b + q_i_b);
                        else if(bergeron >= 2 && q_c_b <= 0.0 && q_i_b <= 0.0 && T < t_0) q_hyp_d = q_Ice_d;
                        else if(ice_entry && q_c_b <= 0.0 && q_i_b <= 0.0){
                            const double cn = T <= t_00 ? 0.0 : (T >= t_0 ? 1.0 : (T - t_00) * t_range_inv);
                            q_hyp_d = cn * q_Rain_d + (1.0 - cn) * q_Ice_d; }
                        else if(q_i_b == 0.0) q_hyp_d = q_Rain_d;
                        else                  q_hyp_d = q_Ice_d;
                        double CNDn = (T - t_00) * t_range_inv;
                        if(T <= t_00) CNDn = 0.0;
                        if(T >= t_0)  CNDn = 1.0;
                        if(berg)      CNDn = 0.0;
                        const double Gf = (lv * CNDn + ls * (1.0 - CNDn)) / (cp_mix * rho_c)
                                        * (q_hyp_d - q_v_hyp) / dT;
                        double wn = 1.0 / (1.0 + stdmax(Gf, 0.0));
                        if(wn < 0.05) wn = 0.05;
                        q_v_hyp = q_v_b + wn * (q_v_hyp - q_v_b);
                    } else {
                        q_v_hyp = 0.5 * (q_v_hyp + q_v_b);
                    }
                }
                nadj++;
                if(!cell_found && !cell_dry) nnc++;
                c[q] = q_v_b; cloud[q] = q_c_b; ice[q] = q_i_b;
                tt[q] = T / t_ref;
            }
        }
    }
    /* final clamp (:673-685) */
    #pragma omp parallel for collapse(2) schedule(static)
    for(int k = 0; k < km; k++) for(int j = 0; j < jm; j++) for(int i = 0; i < im; i++){
        const size_t q = IDX(i,j,k);
        if(c[q]     <= 0.0) c[q]     = 0.0;
        if(cloud[q] <= 0.0) cloud[q] = 0.0;
        if(ice[q]   <= 0.0) ice[q]   = 0.0;
    }
    if(n_adjusted) *n_adjusted = nadj;
    if(n_noconv) *n_noconv = nnc;
    return 0;
}

/* cUranusModel.cpp:1049-1073, ATURAN_RK_SCALAR_SYNC=2 */
int oracle_sync_ncopies(const aturan_params* p, double* const* f){
    const size_t N = (size_t)p->im * p->jm * p->km;
    for(int q = ATURAN_CH4; q <= ATURAN_NH3_ICE; q++) memcpy(f[ATURAN_TN + q], f[q], sizeof(double) * N);
    memcpy(f[ATURAN_TN], f[ATURAN_T], sizeof(double) * N);
    if(p->nh4sh_sync) memcpy(f[ATURAN_NH4SHN], f[ATURAN_NH4SH], sizeof(double) * N);
    return 0;
}

/* cUranusModel.cpp:967-1123, the in-scope calls of one even iteration in their order. */
int oracle_step(const aturan_params* p, double* const* f, int press_kind, double omega,
                int max_sweeps, double tol, double* ref_out){
    if(press_kind == ATURAN_PRESS_GS_LEX) oracle_pressure_gs(p, f);
    else if(press_kind == ATURAN_PRESS_RB_SHARED) oracle_pressure_rb(p, f, max_sweeps);
    else if(press_kind == ATURAN_PRESS_RB_LINE) { int s; double r; oracle_pressure_line(p, f, omega, max_sweeps, tol, &s, &r); }
    else { int s; double r; oracle_pressure_sor(p, f, omega, max_sweeps, tol, 16, &s, &r); }
    for(int g = 0; g < 4; g++) oracle_satadj(p, f, g, NULL, NULL);
    oracle_sync_ncopies(p, f);
    return oracle_rk4(p, f, ref_out);
}

/* ---- after RungeKuttaUran: filters, boundary passes, species clamp (cUranusModel.cpp:1218-1248) ---- */

/* The reference's boundary lists (BC_Uran.cpp:21-88) restricted to the fields the library holds. */
static const int POST_RADIUS[] = { ATURAN_T, ATURAN_U, ATURAN_V, ATURAN_W,
    ATURAN_CH4, ATURAN_CH4_CLOUD, ATURAN_CH4_ICE, ATURAN_H2O, ATURAN_H2O_CLOUD, ATURAN_H2O_ICE,
    ATURAN_H2S, ATURAN_H2S_CLOUD, ATURAN_H2S_ICE, ATURAN_NH3, ATURAN_NH3_CLOUD, ATURAN_NH3_ICE,
    ATURAN_NH4SH, ATURAN_MASSFLUX_H2S, ATURAN_MASSFLUX_NH3, ATURAN_MASSFLUX_NH4SH,
    ATURAN_FLUXLIM_NH4SH, ATURAN_THERMALMASSFLUX, ATURAN_DIFFLUX_H2S, ATURAN_DIFFLUX_NH3, ATURAN_DIFFLUX_NH4SH };
/* BC_Uran.cpp:73-88: the phi list is the radius list without difflux_nh4sh (the last entry above) */
#define POST_NPHI (NELEM(POST_RADIUS) - 1)
static const int POST_THETA_EXTRAP[] = { ATURAN_T, ATURAN_U,
    ATURAN_CH4, ATURAN_CH4_CLOUD, ATURAN_CH4_ICE, ATURAN_H2O, ATURAN_H2O_CLOUD, ATURAN_H2O_ICE,
    ATURAN_H2S, ATURAN_H2S_CLOUD, ATURAN_H2S_ICE, ATURAN_NH3, ATURAN_NH3_CLOUD, ATURAN_NH3_ICE,
    ATURAN_NH4SH, ATURAN_THERMALMASSFLUX };
static const int POST_THETA_ZERO[] = { ATURAN_V, ATURAN_W, ATURAN_MASSFLUX_H2S, ATURAN_MASSFLUX_NH3,
    ATURAN_MASSFLUX_NH4SH, ATURAN_FLUXLIM_NH4SH, ATURAN_DIFFLUX_H2S, ATURAN_DIFFLUX_NH3, ATURAN_DIFFLUX_NH4SH };
/* BC_Uran.h:83-89 (species_fields), the order of the clamp's per-species sums */
static const int POST_SPECIES[ATURAN_NSPECIES] = { ATURAN_H2O, ATURAN_H2O_CLOUD, ATURAN_H2O_ICE,
    ATURAN_H2S, ATURAN_H2S_CLOUD, ATURAN_H2S_ICE, ATURAN_NH3, ATURAN_NH3_CLOUD, ATURAN_NH3_ICE,
    ATURAN_CH4, ATURAN_CH4_CLOUD, ATURAN_CH4_ICE, ATURAN_NH4SH };
#define NELEM(a) ((int)(sizeof(a) / sizeof((a)[0])))

/* BoundaryConditions.h (BCForm::apply) with the model default NEUMANN (cUranusModel.h:397) */
static double bc_form(int form, double a, double b, double c){
    const int f = (form == 0) ? 2 : form;
    if(f == 1) return a;
    if(f == 2) return C43 * a - C13 * b;
    return c - 3.0 * b + 3.0 * a;
}

/* lib/Utils.cpp:224-317, damp_wiggles without a surface (i_surface = nullptr): the 1-2-1 pass
 * along k (periodic ring of km-1 meridians when seam, with k = km-1 the copy of k = 0), then j
 * (clamped at the poles), then i (clamped at the ends), each from a copy of the field. */
static void post_damp(const aturan_params* p, double* x, int along_i, int along_j, int along_k,
                      double strength, int seam_periodic, double* tmp){
    const int im = p->im, jm = p->jm, km = p->km;
    const size_t N = (size_t)im * jm * km;
    const double coeff = strength * 0.25;
    if(along_k){
        memcpy(tmp, x, sizeof(double) * N);
        const int seam = seam_periodic && km > 2;
        const int k_end = seam ? km - 1 : km;
        for(int i = 0; i < im; i++) for(int j = 0; j < jm; j++){
            for(int k = 0; k < k_end; k++){
                const int km1 = seam ? (k == 0 ? km - 2 : k - 1) : (k - 1 + km) % km;
                const int kp1 = seam ? (k == km - 2 ? 0 : k + 1) : (k + 1) % km;
                const double c = tmp[IDX(i,j,k)];
                x[IDX(i,j,k)] = c + coeff * (tmp[IDX(i,j,km1)] - 2.0 * c + tmp[IDX(i,j,kp1)]);
            }
            if(seam) x[IDX(i,j,km-1)] = x[IDX(i,j,0)];
        }
    }
    if(along_j){
        memcpy(tmp, x, sizeof(double) * N);
        for(int i = 0; i < im; i++) for(int j = 0; j < jm; j++){
            const int jm1 = j - 1 < 0 ? 0 : j - 1, jp1 = j + 1 > jm - 1 ? jm - 1 : j + 1;
            for(int k = 0; k < km; k++){
                const double c = tmp[IDX(i,j,k)];
                x[IDX(i,j,k)] = c + coeff * (tmp[IDX(i,jm1,k)] - 2.0 * c + tmp[IDX(i,jp1,k)]);
            }
        }
    }
    if(along_i){
        memcpy(tmp, x, sizeof(double) * N);
        for(int j = 0; j < jm; j++) for(int k = 0; k < km; k++) for(int i = 0; i < im; i++){
            const int im1 = i - 1 < 0 ? 0 : i - 1, ip1 = i + 1 > im - 1 ? im - 1 : i + 1;
            const double c = tmp[IDX(i,j,k)];
            x[IDX(i,j,k)] = c + coeff * (tmp[IDX(im1,j,k)] - 2.0 * c + tmp[IDX(ip1,j,k)]);
        }
    }
}

static double post_max0(double x){ return (0.0 < x) ? x : 0.0; }   /* std::max(0.0, x) */

int oracle_post_step(const aturan_params* p, double* const* f, const aturan_post_params* pp,
                     double* clamp_added, long* clamp_cells){
    const int im = p->im, jm = p->jm, km = p->km;
    const size_t N = (size_t)im * jm * km;
    double* tmp = (double*)malloc(sizeof(double) * N);
    if(!tmp) return -1;
    /* cUranusModel.cpp:1218-1221: the t filter, horizontal passes then the radial one */
    if(pp->damp_t_horiz != 0.0) post_damp(p, f[ATURAN_T], 0, pp->damp_t_j, 1, pp->damp_t_horiz, pp->phi_periodic, tmp);
    if(pp->damp_t_vert != 0.0) post_damp(p, f[ATURAN_T], 1, 0, 0, pp->damp_t_vert, pp->phi_periodic, tmp);
    /* :1236-1240: the velocity filter, u then v then w, each along k, j, i */
    if(pp->vel_shapiro != 0.0)
        for(int q = ATURAN_U; q <= ATURAN_W; q++) post_damp(p, f[q], 1, 1, 1, pp->vel_shapiro, pp->phi_periodic, tmp);
    free(tmp);

    /* BoundaryConditions.h:152-286 (bcRadius; margin 0, no turbulence fields, no lid pin) */
    for(int j = 0; j < jm; j++) for(int k = 0; k < km; k++){
        for(int n = 0; n < NELEM(POST_RADIUS); n++){
            double* F = f[POST_RADIUS[n]];
            const int fb = (pp->bottom_form != 0 && POST_RADIUS[n] != ATURAN_U) ? pp->bottom_form : pp->radius_form;
            F[IDX(0,j,k)] = bc_form(fb, F[IDX(1,j,k)], F[IDX(2,j,k)], F[IDX(3,j,k)]);
            F[IDX(im-1,j,k)] = bc_form(pp->radius_form, F[IDX(im-2,j,k)], F[IDX(im-3,j,k)], F[IDX(im-4,j,k)]);
        }
    }
    if(pp->lid_u != 0)
        for(int j = 0; j < jm; j++) for(int k = 0; k < km; k++){ f[ATURAN_U][IDX(0,j,k)] = 0.0; f[ATURAN_U][IDX(im-1,j,k)] = 0.0; }
    if(pp->top_taper != 0){
        double* v = f[ATURAN_V]; double* w = f[ATURAN_W];
        const int l = im - 1;
        for(int j = 0; j < jm; j++) for(int k = 0; k < km; k++){
            v[IDX(l,j,k)] = 0.0;
            w[IDX(l,j,k)] = 0.0;
            if(pp->top_taper == 2){
                v[IDX(l-1,j,k)] = (1.0 / 3.0) * v[IDX(l-3,j,k)];
                w[IDX(l-1,j,k)] = (1.0 / 3.0) * w[IDX(l-3,j,k)];
                v[IDX(l-2,j,k)] = (2.0 / 3.0) * v[IDX(l-3,j,k)];
                w[IDX(l-2,j,k)] = (2.0 / 3.0) * w[IDX(l-3,j,k)];
            } else {
                v[IDX(l-1,j,k)] *= (1.0 / 3.0);
                w[IDX(l-1,j,k)] *= (1.0 / 3.0);
                v[IDX(l-2,j,k)] *= (2.0 / 3.0);
                w[IDX(l-2,j,k)] *= (2.0 / 3.0);
            }
        }
    }
    /* BC_Uran.h:91-108, floorRadialSpecies */
    if(pp->radius_positive != 0)
        for(int j = 0; j < jm; j++) for(int k = 0; k < km; k++)
            for(int n = 0; n < ATURAN_NSPECIES; n++){
                double* F = f[POST_SPECIES[n]];
                if(F[IDX(0,j,k)] < 0.0) F[IDX(0,j,k)] = (pp->radius_positive == 2) ? post_max0(F[IDX(1,j,k)]) : 0.0;
                if(F[IDX(im-1,j,k)] < 0.0) F[IDX(im-1,j,k)] = (pp->radius_positive == 2) ? post_max0(F[IDX(im-2,j,k)]) : 0.0;
            }
    /* BC_Uran.h:155-170, the lid value of v, w */
    if(pp->lid_vw == 2 || pp->lid_vw == 3){
        double* v = f[ATURAN_V]; double* w = f[ATURAN_W];
        const int a = im - 2, b = im - 3, c = im - 4, l = im - 1;
        for(int j = 0; j < jm; j++) for(int k = 0; k < km; k++){
            if(pp->lid_vw == 2){
                v[IDX(l,j,k)] = 2.0 * v[IDX(a,j,k)] - v[IDX(b,j,k)];
                w[IDX(l,j,k)] = 2.0 * w[IDX(a,j,k)] - w[IDX(b,j,k)];
            } else {
                v[IDX(l,j,k)] = v[IDX(c,j,k)] - 3.0 * v[IDX(b,j,k)] + 3.0 * v[IDX(a,j,k)];
                w[IDX(l,j,k)] = w[IDX(c,j,k)] - 3.0 * w[IDX(b,j,k)] + 3.0 * w[IDX(a,j,k)];
            }
        }
    }
    /* BoundaryConditions.h:293-391 (bcTheta; no pole fill rows for Uranus) */
    for(int k = 0; k < km; k++) for(int i = 0; i < im; i++){
        for(int n = 0; n < NELEM(POST_THETA_ZERO); n++){
            double* F = f[POST_THETA_ZERO[n]];
            F[IDX(i,0,k)] = 0.0;
            F[IDX(i,jm-1,k)] = 0.0;
        }
        for(int n = 0; n < NELEM(POST_THETA_EXTRAP); n++){
            double* F = f[POST_THETA_EXTRAP[n]];
            F[IDX(i,0,k)] = bc_form(pp->pole_form, F[IDX(i,1,k)], F[IDX(i,2,k)], F[IDX(i,3,k)]);
            F[IDX(i,jm-1,k)] = bc_form(pp->pole_form, F[IDX(i,jm-2,k)], F[IDX(i,jm-3,k)], F[IDX(i,jm-4,k)]);
        }
    }
    /* BoundaryConditions.h:398-518 (bcPhi without the seam damping); its list is the radius list
     * without difflux_nh4sh on the fields held */
    for(int i = 0; i < im; i++) for(int j = 0; j < jm; j++)
        for(int n = 0; n < POST_NPHI; n++){
            double* F = f[POST_RADIUS[n]];
            if(pp->phi_periodic) F[IDX(i,j,km-1)] = F[IDX(i,j,0)];
            else {
                const double lo = C43 * F[IDX(i,j,1)] - C13 * F[IDX(i,j,2)];
                const double hi = C43 * F[IDX(i,j,km-2)] - C13 * F[IDX(i,j,km-3)];
                F[IDX(i,j,0)] = F[IDX(i,j,km-1)] = 0.5 * (lo + hi);
            }
        }
    /* BC_Uran.h:110-128, clampNegativeSpecies: this call's clipped sum and count per species */
    for(int n = 0; n < ATURAN_NSPECIES; n++){
        double a = 0.0; long c = 0;
        if(pp->species_clamp){
            double* F = f[POST_SPECIES[n]];
            for(size_t q = 0; q < N; q++)
                if(!(F[q] >= 0.0)){
                    if(isfinite(F[q])){ a -= F[q]; c++; }
                    F[q] = 0.0;
                }
        }
        if(clamp_added) clamp_added[n] = a;
        if(clamp_cells) clamp_cells[n] = c;
    }
    return 0;
}

/* ---- MoistConvectiveAdjustment<cUranusModel>::run (ConvectiveAdjustment.h:402-849) ----
 * With the reference's default knobs: MCA_LEDOUX 1, MCA_LOADING 1, MCA_RELAX 1, MCA_SMOOTH 0
 * (cUranusModel.h:572), MCA_PASSES 64, MCA_PHASE off (SATADJ_BERGERON = 2, cUranusModel.h:586),
 * MCA_INTERIOR 1 (:566), no SeaMount; the gas list and the NH4SH tracer of
 * cUranusModel.cpp:1276-1290. Columns are independent, so they run in parallel. */
#define MCA_NG 4

static double mca_mx(double a, double b){ return (a < b) ? b : a; }            /* std::max(a, b) */

static double* g_cp_H[3];   /* CpH2.h:66-75: the table's running integral, H[0] = cp[0] T_LO */
static const double* cp_H_table(int mode){
    if(g_cp_H[mode]) return g_cp_H[mode];
    const double* t = cp_table(mode);
    double* H = (double*)malloc(sizeof(double) * g_cp_n);
    H[0] = t[0] * CP_T_LO;
    for(int i = 1; i < g_cp_n; i++) H[i] = H[i-1] + 0.5 * CP_DT * (t[i] + t[i-1]);
    g_cp_H[mode] = H;
    return H;
}

/* CpH2.h:94-101 */
static double mca_enth_h2(const aturan_params* p, double T){
    if(p->cp_h2_mode <= 0) return p->cp_h2 * T;
    const double* t = cp_table(p->cp_h2_mode);
    const double* H = cp_H_table(p->cp_h2_mode);
    const int n = g_cp_n;
    if(T <= CP_T_LO) return t[0] * T;
    if(T >= CP_T_HI) return H[n-1] + t[n-1] * (T - CP_T_HI);
    const double x = (T - CP_T_LO) / CP_DT;
    int i = (int)x; if(i > n - 2) i = n - 2;
    const double fr = x - i;
    return H[i] + CP_DT * fr * (t[i] + 0.5 * fr * (t[i+1] - t[i]));
}

/* CpH2.h:135-142 (Lapse::enth) */
static double mca_enth(const aturan_params* p, double T){
    if(!p->cp_dyn) return p->cp_mix * T;
    const double hh = mca_enth_h2(p, T);
    if(p->cp_gas) return (p->r_h2 * hh + (p->r_he * p->cp_he + p->r_ch4 * p->cp_ch4) * T) / (p->r_h2 + p->r_he + p->r_ch4);
    return (p->cp_mix - (p->r_h2 / p->r_mix) * p->cp_h2) * T + (p->r_h2 / p->r_mix) * hh;
}

/* CpH2.h:146-157 (enth_inv: Newton from T0) */
static double mca_enth_inv(const aturan_params* p, double h, double T0){
    if(!p->cp_dyn) return h / p->cp_mix;
    double T = (T0 > 0.0) ? T0 : h / p->cp_mix;
    for(int it = 0; it < 30; it++){
        const double f = mca_enth(p, T) - h, c = oracle_cp_lapse(p, T);
        const double dT = f / c;
        T -= dT; if(T < 1.0) T = 1.0;
        if(fabs(dT) < 1.0e-10 * T) break;
    }
    return T;
}

typedef struct {
    const aturan_params* p;
    const aturan_gas* G[MCA_NG];
    double L_tr;                       /* the NH4SH tracer's heat (ep 0, condensed) */
} mca_ctx;

/* ConvectiveAdjustment.h:437-450 with the phase split off */
static double mca_qsat(const aturan_gas* s, double T, double pr){
    const double E = (T >= s->t_0) ? svp(T, s->C, s->L0, s->R, s->del_alf, s->del_bet)
                                   : svp(T, s->C_i, s->L0_i, s->R, s->del_alf_i, s->del_bet_i);
    const double q = s->ep * E / pr;
    return isfinite(q) ? q : 0.0;
}
static double mca_lat(const aturan_gas* s, double T){ return T >= s->t_0 ? s->lv : s->ls; }

static double mca_fof(const mca_ctx* M, double TT, double hL, const double* qt, double pr, double z){
    double f = mca_enth(M->p, TT) + M->p->g * z - hL;
    for(int g = 0; g < MCA_NG; g++) f -= mca_lat(M->G[g], TT) * mca_mx(0.0, qt[g] - mca_qsat(M->G[g], TT, pr));
    return f;
}

/* :455-488, the equilibrium of (hL, qt) at (p, z) */
static int mca_equil(const mca_ctx* M, double hL, const double* qt, double pr, double z, double* T, double* cond){
    const aturan_params* p = M->p;
    const double cp = p->cp_mix, grav = p->g, tol_T = 1.0e-10;
    const double T_lo = p->cp_dyn ? mca_enth_inv(p, hL - grav * z, 0.0) : (hL - grav * z) / cp;
    if(!(T_lo > 0.0) || !(pr > 0.0)) return 0;
    int any = 0;
    for(int g = 0; g < MCA_NG; g++) if(qt[g] > mca_qsat(M->G[g], T_lo, pr)){ any = 1; break; }
    if(!any){ *T = T_lo; for(int g = 0; g < MCA_NG; g++) cond[g] = 0.0; return 1; }
    double span = 0.0;
    for(int g = 0; g < MCA_NG; g++) span += mca_mx(M->G[g]->lv, M->G[g]->ls) * mca_mx(0.0, qt[g]);
    double a = T_lo, b = p->cp_dyn ? mca_enth_inv(p, mca_enth(p, T_lo) + span, T_lo) + 1.0e-9 : T_lo + span / cp + 1.0e-9;
    double fa = mca_fof(M, a, hL, qt, pr, z), fb = mca_fof(M, b, hL, qt, pr, z);
    int side = 0;
    for(int it = 0; it < 60 && b - a > tol_T; it++){
        double c = (fb - fa != 0.0) ? b - fb * (b - a) / (fb - fa) : 0.5 * (a + b);
        if(!(c > a && c < b)) c = 0.5 * (a + b);
        const double fc = mca_fof(M, c, hL, qt, pr, z);
        if(fc < 0.0){ a = c; fa = fc; if(side == -1) fb *= 0.5; side = -1; }
        else        { b = c; fb = fc; if(side == +1) fa *= 0.5; side = +1; }
        if(fabs(fc) <= cp * tol_T){ a = b = c; break; }
    }
    *T = b;
    for(int g = 0; g < MCA_NG; g++) cond[g] = mca_mx(0.0, qt[g] - mca_qsat(M->G[g], *T, pr));
    return 1;
}

typedef struct {
    int im;
    double *T, *p, *z, *rho, *w, *hL, *qt, *qv, *qc, *qi, *qr, *Teq, *ceq;
    char *touched, *eq_ok, *cen_u, *cen_m;
} mca_col;

static double mca_trE(const mca_ctx* M, const mca_col* C, int i){ double e = 0.0; e += M->L_tr * C->qr[i]; return e; }

/* :613-624, Ledoux virtual temperature with condensate loading */
static double mca_tv(const mca_ctx* M, const mca_col* C, double TT, const double* v_, const double* cnd, int i_tr){
    double f = 1.0;
    for(int g = 0; g < MCA_NG; g++){ f += v_[g] * (1.0 / M->G[g]->ep - 1.0); f -= cnd[g]; }
    f -= C->qr[i_tr];                       /* NH4SH: ep 0, condensed */
    return TT * f;
}

/* :627-644 */
static int mca_unstable(const mca_ctx* M, mca_col* C, int a, int b, int* held, int* moist){
    const double tol_K = 1.0e-7;
    double Tp, pc[MCA_NG], pv[MCA_NG], ec[MCA_NG], ev[MCA_NG];
    if(!mca_equil(M, C->hL[a] + mca_trE(M, C, a), &C->qt[a * MCA_NG], C->p[b], C->z[b], &Tp, pc)) return 0;
    if(!C->eq_ok[b]){
        if(!mca_equil(M, C->hL[b] + mca_trE(M, C, b), &C->qt[b * MCA_NG], C->p[b], C->z[b], &C->Teq[b], &C->ceq[b * MCA_NG])) return 0;
        C->eq_ok[b] = 1;
    }
    const double Tb = C->Teq[b];
    for(int g = 0; g < MCA_NG; g++) ec[g] = C->ceq[b * MCA_NG + g];
    int wet = 0;
    for(int g = 0; g < MCA_NG; g++){ pv[g] = C->qt[a * MCA_NG + g] - pc[g]; if(pc[g] > 0.0) wet = 1; ev[g] = C->qt[b * MCA_NG + g] - ec[g]; }
    const double dTv = mca_tv(M, C, Tp, pv, pc, a) - mca_tv(M, C, Tb, ev, ec, b);
    if(held) *held = (Tp - Tb > tol_K) && !(dTv > tol_K);
    if(moist) *moist = wet;
    return dTv > tol_K;
}

/* :645-661, cell q to equilibrium from hL / qt */
static int mca_settle(const mca_ctx* M, mca_col* C, int q){
    double TT, pc[MCA_NG];
    if(!mca_equil(M, C->hL[q] + mca_trE(M, C, q), &C->qt[q * MCA_NG], C->p[q], C->z[q], &TT, pc)) return 0;
    C->T[q] = TT;
    C->Teq[q] = TT; C->eq_ok[q] = 1;
    for(int g = 0; g < MCA_NG; g++){
        const int x = q * MCA_NG + g;
        C->ceq[x] = pc[g];
        C->qv[x] = C->qt[x] - pc[g];
        if(TT >= M->G[g]->t_0){ C->qc[x] = pc[g]; C->qi[x] = 0.0; } else { C->qi[x] = pc[g]; C->qc[x] = 0.0; }
    }
    C->touched[q] = 1;
    return 1;
}

/* one column (j, k): :555-826 with MCA_SMOOTH 0 and MCA_RELAX 1 */
static void mca_column(const mca_ctx* M, mca_col* C, double* const* f, int j, int k){
    const aturan_params* p = M->p;
    const int im = p->im, jm = p->jm, km = p->km;
    static const int FV[MCA_NG] = { ATURAN_H2O, ATURAN_NH3, ATURAN_H2S, ATURAN_CH4 };
    const int i0 = 1, i1 = im - 2;                          /* MCA_INTERIOR, no SeaMount */
    if(i1 - i0 < 1) return;
    const float hz = (float)(p->L_atm / (im - 1));          /* cUranusModel.h:1205-1208, km per level */
    int ok = 1;
    for(int i = i0; i <= i1 && ok; i++){
        C->T[i] = f[ATURAN_T][IDX(i,j,k)] * p->t_ref;
        C->p[i] = f[ATURAN_P_STAT][IDX(i,j,k)];
        C->z[i] = (double)((float)i * hz) * 1.0e3;
        double rr = p->r_mix;                               /* rho_at, cUranusModel.h:526-531 */
        if(p->local_rho){ const double r_ = f[ATURAN_RHO_MIX][IDX(i,j,k)]; rr = (r_ > 0.0 && isfinite(r_)) ? r_ : p->r_mix; }
        C->rho[i] = rr;
        if(!(C->T[i] > 0.0) || !(C->p[i] > 0.0) || !(C->rho[i] > 0.0) || !isfinite(C->T[i] + C->p[i] + C->rho[i])) ok = 0;
    }
    if(!ok) return;
    for(int i = i0; i <= i1 && ok; i++){
        const double lo = (i > i0) ? 0.5 * (C->z[i-1] + C->z[i]) : C->z[i0];
        const double hi = (i < i1) ? 0.5 * (C->z[i] + C->z[i+1]) : C->z[i1];
        C->w[i] = C->rho[i] * (hi - lo);
        if(!(C->w[i] > 0.0)) ok = 0;
        double h = mca_enth(p, C->T[i]) + p->g * C->z[i];
        for(int g = 0; g < MCA_NG; g++){
            const int x = i * MCA_NG + g;
            C->qv[x] = mca_mx(0.0, f[FV[g]][IDX(i,j,k)]) / C->rho[i];
            C->qc[x] = mca_mx(0.0, f[FV[g] + 1][IDX(i,j,k)]) / C->rho[i];
            C->qi[x] = mca_mx(0.0, f[FV[g] + 2][IDX(i,j,k)]) / C->rho[i];
            C->qt[x] = C->qv[x] + C->qc[x] + C->qi[x];
            h -= M->G[g]->lv * C->qc[x] + M->G[g]->ls * C->qi[x];
        }
        C->qr[i] = f[ATURAN_NH4SH][IDX(i,j,k)] / C->rho[i];
        h -= M->L_tr * C->qr[i];
        C->hL[i] = h;
    }
    if(!ok) return;
    memset(C->touched, 0, im); memset(C->eq_ok, 0, im);
    for(int i = i0; i < i1; i++){
        int held = 0, moist = 0;
        C->cen_u[i] = (char)mca_unstable(M, C, i, i + 1, &held, &moist);
        C->cen_m[i] = (char)moist;
    }
    int passes = 0, changed = 1, fail = 0;
    long layers = 0;
    while(changed && passes < 64 && !fail){
        changed = 0; passes++;
        int i = i0;
        while(i < i1 && !fail){
            int moist = 0, uns;
            if(passes == 1 && !C->touched[i] && !C->touched[i + 1]){ uns = C->cen_u[i]; moist = C->cen_m[i]; }
            else uns = mca_unstable(M, C, i, i + 1, NULL, &moist);
            if(!uns){ i++; continue; }
            int a = i, b = i + 1;
            for(;;){
                double sw = 0.0, sh = 0.0, sq[MCA_NG] = {0.0, 0.0, 0.0, 0.0}, sr = 0.0;
                for(int q = a; q <= b; q++){
                    sw += C->w[q]; sh += C->w[q] * C->hL[q];
                    for(int g = 0; g < MCA_NG; g++) sq[g] += C->w[q] * C->qt[q * MCA_NG + g];
                    sr += C->w[q] * C->qr[q];
                }
                for(int q = a; q <= b; q++){
                    C->hL[q] = sh / sw;
                    for(int g = 0; g < MCA_NG; g++) C->qt[q * MCA_NG + g] = sq[g] / sw;
                    C->qr[q] = sr / sw;
                    if(!mca_settle(M, C, q)){ fail = 1; break; }
                }
                if(fail) break;
                int ext = 0;
                if(a > i0 && mca_unstable(M, C, a - 1, a, NULL, NULL)){ a--; ext = 1; }
                if(b < i1 && mca_unstable(M, C, b, b + 1, NULL, NULL)){ b++; ext = 1; }
                if(!ext) break;
            }
            layers += b - a + 1;
            changed = 1;
            i = b;
        }
    }
    if(fail || layers == 0) return;                         /* nothing written */
    for(int q = i0; q <= i1; q++){
        if(!C->touched[q]) continue;
        f[ATURAN_T][IDX(q,j,k)] = C->T[q] / p->t_ref;
        for(int g = 0; g < MCA_NG; g++){
            const int x = q * MCA_NG + g;
            f[FV[g]][IDX(q,j,k)]     = C->qv[x] * C->rho[q];
            f[FV[g] + 1][IDX(q,j,k)] = C->qc[x] * C->rho[q];
            f[FV[g] + 2][IDX(q,j,k)] = C->qi[x] * C->rho[q];
        }
        f[ATURAN_NH4SH][IDX(q,j,k)] = C->qr[q] * C->rho[q];
    }
}

int oracle_mca(const aturan_params* p, double* const* f){
    mca_ctx M;
    M.p = p;
    M.G[0] = &p->gas[0]; M.G[1] = &p->gas[2]; M.G[2] = &p->gas[1]; M.G[3] = &p->gas[3];   /* H2O NH3 H2S CH4 */
    M.L_tr = p->nh4sh_sync ? 4705.0 * log(10.0) * 8314.46 / 51.1114 : 0.0;             /* ChemistryUran.h:132 */
    if(p->cp_h2_mode > 0){ cp_table(p->cp_h2_mode); cp_H_table(p->cp_h2_mode); }      /* built before the threads */
    const int im = p->im, jm = p->jm, km = p->km;
    #pragma omp parallel
    {
        mca_col C;
        C.im = im;
        double* buf = (double*)malloc(sizeof(double) * (size_t)im * (9 + 6 * MCA_NG));
        char* cb = (char*)malloc((size_t)im * 4);
        double* q = buf;
        C.T = q; q += im; C.p = q; q += im; C.z = q; q += im; C.rho = q; q += im; C.w = q; q += im;
        C.hL = q; q += im; C.qr = q; q += im; C.Teq = q; q += im; q += im;
        C.qt = q; q += im * MCA_NG; C.qv = q; q += im * MCA_NG; C.qc = q; q += im * MCA_NG;
        C.qi = q; q += im * MCA_NG; C.ceq = q; q += im * MCA_NG;
        C.touched = cb; C.eq_ok = cb + im; C.cen_u = cb + 2 * im; C.cen_m = cb + 3 * im;
        #pragma omp for collapse(2) schedule(dynamic, 8)
        for(int j = 0; j < jm; j++) for(int k = 0; k < km; k++) mca_column(&M, &C, f, j, k);
        free(buf); free(cb);
    }
    return 0;
}

/* ---- ChemistryUran (planet/ChemistryUran.h) and FluxLimiter<cUranusModel>::nh4sh (FluxLimiter.h),
 * the equilibrium form with the reference's default knobs ---- */

static double stdmin(double a, double b){ return (b < a) ? b : a; }            /* std::min(a, b) */

/* ChemistryUran.h:132, the van't Hoff enthalpy of K_p [J/kg] */
static double nh4sh_formation_heat(void){ return 4705.0 * log(10.0) * 8314.46 / 51.1114; }
/* ChemistryUran.h:144, Lewis (1969) [Pa^2] */
static double nh4sh_kp(double T){ const double atm = 101325.0; return pow(10.0, 14.82 - 4705.0 / T) * atm * atm; }
/* ChemistryUran.h:154-156 */
static double nh4sh_f(double x, double T0, double heat, double a, double b){
    const double T = T0 + heat * x, RT = 8314.46 * T;
    return (a - x) * (b - x) * RT * RT - nh4sh_kp(T);
}

/* ChemistryUran.h:140-177, equilibrateNH4SHCell: x [kmol/m3] formed (> 0) or decomposed (< 0) */
static double nh4sh_cell(const aturan_params* p, const aturan_chem_params* cp, double* const* f, size_t q){
    const double L_f = nh4sh_formation_heat();
    const double T0 = f[ATURAN_T][q] * p->t_ref;
    if(!(T0 > 0.0)) return 0.0;
    double rho = f[ATURAN_P_STAT][q] * 1e5 / (p->R_mix * T0);
    if(!(rho > 0.0) || !isfinite(rho)) rho = p->r_mix;
    const double a = stdmax(0.0, f[ATURAN_NH3][q]) / cp->m_nh3;
    const double b = stdmax(0.0, f[ATURAN_H2S][q]) / cp->m_h2s;
    const double s = stdmax(0.0, f[ATURAN_NH4SH][q]) / cp->m_nh4sh;
    const double heat = L_f * cp->m_nh4sh / (p->cp_mix * rho);
    const double f0 = nh4sh_f(0.0, T0, heat, a, b);
    double lo, hi;
    if(f0 > 0.0){ lo = 0.0; hi = stdmin(a, b); }
    else if(s > 0.0){
        if(nh4sh_f(-s, T0, heat, a, b) <= 0.0){ lo = hi = -s; }
        else { lo = -s; hi = 0.0; }
    } else return 0.0;
    if(hi > lo) for(int it = 0; it < 80; it++){
        const double xm = 0.5 * (lo + hi);
        if(nh4sh_f(xm, T0, heat, a, b) > 0.0) lo = xm; else hi = xm;
        if(hi - lo <= 1.0e-15 * stdmax(a, stdmax(b, s))) break;
    }
    const double x = (f0 > 0.0) ? lo : hi;
    if(x == 0.0) return 0.0;
    f[ATURAN_NH3][q] = stdmax(0.0, f[ATURAN_NH3][q] - cp->m_nh3 * x);
    f[ATURAN_H2S][q] = stdmax(0.0, f[ATURAN_H2S][q] - cp->m_h2s * x);
    f[ATURAN_NH4SH][q] = stdmax(0.0, f[ATURAN_NH4SH][q] + cp->m_nh4sh * x);
    const double dT = heat * x;
    f[ATURAN_T][q] = (T0 + dT) / p->t_ref;
    return x;
}

/* ChemistryUran.h:210-275, EquilibriumNH4SH("loop"): every cell in place (no SeaMount cells);
 * counts[0] / counts[1] = cells that formed / decomposed NH4SH. */
int oracle_nh4sh_eq(const aturan_params* p, const aturan_chem_params* cp, double* const* f, long* counts){
    const size_t N = (size_t)p->im * p->jm * p->km;
    long nf = 0, nd = 0;
    #pragma omp parallel for reduction(+:nf, nd) schedule(static)
    for(size_t q = 0; q < N; q++){
        const double x = nh4sh_cell(p, cp, f, q);
        if(x > 0.0) nf++;
        else if(x < 0.0) nd++;
    }
    if(counts){ counts[0] = nf; counts[1] = nd; }
    return 0;
}

/* ChemistryUran.h:601-686, derivative_1_order without SeaMount cells: the central differences */
static void chem_d1(const aturan_params* p, const double* c, int i, int j, int k, int per,
                    double* dr_, double* dthe_, double* dphi_){
    const int jm = p->jm, km = p->km;
    const int kw = per ? phi_wrap(k - 1, km) : k - 1, ke = per ? phi_wrap(k + 1, km) : k + 1;
    *dr_ = (c[IDX(i+1,j,k)] - c[IDX(i-1,j,k)]) / (2.0 * p->dr);
    *dthe_ = (c[IDX(i,j+1,k)] - c[IDX(i,j-1,k)]) / (2.0 * p->dthe);
    *dphi_ = (c[IDX(i,j,ke)] - c[IDX(i,j,kw)]) / (2.0 * p->dphi);
}

/* ChemistryUran.h:576-598, laplacian_spherical (coord_stretching false: exp_rm = 1) */
static double chem_laplacian(const aturan_params* p, const aturan_chem_params* cp, const double* c,
                             const double* rad, const double* the, int i, int j, int k, int per){
    const int jm = p->jm, km = p->km;
    const double rm = metric_radius(p, rad[i]);
    const double exp_rm = 1.0, exp_2_rm = exp_rm * exp_rm;
    const double sinthe = sin(the[j]), costhe = cos(the[j]);
    const double rmsinthe = rm * stdmax(sinthe, cp->polar_floor);
    const double x = c[IDX(i,j,k)];
    const double d2cdr2 = (c[IDX(i+1,j,k)] - 2.0 * x + c[IDX(i-1,j,k)]) / (p->dr * p->dr) * exp_2_rm;
    const double d2cdthe2 = (c[IDX(i,j+1,k)] - 2.0 * x + c[IDX(i,j-1,k)]) / (p->dthe * p->dthe);
    const int kw = per ? phi_wrap(k - 1, km) : k - 1, ke = per ? phi_wrap(k + 1, km) : k + 1;
    const double d2cdphi2 = (c[IDX(i,j,ke)] - 2.0 * x + c[IDX(i,j,kw)]) / (p->dphi * p->dphi);
    const double dcdr = (c[IDX(i+1,j,k)] - c[IDX(i-1,j,k)]) / (2.0 * p->dr) * exp_rm;
    const double dcdthe = (c[IDX(i,j+1,k)] - c[IDX(i,j-1,k)]) / (2.0 * p->dthe);
    return d2cdr2 + 2.0 / rm * dcdr + d2cdthe2 / (rm * rm) + costhe / (rm * rmsinthe) * dcdthe
         + d2cdphi2 / (rmsinthe * rmsinthe);
}

/* FluxLimiter.h:68-70 */
static double superbee(double r){ return stdmax(0.0, stdmax(stdmin(2.0 * r, 1.0), stdmin(r, 2.0))); }

/* cUranusModel.cpp:1074-1087: DiffMassFluxUran (ChemistryUran.h:277-427), damp_wiggles on
 * difflux_h2s/nh3/nh4sh and thermalmassflux, ChemMassRateUran (:38-110; w_* = 0 in the
 * equilibrium form), FluxLimiter<cUranusModel>::nh4sh (FluxLimiter.h:89-186), damp_wiggles on
 * massflux_h2s/nh3/nh4sh and fluxlim_nh4sh. The interior rows are written; the boundary rows of
 * the persistent fields are read as they are. */
int oracle_chem_forcing(const aturan_params* p, const aturan_chem_params* cp, double* const* f){
    const int im = p->im, jm = p->jm, km = p->km;
    const size_t N = (size_t)im * jm * km;
    const int per = cp->phi_periodic != 0, k_first = per ? 0 : 1;
    double* rad = (double*)malloc(sizeof(double) * im);
    double* the = (double*)malloc(sizeof(double) * jm);
    double* tmp = (double*)malloc(sizeof(double) * N);
    if(!rad || !the || !tmp){ free(rad); free(the); free(tmp); return -1; }
    oracle_coords(p, rad, the);
    const double nu_mix = p->mue_mix / p->r_mix;
    const double D_nh3 = nu_mix / p->sc_nh3, D_h2s = nu_mix / p->sc_h2s;
    const double DT_nh3 = nu_mix / p->sc_nh3, DT_h2s = nu_mix / p->sc_h2s;
    const double dsign = cp->difflux_plus ? 1.0 : -1.0;
    const double* t = f[ATURAN_T];
    const double *nh3 = f[ATURAN_NH3], *h2s = f[ATURAN_H2S], *nh4sh = f[ATURAN_NH4SH];
    /* ChemistryUran.h:312-320, the local density */
    #pragma omp parallel for schedule(static)
    for(size_t q = 0; q < N; q++) f[ATURAN_RHO_MIX][q] = f[ATURAN_P_STAT][q] * 1e5 / (p->R_mix * t[q] * p->t_ref);
    /* passes 1 and 2 (ChemistryUran.h:322-419): j_* at the cell, thermalmassflux and difflux_* */
    #pragma omp parallel for collapse(2) schedule(static)
    for(int k = k_first; k < km - 1; k++) for(int j = 1; j < jm - 1; j++) for(int i = 1; i < im - 1; i++){
        const size_t q = IDX(i,j,k);
        const double rm = rad[i];
        const double sinthe = stdmax(p->sinthe_min, fabs(sin(the[j])));
        const double rmsinthe = rm * sinthe;
        double dtdr, dtdthe, dtdphi, a_r, a_t, a_p, b_r, b_t, b_p, c_r, c_t, c_p;
        chem_d1(p, t, i, j, k, per, &dtdr, &dtdthe, &dtdphi);
        chem_d1(p, h2s, i, j, k, per, &a_r, &a_t, &a_p);
        chem_d1(p, nh3, i, j, k, per, &b_r, &b_t, &b_p);
        chem_d1(p, nh4sh, i, j, k, per, &c_r, &c_t, &c_p);
        const double jT_nh3 = DT_nh3 / t[q] * dtdr;
        const double jT_h2s = DT_h2s / t[q] * dtdr;
        const double jT_nh4sh = cp->DT_nh4sh / t[q] * dtdr;
        const double d_nh3 = b_r + fabs(b_t) / rm + b_p / rmsinthe;
        const double d_h2s = a_r + fabs(a_t) / rm + a_p / rmsinthe;
        const double d_nh4sh = c_r + fabs(c_t) / rm + c_p / rmsinthe;
        const double j_nh3 = cp->c_mix / p->r_mix * (cp->m_nh3 * D_nh3 * d_nh3 - jT_nh3);
        const double j_h2s = cp->c_mix / p->r_mix * (cp->m_h2s * D_h2s * d_h2s - jT_h2s);
        const double j_nh4sh = cp->c_mix / p->r_mix * (cp->m_nh4sh * cp->D_nh4sh * d_nh4sh - jT_nh4sh);
        f[ATURAN_DIFFLUX_H2S][q] = D_h2s * chem_laplacian(p, cp, h2s, rad, the, i, j, k, per);
        f[ATURAN_DIFFLUX_NH3][q] = D_nh3 * chem_laplacian(p, cp, nh3, rad, the, i, j, k, per);
        f[ATURAN_DIFFLUX_NH4SH][q] = cp->D_nh4sh * chem_laplacian(p, cp, nh4sh, rad, the, i, j, k, per);
        const double w0 = 0.0;   /* w_nh3, w_h2s, w_nh4sh */
        f[ATURAN_THERMALMASSFLUX][q] = (j_nh3 * cp->cp_nh3 + j_h2s * cp->cp_h2s + j_nh4sh * cp->cp_nh4sh)
            * (dtdr + fabs(dtdthe) / rm + dtdphi / rmsinthe)
            + t[q] * (w0 * cp->k_nh3 + w0 * cp->k_h2s + w0 * cp->k_nh4sh);
    }
    post_damp(p, f[ATURAN_DIFFLUX_H2S], 1, 1, 1, 1.0, per, tmp);
    post_damp(p, f[ATURAN_DIFFLUX_NH3], 1, 1, 1, 1.0, per, tmp);
    post_damp(p, f[ATURAN_DIFFLUX_NH4SH], 1, 1, 1, 1.0, per, tmp);
    post_damp(p, f[ATURAN_THERMALMASSFLUX], 1, 1, 1, 1.0, per, tmp);
    /* ChemMassRateUran: massflux = w + sign difflux, w = 0 */
    #pragma omp parallel for collapse(2) schedule(static)
    for(int k = k_first; k < km - 1; k++) for(int j = 1; j < jm - 1; j++) for(int i = 1; i < im - 1; i++){
        const size_t q = IDX(i,j,k);
        f[ATURAN_MASSFLUX_H2S][q] = 0.0 + dsign * f[ATURAN_DIFFLUX_H2S][q];
        f[ATURAN_MASSFLUX_NH3][q] = 0.0 + dsign * f[ATURAN_DIFFLUX_NH3][q];
        f[ATURAN_MASSFLUX_NH4SH][q] = 0.0 + dsign * f[ATURAN_DIFFLUX_NH4SH][q];
    }
    /* the Superbee limiter */
    const double eps = 1.0e-12;
    const double* u = f[ATURAN_U]; const double* v = f[ATURAN_V]; const double* w = f[ATURAN_W];
    #pragma omp parallel for collapse(2) schedule(static)
    for(int k = k_first; k < km - 1; k++) for(int j = 1; j < jm - 1; j++) for(int i = 1; i < im - 1; i++){
        const size_t o = IDX(i,j,k);
        const double q = nh4sh[o], q_rp = nh4sh[IDX(i+1,j,k)], q_rm = nh4sh[IDX(i-1,j,k)];
        const double q_tp = nh4sh[IDX(i,j+1,k)], q_tm = nh4sh[IDX(i,j-1,k)];
        const int kp1 = per ? phi_wrap(k + 1, km) : k + 1, km1 = per ? phi_wrap(k - 1, km) : k - 1;
        const double q_pp = nh4sh[IDX(i,j,kp1)], q_pm = nh4sh[IDX(i,j,km1)];
        const double uu = u[o], vv = v[o], ww = w[o];
        const double rm = metric_radius(p, rad[i]);
        const double sinthe = stdmax(cp->polar_floor, fabs(sin(the[j])));
        const double inv_rm = 1.0 / rm, inv_rmsinthe = 1.0 / (rm * sinthe);
        double corr = 0.0;
        {
            const double df = q_rp - q, db = q - q_rm;
            const double denom = df + (df >= 0.0 ? eps : -eps);
            const double r = (uu >= 0.0) ? db / denom : ((i + 2 < im ? nh4sh[IDX(i+2,j,k)] : q_rp) - q_rp) / denom;
            corr += (1.0 - superbee(r)) * fabs(uu) * (df - db) / (2.0 * p->dr);
        }
        {
            const double df = q_tp - q, db = q - q_tm;
            const double denom = df + (df >= 0.0 ? eps : -eps);
            const double q_far = (j + 2 < jm) ? nh4sh[IDX(i,j+2,k)] : (C43 * q_tp - C13 * q);
            const double r = (vv >= 0.0) ? db / denom : (q_far - q_tp) / denom;
            corr += (1.0 - superbee(r)) * fabs(vv) * inv_rm * (df - db) / (2.0 * p->dthe);
        }
        {
            const double df = q_pp - q, db = q - q_pm;
            const double denom = df + (df >= 0.0 ? eps : -eps);
            const double q2 = per ? nh4sh[IDX(i,j,phi_wrap(k + 2, km))] : (k + 2 < km ? nh4sh[IDX(i,j,k+2)] : q_pp);
            const double r = (ww >= 0.0) ? db / denom : (q2 - q_pp) / denom;
            corr += (1.0 - superbee(r)) * fabs(ww) * inv_rmsinthe * (df - db) / (2.0 * p->dphi);
        }
        f[ATURAN_FLUXLIM_NH4SH][o] = corr;
    }
    post_damp(p, f[ATURAN_MASSFLUX_H2S], 1, 1, 1, 1.0, per, tmp);
    post_damp(p, f[ATURAN_MASSFLUX_NH3], 1, 1, 1, 1.0, per, tmp);
    post_damp(p, f[ATURAN_MASSFLUX_NH4SH], 1, 1, 1, 1.0, per, tmp);
    post_damp(p, f[ATURAN_FLUXLIM_NH4SH], 1, 1, 1, 1.0, per, tmp);
    free(rad); free(the); free(tmp);
    return 0;
}

/* ---- Turbulence<cUranusModel>::run (planet/Turbulence.h:307-331), k-omega SST with the
 * reference's default knobs: TURB_FREE 1, TURB_CLAMP_PASS 1, no land cells, no buoyancy term,
 * no ABL taper, no obstacle (surface_index 0), the closure's fields not in the model's own
 * boundary lists (bc_turb_active false) ---- */

static double clamp3d(double x, double lo, double hi){ return (x < lo) ? lo : ((x > hi) ? hi : x); }   /* Turbulence.h:207-209 */
static double turb_blend(double inner, double outer, double F1){ return F1 * inner + (1.0 - F1) * outer; }   /* :203-205 */

int oracle_turbulence(const aturan_params* p, const aturan_turb_params* tp, double* const* f){
    const int im = p->im, jm = p->jm, km = p->km;
    const int per = tp->phi_periodic != 0, k_first = per ? 0 : 1;
    double* rad = (double*)malloc(sizeof(double) * im);
    double* the = (double*)malloc(sizeof(double) * jm);
    if(!rad || !the){ free(rad); free(the); return -1; }
    oracle_coords(p, rad, the);
    double *tke = f[ATURAN_TKE], *dis = f[ATURAN_DIS], *nue = f[ATURAN_NUE], *prod = f[ATURAN_PROD];
    double *tks = f[ATURAN_TKE_SOURCE], *dss = f[ATURAN_DIS_SOURCE];
    const double *u = f[ATURAN_U], *v = f[ATURAN_V], *w = f[ATURAN_W];
    const double dis_min = 1.0e-10;                                   /* :195 */
    const double L_m = p->L_atm * 1.0e3;                              /* L_atm_m(), :268 */
    const double nue_max = tp->nue_max / (p->u_0 * L_m);
    const double k_bg_nd = tp->k_bg / (p->u_0 * p->u_0);              /* k_bg_of with TURB_FREE, :622-628 */
    /* compute_sources, :614-883; the clamp pass before the loop (:645-650) */
    for(int j = 1; j < jm - 1; j++) for(int k = k_first; k < km - 1; k++) for(int i = 1; i < im - 1; i++){
        const size_t q = IDX(i,j,k);
        tke[q] = stdmax(0.0, tke[q]);
        dis[q] = stdmax(dis_min, dis[q]);
    }
    #pragma omp parallel for collapse(2) schedule(static)
    for(int j = 1; j < jm - 1; j++) for(int k = k_first; k < km - 1; k++){
        const int kw = per ? phi_wrap(k - 1, km) : k - 1, ke = per ? phi_wrap(k + 1, km) : k + 1;
        for(int i = 1; i < im - 1; i++){
            const size_t q = IDX(i,j,k);
            const double rm = metric_radius(p, rad[i]);
            const double exp_rm = 1.0;                                /* coord_stretching false */
            double sinthe = sin(the[j]);
            if(sinthe == 0.0) sinthe = 1.0e-5;
            const double costhe = cos(the[j]);
            const double cotanthe = costhe / sinthe;
            const double inv_rm = 1.0 / rm;
            const double rmsinthe = rm * sinthe;
            const double inv_2dr = 1.0 / (2.0 * p->dr);
            const double inv_2dthe = 1.0 / (2.0 * p->dthe);
            const double inv_2dphi = 1.0 / (2.0 * p->dphi);
            const double inv_rm2dthe = inv_2dthe / rm;
            const double inv_rmsinthe2dphi = inv_2dphi / rmsinthe;
            const double dudr = (u[IDX(i+1,j,k)] - u[IDX(i-1,j,k)]) * inv_2dr * exp_rm;
            const double dvdr = (v[IDX(i+1,j,k)] - v[IDX(i-1,j,k)]) * inv_2dr * exp_rm;
            const double dwdr = (w[IDX(i+1,j,k)] - w[IDX(i-1,j,k)]) * inv_2dr * exp_rm;
            const double dudthe = (u[IDX(i,j+1,k)] - u[IDX(i,j-1,k)]) * inv_rm2dthe;
            const double dvdthe = (v[IDX(i,j+1,k)] - v[IDX(i,j-1,k)]) * inv_rm2dthe;
            const double dwdthe = (w[IDX(i,j+1,k)] - w[IDX(i,j-1,k)]) * inv_rm2dthe;
            const double dudphi = (u[IDX(i,j,ke)] - u[IDX(i,j,kw)]) * inv_rmsinthe2dphi;
            const double dvdphi = (v[IDX(i,j,ke)] - v[IDX(i,j,kw)]) * inv_rmsinthe2dphi;
            const double dwdphi = (w[IDX(i,j,ke)] - w[IDX(i,j,kw)]) * inv_rmsinthe2dphi;
            const double dtkedr = (tke[IDX(i+1,j,k)] - tke[IDX(i-1,j,k)]) * inv_2dr * exp_rm;
            const double ddisdr = (dis[IDX(i+1,j,k)] - dis[IDX(i-1,j,k)]) * inv_2dr * exp_rm;
            /* the production tensor, :697-760 */
            double cnue;
            {
                const double dis_here = stdmax(dis[q], dis_min);
                const double tke_here = stdmax(tke[q], 0.0);
                cnue = tke_here / dis_here;
                cnue = stdmin(cnue, nue_max);
            }
            const int curv = tp->curv != 0;
            const double u_r = curv ? u[q] * inv_rm : 0.0;
            const double v_r = curv ? v[q] * inv_rm : 0.0;
            const double w_r = curv ? w[q] * inv_rm : 0.0;
            const double v_cot_r = v_r * cotanthe;
            const double w_cot_r = w_r * cotanthe;
            const double g_rr = dudr, g_rt = dudthe - v_r, g_rp = dudphi - w_r;
            const double g_tr = dvdr, g_tt = dvdthe + u_r, g_tp = dvdphi - w_cot_r;
            const double g_pr = dwdr, g_pt = dwdthe, g_pp = dwdphi + u_r + v_cot_r;
            const double der = 0.66667 * (g_rr + g_tt + g_pp);
            const double tk = tke[q];
            prod[q] = stdmax(0.0,
                  (cnue * (2.0 * g_rr - der) - 0.66667 * tk) * g_rr
                + (cnue * (g_rt + g_tr)) * g_rt
                + (cnue * (g_rp + g_pr)) * g_rp
                + (cnue * (2.0 * g_tt - der) - 0.66667 * tk) * g_tt
                + (cnue * (g_tr + g_rt)) * g_tr
                + (cnue * (g_tp + g_pt)) * g_tp
                + (cnue * (2.0 * g_pp - der) - 0.66667 * tk) * g_pp
                + (cnue * (g_pr + g_rp)) * g_pr
                + (cnue * (g_pt + g_tp)) * g_pt);
            const double W12 = g_rt - g_tr, W13 = g_rp - g_pr, W23 = g_tp - g_pt;
            const double Omega = sqrt(W12 * W12 + W13 * W13 + W23 * W23);
            /* compute_k_omega_SST, :1020-1100, with no land cells and no wall */
            const double a1 = 0.31, bet_star = 0.09, bet1 = 0.0333, bet2 = 0.0368;
            const double gam1 = 0.413, gam2 = 0.2, sig_w2 = 1.168;
            const double nue_air_nd = tp->nue_air / (p->u_0 * L_m);
            const double y_phys = 1.0e20;                             /* free_wall_dist(), :147 */
            const double y_star = y_phys / L_m;
            const double rms = rm * sinthe;
            const double dtkedthe_neu = (tke[IDX(i,j+1,k)] - tke[IDX(i,j-1,k)]) / (rm * 2.0 * p->dthe);
            const double ddisdthe_neu = (dis[IDX(i,j+1,k)] - dis[IDX(i,j-1,k)]) / (rm * 2.0 * p->dthe);
            const double dtkedphi_neu = (tke[IDX(i,j,ke)] - tke[IDX(i,j,kw)]) / (rms * 2.0 * p->dphi);
            const double ddisdphi_neu = (dis[IDX(i,j,ke)] - dis[IDX(i,j,kw)]) / (rms * 2.0 * p->dphi);
            const double grad_dot = dtkedr * ddisdr + dtkedthe_neu * ddisdthe_neu + dtkedphi_neu * ddisdphi_neu;
            const double CD_kw = stdmax(2.0 * sig_w2 / stdmax(dis[q], 1.0e-20) * grad_dot, 1.0e-20);
            const double dis_safe = stdmax(dis[q], 1.0e-20);
            const double arg1 = stdmin(
                stdmax(sqrt(tk) / (bet_star * dis_safe * y_star), 500.0 * nue_air_nd / (y_star * y_star * dis_safe)),
                4.0 * sig_w2 * tk / (CD_kw * y_star * y_star));
            const double arg2 = stdmax(2.0 * sqrt(tk) / (bet_star * dis_safe * y_star),
                                       500.0 * nue_air_nd / (y_star * y_star * dis_safe));
            const double F1 = tanh(pow(arg1, 4));
            const double F2 = tanh(pow(arg2, 2));
            nue[q] = a1 * tk / stdmax(a1 * dis_safe, Omega * F2);
            const double tke_safe = stdmax(tk, 1.0e-20);
            const double P_k = stdmin(prod[q], 20.0 * bet_star * tke_safe * dis_safe);
            const double Y_k = bet_star * tke_safe * dis_safe;
            const double P_w = turb_blend(gam1, gam2, F1) * P_k * dis_safe / tke_safe;
            const double Y_w = turb_blend(bet1, bet2, F1) * dis_safe * dis_safe;
            const double D_w = 2.0 * (1.0 - F1) * sig_w2 / dis_safe * grad_dot;
            tks[q] = P_k - Y_k;
            dss[q] = P_w - Y_w + D_w;
        }
    }
    /* the floor and the caps after the loop (:862-869, clamp_out :631-643) */
    for(int j = 1; j < jm - 1; j++) for(int k = k_first; k < km - 1; k++) for(int i = 1; i < im - 1; i++){
        const size_t q = IDX(i,j,k);
        tke[q] = stdmax(k_bg_nd, tke[q]);
        dis[q] = stdmax(dis_min, dis[q]);
        nue[q] = clamp3d(nue[q], 0.0, nue_max);
        const double dis_src_max = 20.0 * dis[q] * dis[q];
        dss[q] = clamp3d(dss[q], -dis_src_max, dis_src_max);
        const double tke_src_max = 20.0 * tke[q] * dis[q];
        tks[q] = clamp3d(tks[q], -tke_src_max, tke_src_max);
    }
    /* apply_wall_bc with TURB_FREE (:383-424): the zero-gradient copy at i = 0 in every column */
    for(int j = 0; j < jm; j++) for(int k = 0; k < km; k++){
        tke[IDX(0,j,k)] = tke[IDX(1,j,k)];
        dis[IDX(0,j,k)] = dis[IDX(1,j,k)];
        nue[IDX(0,j,k)] = nue[IDX(1,j,k)];
    }
    /* clamp_nue without the taper (:565-589) */
    for(size_t q = 0; q < (size_t)im * jm * km; q++) nue[q] = clamp3d(nue[q], 0.0, nue_max) * 1.0;
    /* seam_copy (:543-562) and fill_lid_corners for a model without the closure's fields in its own
     * boundary lists (:511-540): the lid row from im-2, then the pole rows from 1 and jm-2 */
    double* arr[8] = { tke, dis, f[ATURAN_TKEN], f[ATURAN_DISN], nue, prod, tks, dss };
    if(per)
        for(int i = 0; i < im; i++) for(int j = 0; j < jm; j++)
            for(int n = 0; n < 8; n++) arr[n][IDX(i,j,km-1)] = arr[n][IDX(i,j,0)];
    for(int j = 1; j < jm - 1; j++) for(int k = 0; k < km; k++)
        for(int n = 0; n < 8; n++) arr[n][IDX(im-1,j,k)] = arr[n][IDX(im-2,j,k)];
    for(int i = 0; i < im; i++) for(int k = 0; k < km; k++)
        for(int n = 0; n < 8; n++){
            arr[n][IDX(i,0,k)] = arr[n][IDX(i,1,k)];
            arr[n][IDX(i,jm-1,k)] = arr[n][IDX(i,jm-2,k)];
        }
    free(rad); free(the);
    return 0;
}

/* ---- Precipitation<cUranusModel>::run (planet/Precipitation.h:192-277) and its column solver
 * (:280-446) for H2O, NH3, CH4 and H2S (cUranusModel.h:280-297), no land cells. The fluxes
 * P_rain, P_snow, P_graupel of a column are carried down the column in locals; they, the NH4SH
 * settling flux and the surface maps are diagnostics the hot path does not keep. ---- */

/* cUranusModel.h:1199-1210 and :372-375: float layer heights i * (L_atm / (im-1)), thickness in m */
static double precip_dz(const aturan_params* p, int i){
    if(i < 0 || i > p->im - 2) return 0.0;
    const float h = (float)(p->L_atm / (p->im - 1));
    const float hi = (float)(i + 1) * h, lo = (float)i * h;
    return (double)(hi - lo) * 1.0e3;
}

/* one species, every column (Precipitation.h:281-446) */
static void precip_column(const aturan_params* p, const aturan_precip_params* pp, double* const* f,
                          const aturan_gas* s, int fv, int fc, int fi, int sv, int sc, int si){
    const int im = p->im, jm = p->jm, km = p->km;
    const double c_c_au = 2.0e-8, c_i_au = 5.0e-8, q_c_crit = 5.0e-4, c_ac = 1.0e-7, c_rim = 1.0e-8;
    const double z_csg = 2.5e-8, a_ev = 2.76e-3, c_melt_K = 0.2, c_frz_K = 0.2, P_ref = 1.0e-4;
    const double v_fall = 2.0;
    const double t_ref = p->t_ref;
    const double Lf = s->ls - s->lv;
    const double P_max_flux = 1.0e-4, dep_frac = 1.0, ratio_cap = 5.0;
    const double rs = pp->rate_scale;
    #pragma omp parallel for collapse(2) schedule(static)
    for(int j = 0; j < jm; j++) for(int k = 0; k < km; k++){
        double Pr = 0.0, Ps = 0.0, Pg = 0.0;                    /* the fluxes at i + 1 */
        for(int i = im - 2; i >= 0; i--){
            const size_t q = IDX(i,j,k);
            const double T = f[ATURAN_T][q] * t_ref;
            const double p_u = f[ATURAN_P_STAT][q];
            const double q_v = stdmax(0.0, f[fv][q]);
            const double q_c = stdmax(0.0, f[fc][q]);
            const double q_i = stdmax(0.0, f[fi][q]);
            const double E_r = svp(T, s->C, s->L0, s->R, s->del_alf, s->del_bet);
            double rho = p->r_mix;                                 /* rho_at, cUranusModel.h:526-531 */
            if(p->local_rho){ const double r = f[ATURAN_RHO_MIX][q]; rho = (r > 0.0 && isfinite(r)) ? r : p->r_mix; }
            const double q_sat = (p_u > E_r) ? rho * s->ep * E_r / p_u : q_v;
            const double dz = stdmax(0.0, precip_dz(p, i));
            if(dz <= 0.0) continue;                                /* the fluxes pass through */
            const double F_r_in = Pr, F_s_in = Ps, F_g_in = Pg;
            const double Rain = stdmin(ratio_cap, F_r_in / P_ref);
            const double Snow = stdmin(ratio_cap, F_s_in / P_ref);
            const double Graupel = stdmin(ratio_cap, F_g_in / P_ref);
            const double Rain_79 = (Rain > 0.0) ? pow(Rain, 7.0 / 9.0) : 0.0;
            const double Rain_49 = (Rain > 0.0) ? pow(Rain, 4.0 / 9.0) : 0.0;
            const int warm = (T >= s->t_0);
            const double S_c_au = (warm && q_c > q_c_crit) ? (rs * c_c_au) * (q_c - q_c_crit) : 0.0;
            const double S_i_au = (!warm && T >= s->t_00) ? (rs * c_i_au) * q_i : 0.0;
            const double S_ac = warm ? (rs * c_ac) * q_c * Rain_79 : 0.0;
            const double S_s_rim = !warm ? (rs * c_rim) * q_c * Snow : 0.0;
            const double S_g_rim = !warm ? (rs * c_rim) * q_c * Graupel : 0.0;
            const double S_csg = (!warm && q_c > q_c_crit) ? (rs * z_csg) * q_c * Snow : 0.0;
            const double f_melt = warm ? stdmin(1.0, c_melt_K * (T - s->t_0)) : 0.0;
            const double f_frz = warm ? 0.0 : stdmin(1.0, c_frz_K * (s->t_0 - T));
            const double F_s_melt = f_melt * F_s_in;
            const double F_g_melt = f_melt * F_g_in;
            const double F_r_frz = f_frz * F_r_in;
            const double F_r_avail = stdmax(0.0, F_r_in - F_r_frz + F_s_melt + F_g_melt + (S_c_au + S_ac) * dz);
            const double S_ev_raw = (warm && Rain > 0.0 && q_v < q_sat) ? a_ev * (q_sat - q_v) * Rain_49 : 0.0;
            const double F_ev_sat = stdmax(0.0, q_sat - q_v) * v_fall;
            const double F_ev = stdmin(stdmin(S_ev_raw * dz, F_r_avail), F_ev_sat);
            const double S_ev = F_ev / dz;
            f[ATURAN_Q_PRECIP][q] += Lf * (S_s_rim + S_g_rim + S_csg)
                                   + Lf * (F_r_frz - F_s_melt - F_g_melt) / dz
                                   - s->lv * F_ev / dz;
            const double tau = dz / v_fall;
            const double d_c = stdmin(dep_frac * q_c, (S_c_au + S_ac + S_s_rim + S_g_rim + S_csg) * tau);
            const double d_i = stdmin(dep_frac * q_i, S_i_au * tau);
            if(pp->coupling){
                const double nd = (p->L_atm * 1.0e3) / p->u_0;
                f[sc][q] = -stdmax(0.0, d_c) / tau * nd;
                f[si][q] = -stdmax(0.0, d_i) / tau * nd;
                f[sv][q] = +S_ev * nd;
            } else {
                f[fc][q] = q_c - stdmax(0.0, d_c);
                f[fi][q] = q_i - stdmax(0.0, d_i);
                f[fv][q] = q_v + S_ev * tau;
            }
            const double F_r = F_r_in - F_r_frz + F_s_melt + F_g_melt - F_ev + (S_c_au + S_ac) * dz;
            const double F_s = F_s_in - F_s_melt + (S_i_au + S_s_rim - S_csg) * dz;
            const double F_g = F_g_in - F_g_melt + F_r_frz + (S_g_rim + S_csg) * dz;
            Pr = stdmin(P_max_flux, stdmax(0.0, F_r));
            Ps = stdmin(P_max_flux, stdmax(0.0, F_s));
            Pg = stdmin(P_max_flux, stdmax(0.0, F_g));
        }
    }
}

int oracle_precipitation(const aturan_params* p, const aturan_precip_params* pp, double* const* f){
    const size_t N = (size_t)p->im * p->jm * p->km;
    /* Precipitation.h:199-212 */
    static const int zero_me[] = { ATURAN_Q_PRECIP, ATURAN_S_PRECIP_H2O, ATURAN_S_PRECIP_H2O_CLOUD,
        ATURAN_S_PRECIP_H2O_ICE, ATURAN_S_PRECIP_NH3, ATURAN_S_PRECIP_NH3_CLOUD, ATURAN_S_PRECIP_NH3_ICE,
        ATURAN_S_PRECIP_CH4, ATURAN_S_PRECIP_CH4_CLOUD, ATURAN_S_PRECIP_CH4_ICE };
    for(int n = 0; n < 10; n++) memset(f[zero_me[n]], 0, sizeof(double) * N);
    /* the params' gas order is H2O, H2S, NH3, CH4 */
    precip_column(p, pp, f, &p->gas[0], ATURAN_H2O, ATURAN_H2O_CLOUD, ATURAN_H2O_ICE,
                  ATURAN_S_PRECIP_H2O, ATURAN_S_PRECIP_H2O_CLOUD, ATURAN_S_PRECIP_H2O_ICE);
    precip_column(p, pp, f, &p->gas[2], ATURAN_NH3, ATURAN_NH3_CLOUD, ATURAN_NH3_ICE,
                  ATURAN_S_PRECIP_NH3, ATURAN_S_PRECIP_NH3_CLOUD, ATURAN_S_PRECIP_NH3_ICE);
    precip_column(p, pp, f, &p->gas[3], ATURAN_CH4, ATURAN_CH4_CLOUD, ATURAN_CH4_ICE,
                  ATURAN_S_PRECIP_CH4, ATURAN_S_PRECIP_CH4_CLOUD, ATURAN_S_PRECIP_CH4_ICE);
    /* cUranusModel.h:280-297, precip_extra_species */
    memset(f[ATURAN_S_PRECIP_H2S], 0, sizeof(double) * N);
    memset(f[ATURAN_S_PRECIP_H2S_CLOUD], 0, sizeof(double) * N);
    memset(f[ATURAN_S_PRECIP_H2S_ICE], 0, sizeof(double) * N);
    if(pp->h2s)
        precip_column(p, pp, f, &p->gas[1], ATURAN_H2S, ATURAN_H2S_CLOUD, ATURAN_H2S_ICE,
                      ATURAN_S_PRECIP_H2S, ATURAN_S_PRECIP_H2S_CLOUD, ATURAN_S_PRECIP_H2S_ICE);
    return 0;
}

/* ---- one iteration of cUranusModel::Run's loop (cUranusModel.cpp:952-1296) with the default
 * knobs, composed of the functions above in the loop's order ---- */
int oracle_iteration(const aturan_params* p, const aturan_iter_params* ip, double* const* f, int iter_n){
    const size_t N = (size_t)p->im * p->jm * p->km;
    if(iter_n % 2 == 0){
        /* :967-973 */
        if(ip->press_kind == ATURAN_PRESS_GS_LEX) oracle_pressure_gs(p, f);
        else if(ip->press_kind == ATURAN_PRESS_RB_SHARED) oracle_pressure_rb(p, f, ip->max_sweeps);
        else if(ip->press_kind == ATURAN_PRESS_RB_LINE){ int s; double r; oracle_pressure_line(p, f, ip->omega, ip->max_sweeps, ip->tol, &s, &r); }
        else { int s; double r; oracle_pressure_sor(p, f, ip->omega, ip->max_sweeps, ip->tol, 16, &s, &r); }
        /* :975-984, the p_dyn filter */
        double* tmp = (double*)malloc(sizeof(double) * N);
        if(!tmp) return -1;
        const int per = ip->post.phi_periodic;
        if(ip->damp_p_horiz == 1.0) post_damp(p, f[ATURAN_P_DYN], 1, 1, 1, 1.0, per, tmp);
        else {
            if(ip->damp_p_horiz != 0.0) post_damp(p, f[ATURAN_P_DYN], 0, 1, 1, ip->damp_p_horiz, per, tmp);
            post_damp(p, f[ATURAN_P_DYN], 1, 0, 0, 1.0, per, tmp);
        }
        free(tmp);
        /* :997-1030, H2O, H2S, NH3, CH4 */
        for(int g = 0; g < 4; g++) oracle_satadj(p, f, g, NULL, NULL);
        /* :1034, :1037 */
        if(ip->chemistry) oracle_nh4sh_eq(p, &ip->chem, f, NULL);
        if(ip->precipitation) oracle_precipitation(p, &ip->precip, f);
        /* :1049-1073 */
        oracle_sync_ncopies(p, f);
        /* :1074-1087 */
        if(ip->chemistry) oracle_chem_forcing(p, &ip->chem, f);
    }
    /* :1123 */
    double ref[1024];
    if(p->im > 1024) return -1;
    oracle_rk4(p, f, ref);
    /* :1199-1248 */
    oracle_post_step(p, f, &ip->post, NULL, NULL);
    /* :1264, restoreVar(1.0) */
    for(int q = 0; q < ATURAN_NPROG; q++) memcpy(f[ATURAN_TN + q], f[q], sizeof(double) * N);
    /* :1270-1296 */
    if(ip->turbulence) oracle_turbulence(p, &ip->turb, f);
    if(ip->mca_stride > 0 && iter_n % ip->mca_stride == 0) oracle_mca(p, f);
    return 0;
}
