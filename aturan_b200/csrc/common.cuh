// Device layout, per-(i,j) geometry and derived constants shared by every aturan_b200 kernel.
//
// HBM layout: one field is a block [i][j][kp] with the longitude row padded from km to kp (a
// multiple of 32 elements) so that every row starts on a 256-byte boundary for FP64 (128-byte
// for FP32) and a warp's 32 consecutive k land in whole sectors. Field f of an arena starts at
// base + f * fstride. k = km-1 is the seam copy of k = 0; padding columns are never read.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>
#include "aturan_b200.h"

namespace aturan {

struct Grid {
    int im, jm, km, kp;
    size_t fstride;            // elements per field (im * jm * kp)
};

__host__ __device__ __forceinline__ size_t gidx(const Grid& g, int i, int j, int k){
    return ((size_t)i * g.jm + j) * g.kp + k;
}

// ATPhys.h:135-139, the periodic seam: ring of km-1 distinct meridians.
__host__ __device__ __forceinline__ int phi_wrap(int kk, int km){
    const int n = km - 1;
    return kk < 0 ? kk + n : (kk >= n ? kk - n : kk);
}

// Per-(i,j) metric of RungeKutta_Uran_Turb.cpp:258-283 plus the products of it the RHS forms
// (RHS_Uran_Turb.cpp:224-331), computed once on the host in FP64 in the reference's operand
// order and uploaded, so the device reads exactly the CPU's values.
template <typename T>
struct GeoIJ {
    T inv_rm, inv_rm2, inv_rmsinthe, inv_rm2sinthe, inv_rm2sinthe2, costhe_inv_rm2sinthe;
    T costhe, cotanthe, v_metric, two_inv_rm, sinthe_bf, cent_rad, cent_the, sponge;
};

// Scalars of the RHS and the RK4 update, precomputed on the host in the operand order in which
// the reference forms them (each product noted beside its field).
template <typename T>
struct RhsConst {
    T inv_2dr, inv_2dthe, inv_2dphi, inv_dr2, inv_dthe2, inv_dphi2;
    T ce_sp;            // coeff_energy_p * scale_p
    T scale_p;
    T m2om, p2om;       // -2 omega, +2 omega
    T cor_sc;           // Coriolis * scale_Cor
    T cor_rad_f;        // cor_rad_on * Coriolis * scale_Cor  (0: CORIOLIS_SPLIT)
    T cen_f;            // 1.0 * centrifugal * cent_mom * scale_cen
    T re, re_pr, re_eff, inv_re;
    T turb_coupling, precip_coupling, chemical_reaction;
    T tmf;              // tmf_scale * chemical_reaction
    T precip_L;         // L_atm * 1e3
    T precip_den;       // r_mix * cp_mix * u_0 * t_ref
    T sc_re[5];         // sc * re for ch4, h2o, h2s, nh3, nh4sh
    T stokes_a;         // (2/9) r_p r_p
    T rho_cond_nh4sh, g, mue_mix, u_0;
    T cp_mix, t_ref;
    T cp_rh2, cp_he_term, cp_ch4_term, cp_rsum, cp_h2_const;   // cp(T), CpH2.h:122-134
    T tke_max, dis_min, t_min, t_max, dt;
    T heat_scale;       // (L_atm * 1e3 / u_0) / t_ref: a heating rate in K/s as a tendency of t
    // reciprocals of the divisors above, for the mixed form's multiplications (qdiv)
    T inv_re_eff, inv_re_pr, inv_sc_re[5], inv_mue_mix, inv_u_0, inv_precip_den, inv_cp_rsum;
    int cp_dyn, cp_gas, cp_mode, turb_active;
};

// Constants of the buoyancy reference level and the hydrostatic column integral
// (RungeKutta_Uran_Turb.cpp:18-177).
struct HydroConst {
    double g, rR, t_ref;       // b = g p / (rR T t_ref), rR = r_mix * R_mix
    double m_nd_rel_b;         // -nd_rel * buoy_scale * buoyancy (buoy_scale = 1)
    double dr, follow_tau;
    int follow_on;
};

// Scratch of the exact (reference-order) level means: the terms, per-chunk sums and flags, and the
// per-chunk binades and units (rk4.cuh, buoy_terms_kernel to buoy_serial_pass_kernel).
struct BuoyScratch {
    double* terms;          // [im][2][jm*km]
    double* bpart;          // [im][nbx][3]
    int* bexp;              // [im][nbx][2]
    long long* bunits;      // [im][nbx][4]
    int nbx;                // chunks per level
};

constexpr int CP_TABLE_N = 2991;   // (1500 - 5) / 0.5 + 1, CpH2.h:66-75

// The mixed form carries the temperature (t and its start-of-step copy tn) as an FP32 pair: the
// stored FP32 value hi, which every stencil reads, and lo = the FP32-rounded remainder T - hi, so
// that T = hi + lo to about 2^-48 relative. The kernels that write T (the RK4 final update, the
// saturation adjustment, the passes after RK4, the layout kernels) form it in FP64 from hi + lo
// and store both halves. Without lo the FP32 rounding of T (~6e-8) moves the adjustment's
// relative 1e-3 stopping test (SaturationAdjustment.h:250-251) to another pass in some cells of
// the CH4 band, a jump of ~1e-5 in T there. lo is null in an FP64 context (and ignored).
template <typename S>
__device__ __forceinline__ double t_ld(const S* hi, const float* lo, size_t q){
    double v = (double)hi[q];
    if(lo) v += (double)lo[q];
    return v;
}
template <typename S>
__device__ __forceinline__ void t_st(S* hi, float* lo, size_t q, double v){
    const S h = (S)v;
    hi[q] = h;
    if(lo) lo[q] = (float)(v - (double)h);
}

}  // namespace aturan
