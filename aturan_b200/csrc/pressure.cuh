// Poisson pressure solves of the dynamic pressure p_dyn (always FP64 on the device).
//
// GS_LEX reproduces PressureSolverUran::run() (planet/PressureSolverUran.h:33-250): ONE
// lexicographic Gauss-Seidel sweep i -> j -> k over the interior, in place. A serial sweep
// makes cell (i,j,k) see the NEW values of (i-1,j,k), (i,j-1,k), (i,j,k-1) and the OLD values of
// (i+1,j,k), (i,j+1,k), (i,j,k+1); at the seam k = 0 reads the old k = km-2 and k = km-2 reads
// the new k = 0. Every one of those relations is preserved by sweeping the hyperplanes
// s = i + j + k in increasing order, all cells of one hyperplane in parallel: a neighbour with a
// smaller coordinate sum is already new, one with a larger sum is still old (the seam pair
// included: k = km-2 lies km-2 hyperplanes after k = 0). So the wavefront computes exactly the
// serial sweep's values, cell for cell, with no change in any arithmetic.
//
// RB_SHARED reproduces PressureSolver<Planet>::run() (planet/PressureSolver.h:145-766) with
// N sweeps: red-black colouring on (i+j+k)&1, the div(aux) source clamped at den*p_dyn_cap, the
// model's projection boundaries first (planet/Pressure_Uran.cpp:30-146) and the p_dyn boundary
// passes inside the sweep loop.
#pragma once
#include "common.cuh"

namespace aturan {

constexpr double C43 = 4.0 / 3.0, C13 = 1.0 / 3.0;   // cUranusModel.h:866

// Per-(i,j) weights of PressureSolverUran (sweep and defect-correction source; :139-199).
struct GSW {
    double num1, num2, num3, inv_denom;           // sweep, :180-190
    double inv_rm, inv_rmsinthe;                  // both sources
    double n1, n2, n3, denom;                     // incr_src, :151-157
};

// Per-(i,j) weights of the shared solver (:326-353) and its clamp bound den * p_dyn_cap.
struct RBW {
    double num1, num2, num3, den, inv_rm, inv_rmsinthe, src_max;
};

struct PressConst {
    double inv_2dr, inv_2dthe, inv_2dphi, two_dr, two_dthe, two_dphi, src_scale;
    int press_incr;
};

// ---- PressureSolverUran.h:70-81: aux radial planes ----
template <typename S>
__global__ void gs_aux_bc_kernel(Grid g, S* au, S* av, S* aw){
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    if(k > g.km - 2 || j > g.jm - 2) return;
    S* A[3] = {au, av, aw};
    for(int q = 0; q < 3; q++){
        S* a = A[q];
        a[gidx(g, 0, j, k)]        = (S)(C43 * (double)a[gidx(g, 1, j, k)] - C13 * (double)a[gidx(g, 2, j, k)]);
        a[gidx(g, g.im - 1, j, k)] = (S)(C43 * (double)a[gidx(g, g.im - 2, j, k)] - C13 * (double)a[gidx(g, g.im - 3, j, k)]);
    }
}

// ---- PressureSolverUran.h:139-175: incr_src = src_scale div(rhs) + Lc(p_old), the radial
// end planes of rhs_u read as their 2-point extrapolation ----
template <typename S>
__global__ void gs_incr_kernel(Grid g, const S* ru, const S* rv, const S* rw, const double* P,
                               const GSW* w, PressConst c, double* incr){
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    const int i = 1 + blockIdx.z;
    if(k > g.km - 2 || j > g.jm - 2) return;
    const GSW W = w[i * g.jm + j];
    const int kw = phi_wrap(k - 1, g.km), ke = phi_wrap(k + 1, g.km);
    auto RU = [&](int ii) -> double {
        if(ii == 0) return C43 * (double)ru[gidx(g, 1, j, k)] - C13 * (double)ru[gidx(g, 2, j, k)];
        if(ii == g.im - 1) return C43 * (double)ru[gidx(g, g.im - 2, j, k)] - C13 * (double)ru[gidx(g, g.im - 3, j, k)];
        return (double)ru[gidx(g, ii, j, k)];
    };
    const double div_rhs =
          (RU(i + 1) - RU(i - 1)) / c.two_dr
        + ((double)rv[gidx(g, i, j + 1, k)] - (double)rv[gidx(g, i, j - 1, k)]) / c.two_dthe * W.inv_rm
        + ((double)rw[gidx(g, i, j, ke)] - (double)rw[gidx(g, i, j, kw)]) / c.two_dphi * W.inv_rmsinthe;
    const double lc_old =
          (P[gidx(g, i + 1, j, k)] + P[gidx(g, i - 1, j, k)]) * W.n1
        + (P[gidx(g, i, j + 1, k)] + P[gidx(g, i, j - 1, k)]) * W.n2
        + (P[gidx(g, i, j, ke)] + P[gidx(g, i, j, kw)]) * W.n3
        - W.denom * P[gidx(g, i, j, k)];
    incr[gidx(g, i, j, k)] = c.src_scale * div_rhs + lc_old;
}

// ---- PressureSolverUran.h:177-211: one hyperplane s = i + j + k of the lexicographic sweep ----
template <typename S>
__global__ void __launch_bounds__(256) gs_hyperplane_kernel(Grid g, double* P, const double* incr,
                                                            const S* au, const S* av, const S* aw,
                                                            const GSW* w, PressConst c, int s){
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int nj = g.jm - 2;
    if(t >= (g.im - 2) * nj) return;
    const int i = 1 + t / nj, j = 1 + (t - (i - 1) * nj);
    const int k = s - i - j;
    if(k < 0 || k > g.km - 2) return;
    const GSW W = w[i * g.jm + j];
    const int kw = phi_wrap(k - 1, g.km), ke = phi_wrap(k + 1, g.km);
    double src;
    if(c.press_incr) src = incr[gidx(g, i, j, k)];
    else {
        const double du_dr   = ((double)au[gidx(g, i + 1, j, k)] - (double)au[gidx(g, i - 1, j, k)]) * c.inv_2dr;
        const double dv_dthe = ((double)av[gidx(g, i, j + 1, k)] - (double)av[gidx(g, i, j - 1, k)]) * c.inv_2dthe * W.inv_rm;
        const double dw_dphi = ((double)aw[gidx(g, i, j, ke)] - (double)aw[gidx(g, i, j, kw)]) * c.inv_2dphi * W.inv_rmsinthe;
        src = c.src_scale * (du_dr + dv_dthe + dw_dphi);
    }
    P[gidx(g, i, j, k)] =
        ((P[gidx(g, i + 1, j, k)] + P[gidx(g, i - 1, j, k)]) * W.num1
       + (P[gidx(g, i, j + 1, k)] + P[gidx(g, i, j - 1, k)]) * W.num2
       + (P[gidx(g, i, j, ke)] + P[gidx(g, i, j, kw)]) * W.num3
       - src) * W.inv_denom;
}

// ---- p_dyn boundary passes, in the reference's order: radial planes over every (j,k), then
// the polar rows over every (i,k), then the seam copy (PressureSolverUran.h:213-244,
// PressureSolver.h:718-746) ----
static __global__ void pdyn_bc_r_kernel(Grid g, double* P){
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if(k >= g.km) return;
    P[gidx(g, 0, j, k)]        = C43 * P[gidx(g, 1, j, k)] - C13 * P[gidx(g, 2, j, k)];
    P[gidx(g, g.im - 1, j, k)] = C43 * P[gidx(g, g.im - 2, j, k)] - C13 * P[gidx(g, g.im - 3, j, k)];
}
static __global__ void pdyn_bc_t_kernel(Grid g, double* P){
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if(k >= g.km) return;
    P[gidx(g, i, 0, k)]        = C43 * P[gidx(g, i, 1, k)] - C13 * P[gidx(g, i, 2, k)];
    P[gidx(g, i, g.jm - 1, k)] = C43 * P[gidx(g, i, g.jm - 2, k)] - C13 * P[gidx(g, i, g.jm - 3, k)];
}
static __global__ void pdyn_bc_p_kernel(Grid g, double* P){
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if(c >= g.im * g.jm) return;
    const int i = c / g.jm, j = c - i * g.jm;
    P[gidx(g, i, j, g.km - 1)] = P[gidx(g, i, j, 0)];
}

// ---- Pressure_Uran.cpp:30-146, prepareProjectionBoundaries(rigid_lid), periodic phi.
// The radial and polar passes touch disjoint cells and read only interior ones, so they may
// run in one launch; the seam copy follows. ----
template <typename S>
__global__ void prep_rt_kernel(Grid g, S* au, S* av, S* aw, S* ru, S* rv, S* rw, int rigid_lid){
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;                       // y < jm-2: radial pass row j = y+1, else polar pass level
    if(k > g.km - 2) return;
    S* A[6] = {au, av, aw, ru, rv, rw};
    auto cub = [&](S* X, size_t a3, size_t a2, size_t a1) -> S {
        return (S)((double)X[a3] - 3.0 * (double)X[a2] + 3.0 * (double)X[a1]);
    };
    if(y < g.jm - 2){
        const int j = y + 1;
        for(int q = 0; q < 6; q++){
            S* X = A[q];
            if(q == 0 && rigid_lid){
                X[gidx(g, 0, j, k)] = (S)0.0; X[gidx(g, g.im - 1, j, k)] = (S)0.0;
            } else {
                X[gidx(g, 0, j, k)] = cub(X, gidx(g, 3, j, k), gidx(g, 2, j, k), gidx(g, 1, j, k));
                X[gidx(g, g.im - 1, j, k)] = cub(X, gidx(g, g.im - 4, j, k), gidx(g, g.im - 3, j, k), gidx(g, g.im - 2, j, k));
            }
        }
    } else {
        const int i = y - (g.jm - 2) + 1;
        if(i > g.im - 2) return;
        for(int q = 0; q < 6; q += 3){              // aux_u / rhs_u: cubic; v, w: zero at the poles
            S* X = A[q];
            X[gidx(g, i, 0, k)] = cub(X, gidx(g, i, 3, k), gidx(g, i, 2, k), gidx(g, i, 1, k));
            X[gidx(g, i, g.jm - 1, k)] = cub(X, gidx(g, i, g.jm - 4, k), gidx(g, i, g.jm - 3, k), gidx(g, i, g.jm - 2, k));
            A[q + 1][gidx(g, i, 0, k)] = (S)0.0; A[q + 2][gidx(g, i, 0, k)] = (S)0.0;
            A[q + 1][gidx(g, i, g.jm - 1, k)] = (S)0.0; A[q + 2][gidx(g, i, g.jm - 1, k)] = (S)0.0;
        }
    }
}
template <typename S>
__global__ void prep_seam_kernel(Grid g, S* au, S* av, S* aw, S* ru, S* rv, S* rw){
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if(c >= g.im * g.jm) return;
    const int i = c / g.jm, j = c - i * g.jm;
    S* A[6] = {au, av, aw, ru, rv, rw};
    for(int q = 0; q < 6; q++) A[q][gidx(g, i, j, g.km - 1)] = A[q][gidx(g, i, j, 0)];
}

// ---- PressureSolver.h:370-487: div(aux) source, clamped, non-finite guard ----
template <typename S>
__global__ void rb_src_kernel(Grid g, const S* au, const S* av, const S* aw, const RBW* w,
                              PressConst c, double* src){
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    const int i = 1 + blockIdx.z;
    if(k > g.km - 2 || j > g.jm - 2) return;
    const RBW W = w[i * g.jm + j];
    const int kw = phi_wrap(k - 1, g.km), ke = phi_wrap(k + 1, g.km);
    const double du_dr   = ((double)au[gidx(g, i + 1, j, k)] - (double)au[gidx(g, i - 1, j, k)]) * c.inv_2dr;
    const double dv_dthe = ((double)av[gidx(g, i, j + 1, k)] - (double)av[gidx(g, i, j - 1, k)]) * c.inv_2dthe;
    const double dw_dphi = ((double)aw[gidx(g, i, j, ke)] - (double)aw[gidx(g, i, j, kw)]) * c.inv_2dphi;
    double d = du_dr * 1.0 + dv_dthe * W.inv_rm + dw_dphi * W.inv_rmsinthe;
    if(!isfinite(d)) d = 0.0;
    else if(d >  W.src_max) d =  W.src_max;
    else if(d < -W.src_max) d = -W.src_max;
    src[gidx(g, i, j, k)] = d;
}

// ---- PressureSolver.h:320-495: one colour of the red-black relaxation. omega = 1 is the
// reference's update p = (acc - src) / den; other omega over-relax it (RB_SOR). ----
static __global__ void __launch_bounds__(256) rb_colour_kernel(Grid g, double* P, const double* src, const RBW* w,
                                                        int colour, double omega){
    const int half = g.km / 2;                       // km-1 even: each row holds half of each colour
    const int k2 = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    const int i = 1 + blockIdx.z;
    if(k2 >= half || j > g.jm - 2) return;
    const int k = 2 * k2 + ((i + j + colour) & 1);
    if(k > g.km - 2) return;
    const RBW W = w[i * g.jm + j];
    const int kw = phi_wrap(k - 1, g.km), ke = phi_wrap(k + 1, g.km);
    const size_t o = gidx(g, i, j, k);
    const double acc = (P[o + (size_t)g.jm * g.kp] + P[o - (size_t)g.jm * g.kp]) * W.num1
                     + (P[o + g.kp] + P[o - g.kp]) * W.num2
                     + (P[o - k + ke] + P[o - k + kw]) * W.num3;
    const double pn = (acc - src[o]) / W.den;
    P[o] = (omega == 1.0) ? pn : P[o] + omega * (pn - P[o]);
}

}  // namespace aturan
