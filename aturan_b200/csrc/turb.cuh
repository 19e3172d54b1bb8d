// The turbulence closure (planet/Turbulence.h, Turbulence<cUranusModel>::run, :307-331), k-omega
// SST with the reference's default knobs: TURB_FREE (no wall law, the background k floor, the
// free-flow wall distance), TURB_CLAMP_PASS (the clamps as passes around the source loop), no land
// cells, no buoyancy term, no ABL taper, and the closure's fields outside the model's own boundary
// lists (the edges copied from their neighbours).
//
// Three launches:
//   turb_sources_kernel  one thread per interior cell: the production tensor from the 7-point
//                        gradients of u, v, w and of k*, omega* (the clamp pass applied on the fly
//                        to every interior value it reads), the SST eddy viscosity and sources, and
//                        the caps of the clamp pass after the loop (which read only the cell);
//   turb_column_kernel   one thread per (j, k) column: the floors of k* and omega* on the interior
//                        (after every read of the source loop), the zero-gradient copy at i = 0 and
//                        the eddy-viscosity clamp on the whole column;
//   turb_edges_kernel    the seam copy, the lid row and the pole rows of the eight fields, each edge
//                        cell read from where the three copies in the reference's order take it.
// Arithmetic is FP64 on the stored values in the reference's operand order; the metric radius and
// sin, cos of the colatitude come from the host table the chemistry uses (host libm), so all of it
// but the SST blending's tanh and pow matches the CPU bit for bit; with TURB_FREE's wall distance
// of 1e20 m the blending arguments are ~1e-20 and F1, F2 vanish against 1, so in practice that
// holds there as well.
#pragma once
#include "common.cuh"

namespace aturan {

struct TurbConst {
    double dis_min, nue_max, k_bg_nd, nue_air_nd, y_star;
    double dr, dthe, dphi;
    int curv, per;
};

template <typename S>
struct TurbArgs {
    Grid g;
    S *tke, *dis, *tken, *disn, *nue, *prod, *tks, *dss;
    const S *u, *v, *w;
    const double *rmm, *sin, *cos;      // metric radius (im), sin and cos of the colatitude (jm)
    TurbConst c;
};

__device__ __forceinline__ double turb_max(double a, double b){ return (a < b) ? b : a; }   // std::max
__device__ __forceinline__ double turb_min(double a, double b){ return (b < a) ? b : a; }   // std::min
__device__ __forceinline__ double turb_clamp3(double x, double lo, double hi){            // Turbulence.h:207-209
    return (x < lo) ? lo : ((x > hi) ? hi : x);
}
__device__ __forceinline__ double turb_blend(double inner, double outer, double F1){       // :203-205
    return F1 * inner + (1.0 - F1) * outer;
}

template <typename S>
__global__ void __launch_bounds__(128) turb_sources_kernel(TurbArgs<S> a){
    const Grid& g = a.g;
    const TurbConst& c = a.c;
    const int kf = c.per ? 0 : 1;
    const int k = kf + blockIdx.x * blockDim.x + threadIdx.x, j = 1 + blockIdx.y, i = 1 + blockIdx.z;
    if(k > g.km - 2) return;
    const size_t q = gidx(g, i, j, k), pl = (size_t)g.jm * g.kp, kp = (size_t)g.kp;
    int kw, ke;
    if(c.per){ kw = phi_wrap(k - 1, g.km); ke = phi_wrap(k + 1, g.km); }
    else { kw = k - 1; ke = k + 1; }
    const size_t qw = q - k + kw, qe = q - k + ke;
    // the clamp pass before the loop (:645-650) acts on the interior only: a neighbour on the
    // boundary is read as it is
    const bool in_im = i - 1 >= 1, in_ip = i + 1 <= g.im - 2, in_jm = j - 1 >= 1, in_jp = j + 1 <= g.jm - 2;
    const bool in_kw = kw >= kf && kw <= g.km - 2, in_ke = ke >= kf && ke <= g.km - 2;
    auto tk = [&](size_t o, bool in) -> double { const double x = (double)a.tke[o]; return in ? turb_max(0.0, x) : x; };
    auto ds = [&](size_t o, bool in) -> double { const double x = (double)a.dis[o]; return in ? turb_max(c.dis_min, x) : x; };
    const double tk0 = tk(q, true), ds0 = ds(q, true);

    const double rm = a.rmm[i];
    const double exp_rm = 1.0;                                 // coord_stretching false
    double sinthe = a.sin[j];
    if(sinthe == 0.0) sinthe = 1.0e-5;
    const double costhe = a.cos[j];
    const double cotanthe = costhe / sinthe;
    const double inv_rm = 1.0 / rm;
    const double rmsinthe = rm * sinthe;
    const double inv_2dr = 1.0 / (2.0 * c.dr);
    const double inv_2dthe = 1.0 / (2.0 * c.dthe);
    const double inv_2dphi = 1.0 / (2.0 * c.dphi);
    const double inv_rm2dthe = inv_2dthe / rm;
    const double inv_rmsinthe2dphi = inv_2dphi / rmsinthe;
    auto d_r = [&](const S* x){ return ((double)x[q + pl] - (double)x[q - pl]) * inv_2dr * exp_rm; };
    auto d_t = [&](const S* x){ return ((double)x[q + kp] - (double)x[q - kp]) * inv_rm2dthe; };
    auto d_p = [&](const S* x){ return ((double)x[qe] - (double)x[qw]) * inv_rmsinthe2dphi; };
    const double dudr = d_r(a.u), dvdr = d_r(a.v), dwdr = d_r(a.w);
    const double dudthe = d_t(a.u), dvdthe = d_t(a.v), dwdthe = d_t(a.w);
    const double dudphi = d_p(a.u), dvdphi = d_p(a.v), dwdphi = d_p(a.w);
    const double dtkedr = (tk(q + pl, in_ip) - tk(q - pl, in_im)) * inv_2dr * exp_rm;
    const double ddisdr = (ds(q + pl, in_ip) - ds(q - pl, in_im)) * inv_2dr * exp_rm;

    // the production tensor (:697-760)
    double cnue;
    {
        const double dis_here = turb_max(ds0, c.dis_min);
        const double tke_here = turb_max(tk0, 0.0);
        cnue = tke_here / dis_here;
        cnue = turb_min(cnue, c.nue_max);
    }
    const double u0 = (double)a.u[q], v0 = (double)a.v[q], w0 = (double)a.w[q];
    const double u_r = c.curv ? u0 * inv_rm : 0.0;
    const double v_r = c.curv ? v0 * inv_rm : 0.0;
    const double w_r = c.curv ? w0 * inv_rm : 0.0;
    const double v_cot_r = v_r * cotanthe;
    const double w_cot_r = w_r * cotanthe;
    const double g_rr = dudr, g_rt = dudthe - v_r, g_rp = dudphi - w_r;
    const double g_tr = dvdr, g_tt = dvdthe + u_r, g_tp = dvdphi - w_cot_r;
    const double g_pr = dwdr, g_pt = dwdthe, g_pp = dwdphi + u_r + v_cot_r;
    const double der = 0.66667 * (g_rr + g_tt + g_pp);
    const double prod = turb_max(0.0,
          (cnue * (2.0 * g_rr - der) - 0.66667 * tk0) * g_rr
        + (cnue * (g_rt + g_tr)) * g_rt
        + (cnue * (g_rp + g_pr)) * g_rp
        + (cnue * (2.0 * g_tt - der) - 0.66667 * tk0) * g_tt
        + (cnue * (g_tr + g_rt)) * g_tr
        + (cnue * (g_tp + g_pt)) * g_tp
        + (cnue * (2.0 * g_pp - der) - 0.66667 * tk0) * g_pp
        + (cnue * (g_pr + g_rp)) * g_pr
        + (cnue * (g_pt + g_tp)) * g_pt);
    const double W12 = g_rt - g_tr, W13 = g_rp - g_pr, W23 = g_tp - g_pt;
    const double Omega = sqrt(W12 * W12 + W13 * W13 + W23 * W23);

    // compute_k_omega_SST (:1020-1100), no land cells, no wall
    const double a1 = 0.31, bet_star = 0.09, bet1 = 0.0333, bet2 = 0.0368;
    const double gam1 = 0.413, gam2 = 0.2, sig_w2 = 1.168;
    const double y_star = c.y_star;
    const double dtkedthe_neu = (tk(q + kp, in_jp) - tk(q - kp, in_jm)) / (rm * 2.0 * c.dthe);
    const double ddisdthe_neu = (ds(q + kp, in_jp) - ds(q - kp, in_jm)) / (rm * 2.0 * c.dthe);
    const double dtkedphi_neu = (tk(qe, in_ke) - tk(qw, in_kw)) / (rmsinthe * 2.0 * c.dphi);
    const double ddisdphi_neu = (ds(qe, in_ke) - ds(qw, in_kw)) / (rmsinthe * 2.0 * c.dphi);
    const double grad_dot = dtkedr * ddisdr + dtkedthe_neu * ddisdthe_neu + dtkedphi_neu * ddisdphi_neu;
    const double CD_kw = turb_max(2.0 * sig_w2 / turb_max(ds0, 1.0e-20) * grad_dot, 1.0e-20);
    const double dis_safe = turb_max(ds0, 1.0e-20);
    const double arg1 = turb_min(
        turb_max(sqrt(tk0) / (bet_star * dis_safe * y_star), 500.0 * c.nue_air_nd / (y_star * y_star * dis_safe)),
        4.0 * sig_w2 * tk0 / (CD_kw * y_star * y_star));
    const double arg2 = turb_max(2.0 * sqrt(tk0) / (bet_star * dis_safe * y_star),
                                 500.0 * c.nue_air_nd / (y_star * y_star * dis_safe));
    const double F1 = tanh(pow(arg1, 4.0));
    const double F2 = tanh(pow(arg2, 2.0));
    const double nue = a1 * tk0 / turb_max(a1 * dis_safe, Omega * F2);
    const double tke_safe = turb_max(tk0, 1.0e-20);
    const double P_k = turb_min(prod, 20.0 * bet_star * tke_safe * dis_safe);
    const double Y_k = bet_star * tke_safe * dis_safe;
    const double P_w = turb_blend(gam1, gam2, F1) * P_k * dis_safe / tke_safe;
    const double Y_w = turb_blend(bet1, bet2, F1) * dis_safe * dis_safe;
    const double D_w = 2.0 * (1.0 - F1) * sig_w2 / dis_safe * grad_dot;
    const double tks = P_k - Y_k;
    const double dss = P_w - Y_w + D_w;

    // the caps of the pass after the loop (:631-643), on the cell's floored k* and omega*
    const double tke_f = turb_max(c.k_bg_nd, tk0), dis_f = turb_max(c.dis_min, ds0);
    const double dis_src_max = 20.0 * dis_f * dis_f;
    const double tke_src_max = 20.0 * tke_f * dis_f;
    a.prod[q] = (S)prod;
    a.nue[q] = (S)turb_clamp3(nue, 0.0, c.nue_max);
    a.dss[q] = (S)turb_clamp3(dss, -dis_src_max, dis_src_max);
    a.tks[q] = (S)turb_clamp3(tks, -tke_src_max, tke_src_max);
}

// Per (j, k) column: the floors of the pass after the loop on the interior, apply_wall_bc's copy at
// i = 0 (:414-419), clamp_nue on every level (:565-589).
template <typename S>
__global__ void __launch_bounds__(128) turb_column_kernel(TurbArgs<S> a){
    const Grid& g = a.g;
    const TurbConst& c = a.c;
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if(k >= g.km) return;
    const size_t pl = (size_t)g.jm * g.kp, o = gidx(g, 0, j, k);
    const int kf = c.per ? 0 : 1;
    // CH levels at a time, every load of a chunk before its stores (a store could alias the next
    // level's load as far as the compiler knows); the same operations per cell, in the same order
    constexpr int CH = 8;
    if(j >= 1 && j <= g.jm - 2 && k >= kf && k <= g.km - 2)
        for(int i0 = 1; i0 < g.im - 1; i0 += CH){
            S tk[CH], ds[CH];
#pragma unroll
            for(int u = 0; u < CH; u++)
                if(i0 + u < g.im - 1){ const size_t q = o + (size_t)(i0 + u) * pl; tk[u] = a.tke[q]; ds[u] = a.dis[q]; }
#pragma unroll
            for(int u = 0; u < CH; u++)
                if(i0 + u < g.im - 1){
                    const size_t q = o + (size_t)(i0 + u) * pl;
                    a.tke[q] = (S)turb_max(c.k_bg_nd, turb_max(0.0, (double)tk[u]));
                    a.dis[q] = (S)turb_max(c.dis_min, turb_max(c.dis_min, (double)ds[u]));
                }
        }
    a.tke[o] = a.tke[o + pl];
    a.dis[o] = a.dis[o + pl];
    a.nue[o] = a.nue[o + pl];
    for(int i0 = 0; i0 < g.im; i0 += CH){
        S nu[CH];
#pragma unroll
        for(int u = 0; u < CH; u++) if(i0 + u < g.im) nu[u] = a.nue[o + (size_t)(i0 + u) * pl];
#pragma unroll
        for(int u = 0; u < CH; u++)
            if(i0 + u < g.im) a.nue[o + (size_t)(i0 + u) * pl] = (S)(turb_clamp3((double)nu[u], 0.0, c.nue_max) * 1.0);
    }
}

// seam_copy (:543-562), then fill_lid_corners without the model's own boundary lists (:511-540):
// the lid row from i = im-2 (j = 1..jm-2), then the pole rows from j = 1 and jm-2 (every i). Each
// edge cell takes its value from where that sequence takes it; those source cells are never edge
// cells, so one launch holds no read-after-write hazard. Segments of the flat index: the seam
// cells off the lid and pole rows, the lid row, the pole pairs.
template <typename S>
__global__ void __launch_bounds__(128) turb_edges_kernel(TurbArgs<S> a){
    const Grid& g = a.g;
    const int im = g.im, jm = g.jm, km = g.km;
    const long nseam = a.c.per ? (long)(im - 1) * (jm - 2) : 0;
    const long nlid = (long)(jm - 2) * km, npole = (long)im * km;
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    // the value after the seam copy of (i, j, k)
    auto seam_src = [&](int i, int j, int k) -> size_t {
        return gidx(g, i, j, (a.c.per && k == km - 1) ? 0 : k);
    };
    // the value after the lid copy of (i, j, k), 1 <= j <= jm-2
    auto lid_src = [&](int i, int j, int k) -> size_t {
        return seam_src(i == im - 1 ? im - 2 : i, j, k);
    };
    S* f[8] = {a.tke, a.dis, a.tken, a.disn, a.nue, a.prod, a.tks, a.dss};
    if(t < nseam){
        const int i = (int)(t / (jm - 2)), j = 1 + (int)(t % (jm - 2));
        const size_t d = gidx(g, i, j, km - 1), s = gidx(g, i, j, 0);
#pragma unroll
        for(int n = 0; n < 8; n++) f[n][d] = f[n][s];
        return;
    }
    t -= nseam;
    if(t < nlid){
        const int j = 1 + (int)(t / km), k = (int)(t % km);
        const size_t d = gidx(g, im - 1, j, k), s = lid_src(im - 1, j, k);
#pragma unroll
        for(int n = 0; n < 8; n++) f[n][d] = f[n][s];
        return;
    }
    t -= nlid;
    if(t < npole){
        const int i = (int)(t / km), k = (int)(t % km);
        const size_t d0 = gidx(g, i, 0, k), s0 = lid_src(i, 1, k);
        const size_t d1 = gidx(g, i, jm - 1, k), s1 = lid_src(i, jm - 2, k);
#pragma unroll
        for(int n = 0; n < 8; n++){ f[n][d0] = f[n][s0]; f[n][d1] = f[n][s1]; }
    }
}

}  // namespace aturan
