// Definitions of the launch wrappers declared in launch.h, instantiated per storage/compute type
// by the translation unit that includes this file (fp64.cu, mixed.cu).
#pragma once
#include "rk4.cuh"
#include "satadj.cuh"
#include "pressure.cuh"
#include "post.cuh"
#include "chem.cuh"
#include "turb.cuh"
#include "precip.cuh"
#include "mca.cuh"

namespace aturan {
// Stage launch configuration per storage type, measured on B200 at 41x181x361: resident blocks per
// SM of the momentum launch (MINB1) and of the scalar launch (MINB2), and the scalar launch's
// prefetch depth (PD fields ahead). The scalar launch takes two cells per thread
// (rk_scalar_pair_kernel): 5 % faster than one cell per thread in FP64, 15 % in FP32.
// AD > 0: the scalar launch stages its loads through a ring of AD shared-memory slots
// (rk_scalar_async_kernel) at AMINB resident blocks per SM instead of the register ring. FP64:
// 6-9 % faster than the register ring at 3 or 4 blocks per SM; FP32: 3-25 % slower at every
// depth and occupancy tried, so the register ring stays, one field ahead at 6 blocks per SM
// (80 registers; 9 % faster than 4 blocks with two fields ahead).
// MP > 0: the momentum launch takes two cells per thread (rk_stage_pair_kernel) at MP resident
// blocks per SM instead of one cell per thread at MINB1. FP32: 128 registers at 4 blocks per SM,
// a 1.5 % faster stage than one cell per thread at 7 (3 blocks per SM: 2 % slower). FP64: the
// pair form spills at 3-5 blocks per SM, so it keeps one cell per thread.
template <typename S> struct StageCfg { static constexpr int MINB1 = 5, MP = 0, PD = 1, MINB2 = 3, AD = 2, AMINB = 3; };
template <> struct StageCfg<float> { static constexpr int MINB1 = 7, MP = 4, PD = 1, MINB2 = 6, AD = 0, AMINB = 4; };
// The saturation adjustment has no shared memory of its own, so left to itself it runs with the
// smallest shared-memory split of each SM's L1, and a kernel that needs shared memory (the pressure
// solve's, beside it in aturan_step) cannot start on that SM until all its blocks have left.
// Preferring the largest split lets the solve's blocks take each slot the adjustment frees.
template <typename K>
inline void prefer_max_shared(K* kernel){
    if(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                            (int)cudaSharedmemCarveoutMaxShared) != cudaSuccess)
        cudaGetLastError();                       // a hint: carry on without it
}
// Saturation adjustment: threads per block (one row segment of NT cells along k).
template <typename S> struct SatCfg { static constexpr int NT = 128; };
template <typename S, typename C>
void launch_scalars(const StageArgs<S, C>& a, dim3 grid2, cudaStream_t st){
    if constexpr(StageCfg<S>::AD > 0){
        constexpr int D = StageCfg<S>::AD;
        auto kern = rk_scalar_async_kernel<S, C, D, StageCfg<S>::AMINB>;
        const int sm = D * (int)sizeof(AsyncSlot<S>);
        static const bool attr = (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, sm) == cudaSuccess)
                                 || (cudaGetLastError(), false);
        (void)attr;
        kern<<<grid2, dim3(32, 4), sm, st>>>(a);
    } else {
        rk_scalar_pair_kernel<S, C, StageCfg<S>::PD, StageCfg<S>::MINB2><<<grid2, dim3(32, 4), 0, st>>>(a);
    }
}
template <typename S, typename C>
void launch_momentum(const StageArgs<S, C>& a, dim3 grid2, cudaStream_t st){
    if constexpr(StageCfg<S>::MP > 0){
        rk_stage_pair_kernel<S, C, StageCfg<S>::MP><<<grid2, dim3(32, 4), 0, st>>>(a);
    } else {
        const Grid& g = a.g;
        const dim3 grid((g.km - 1 + 31) / 32, (g.jm - 2 + 3) / 4, g.im - 2);
        rk_stage_kernel<S, C, StageCfg<S>::MINB1><<<grid, dim3(32, 4), 0, st>>>(a);
    }
}
// damp_wiggles (lib/Utils.cpp:224-317) on x along the axes selected, k then j then i; lo: the low
// part of the mixed form's temperature pair when x is t (common.cuh), else null. Returns the
// number of launches.
template <typename S>
int launch_filter(const Grid& g, S* x, float* lo, bool ai, bool aj, bool ak, double strength, int phi_periodic,
                  cudaStream_t st){
    const double coeff = strength * 0.25;                 // lib/Utils.cpp:232
    const dim3 cols_k((g.km + 127) / 128);
    int n = 0;
    if(ak){
        // four rows (warps) per block while they fit the default 48 KB, else one row per block
        // with the opt-in size (rows of up to 8192 values)
        const int R = 4 * g.km * (int)sizeof(double) <= 48 * 1024 ? 4 : 1;
        const int sm = R * g.km * (int)sizeof(double), rows = g.im * g.jm;
        static const bool big = (cudaFuncSetAttribute(post_filter_k_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                      8192 * (int)sizeof(double)) == cudaSuccess) || (cudaGetLastError(), false);
        (void)big;
        post_filter_k_kernel<S><<<(rows + R - 1) / R, dim3(32, R), sm, st>>>(g, x, lo, coeff, phi_periodic && g.km > 2, rows);
        n++;
    }
    if(aj){ post_filter_j_kernel<S><<<dim3(cols_k.x, g.im), 128, 0, st>>>(g, x, lo, coeff); n++; }
    if(ai){ post_filter_i_kernel<S><<<dim3(cols_k.x, g.jm), 128, 0, st>>>(g, x, lo, coeff); n++; }
    return n;
}
// damp_wiggles on x along all three axes in one fused pass into the scratch field y, copied back
// over x (post_filter3_kernel); returns the launches.
template <typename S>
int launch_filter3(const Grid& g, S* x, S* y, double strength, int phi_periodic, cudaStream_t st){
    const double coeff = strength * 0.25;                 // lib/Utils.cpp:232
    const dim3 grid((g.km + FT_K - 1) / FT_K, (g.jm + FT_J - 1) / FT_J, (g.im + FT_I - 1) / FT_I);
    post_filter3_kernel<S><<<grid, dim3(32, 8), 0, st>>>(g, x, y, coeff, phi_periodic && g.km > 2);
    cudaMemcpyAsync(x, y, g.fstride * sizeof(S), cudaMemcpyDeviceToDevice, st);
    return 1;
}
// The passes after RK4 in the reference's order; returns the number of launches.
template <typename S>
int launch_post_impl(const PostArgs<S>& a, const PostPlan& pl, S* t, float* tlo, cudaStream_t st){
    const Grid& g = a.g;
    const dim3 cols_k((g.km + 127) / 128);
    int n = 0;
    auto filt = [&](S* x, float* lo, bool ai, bool aj, bool ak, double strength){
        n += launch_filter<S>(g, x, lo, ai, aj, ak, strength, a.phi_periodic, st);
    };
    if(pl.damp_t_horiz != 0.0) filt(t, tlo, false, pl.damp_t_j != 0, true, pl.damp_t_horiz);
    if(pl.damp_t_vert != 0.0) filt(t, tlo, true, false, false, pl.damp_t_vert);
    if(pl.vel_shapiro != 0.0){ filt(a.u, nullptr, true, true, true, pl.vel_shapiro); filt(a.v, nullptr, true, true, true, pl.vel_shapiro);
                               filt(a.w, nullptr, true, true, true, pl.vel_shapiro); }
    post_bc_radius_kernel<S><<<dim3(cols_k.x, g.jm, POST_NRAD), 128, 0, st>>>(a);
    post_bc_theta_kernel<S><<<dim3(cols_k.x, g.im, POST_NTHZ + POST_NTHX), 128, 0, st>>>(a);
    post_bc_phi_kernel<S><<<dim3((g.im * g.jm + 127) / 128, POST_NPHI), 128, 0, st>>>(a);
    n += 3;
    if(pl.species_clamp){
        post_clamp_kernel<S><<<dim3(pl.nb, POST_NSP), POST_CLAMP_NT, 0, st>>>(a, pl.part);
        post_clamp_finish_kernel<<<POST_NSP, POST_CLAMP_NT, 0, st>>>(pl.part, pl.nb, pl.out);
        n += 2;
    }
    return n;
}
// The chemistry (chem.cuh): NH4SH_EQ (1) then FORCING (2) as selected in `what`; returns the
// number of launches.
template <typename S>
int launch_chem_impl(const ChemArgs<S>& a, int what, cudaStream_t st){
    const Grid& g = a.g;
    const dim3 cols((g.km + 127) / 128, g.jm, g.im);
    int n = 0;
    if(what & 1){ nh4sh_eq_kernel<S><<<cols, 128, 0, st>>>(a); n++; }
    if(what & 2){
        chem_diff_kernel<S><<<cols, 128, 0, st>>>(a);
        n++;
        S* f1[4] = {a.df_h2s, a.df_nh3, a.df_nh4sh, a.tmf};
        for(S* x : f1) n += launch_filter3<S>(g, x, a.scratch, 1.0, a.c.per, st);
        const int kn = g.km - 1 - (a.c.per ? 0 : 1);
        chem_limit_kernel<S><<<dim3((kn + 127) / 128, g.jm - 2, g.im - 2), 128, 0, st>>>(a);
        n++;
        S* f2[4] = {a.mf_h2s, a.mf_nh3, a.mf_nh4sh, a.fl};
        for(S* x : f2) n += launch_filter3<S>(g, x, a.scratch, 1.0, a.c.per, st);
    }
    return n;
}
// The turbulence closure (turb.cuh); returns the number of launches.
template <typename S>
int launch_turb_impl(const TurbArgs<S>& a, cudaStream_t st){
    const Grid& g = a.g;
    const int kn = g.km - 1 - (a.c.per ? 0 : 1);
    turb_sources_kernel<S><<<dim3((kn + 127) / 128, g.jm - 2, g.im - 2), 128, 0, st>>>(a);
    turb_column_kernel<S><<<dim3((g.km + 127) / 128, g.jm), 128, 0, st>>>(a);
    const long nedge = (a.c.per ? (long)(g.im - 1) * (g.jm - 2) : 0) + (long)(g.jm - 2) * g.km + (long)g.im * g.km;
    turb_edges_kernel<S><<<(unsigned)((nedge + 127) / 128), 128, 0, st>>>(a);
    return 3;
}
// The precipitation (precip.cuh): one thread per column; returns the number of launches.
template <typename S>
int launch_precip_impl(const PrecipArgs<S>& a, cudaStream_t st){
    precip_kernel<S><<<dim3((a.g.km + 31) / 32, a.g.jm), 128, 0, st>>>(a);
    return 1;
}
// The moist convective adjustment (mca.cuh): one warp per column, W warps per block, W = 4 halved
// until the block's slices fit the shared memory; returns the launches, or -1 if one column's slice
// does not fit.
template <typename S>
int launch_mca_impl(const McaArgs<S>& a, cudaStream_t st){
    const size_t per = mca_warp_bytes(a.g.im);
    int W = 4;
    while(W > 1 && (size_t)W * per > MCA_SMEM_MAX) W /= 2;
    if((size_t)W * per > MCA_SMEM_MAX) return -1;
    const size_t sm = (size_t)W * per;
    if(sm > 48 * 1024 &&
       cudaFuncSetAttribute(mca_warp_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess){
        cudaGetLastError();
        return -1;
    }
    const long cols = (long)a.g.jm * a.g.km;
    mca_warp_kernel<S><<<(unsigned)((cols + W - 1) / W), dim3(32, W), sm, st>>>(a);
    return 1;
}
// Hydrostatic integral: threads per column (ROWS) and resident blocks per SM (MINB), measured.
template <typename S> struct HydCfg { static constexpr int ROWS = 8, MINB = 2; };
template <> struct HydCfg<float> { static constexpr int ROWS = 16, MINB = 2; };
}  // namespace aturan

#define ATURAN_DEFINE_LAUNCHERS(S, C)                                                                     \
void launch_stage(const StageArgs<S, C>& a, cudaStream_t st, cudaStream_t side, cudaEvent_t ef,           \
                  cudaEvent_t ej){                                                                        \
    const Grid& g = a.g;                                                                                  \
    const dim3 grid2((g.km - 1 + 63) / 64, (g.jm - 2 + 3) / 4, g.im - 2);                                 \
    if(!side){                                                                                            \
        launch_momentum(a, grid2, st);                                                                    \
        launch_scalars(a, grid2, st);                                                                     \
        return;                                                                                           \
    }                                                                                                     \
    cudaEventRecord(ef, st);                                                                              \
    cudaStreamWaitEvent(side, ef, 0);                                                                     \
    launch_momentum(a, grid2, side);                                                                      \
    launch_scalars(a, grid2, st);                                                                         \
    cudaEventRecord(ej, side);                                                                            \
    cudaStreamWaitEvent(st, ej, 0);                                                                       \
}                                                                                                         \
void launch_buoy(Grid g, const S* t, const S* ps, const double* wsin, HydroConst h, double* part_sum,     \
                 double* part_w, int nblk, double* ref, int exact, const BuoyScratch& bx, cudaStream_t st){ \
    if(exact){                                                                                            \
        buoy_terms_kernel<S><<<dim3(bx.nbx, g.im), BX_CH, 0, st>>>(g, t, ps, wsin, h, bx.terms, bx.bpart, bx.nbx); \
        buoy_predict_kernel<<<g.im, 256, 0, st>>>(bx.nbx, bx.bpart, bx.bexp);                               \
        buoy_units_kernel<<<dim3(bx.nbx, g.im), BX_CH, 0, st>>>(g, bx.nbx, bx.terms, bx.bexp, bx.bunits);  \
        buoy_serial_pass_kernel<<<g.im, 32, 0, st>>>(g, bx.nbx, bx.terms, bx.bexp, bx.bunits, ref);         \
        return;                                                                                           \
    }                                                                                                     \
    buoy_partial_kernel<S><<<dim3(nblk, g.im), 256, 0, st>>>(g, t, ps, wsin, h, part_sum, part_w, nblk); \
    buoy_finish_kernel<<<(g.im + 63) / 64, 64, 0, st>>>(g.im, nblk, part_sum, part_w, ref);               \
}                                                                                                         \
void launch_hydro(Grid g, const S* t, const S* ps, const S* v, const S* w, const double* ref,              \
                  const double* rm_i, const double* cor_j, const double* pbaro, const double* pb0,         \
                  double* pbf, double* ph, HydroConst h, int advance, cudaStream_t st){                    \
    const int n = g.jm * g.km;                                                                            \
    constexpr int R = HydCfg<S>::ROWS;                                                                    \
    hydro_kernel<S, R, HydCfg<S>::MINB><<<(n + 31) / 32, dim3(32, R), 0, st>>>(g, t, ps, v, w, ref, rm_i,   \
                                                                  cor_j, pbaro, pb0, pbf, ph, h, advance); \
}                                                                                                         \
void launch_satadj(const SatArgs<S>& a, cudaStream_t st){                                                  \
    constexpr int NT = SatCfg<S>::NT;                                                                     \
    static const bool carve = (prefer_max_shared(satadj_kernel<S, NT>), true);                            \
    (void)carve;                                                                                          \
    dim3 grid((a.g.km + NT - 1) / NT, a.g.jm, a.g.im);                                                    \
    satadj_kernel<S, NT><<<grid, NT, 0, st>>>(a);                                                         \
}                                                                                                         \
void launch_gs_pre(Grid g, S* au, S* av, S* aw, const S* ru, const S* rv, const S* rw, const double* P,    \
                   const GSW* w, PressConst c, double* incr, cudaStream_t st){                             \
    gs_aux_bc_kernel<S><<<dim3((g.km - 1 + 127) / 128, g.jm - 2), 128, 0, st>>>(g, au, av, aw);           \
    if(c.press_incr)                                                                                      \
        gs_incr_kernel<S><<<dim3((g.km - 1 + 127) / 128, g.jm - 2, g.im - 2), 128, 0, st>>>(              \
            g, ru, rv, rw, P, w, c, incr);                                                                \
}                                                                                                         \
void launch_gs_plane(Grid g, double* P, const double* incr, const S* au, const S* av, const S* aw,         \
                     const GSW* w, PressConst c, int s, cudaStream_t st){                                   \
    const int n = (g.im - 2) * (g.jm - 2);                                                                \
    gs_hyperplane_kernel<S><<<(n + 255) / 256, 256, 0, st>>>(g, P, incr, au, av, aw, w, c, s);            \
}                                                                                                         \
void launch_rb_prep(Grid g, S* au, S* av, S* aw, S* ru, S* rv, S* rw, int rigid_lid,                       \
                    const RBW* w, PressConst c, double* src, cudaStream_t st){                             \
    prep_rt_kernel<S><<<dim3((g.km - 1 + 127) / 128, (g.jm - 2) + (g.im - 2)), 128, 0, st>>>(             \
        g, au, av, aw, ru, rv, rw, rigid_lid);                                                            \
    prep_seam_kernel<S><<<(g.im * g.jm + 255) / 256, 256, 0, st>>>(g, au, av, aw, ru, rv, rw);            \
    rb_src_kernel<S><<<dim3((g.km - 1 + 127) / 128, g.jm - 2, g.im - 2), 128, 0, st>>>(                   \
        g, au, av, aw, w, c, src);                                                                        \
}                                                                                                         \
int launch_post(const PostArgs<S>& a, const PostPlan& pl, S* t, float* tlo, cudaStream_t st){              \
    return launch_post_impl<S>(a, pl, t, tlo, st);                                                        \
}                                                                                                         \
int launch_chem(const ChemArgs<S>& a, int what, cudaStream_t st){                                         \
    return launch_chem_impl<S>(a, what, st);                                                              \
}                                                                                                         \
int launch_turb(const TurbArgs<S>& a, cudaStream_t st){                                                   \
    return launch_turb_impl<S>(a, st);                                                                    \
}                                                                                                         \
int launch_precip(const PrecipArgs<S>& a, cudaStream_t st){                                               \
    return launch_precip_impl<S>(a, st);                                                                  \
}                                                                                                         \
int launch_mca(const McaArgs<S>& a, cudaStream_t st){                                                     \
    return launch_mca_impl<S>(a, st);                                                                     \
}
