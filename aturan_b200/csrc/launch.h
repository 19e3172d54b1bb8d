// Host-side launch wrappers. Each kernel family is instantiated in the translation unit whose
// compiler flags it needs: fp64.cu (FP64 state, no FMA contraction: the parity path) and
// mixed.cu (FP32 state with FMA). api.cu holds the host logic and calls these.
#pragma once
#include "common.cuh"

namespace aturan {

template <typename S, typename C> struct StageArgs;
template <typename S> struct SatArgs;
template <typename S> struct PostArgs;
template <typename S> struct ChemArgs;
template <typename S> struct TurbArgs;
template <typename S> struct PrecipArgs;
template <typename S> struct McaArgs;
struct GSW; struct RBW; struct PressConst; struct PostPlan;

// launch_stage: one RK4 stage, the momentum + T launch and then the scalar launch on st; given a
// side stream (and two events), the momentum launch runs on side beside the scalar launch on st
// (the two read the stage input and write disjoint fields) and st waits for it.
#define ATURAN_DECLARE_LAUNCHERS(S, C)                                                                     \
void launch_stage(const StageArgs<S, C>& a, cudaStream_t st, cudaStream_t side = nullptr,                   \
                  cudaEvent_t ef = nullptr, cudaEvent_t ej = nullptr);                                     \
void launch_buoy(Grid g, const S* t, const S* ps, const double* wsin, HydroConst h, double* part_sum,     \
                 double* part_w, int nblk, double* ref, int exact, const BuoyScratch& bx, cudaStream_t st);                       \
void launch_hydro(Grid g, const S* t, const S* ps, const S* v, const S* w, const double* ref,              \
                  const double* rm_i, const double* cor_j, const double* pbaro, const double* pb0,         \
                  double* pbf, double* ph, HydroConst h, int advance, cudaStream_t st);                    \
void launch_satadj(const SatArgs<S>& a, cudaStream_t st);                                                  \
void launch_gs_pre(Grid g, S* au, S* av, S* aw, const S* ru, const S* rv, const S* rw, const double* P,    \
                   const GSW* w, PressConst c, double* incr, cudaStream_t st);                             \
void launch_gs_plane(Grid g, double* P, const double* incr, const S* au, const S* av, const S* aw,         \
                     const GSW* w, PressConst c, int s, cudaStream_t st);                                   \
void launch_rb_prep(Grid g, S* au, S* av, S* aw, S* ru, S* rv, S* rw, int rigid_lid,                       \
                    const RBW* w, PressConst c, double* src, cudaStream_t st);                             \
int launch_post(const PostArgs<S>& a, const PostPlan& pl, S* t, float* tlo, cudaStream_t st);               \
int launch_chem(const ChemArgs<S>& a, int what, cudaStream_t st);                                         \
int launch_turb(const TurbArgs<S>& a, cudaStream_t st);                                                   \
int launch_precip(const PrecipArgs<S>& a, cudaStream_t st);                                               \
int launch_mca(const McaArgs<S>& a, cudaStream_t st);

ATURAN_DECLARE_LAUNCHERS(double, double)
ATURAN_DECLARE_LAUNCHERS(float, float)
#undef ATURAN_DECLARE_LAUNCHERS

// The moist convective adjustment's cp-table integral (CpH2.h:66-75), formed once per context.
void launch_mca_H(const double* cp_tab, double* H, cudaStream_t st);

// FP64-only kernels (p_dyn is FP64 in both precisions).
void launch_pdyn_bcs(Grid g, double* P, cudaStream_t st);
// damp_wiggles on an FP64 field (p_dyn) in either precision; returns the launches.
int launch_filter_f64(const Grid& g, double* x, bool ai, bool aj, bool ak, double strength, int phi_periodic, cudaStream_t st);
void launch_scale_copy_f64(const double* in, double* out, size_t n, double coeff, cudaStream_t st);
void launch_scale_copy_f32(const float* in, float* out, size_t n, double coeff, cudaStream_t st);
void launch_rb_colour(Grid g, double* P, const double* src, const RBW* w, int colour, double omega, cudaStream_t st);

// Layout conversions for the mixed-precision context (FP64 exchange <-> FP32 storage).
void launch_f64_to_f32(const double* in, float* out, size_t n, cudaStream_t st);
void launch_pack_in_f64(const double* in, double* out, int km, int kp, size_t rows, cudaStream_t st);
void launch_pack_in_f32(const double* in, float* out, int km, int kp, size_t rows, cudaStream_t st);
void launch_pack_out_f64(const double* in, double* out, int km, int kp, size_t rows, cudaStream_t st);
void launch_pack_out_f32(const float* in, double* out, int km, int kp, size_t rows, cudaStream_t st);
void launch_f32_to_f64(const float* in, double* out, size_t n, cudaStream_t st);
// The mixed form's temperature pair (common.cuh): FP64 exchange <-> (hi, lo) FP32 storage.
void launch_pack_in_pair(const double* in, float* hi, float* lo, int km, int kp, size_t rows, cudaStream_t st);
void launch_pack_out_pair(const float* hi, const float* lo, double* out, int km, int kp, size_t rows, cudaStream_t st);
void launch_scale_copy_pair(const float* hi, const float* lo, float* ohi, float* olo, size_t n, double coeff, cudaStream_t st);

}  // namespace aturan
