// The passes that follow RungeKuttaUran in one iteration (planet/cUranusModel.cpp:1218-1248): the
// 1-2-1 filters of lib/Utils.cpp:224-317 (damp_wiggles), the boundary passes of
// BoundaryConditions.h:152-518 as BC_Uran.h:140-173 runs them for Uranus (margin 0, Neumann
// default, no turbulence fields, no pole fill rows), the species floor of the radial planes and
// the species clamp (BC_Uran.h:91-128).
//
// All of it is streaming work on a few planes of the state, bound by HBM. The filters update a
// field in place: along k one warp holds a row in shared memory; along j and i one thread walks
// a column, keeping the old values of the cell and its lower neighbour in registers, so every old
// value is read before it is overwritten, as the reference's copy of the field guarantees. The
// boundary passes are column-local (radius: per (j,k), theta: per (i,k), phi: per (i,j)) and
// field-local, so a thread applies every step of one field's column in the reference's order,
// and one launch per pass keeps the reference's order between passes. Arithmetic is FP64 on the stored values (FP32
// storage in the mixed form is widened, computed in FP64 and rounded back).
#pragma once
#include "common.cuh"
#include "pressure.cuh"

namespace aturan {

// Field tables: the reference's lists (BC_Uran.cpp:21-88) restricted to the fields the context
// holds. The phi list is the radius list's first POST_NPHI fields: all but difflux_nh4sh.
constexpr int POST_NRAD = 25, POST_NPHI = 24, POST_NTHX = 16, POST_NTHZ = 9, POST_NSP = 13;

// Which filter passes run and the clamp's scratch: part holds 2 nb doubles per species, out 2 x 13.
struct PostPlan {
    double damp_t_horiz, damp_t_vert, vel_shapiro;
    int damp_t_j, species_clamp, nb;
    double *part, *out;
};

template <typename S>
struct PostArgs {
    Grid g;
    S* rad[POST_NRAD];           // radius and phi passes: t, u, v, w, the species (4..16), the fluxes, difflux
    S* thx[POST_NTHX];           // theta pass, extrapolated to the poles
    S* thz[POST_NTHZ];           // theta pass, zeroed at the poles (v, w first)
    S* sp[POST_NSP];             // species for the clamp, in BC_Uran.h:83-89's order
    S *u, *v, *w;
    float* tlo;                  // the mixed form's temperature pair (common.cuh): t's low part, else null
    int radius_form, bottom_form, pole_form, lid_u, top_taper, lid_vw, positive, phi_periodic;
};

// BCForm::apply with the model default NEUMANN (BoundaryConditions.h, cUranusModel.h:397)
__device__ __forceinline__ double post_form(int form, double a, double b, double c){
    const int f = (form == 0) ? 2 : form;
    if(f == 1) return a;
    if(f == 2) return C43 * a - C13 * b;
    return c - 3.0 * b + 3.0 * a;
}
__device__ __forceinline__ double post_max0(double x){ return (0.0 < x) ? x : 0.0; }   // std::max(0.0, x)

// ---- damp_wiggles (lib/Utils.cpp:224-317), one axis per launch ----

// Along k: one warp per (i, j) row (blockDim.y rows per block), the row's old values in the warp's
// own slice of shared memory, ~km/32 loads in flight per lane. With the periodic seam the ring is
// k = 0..km-2 and k = km-1 takes the new k = 0; otherwise k wraps over all km. lo: the low part of
// the mixed form's temperature pair when x is its t (common.cuh), else null.
template <typename S>
__global__ void __launch_bounds__(128) post_filter_k_kernel(Grid g, S* x, float* lo, double coeff, int seam, int rows){
    extern __shared__ double sm[];
    const int r = blockIdx.x * blockDim.y + threadIdx.y;
    if(r >= rows) return;                          // a whole warp: only warp-level syncs below
    const int km = g.km;
    double* row = sm + (size_t)threadIdx.y * km;
    const size_t o = (size_t)r * g.kp;
    for(int k = threadIdx.x; k < km; k += 32) row[k] = t_ld(x, lo, o + k);
    __syncwarp();
    const int k_end = seam ? km - 1 : km;
    for(int k = threadIdx.x; k < k_end; k += 32){
        const int km1 = seam ? (k == 0 ? km - 2 : k - 1) : (k - 1 + km) % km;
        const int kp1 = seam ? (k == km - 2 ? 0 : k + 1) : (k + 1) % km;
        const double c = row[k];
        const double y = c + coeff * (row[km1] - 2.0 * c + row[kp1]);
        t_st(x, lo, o + k, y);
        if(seam && k == 0) t_st(x, lo, o + km - 1, y);
    }
}

// Along a column of n cells at stride st from x0 (j: clamped at the poles; i: at the ends).
template <typename S>
__device__ __forceinline__ void post_walk(S* x0, float* lo0, size_t st, int n, double coeff){
    double pm = t_ld(x0, lo0, 0), c = pm;
    for(int q = 0; q < n; q++){
        const double nx = (q + 1 < n) ? t_ld(x0, lo0, (size_t)(q + 1) * st) : c;
        t_st(x0, lo0, (size_t)q * st, c + coeff * (pm - 2.0 * c + nx));
        pm = c;
        c = nx;
    }
}
template <typename S>
__global__ void __launch_bounds__(128) post_filter_j_kernel(Grid g, S* x, float* lo, double coeff){
    const int k = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if(k >= g.km) return;
    const size_t o = gidx(g, i, 0, k);
    post_walk(x + o, lo ? lo + o : nullptr, (size_t)g.kp, g.jm, coeff);
}
template <typename S>
__global__ void __launch_bounds__(128) post_filter_i_kernel(Grid g, S* x, float* lo, double coeff){
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if(k >= g.km) return;
    const size_t o = gidx(g, 0, j, k);
    post_walk(x + o, lo ? lo + o : nullptr, (size_t)g.jm * g.kp, g.im, coeff);
}

// ---- damp_wiggles along k, j and i in one pass, out of place (x -> y) ----
// The three 1-2-1 passes of damp_wiggles with all axes on, fused over a tile of FT_I x FT_J x FT_K
// outputs: the k pass of the tile and its one-cell i and j halo is formed from global memory (the
// k neighbours are the row's own, L1 hits), the j pass of the tile and its i halo from that, the i
// pass from that. The halo rows and planes are the clamped ones the passes use at the poles and
// the ends (j - 1 of j = 0 is j = 0, and likewise), so every output is formed from exactly the
// values, and by exactly the arithmetic, of the three passes in turn. With the periodic seam the
// k pass of k = km-1 is that of k = 0 (the pass's copy), and so the j and i passes there too. The
// result goes to y, which the launcher copies back over x: the passes read every neighbour's old
// value, which an in-place tile could overwrite before its neighbour tile reads it.
constexpr int FT_K = 32, FT_J = 8, FT_I = 4;
template <typename S>
__global__ void __launch_bounds__(256) post_filter3_kernel(Grid g, const S* __restrict__ x, S* __restrict__ y, double coeff, int seam){
    __shared__ double YK[FT_I + 2][FT_J + 2][FT_K];
    __shared__ double YJ[FT_I + 2][FT_J][FT_K];
    const int tk = threadIdx.x, ty = threadIdx.y;              // 32 x 8
    const int k = blockIdx.x * FT_K + tk, j0 = blockIdx.y * FT_J, i0 = blockIdx.z * FT_I;
    const int km = g.km;
    const bool kin = k < km;
    // the k pass's own index and neighbours (damp_wiggles, lib/Utils.cpp:250-265)
    int kc = k, km1 = 0, kp1 = 0;
    if(kin){
        if(seam && k == km - 1) kc = 0;
        km1 = seam ? (kc == 0 ? km - 2 : kc - 1) : (kc - 1 + km) % km;
        kp1 = seam ? (kc == km - 2 ? 0 : kc + 1) : (kc + 1) % km;
    }
    for(int r = ty; r < (FT_I + 2) * (FT_J + 2); r += 8){
        const int ii = r / (FT_J + 2), jj = r % (FT_J + 2);
        const int i = min(max(i0 - 1 + ii, 0), g.im - 1), j = min(max(j0 - 1 + jj, 0), g.jm - 1);
        double v = 0.0;
        if(kin){
            const S* row = x + gidx(g, i, j, 0);
            const double c = (double)__ldg(row + kc);
            v = c + coeff * ((double)__ldg(row + km1) - 2.0 * c + (double)__ldg(row + kp1));
        }
        YK[ii][jj][tk] = v;
    }
    __syncthreads();
    for(int r = ty; r < (FT_I + 2) * FT_J; r += 8){
        const int ii = r / FT_J, jj = r % FT_J;
        const int j = j0 + jj;
        // j - 1 and j + 1 clamped to the poles: the halo rows hold the clamped rows already
        const double c = YK[ii][jj + 1][tk];
        YJ[ii][jj][tk] = c + coeff * (YK[ii][jj][tk] - 2.0 * c + YK[ii][jj + 2][tk]);
        (void)j;
    }
    __syncthreads();
    if(!kin) return;
    for(int r = ty; r < FT_I * FT_J; r += 8){
        const int ii = r / FT_J, jj = r % FT_J;
        const int i = i0 + ii, j = j0 + jj;
        if(i >= g.im || j >= g.jm) continue;
        const double c = YJ[ii + 1][jj][tk];
        y[gidx(g, i, j, k)] = (S)(c + coeff * (YJ[ii][jj][tk] - 2.0 * c + YJ[ii + 2][jj][tk]));
    }
}

// ---- bcRadius (BoundaryConditions.h:152-286), floorRadialSpecies and the lid v, w (BC_Uran.h:91-170) ----
// One thread per (j, k) column of one field (blockIdx.z = the field's place in rad): the field's
// two end values, then what the reference does afterwards to that same column -- u = 0 at the
// ends (lid_u), the top taper and the lid form of v and w, the species floor. Every later step
// reads and writes only its own field's column, so the fields run side by side.
template <typename S>
__global__ void __launch_bounds__(128) post_bc_radius_kernel(PostArgs<S> a){
    const Grid& g = a.g;
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, n = blockIdx.z;
    if(k >= g.km) return;
    const int im = g.im;
    const size_t pl = (size_t)g.jm * g.kp;
    S* F = a.rad[n] + gidx(g, 0, j, k);
    auto at = [&](int i) -> S& { return F[(size_t)i * pl]; };
    const int fb = (a.bottom_form != 0 && n != 1) ? a.bottom_form : a.radius_form;
    if(n == 0 && a.tlo){                            // t as the mixed form's pair: its two end values, in order
        float* L = a.tlo + gidx(g, 0, j, k);
        auto get = [&](int i) -> double { return t_ld(F, L, (size_t)i * pl); };
        t_st(F, L, 0, post_form(fb, get(1), get(2), get(3)));
        t_st(F, L, (size_t)(im - 1) * pl, post_form(a.radius_form, get(im - 2), get(im - 3), get(im - 4)));
        return;
    }
    const bool species = n >= 4 && n <= 16;        // the twelve condensables and nh4sh
    if(im >= 8){
        // planes 1..3 and im-4..im-2 are disjoint from each other and from 0 and im-1: every
        // value is loaded up front (the third plane only for the cubic form), one round trip
        auto cubic = [](int f){ return f != 0 && f != 1 && f != 2; };
        const double b1 = (double)at(1), b2 = (double)at(2), b3 = cubic(fb) ? (double)at(3) : 0.0;
        const double t1 = (double)at(im - 2), t2 = (double)at(im - 3);
        const double t3 = cubic(a.radius_form) ? (double)at(im - 4) : 0.0;
        S y0 = (S)post_form(fb, b1, b2, b3), yl = (S)post_form(a.radius_form, t1, t2, t3);
        if(n == 1 && a.lid_u != 0){ y0 = (S)0.0; yl = (S)0.0; }
        if(species && a.positive != 0){          // the floor reads planes 1 and im-2, unchanged
            if((double)y0 < 0.0) y0 = (S)((a.positive == 2) ? post_max0(b1) : 0.0);
            if((double)yl < 0.0) yl = (S)((a.positive == 2) ? post_max0(t1) : 0.0);
        }
        at(0) = y0;
        at(im - 1) = yl;
        if(n != 2 && n != 3) return;
    } else {
        // in the reference's order, through memory (the planes overlap when im < 8)
        at(0) = (S)post_form(fb, (double)at(1), (double)at(2), (double)at(3));
        at(im - 1) = (S)post_form(a.radius_form, (double)at(im - 2), (double)at(im - 3), (double)at(im - 4));
        if(n == 1 && a.lid_u != 0){ at(0) = (S)0.0; at(im - 1) = (S)0.0; }
    }
    if(n == 2 || n == 3){                         // v, w
        const int l = im - 1;
        if(a.top_taper != 0){
            at(l) = (S)0.0;
            if(a.top_taper == 2){
                at(l - 1) = (S)((1.0 / 3.0) * (double)at(l - 3));
                at(l - 2) = (S)((2.0 / 3.0) * (double)at(l - 3));
            } else {
                at(l - 1) = (S)((double)at(l - 1) * (1.0 / 3.0));
                at(l - 2) = (S)((double)at(l - 2) * (2.0 / 3.0));
            }
        }
        if(a.lid_vw == 2)
            at(l) = (S)(2.0 * (double)at(l - 1) - (double)at(l - 2));
        else if(a.lid_vw == 3)
            at(l) = (S)((double)at(l - 3) - 3.0 * (double)at(l - 2) + 3.0 * (double)at(l - 1));
    } else if(species && a.positive != 0){
        if((double)at(0) < 0.0) at(0) = (S)((a.positive == 2) ? post_max0((double)at(1)) : 0.0);
        if((double)at(im - 1) < 0.0) at(im - 1) = (S)((a.positive == 2) ? post_max0((double)at(im - 2)) : 0.0);
    }
}

// ---- bcTheta (BoundaryConditions.h:293-391): one thread per (i, k) column of one field; fields
// 0..POST_NTHZ-1 are zeroed at the poles, the others extrapolated. ----
template <typename S>
__global__ void __launch_bounds__(128) post_bc_theta_kernel(PostArgs<S> a){
    const Grid& g = a.g;
    const int k = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y, n = blockIdx.z;
    if(k >= g.km) return;
    const int jm = g.jm;
    const size_t kp = (size_t)g.kp, o = gidx(g, i, 0, k);
    if(n < POST_NTHZ){
        S* F = a.thz[n] + o;
        F[0] = (S)0.0;
        F[(size_t)(jm - 1) * kp] = (S)0.0;
        return;
    }
    S* F = a.thx[n - POST_NTHZ] + o;
    if(n == POST_NTHZ && a.tlo){                    // t as the mixed form's pair
        float* L = a.tlo + o;
        auto get = [&](int j) -> double { return t_ld(F, L, (size_t)j * kp); };
        t_st(F, L, 0, post_form(a.pole_form, get(1), get(2), get(3)));
        t_st(F, L, (size_t)(jm - 1) * kp, post_form(a.pole_form, get(jm - 2), get(jm - 3), get(jm - 4)));
        return;
    }
    auto at = [&](int j) -> S& { return F[(size_t)j * kp]; };
    at(0) = (S)post_form(a.pole_form, (double)at(1), (double)at(2), (double)at(3));     // in order (jm < 5 overlaps)
    at(jm - 1) = (S)post_form(a.pole_form, (double)at(jm - 2), (double)at(jm - 3), (double)at(jm - 4));
}

// ---- bcPhi (BoundaryConditions.h:398-455, without the seam damping): one thread per (i, j) row
// of one field ----
template <typename S>
__global__ void __launch_bounds__(128) post_bc_phi_kernel(PostArgs<S> a){
    const Grid& g = a.g;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;      // row (i, j)
    if(r >= g.im * g.jm) return;
    const int km = g.km;
    S* F = a.rad[blockIdx.y] + (size_t)r * g.kp;
    if(blockIdx.y == 0 && a.tlo){                   // t as the mixed form's pair
        float* L = a.tlo + (size_t)r * g.kp;
        if(a.phi_periodic){ F[km - 1] = F[0]; L[km - 1] = L[0]; }
        else {
            const double y = 0.5 * ((C43 * t_ld(F, L, 1) - C13 * t_ld(F, L, 2)) + (C43 * t_ld(F, L, km - 2) - C13 * t_ld(F, L, km - 3)));
            t_st(F, L, 0, y);
            t_st(F, L, km - 1, y);
        }
        return;
    }
    if(a.phi_periodic) F[km - 1] = F[0];
    else {
        const double lo = C43 * (double)F[1] - C13 * (double)F[2];
        const double hi = C43 * (double)F[km - 2] - C13 * (double)F[km - 3];
        const S y = (S)(0.5 * (lo + hi));
        F[0] = y;
        F[km - 1] = y;
    }
}

// ---- clampNegativeSpecies (BC_Uran.h:110-128) ----
// Block (b, n) clamps a block-stride share of species n's padded field, read as 16-byte vectors
// (a vector never straddles a row: the row pitch is a multiple of 32 values), four vectors in
// flight per thread; values in the row padding are skipped. It writes its clipped sum and count
// (as doubles, exact for any count below 2^53) to part[2 (n nb + b)] in a fixed tree order, and
// post_clamp_finish_kernel adds a species' nb partials in a fixed order. Deterministic run to
// run; the reference's OpenMP reduction order differs, so the sum agrees to its rounding.
constexpr int POST_CLAMP_NT = 256;
template <typename S> struct Vec16;
template <> struct Vec16<float>  { using T = float4;  static constexpr int N = 4; };
template <> struct Vec16<double> { using T = double2; static constexpr int N = 2; };

template <typename S>
__device__ __forceinline__ void post_clamp_one(S* R, int k, int km, double x, double& s, double& c){
    if(k < km && !(x >= 0.0)){                     // catches a NaN too
        if(isfinite(x)){ s -= x; c += 1.0; }
        R[k] = (S)0.0;
    }
}

template <typename S>
__global__ void __launch_bounds__(POST_CLAMP_NT) post_clamp_kernel(PostArgs<S> a, double* part){
    using V = typename Vec16<S>::T;
    constexpr int NV = Vec16<S>::N, U = 4;
    const Grid& g = a.g;
    const int n = blockIdx.y, nb = gridDim.x;
    S* F = a.sp[n];
    const int vpr = g.kp / NV;                                    // vectors per row
    const long long nvec = (long long)g.im * g.jm * vpr;
    const long long step = (long long)nb * POST_CLAMP_NT;
    double s = 0.0, c = 0.0;
    for(long long q0 = (long long)blockIdx.x * POST_CLAMP_NT + threadIdx.x; q0 < nvec; q0 += U * step){
        V v[U];
#pragma unroll
        for(int u = 0; u < U; u++){
            const long long q = q0 + u * step;
            if(q < nvec) v[u] = reinterpret_cast<const V*>(F)[q];
        }
#pragma unroll
        for(int u = 0; u < U; u++){
            const long long q = q0 + u * step;
            if(q >= nvec) break;
            const long long r = q / vpr;
            const int k0 = (int)(q - r * vpr) * NV;
            S* R = F + r * g.kp;
            const S* e = reinterpret_cast<const S*>(&v[u]);
#pragma unroll
            for(int m = 0; m < NV; m++) post_clamp_one(R, k0 + m, g.km, (double)e[m], s, c);
        }
    }
    __shared__ double ss[POST_CLAMP_NT], sc[POST_CLAMP_NT];
    ss[threadIdx.x] = s; sc[threadIdx.x] = c;
    __syncthreads();
    for(int st = POST_CLAMP_NT / 2; st > 0; st >>= 1){
        if((int)threadIdx.x < st){ ss[threadIdx.x] += ss[threadIdx.x + st]; sc[threadIdx.x] += sc[threadIdx.x + st]; }
        __syncthreads();
    }
    if(threadIdx.x == 0){ part[2 * ((size_t)n * nb + blockIdx.x)] = ss[0]; part[2 * ((size_t)n * nb + blockIdx.x) + 1] = sc[0]; }
}

// One block per species: thread t adds partials t, t + 256, ... in order, then a fixed tree.
static __global__ void __launch_bounds__(POST_CLAMP_NT) post_clamp_finish_kernel(const double* part, int nb, double* out){
    const int n = blockIdx.x;
    double s = 0.0, c = 0.0;
    for(int b = threadIdx.x; b < nb; b += POST_CLAMP_NT){ s += part[2 * ((size_t)n * nb + b)]; c += part[2 * ((size_t)n * nb + b) + 1]; }
    __shared__ double ss[POST_CLAMP_NT], sc[POST_CLAMP_NT];
    ss[threadIdx.x] = s; sc[threadIdx.x] = c;
    __syncthreads();
    for(int st = POST_CLAMP_NT / 2; st > 0; st >>= 1){
        if((int)threadIdx.x < st){ ss[threadIdx.x] += ss[threadIdx.x + st]; sc[threadIdx.x] += sc[threadIdx.x + st]; }
        __syncthreads();
    }
    if(threadIdx.x == 0){ out[n] = ss[0]; out[POST_NSP + n] = sc[0]; }
}

}  // namespace aturan
