// Poisson solve of the shared solver's equation to a relative residual: red-black SOR plus an
// exact correction of the column-uniform (barotropic) mode. No reference oracle exists for this
// (the reference sweeps a fixed count with omega = 1); it is checked against the CPU
// restatement in oracle/aturan_oracle.c and against its own residual.
//
// The equation is the one PressureSolver<Planet>::run relaxes (PressureSolver.h:318-495):
// Lc p = src over the interior, Lc the compact 7-point operator with the 2-point Neumann folds
// p0 = c43 p1 - c13 p2 on the radial and polar ends and the periodic phi ring, src the clamped
// div(aux). The operator is ~6000:1 anisotropic (num1 = 1/dr^2 = 1600 against horizontal weights
// ~0.26), so a pointwise sweep damps a column-uniform error component by ~1e-4 of its size; the
// reference records that such a mode needs ~2e8 sweeps (PressureSolver.h:51-56).
//
// THE COLUMN-UNIFORM CORRECTION. For the folded radial operator T_r the row vector
// y = (3/2, 1, ..., 1, 3/2) satisfies y^T T_r = 0, so the y-weighted column sum of the residual
// sees only the horizontal part of Lc. Adding a column-uniform q(j,k) to every level changes that
// weighted sum by A2y L2(q), A2y = sum_i y_i / rm_i^2, L2 the horizontal stencil of Lc. Solving
// A2y L2(q) = sum_i y_i r_i exactly (a DFT in phi, then one tridiagonal solve in theta per
// Fourier mode, the theta ends folded) is the Galerkin coarse correction onto column-uniform
// functions. It is the reference's PRESS_BAROTROPIC (PressureSolver.h:572-708) with the weights
// of the folded operator's left null vector, which makes it exact. With it, red-black SOR only
// has to converge the radially structured modes, whose damping is set by num1.
//
// Compatibility: the all-Neumann operator is singular with left null vector y_i y_j (times the
// phi ring's ones); the source's component along it is removed by a constant shift before the
// solve (the shift leaves every gradient unchanged).
#pragma once
#include "common.cuh"
#include "pressure.cuh"

namespace aturan {

struct SorConst {
    int J, N, NM;          // rows j = 1..jm-2, meridians k = 0..km-2, modes 0..N/2
    double inv_dthe2, A2y;
};

// Host-factored tridiagonal of one Fourier mode of the column correction (rows q = 0..J-1):
// forward y_q = (d_q - a_q y_{q-1}) * idn_q, back x_q = y_q - cf_q x_{q+1}. Mode 0 carries the pin
// q_0 = 0 in its first row.
struct ModeLU { const double *a, *cf, *idn; };

__device__ __forceinline__ double ywt(int n, int lo, int hi){ return (n == lo || n == hi) ? 1.5 : 1.0; }

// The shared solver's operator with the 2-point Neumann folds substituted into the rows (at i = 1
// the boundary value c43 p[1] - c13 p[2] puts c43 num1 on the diagonal and -c13 num1 on p[2];
// likewise at i = im-2, j = 1, j = jm-2), instead of boundary rows refreshed after each sweep as
// the reference does. Same operator on the interior unknowns, hence the same solution; but every
// row couples only to the other colour, so red-black SOR keeps its consistently-ordered rate
// (with the lagged rows the radially structured modes converge at ~0.955 per sweep at omega 1.9
// instead of ~0.9). Returns the off-diagonal sum; *diag receives the diagonal.
// The weights a row reads, through the read-only path (the tables never change inside a launch).
struct RBW4 { double num1, num2, num3, den; };
__device__ __forceinline__ RBW4 ldw(const RBW* w){
    RBW4 r; r.num1 = __ldg(&w->num1); r.num2 = __ldg(&w->num2); r.num3 = __ldg(&w->num3); r.den = __ldg(&w->den);
    return r;
}

template <typename T>
__device__ __forceinline__ double folded_acc(const Grid& g, const T* P, size_t o, int i, int j, int k,
                                             const RBW4& W, double* diag){
    const size_t si = (size_t)g.jm * g.kp, sj = g.kp;
    const int kw = phi_wrap(k - 1, g.km), ke = phi_wrap(k + 1, g.km);
    auto p = [&](size_t q){ return (double)__ldg(P + q); };
    double d = W.den;
    double aim, aip, ajm, ajp;
    if(i == 1)        { d -= C43 * W.num1; aim = -C13 * p(o + si); } else aim = p(o - si);
    if(i == g.im - 2) { d -= C43 * W.num1; aip = -C13 * p(o - si); } else aip = p(o + si);
    if(j == 1)        { d -= C43 * W.num2; ajm = -C13 * p(o + sj); } else ajm = p(o - sj);
    if(j == g.jm - 2) { d -= C43 * W.num2; ajp = -C13 * p(o - sj); } else ajp = p(o + sj);
    *diag = d;
    return (aip + aim) * W.num1 + (ajp + ajm) * W.num2
         + (p(o - k + ke) + p(o - k + kw)) * W.num3;
}

// The transposed folded operator (the pressure solve's adjoint): the gather of every row's
// coefficient on (i,j,k). Row (1,j,k) of Lc puts num1 (1 - c13) on (2,j,k) and nothing on
// (0,j,k), so row (2,j,k) of Lc^T takes num1 (1 - c13) from (1,j,k); likewise at i = im-2 and in
// theta at j = 1, jm-2, with the neighbouring row's own weights. The diagonal is Lc's.
template <typename T>
__device__ __forceinline__ double folded_accT(const Grid& g, const T* P, size_t o, int i, int j, int k,
                                              const RBW* w, double* diag){
    const size_t si = (size_t)g.jm * g.kp, sj = g.kp;
    const int kw = phi_wrap(k - 1, g.km), ke = phi_wrap(k + 1, g.km);
    const RBW4 W = ldw(w + i * g.jm + j);
    double d = W.den;
    if(i == 1)        d -= C43 * W.num1;
    if(i == g.im - 2) d -= C43 * W.num1;
    if(j == 1)        d -= C43 * W.num2;
    if(j == g.jm - 2) d -= C43 * W.num2;
    *diag = d;
    auto p = [&](size_t q){ return (double)__ldg(P + q); };
    double acc = (p(o - k + ke) + p(o - k + kw)) * W.num3;
    if(i - 1 >= 1)        acc += __ldg(&w[(i - 1) * g.jm + j].num1) * (i - 1 == 1 ? 1.0 - C13 : 1.0) * p(o - si);
    if(i + 1 <= g.im - 2) acc += __ldg(&w[(i + 1) * g.jm + j].num1) * (i + 1 == g.im - 2 ? 1.0 - C13 : 1.0) * p(o + si);
    if(j - 1 >= 1)        acc += __ldg(&w[i * g.jm + j - 1].num2) * (j - 1 == 1 ? 1.0 - C13 : 1.0) * p(o - sj);
    if(j + 1 <= g.jm - 2) acc += __ldg(&w[i * g.jm + j + 1].num2) * (j + 1 == g.jm - 2 ? 1.0 - C13 : 1.0) * p(o + sj);
    return acc;
}

// Row of Lc (TR = false) or Lc^T (TR = true): the off-diagonal sum, *diag the diagonal.
template <bool TR, typename T>
__device__ __forceinline__ double row_acc(const Grid& g, const T* P, size_t o, int i, int j, int k,
                                          const RBW* w, double* diag){
    if constexpr(TR) return folded_accT<T>(g, P, o, i, j, k, w, diag);
    else return folded_acc<T>(g, P, o, i, j, k, ldw(w + i * g.jm + j), diag);
}

// Residual r = src - Lc p of the folded operator (or src - Lc^T p, TR): per (j,k) column its
// y-weighted (TR: plain) sum over the interior levels (and, given r32/e32, r rounded to FP32 with
// e = 0 on the interior for the mixed form's correction solve), and per-block partial sums of r^2 and src^2. A block is 32 meridians x 8 level
// groups; the groups' column sums are added in group order and the block's norms in a fixed tree
// order, so the result is deterministic. P and src of type T (double: FP64 solve; float: the
// correction solve of the mixed form). Given shift (the source's compatibility shift, FP64 only),
// the pass first applies src -= shift to each interior cell it reads and writes the shifted value
// back through src_w (the same array): sor_shift_kernel's work, folded into the solve's first pass.
template <typename T, bool TR = false>
__global__ void __launch_bounds__(256) sor_colsum_kernel(Grid g, const T* P, const T* src, const RBW* w,
                                                         double* colR, double* part, int want_col,
                                                         float* r32 = nullptr, float* e32 = nullptr,
                                                         double* src_w = nullptr, const double* shift = nullptr){
    const int N = g.km - 1;
    const int k = blockIdx.x * 32 + threadIdx.x;
    const int j = 1 + blockIdx.y;
    const int grp = threadIdx.y;
    double R = 0.0, rr = 0.0, ss = 0.0;
    const double sh = shift ? *shift : 0.0;
    if(k < N){
        // CH levels at a time: every load of the chunk before its stores (which the compiler must
        // otherwise assume to alias the next level's loads); sums in level order as before
        constexpr int CH = 5;
        for(int i0 = 1 + grp; i0 < g.im - 1; i0 += 8 * CH){
            double rv[CH], sv[CH];
#pragma unroll
            for(int c = 0; c < CH; c++){
                const int i = i0 + 8 * c;
                if(i < g.im - 1){
                    const size_t o = gidx(g, i, j, k);
                    double diag;
                    const double acc = row_acc<TR, T>(g, P, o, i, j, k, w, &diag);
                    const double lc = acc - diag * (double)__ldg(P + o);
                    // the same subtraction as sor_shift_kernel
                    const double s = shift ? (double)src[o] - sh : (double)__ldg(src + o);
                    sv[c] = s;
                    rv[c] = s - lc;
                }
            }
#pragma unroll
            for(int c = 0; c < CH; c++){
                const int i = i0 + 8 * c;
                if(i < g.im - 1){
                    const size_t o = gidx(g, i, j, k);
                    const double r = rv[c], s = sv[c];
                    if(shift) src_w[o] = s;
                    if(r32){ r32[o] = (float)r; e32[o] = 0.0f; }  // the mixed form's next correction solve
                    R += (TR ? 1.0 : ywt(i, 1, g.im - 2)) * r;    // the radial block's left null vector
                    rr += r * r;
                    ss += s * s;
                }
            }
        }
    }
    __shared__ double sR[8][32], sr[256], sq[256];
    const int t = threadIdx.y * 32 + threadIdx.x;
    sR[grp][threadIdx.x] = R; sr[t] = rr; sq[t] = ss;
    __syncthreads();
    if(grp == 0 && want_col && k < N){
        double c = 0.0;
        for(int q = 0; q < 8; q++) c += sR[q][threadIdx.x];
        colR[(size_t)(j - 1) * N + k] = c;
    }
    for(int st = 128; st > 0; st >>= 1){
        if(t < st){ sr[t] += sr[t + st]; sq[t] += sq[t + st]; }
        __syncthreads();
    }
    if(t == 0){
        const int b = blockIdx.y * gridDim.x + blockIdx.x;
        part[2 * b] = sr[0]; part[2 * b + 1] = sq[0];
    }
}

// The two transforms of the correction are small dense products (J x N by N x (N/2+1) and back),
// so they run as one tiled FP64 product kernel computing P1 = A1 B1 and P2 = A2 B2 at once, every
// operand addressed by (row, column) strides; it writes C1 = scale P1 and C2 = scale P2, or, with
// no C2, C1 = scale (P1 + P2). A block computes a 32 x 32 tile from 32-wide k-chunks of the
// operands staged in shared memory (rows padded to 33: no bank conflicts); each operand tile is
// loaded along whichever of its two indices has unit stride.
//   forward:  Ac^T = (colR / A2y) . ctT  and  As^T = (colR / A2y) . stT  (one launch, A shared)
//   inverse:  q = Ac^T . ct + As^T . st,  Ac/As carrying the weights w_m / N (tridiagonal write-back)
// ct/st are host-built with the (m k mod N) argument reduction of PressureSolver.h:614-617.
struct MatRef { const double* p; long rs, cs; };      // element (r, c) at p[r * rs + c * cs]

__device__ __forceinline__ void gemm_stage(double (*t)[33], const MatRef& A, int r0, int k0, int R, int K){
    const bool kfast = (A.cs == 1);
#pragma unroll 4
    for(int idx = threadIdx.x; idx < 32 * 32; idx += blockDim.x){
        const int a = idx >> 5, b = idx & 31;          // b runs along the unit-stride index
        const int r = kfast ? a : b, k = kfast ? b : a;
        const int gr = r0 + r, gk = k0 + k;
        t[r][k] = (gr < R && gk < K) ? A.p[(long)gr * A.rs + (long)gk * A.cs] : 0.0;
    }
}

// Split K: block z sums k in [z kc, (z + 1) kc) and writes its partial products at C + z * cz; the
// consumer (the tridiagonal kernel, the add kernel) sums the gridDim.z partials in order.
__global__ void __launch_bounds__(256) sor_gemm_kernel(int M, int Nn, int K, MatRef A1, MatRef B1, MatRef A2,
                                                       MatRef B2, double scale, double* C1, double* C2,
                                                       long crs, long ccs, int kc, long cz){
    __shared__ double sa1[32][33], sb1[32][33], sa2[32][33], sb2[32][33];   // sa[r][k], sb[c][k]
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    const int kb = blockIdx.z * kc, ke = min(K, kb + kc);
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const bool sharedA = (A2.p == A1.p && A2.rs == A1.rs && A2.cs == A1.cs);
    const MatRef Bt1{B1.p, B1.cs, B1.rs}, Bt2{B2.p, B2.cs, B2.rs};   // B^T: (c, k)
    double acc1[4] = {0.0, 0.0, 0.0, 0.0}, acc2[4] = {0.0, 0.0, 0.0, 0.0};
    for(int k0 = kb; k0 < ke; k0 += 32){
        gemm_stage(sa1, A1, r0, k0, M, ke);
        if(!sharedA) gemm_stage(sa2, A2, r0, k0, M, ke);
        gemm_stage(sb1, Bt1, c0, k0, Nn, ke);
        gemm_stage(sb2, Bt2, c0, k0, Nn, ke);
        __syncthreads();
        double (*a2)[33] = sharedA ? sa1 : sa2;
#pragma unroll 8
        for(int k = 0; k < 32; k++){
            const double b1 = sb1[tx][k], b2 = sb2[tx][k];
#pragma unroll
            for(int q = 0; q < 4; q++){
                acc1[q] += sa1[ty + 8 * q][k] * b1;
                acc2[q] += a2[ty + 8 * q][k] * b2;
            }
        }
        __syncthreads();
    }
    const int c = c0 + tx;
#pragma unroll
    for(int q = 0; q < 4; q++){
        const int r = r0 + ty + 8 * q;
        if(r < M && c < Nn){
            const long off = (long)r * crs + (long)c * ccs + (long)blockIdx.z * cz;
            if(C2){ C1[off] = scale * acc1[q]; C2[off] = scale * acc2[q]; }
            else C1[off] = scale * (acc1[q] + acc2[q]);
        }
    }
}

// One tridiagonal solve per (mode, cos/sin part) in theta:
//   (q[j+1] - 2 q[j] + q[j-1]) / dthe^2 - lam_m / s_j^2 q[j] = rhs[j],  lam_m = 4 sin^2(pi m/N)/dphi^2,
// the ends folded with q0 = c43 q1 - c13 q2, factored on the host once per context (ModeLU). Every
// row is diagonally dominant, so the factorisation needs no pivoting. Mode 0 is singular: its
// source is made consistent with the left null vector (3/2, 1, ..., 1, 3/2), q pinned at the first
// row, and q returned with zero weighted mean. For the transposed system (tr) the null vectors
// swap: the source is made zero-sum and the pinned row alone fixes q's free multiple of y. The result is written back times the inverse
// transform's weight w_m / N (w = 1 for m = 0 and m = N/2, else 2).
//
// A block takes pm modes (2 pm problems, problem t = 2 m + part): all of its threads stage the
// right-hand sides (the sum of the transform's nsplit partials) into shared memory as [q][t] (row stride 2 pm + 1: conflict-free) and the
// modes' factors as [q][m] (stride pm + 1); then one thread per problem runs the two dependent
// recurrences on shared-memory latency, in place, and the block writes back. Shared memory:
// 8 J (5 pm + 4) bytes.
__global__ void __launch_bounds__(128) sor_tridiag_kernel(SorConst s, ModeLU lu, double* Ac, double* As, int pm,
                                                          int tr, int nsplit, long split_stride){
    extern __shared__ double sm[];
    const int J = s.J, np = 2 * pm, ldr = np + 1, ldf = pm + 1;
    double* sd = sm;                                     // [J][ldr]
    double* fa = sd + (size_t)J * ldr;                   // [J][ldf] each
    double* fc = fa + (size_t)J * ldf;
    double* fi = fc + (size_t)J * ldf;
    const int nmode = s.NM + 1;
    const int m0 = blockIdx.x * pm;
#pragma unroll 4
    for(int idx = threadIdx.x; idx < pm * J; idx += blockDim.x){
        const int lm = idx / J, q = idx - lm * J;
        const int m = m0 + lm;
        double c = 0.0, sn = 0.0, va = 0.0, vc = 0.0, vi = 0.0;
        if(m < nmode){
            const size_t g = (size_t)m * J + q;
            for(int z = 0; z < nsplit; z++){ c += Ac[g + z * split_stride]; sn += As[g + z * split_stride]; }
            va = lu.a[g]; vc = lu.cf[g]; vi = lu.idn[g];
        }
        sd[q * ldr + 2 * lm] = c; sd[q * ldr + 2 * lm + 1] = sn;
        fa[q * ldf + lm] = va; fc[q * ldf + lm] = vc; fi[q * ldf + lm] = vi;
    }
    __syncthreads();
    const int lt = threadIdx.x;
    const int lm = lt >> 1, part = lt & 1, m = m0 + lm;
    if(lt < np && m < nmode){
        double* d = sd + lt;
        if(part == 1 && (m == 0 || 2 * m == s.N)){
            for(int q = 0; q < J; q++) d[q * ldr] = 0.0;
        } else {
            const double* a = fa + lm;
            const double* cf = fc + lm;
            const double* idn = fi + lm;
            if(m == 0){                                       // compatible with the left null vector
                double yr = 0.0, ys = 0.0;
                for(int q = 0; q < J; q++){ const double wq = tr ? 1.0 : ywt(q, 0, J - 1); yr += wq * d[q * ldr]; ys += wq; }
                const double sh = yr / ys;
                for(int q = 0; q < J; q++) d[q * ldr] -= sh;
                d[0] = 0.0;                                   // the pinned row
            }
            double yp = 0.0;
#pragma unroll 4
            for(int q = 0; q < J; q++){ yp = (d[q * ldr] - a[q * ldf] * yp) * idn[q * ldf]; d[q * ldr] = yp; }
            double x = d[(J - 1) * ldr];
#pragma unroll 4
            for(int q = J - 2; q >= 0; q--){ x = d[q * ldr] - cf[q * ldf] * x; d[q * ldr] = x; }
            if(m == 0 && !tr){                                // the free constant: zero y-weighted mean
                double yq = 0.0, ys = 0.0;
                for(int q = 0; q < J; q++){ const double wq = ywt(q, 0, J - 1); yq += wq * d[q * ldr]; ys += wq; }
                const double sh = yq / ys;
                for(int q = 0; q < J; q++) d[q * ldr] -= sh;
            }
        }
    }
    __syncthreads();
    for(int idx = threadIdx.x; idx < pm * J; idx += blockDim.x){
        const int lm2 = idx / J, q = idx - lm2 * J;
        const int m2 = m0 + lm2;
        if(m2 < nmode){
            const double wm = ((m2 == 0 || 2 * m2 == s.N) ? 1.0 : 2.0) / s.N;   // inverse-transform weight
            const size_t g = (size_t)m2 * J + q;
            Ac[g] = wm * sd[q * ldr + 2 * lm2];
            As[g] = wm * sd[q * ldr + 2 * lm2 + 1];
        }
    }
}

// Onto every interior level of the column: P[i][j][k] += q(j,k).
// (TR: y_i q, the trial functions of the transposed system's correction.)
template <typename T, bool TR = false>
__global__ void __launch_bounds__(128) sor_add_kernel(Grid g, const double* qbuf, T* P, int nsplit, long split_stride){
    const int N = g.km - 1;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    if(k >= N) return;
    double q = 0.0;
    for(int z = 0; z < nsplit; z++) q += qbuf[(size_t)(j - 1) * N + k + z * split_stride];   // the partials
    // one thread per column: the levels' loads of a chunk before its stores
    constexpr int CH = 8;
    for(int i0 = 1; i0 < g.im - 1; i0 += CH){
        T v[CH];
#pragma unroll
        for(int c = 0; c < CH; c++) if(i0 + c < g.im - 1) v[c] = P[gidx(g, i0 + c, j, k)];
#pragma unroll
        for(int c = 0; c < CH; c++){
            const int i = i0 + c;
            if(i < g.im - 1) P[gidx(g, i, j, k)] = (T)((double)v[c] + (TR ? ywt(i, 1, g.im - 2) * q : q));
        }
    }
}

// Red-black SOR colour pass of the folded operator, Lc e = r, for T = double (the FP64 solve) or
// float (the correction solve of the mixed form: e and r in FP32, the row assembled in FP64 and
// rounded once).
template <typename T, bool TR = false>
__global__ void __launch_bounds__(256) sor_colour_kernel(Grid g, T* E, const T* R, const RBW* w, int colour, double omega){
    const int half = g.km / 2;
    const int k2 = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    const int i = 1 + blockIdx.z;
    if(k2 >= half || j > g.jm - 2) return;
    const int k = 2 * k2 + ((i + j + colour) & 1);
    if(k > g.km - 2) return;
    const size_t o = gidx(g, i, j, k);
    double diag;
    const double acc = row_acc<TR, T>(g, E, o, i, j, k, w, &diag);
    const double e0 = (double)E[o];
    const double pn = (acc - (double)__ldg(R + o)) / diag;
    E[o] = (T)(e0 + omega * (pn - e0));
}

// One colour of red-black LINE relaxation of the folded operator: every column (j,k) with
// (j + k) & 1 == colour is solved exactly in r, its horizontal neighbours (the other colour, or the
// column itself through the theta fold) held at their current values, then over-relaxed,
// p += omega (p_line - p) -- the reference's PRESS_LINE (PressureSolver.h:497-570) on the folded
// operator. The radial tridiagonal of each column (radial ends folded as :547-550) is factored on
// the host: per (i,j) the row's sub-diagonal `la`, the factor `lcf` and the pivot reciprocal `lidn`
// (the theta fold changes the diagonal on the first and last rows). TR relaxes Lc^T instead: the
// transposed theta couplings and the host-factored transposed column tridiagonals.
//
// A block takes 64 columns of one colour in one row j (lane l: columns l and l + 32). Its 8 warps
// form the right-hand sides of all levels in parallel (coalesced along k, one level of 32 columns
// per warp at a time) into shared memory [level][column] and stage the row's factors beside them;
// warp 0 then runs the recurrences of each lane's two columns interleaved (two independent
// dependency chains per lane), entirely on shared-memory latency, in place; all warps write the
// relaxed columns back. Shared memory: (im - 2) * (LINE_COLS + 3) doubles. With 64 columns the
// default grid's 537 blocks are resident at once (one wave).
constexpr int LINE_COLS = 64;
// Arithmetic of the right-hand sides and recurrences: FP64 for both the FP64 solve and the mixed
// form's FP32 correction solves (FP32 recurrences were no faster per solve and took more sweeps in
// the first steps: the column tridiagonals are strongly anisotropic). LV: levels per warp per pass
// of phases 1 and 3, whose loads all come first; sized so that 4 blocks of 256 threads (64
// registers) stay resident without spills.
template <typename T> struct LineArith { using A = double; static constexpr int LV = 3; };
template <> struct LineArith<float> { using A = double; static constexpr int LV = 5; };

template <typename T, bool TR = false>
__global__ void __launch_bounds__(256, 4) sor_line_kernel(Grid g, T* P, const T* R, const RBW* w, const double* la,
                                                       const double* lcf, const double* lidn, int colour, double omega){
    using A = typename LineArith<T>::A;
    constexpr int LINE_LV = LineArith<T>::LV;
    extern __shared__ __align__(16) unsigned char line_raw[];
    A* ds = reinterpret_cast<A*>(line_raw);
    const int n = g.im - 2;
    A* fa = ds + (size_t)n * LINE_COLS;                // the row's factors by level
    A* fc = fa + n;
    A* fi = fc + n;
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const int j = 1 + blockIdx.y;
    const size_t sj = g.kp;
    for(int i = threadIdx.x; i < n; i += blockDim.x){
        const size_t f = (size_t)(i + 1) * g.jm + j;
        fa[i] = (A)la[f]; fc[i] = (A)lcf[f]; fi[i] = (A)lidn[f];
    }
    int kk[2]; bool valid[2];
#pragma unroll
    for(int h = 0; h < 2; h++){
        const int k2 = blockIdx.x * LINE_COLS + h * 32 + lane;
        kk[h] = 2 * k2 + ((j + colour) & 1);
        valid[h] = k2 < g.km / 2 && kk[h] <= g.km - 2;
    }
    // phase 1: right-hand sides. It reads only the other colour's cells, which this launch does not
    // write (read-only path); per pass, every load of the warp's LINE_LV levels comes first.
    for(int i0 = 1 + wp; i0 <= n; i0 += 8 * LINE_LV){
#pragma unroll
        for(int h = 0; h < 2; h++){
            T vjm[LINE_LV], vjp[LINE_LV], vke[LINE_LV], vkw[LINE_LV], vr[LINE_LV];
            double n2[LINE_LV], n3[LINE_LV], n2m[LINE_LV], n2p[LINE_LV];
            const int k = kk[h];
            const int kw = phi_wrap(k - 1, g.km), ke = phi_wrap(k + 1, g.km);
#pragma unroll
            for(int q = 0; q < LINE_LV; q++){
                const int i = i0 + 8 * q;
                if(i <= n && valid[h]){
                    const size_t o = gidx(g, i, j, k);
                    vjm[q] = __ldg(P + (o - sj)); vjp[q] = __ldg(P + (o + sj));
                    vke[q] = __ldg(P + (o - k + ke)); vkw[q] = __ldg(P + (o - k + kw));
                    vr[q] = __ldg(R + o);
                    n2[q] = __ldg(&w[i * g.jm + j].num2); n3[q] = __ldg(&w[i * g.jm + j].num3);
                    if constexpr(TR){
                        n2m[q] = (j - 1 >= 1) ? __ldg(&w[i * g.jm + j - 1].num2) : 0.0;
                        n2p[q] = (j + 1 <= g.jm - 2) ? __ldg(&w[i * g.jm + j + 1].num2) : 0.0;
                    }
                }
            }
#pragma unroll
            for(int q = 0; q < LINE_LV; q++){
                const int i = i0 + 8 * q;
                if(i > n) break;
                A d = A(0);
                if(valid[h]){
                    // at j = 1 and jm - 2 one theta neighbour is the boundary row, which lies in the
                    // row itself through the theta fold: the other row (o + sj or o - sj) enters
                    const A pjm = (A)vjm[q], pjp = (A)vjp[q];
                    A hsum;
                    if constexpr(TR){                  // the transposed theta couplings (folded_accT)
                        hsum = ((A)vke[q] + (A)vkw[q]) * (A)n3[q];
                        if(j - 1 >= 1)        hsum += (A)n2m[q] * (A)(j - 1 == 1 ? 1.0 - C13 : 1.0) * pjm;
                        if(j + 1 <= g.jm - 2) hsum += (A)n2p[q] * (A)(j + 1 == g.jm - 2 ? 1.0 - C13 : 1.0) * pjp;
                    } else {
                        const A ajm = (j == 1)        ? (A)(-C13) * pjp : pjm;
                        const A ajp = (j == g.jm - 2) ? (A)(-C13) * pjm : pjp;
                        hsum = (ajp + ajm) * (A)n2[q] + ((A)vke[q] + (A)vkw[q]) * (A)n3[q];
                    }
                    d = hsum - (A)vr[q];
                }
                ds[(i - 1) * LINE_COLS + h * 32 + lane] = d;
            }
        }
    }
    __syncthreads();
    // phase 2: the host-factored Thomas recurrences, two independent chains per lane
    if(wp == 0){
        A* c0 = ds + lane;
        A* c1 = ds + 32 + lane;
        A y0 = A(0), y1 = A(0);
#pragma unroll 4
        for(int i = 0; i < n; i++){
            const A a_ = fa[i], r_ = fi[i];
            y0 = (c0[i * LINE_COLS] - a_ * y0) * r_;
            y1 = (c1[i * LINE_COLS] - a_ * y1) * r_;
            c0[i * LINE_COLS] = y0;
            c1[i * LINE_COLS] = y1;
        }
        A x0 = c0[(n - 1) * LINE_COLS], x1 = c1[(n - 1) * LINE_COLS];
#pragma unroll 4
        for(int i = n - 2; i >= 0; i--){
            const A c_ = fc[i];
            x0 = c0[i * LINE_COLS] - c_ * x0;
            x1 = c1[i * LINE_COLS] - c_ * x1;
            c0[i * LINE_COLS] = x0;
            c1[i * LINE_COLS] = x1;
        }
    }
    __syncthreads();
    // phase 3: over-relax the columns in place, loads first
#pragma unroll
    for(int h = 0; h < 2; h++){
        if(!valid[h]) continue;
        for(int i0 = 1 + wp; i0 <= n; i0 += 8 * LINE_LV){
            T pv[LINE_LV];
#pragma unroll
            for(int q = 0; q < LINE_LV; q++){
                const int i = i0 + 8 * q;
                if(i <= n) pv[q] = P[gidx(g, i, j, kk[h])];
            }
#pragma unroll
            for(int q = 0; q < LINE_LV; q++){
                const int i = i0 + 8 * q;
                if(i > n) break;
                const double p0 = (double)pv[q];
                P[gidx(g, i, j, kk[h])] = (T)(p0 + omega * ((double)ds[(i - 1) * LINE_COLS + h * 32 + lane] - p0));
            }
        }
    }
}

// Compatibility: per-block partial sums of y_i y_j src and y_i y_j over the interior (plain: of
// src and 1, the transposed operator's left null vector being the constant).
__global__ void __launch_bounds__(256) sor_ysum_kernel(Grid g, const double* src, double* part, int plain){
    const int J = g.jm - 2, N = g.km - 1;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    double a = 0.0, b = 0.0;
    if(c < J * N){
        const int j = 1 + c / N, k = c - (j - 1) * N;
        const double yj = plain ? 1.0 : ywt(j, 1, g.jm - 2);
        for(int i = 1; i < g.im - 1; i++){
            const double y = plain ? 1.0 : ywt(i, 1, g.im - 2) * yj;
            a += y * src[gidx(g, i, j, k)];
            b += y;
        }
    }
    __shared__ double sa[256], sb[256];
    sa[threadIdx.x] = a; sb[threadIdx.x] = b;
    __syncthreads();
    for(int st = 128; st > 0; st >>= 1){
        if(threadIdx.x < st){ sa[threadIdx.x] += sa[threadIdx.x + st]; sb[threadIdx.x] += sb[threadIdx.x + st]; }
        __syncthreads();
    }
    if(threadIdx.x == 0){ part[2 * blockIdx.x] = sa[0]; part[2 * blockIdx.x + 1] = sb[0]; }
}

// The shift = sum(y y src) / sum(y y) from the partials, in a fixed tree order (one block).
__global__ void __launch_bounds__(256) sor_shift_finish_kernel(const double* part, int nblk, double* shift){
    __shared__ double sa[256], sb[256];
    double a = 0.0, b = 0.0;
    for(int n = threadIdx.x; n < nblk; n += 256){ a += part[2 * n]; b += part[2 * n + 1]; }
    sa[threadIdx.x] = a; sb[threadIdx.x] = b;
    __syncthreads();
    for(int st = 128; st > 0; st >>= 1){
        if(threadIdx.x < st){ sa[threadIdx.x] += sa[threadIdx.x + st]; sb[threadIdx.x] += sb[threadIdx.x + st]; }
        __syncthreads();
    }
    if(threadIdx.x == 0) *shift = sa[0] / sb[0];
}

// src -= shift on the interior (the shift is read from device memory: no host round trip).
__global__ void sor_shift_kernel(Grid g, double* src, const double* shift_p){
    const double shift = *shift_p;
    const int J = g.jm - 2, N = g.km - 1;
    for(int c = blockIdx.x * blockDim.x + threadIdx.x; c < J * N; c += gridDim.x * blockDim.x){
        const int j = 1 + c / N, k = c - (j - 1) * N;
        for(int i = 1; i < g.im - 1; i++) src[gidx(g, i, j, k)] -= shift;
    }
}

// Mixed form: p += e over every cell (e is zero on the boundary rows and the seam column, which no
// correction solve writes).
__global__ void sor_axpy_kernel(size_t n, double* P, const float* e){
    for(size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        P[t] += (double)e[t];
}

}  // namespace aturan
