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

__device__ __forceinline__ double ywt(int n, int lo, int hi){ return (n == lo || n == hi) ? 1.5 : 1.0; }

// The shared solver's operator with the 2-point Neumann folds substituted into the rows (at i = 1
// the boundary value c43 p[1] - c13 p[2] puts c43 num1 on the diagonal and -c13 num1 on p[2];
// likewise at i = im-2, j = 1, j = jm-2), instead of boundary rows refreshed after each sweep as
// the reference does. Same operator on the interior unknowns, hence the same solution; but every
// row couples only to the other colour, so red-black SOR keeps its consistently-ordered rate
// (with the lagged rows the radially structured modes converge at ~0.955 per sweep at omega 1.9
// instead of ~0.9). Returns the off-diagonal sum; *diag receives the diagonal.
template <typename T>
__device__ __forceinline__ double folded_acc(const Grid& g, const T* P, size_t o, int i, int j, int k,
                                             const RBW& W, double* diag){
    const size_t si = (size_t)g.jm * g.kp, sj = g.kp;
    const int kw = phi_wrap(k - 1, g.km), ke = phi_wrap(k + 1, g.km);
    double d = W.den;
    double aim, aip, ajm, ajp;
    if(i == 1)        { d -= C43 * W.num1; aim = -C13 * (double)P[o + si]; } else aim = (double)P[o - si];
    if(i == g.im - 2) { d -= C43 * W.num1; aip = -C13 * (double)P[o - si]; } else aip = (double)P[o + si];
    if(j == 1)        { d -= C43 * W.num2; ajm = -C13 * (double)P[o + sj]; } else ajm = (double)P[o - sj];
    if(j == g.jm - 2) { d -= C43 * W.num2; ajp = -C13 * (double)P[o - sj]; } else ajp = (double)P[o + sj];
    *diag = d;
    return (aip + aim) * W.num1 + (ajp + ajm) * W.num2
         + ((double)P[o - k + ke] + (double)P[o - k + kw]) * W.num3;
}

// Per (j,k) column: y-weighted sum of r = src - Lc p over the interior levels, and per-block
// partial sums of r^2 and src^2 (fixed tree order). P of type T (double for the FP64 solve,
// float for the correction solve of the mixed form), src of type T.
template <typename T>
__global__ void __launch_bounds__(256) sor_colsum_kernel(Grid g, const T* P, const T* src, const RBW* w,
                                                         double* colR, double* part, int want_col){
    const int J = g.jm - 2, N = g.km - 1;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    double rr = 0.0, ss = 0.0;
    if(c < J * N){
        const int j = 1 + c / N, k = c - (j - 1) * N;
        const int kw = phi_wrap(k - 1, g.km), ke = phi_wrap(k + 1, g.km);
        double R = 0.0;
        (void)kw; (void)ke;
        for(int i = 1; i < g.im - 1; i++){
            const RBW W = w[i * g.jm + j];
            const size_t o = gidx(g, i, j, k);
            double diag;
            const double acc = folded_acc<T>(g, P, o, i, j, k, W, &diag);
            const double lc = acc - diag * (double)P[o];
            const double s = (double)src[o];
            const double r = s - lc;
            R += ywt(i, 1, g.im - 2) * r;
            rr += r * r;
            ss += s * s;
        }
        if(want_col) colR[(size_t)(j - 1) * N + k] = R;
    }
    __shared__ double sr[256], sq[256];
    sr[threadIdx.x] = rr; sq[threadIdx.x] = ss;
    __syncthreads();
    for(int st = 128; st > 0; st >>= 1){
        if(threadIdx.x < st){ sr[threadIdx.x] += sr[threadIdx.x + st]; sq[threadIdx.x] += sq[threadIdx.x + st]; }
        __syncthreads();
    }
    if(threadIdx.x == 0){ part[2 * blockIdx.x] = sr[0]; part[2 * blockIdx.x + 1] = sq[0]; }
}

// DFT in phi of colR / A2y: Ac[m][j] = sum_k R cos(2 pi m k / N), As likewise with sin.
// ct/st are host-built tables with the (m k mod N) reduction of PressureSolver.h:614-617.
__global__ void sor_dft_kernel(SorConst s, const double* colR, const double* ct, const double* st,
                               double* Ac, double* As){
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if(t >= (s.NM + 1) * s.J) return;
    const int m = t / s.J, jj = t - m * s.J;
    const double* r = colR + (size_t)jj * s.N;
    const double* c = ct + (size_t)m * s.N;
    const double* sn = st + (size_t)m * s.N;
    double sc = 0.0, ss = 0.0;
    for(int k = 0; k < s.N; k++){ const double v = r[k] / s.A2y; sc += v * c[k]; ss += v * sn[k]; }
    Ac[(size_t)m * s.J + jj] = sc;
    As[(size_t)m * s.J + jj] = ss;
}

// One tridiagonal solve per (mode, cos/sin part) in theta:
//   (q[j+1] - 2 q[j] + q[j-1]) / dthe^2 - lam_m / s_j^2 q[j] = rhs[j],  lam_m = 4 sin^2(pi m/N)/dphi^2,
// the ends folded with q0 = c43 q1 - c13 q2. Mode 0 is singular: its source is made consistent
// with the left null vector (3/2, 1, ..., 1, 3/2) and q pinned to zero mean with those weights.
// Thomas needs no pivoting: every row is diagonally dominant (|b| >= |a| + |c|, strictly for
// m > 0; the folded end rows keep 2/3 e against 2/3 e).
__global__ void sor_tridiag_kernel(SorConst s, const double* lam, const double* sj, double* Ac, double* As,
                                   double* work){
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if(t >= 2 * (s.NM + 1)) return;
    const int m = t >> 1, part = t & 1;
    if(part == 1 && (m == 0 || 2 * m == s.N)) { if(part == 1){ double* d = As + (size_t)m * s.J; for(int q = 0; q < s.J; q++) d[q] = 0.0; } return; }
    double* d = (part == 0 ? Ac : As) + (size_t)m * s.J;
    double* cp = work + (size_t)t * 2 * s.J;
    double* dp = cp + s.J;
    const int J = s.J;
    const double e = s.inv_dthe2;
    if(m == 0){
        double yr = 0.0, ys = 0.0;
        for(int q = 0; q < J; q++){ const double y = ywt(q, 0, J - 1); yr += y * d[q]; ys += y; }
        for(int q = 0; q < J; q++) d[q] -= yr / ys;
    }
    auto A = [&](int q){ double a = e; if(q == 0) a = 0.0; if(q == J - 1) a -= C13 * e; return a; };
    auto B = [&](int q){ double b = -2.0 * e - lam[m] / (sj[q] * sj[q]); if(q == 0 || q == J - 1) b += C43 * e; return b; };
    auto Cc = [&](int q){ double c = e; if(q == J - 1) c = 0.0; if(q == 0) c -= C13 * e; return c; };
    double b0 = B(0), c0 = Cc(0), d0 = d[0];
    if(m == 0){ b0 = 1.0; c0 = 0.0; d0 = 0.0; }           // pin q at j = 1
    cp[0] = c0 / b0; dp[0] = d0 / b0;
    for(int q = 1; q < J; q++){
        const double dn = B(q) - A(q) * cp[q - 1];
        cp[q] = Cc(q) / dn;
        dp[q] = (d[q] - A(q) * dp[q - 1]) / dn;
    }
    d[J - 1] = dp[J - 1];
    for(int q = J - 2; q >= 0; q--) d[q] = dp[q] - cp[q] * d[q + 1];
    if(m == 0){                                           // zero y-weighted mean
        double yq = 0.0, ys = 0.0;
        for(int q = 0; q < J; q++){ const double y = ywt(q, 0, J - 1); yq += y * d[q]; ys += y; }
        for(int q = 0; q < J; q++) d[q] -= yq / ys;
    }
}

// Back to phi and onto every interior level of the column: P[i][j][k] += q(j,k).
template <typename T>
__global__ void sor_idft_add_kernel(Grid g, SorConst s, const double* Ac, const double* As, const double* ct,
                                    const double* st, T* P){
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if(c >= s.J * s.N) return;
    const int jj = c / s.N, k = c - jj * s.N;
    double q = 0.0;
    for(int m = 0; m <= s.NM; m++){
        const bool edge = (m == 0 || 2 * m == s.N);
        const double w_ = edge ? 1.0 : 2.0;
        q += w_ * (Ac[(size_t)m * s.J + jj] * ct[(size_t)m * s.N + k]
                   + (edge ? 0.0 : As[(size_t)m * s.J + jj] * st[(size_t)m * s.N + k]));
    }
    q /= s.N;
    for(int i = 1; i < g.im - 1; i++){
        const size_t o = gidx(g, i, jj + 1, k);
        P[o] = (T)((double)P[o] + q);
    }
}

// Red-black SOR colour pass of the folded operator, Lc e = r, for T = double (the FP64 solve) or
// float (the correction solve of the mixed form: e and r in FP32, the row assembled in FP64 and
// rounded once).
template <typename T>
__global__ void __launch_bounds__(256) sor_colour_kernel(Grid g, T* E, const T* R, const RBW* w, int colour, double omega){
    const int half = g.km / 2;
    const int k2 = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    const int i = 1 + blockIdx.z;
    if(k2 >= half || j > g.jm - 2) return;
    const int k = 2 * k2 + ((i + j + colour) & 1);
    if(k > g.km - 2) return;
    const RBW W = w[i * g.jm + j];
    const size_t o = gidx(g, i, j, k);
    double diag;
    const double acc = folded_acc<T>(g, E, o, i, j, k, W, &diag);
    const double e0 = (double)E[o];
    const double pn = (acc - (double)R[o]) / diag;
    E[o] = (T)(e0 + omega * (pn - e0));
}

// The folded boundary passes for any T (same order as pdyn_bc_*).
template <typename T>
__global__ void bc_r_kernel(Grid g, T* P){
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if(k >= g.km) return;
    P[gidx(g, 0, j, k)]        = (T)(C43 * (double)P[gidx(g, 1, j, k)] - C13 * (double)P[gidx(g, 2, j, k)]);
    P[gidx(g, g.im - 1, j, k)] = (T)(C43 * (double)P[gidx(g, g.im - 2, j, k)] - C13 * (double)P[gidx(g, g.im - 3, j, k)]);
}
template <typename T>
__global__ void bc_t_kernel(Grid g, T* P){
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if(k >= g.km) return;
    P[gidx(g, i, 0, k)]        = (T)(C43 * (double)P[gidx(g, i, 1, k)] - C13 * (double)P[gidx(g, i, 2, k)]);
    P[gidx(g, i, g.jm - 1, k)] = (T)(C43 * (double)P[gidx(g, i, g.jm - 2, k)] - C13 * (double)P[gidx(g, i, g.jm - 3, k)]);
}
template <typename T>
__global__ void bc_p_kernel(Grid g, T* P){
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if(c >= g.im * g.jm) return;
    const int i = c / g.jm, j = c - i * g.jm;
    P[gidx(g, i, j, g.km - 1)] = P[gidx(g, i, j, 0)];
}

// Compatibility: per-block partial sums of y_i y_j src and y_i y_j over the interior.
__global__ void __launch_bounds__(256) sor_ysum_kernel(Grid g, const double* src, double* part){
    const int J = g.jm - 2, N = g.km - 1;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    double a = 0.0, b = 0.0;
    if(c < J * N){
        const int j = 1 + c / N, k = c - (j - 1) * N;
        const double yj = ywt(j, 1, g.jm - 2);
        for(int i = 1; i < g.im - 1; i++){
            const double y = ywt(i, 1, g.im - 2) * yj;
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

// src -= shift on the interior (the shift is read from device memory: no host round trip).
__global__ void sor_shift_kernel(Grid g, double* src, const double* part, int nblk){
    __shared__ double shift;
    if(threadIdx.x == 0){
        double a = 0.0, b = 0.0;
        for(int n = 0; n < nblk; n++){ a += part[2 * n]; b += part[2 * n + 1]; }
        shift = a / b;
    }
    __syncthreads();
    const int J = g.jm - 2, N = g.km - 1;
    for(int c = blockIdx.x * blockDim.x + threadIdx.x; c < J * N; c += gridDim.x * blockDim.x){
        const int j = 1 + c / N, k = c - (j - 1) * N;
        for(int i = 1; i < g.im - 1; i++) src[gidx(g, i, j, k)] -= shift;
    }
}

// Mixed form: r = src - Lc p in FP64, stored as FP32 for the correction solve; e cleared.
__global__ void sor_resid32_kernel(Grid g, const double* P, const double* src, const RBW* w, float* r32, float* e32){
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int i = blockIdx.z;
    if(k >= g.km) return;
    const size_t o = gidx(g, i, j, k);
    e32[o] = 0.0f;
    if(i == 0 || i == g.im - 1 || j == 0 || j == g.jm - 1 || k == g.km - 1){ r32[o] = 0.0f; return; }
    const RBW W = w[i * g.jm + j];
    double diag;
    const double acc = folded_acc<double>(g, P, o, i, j, k, W, &diag);
    const double lc = acc - diag * P[o];
    r32[o] = (float)(src[o] - lc);
}

// Mixed form: p += e over every cell (e carries its own folded boundary rows).
__global__ void sor_axpy_kernel(size_t n, double* P, const float* e){
    for(size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        P[t] += (double)e[t];
}

}  // namespace aturan
