// The moist convective adjustment (planet/ConvectiveAdjustment.h:402-849,
// MoistConvectiveAdjustment<cUranusModel>::run) with the reference's default knobs: Ledoux test
// with condensate loading, relaxation 1, no latitude smoothing (cUranusModel.h:572), at most 64
// sweeps, no phase split (SATADJ_BERGERON = 2), interior levels only (cUranusModel.h:566); the gas
// list H2O, NH3, H2S (its liquid set for both phases), CH4 and the NH4SH tracer of
// cUranusModel.cpp:1276-1290.
//
// Every (j, k) column is independent. One warp takes one column and keeps its state in its own
// slice of shared memory (16 values and 4 flags per level, two parcel slots): the lanes load,
// convert and write back the levels in parallel, and run in parallel everything of a sweep that
// does not depend on what the sweep has done before it:
//   * at the start of each sweep every pair test (i, i+1) is evaluated, one pair per lane; while
//     the sweep walks up the column a pair is re-tested only if one of its two cells has been
//     mixed in this sweep, which is exactly when its inputs differ from the start's (the
//     reference's first sweep makes the same reuse with its cached test of untouched pairs); the
//     re-test's two equilibria (the parcel, the upper cell's own) are solved on two lanes at once;
//   * a segment's mass-weighted means are summed by lane 0 in the reference's order; then one
//     round of equilibria settles each of its cells on its own lane and, on further lanes, solves
//     what the two growth tests (below and above) need, since none of those solves reads another's
//     result (the lower neighbour lifted to the segment's bottom level, the mixed top cell lifted
//     to the level above, that level's own equilibrium); the tests' decisions follow.
// Each solve is a cell's equilibrium by Illinois regula falsi, so the arithmetic is FP64 whatever
// the storage (FP32 storage in the mixed form is widened, T read as its FP32 pair). The solve, the
// decision, the energy balance and the enthalpy inverse are out-of-line functions, and every round
// reaches the solve through one call site: inlined at each call site the kernel's code outgrew the
// instruction cache and most issue slots went unused for want of an instruction.
// Every loop is bounded: 60 regula-falsi steps, 30 Newton steps of the enthalpy inverse, 64
// sweeps, and a segment grows by one level per step within the column.
#pragma once
#include "common.cuh"

namespace aturan {

constexpr int MCA_NG = 4;
constexpr double CP_T_LO_D = 5.0, CP_T_HI_D = 1500.0, CP_DT_D = 0.5;   // CpH2.h:13

struct McaGas { double ep, lv, ls, t_0, C, L0, R, del_alf, del_bet, C_i, L0_i, del_alf_i, del_bet_i; };

struct McaConst {
    McaGas G[MCA_NG];                // H2O, NH3, H2S, CH4
    double L_tr, t_ref, grav, cp_mix, r_mix, cp_h2, r_h2, r_he, r_ch4, cp_he, cp_ch4;
    float hz;                        // level spacing [km] as the model stores it (float)
    int cp_dyn, cp_mode, cp_gas, local_rho;
    const double *cp_tab, *H_tab;    // H2 cp table and its running integral (CpH2.h:66-75)
};

template <typename S>
struct McaArgs {
    Grid g;
    McaConst c;
    S* t;
    float* tlo;                      // the mixed form's temperature pair (common.cuh), else null
    S* sp[MCA_NG][3];                // vapour, cloud, ice
    S* nh4sh;
    const S *ps, *rho;
};

__device__ __forceinline__ double mca_mx(double a, double b){ return (a < b) ? b : a; }   // std::max

// CpH2.h:88-101, 122-157
static __device__ double mca_cp_h2(const McaConst& A, double T){
    if(A.cp_mode <= 0) return A.cp_h2;
    const double Tc = T < CP_T_LO_D ? CP_T_LO_D : T;
    const double x = ((Tc > CP_T_HI_D ? CP_T_HI_D : Tc) - CP_T_LO_D) / CP_DT_D;
    int i = (int)x; if(i > CP_TABLE_N - 2) i = CP_TABLE_N - 2;
    const double f = x - i;
    return A.cp_tab[i] + f * (A.cp_tab[i + 1] - A.cp_tab[i]);
}
static __device__ double mca_enth_h2(const McaConst& A, double T){
    if(A.cp_mode <= 0) return A.cp_h2 * T;
    const int n = CP_TABLE_N;
    if(T <= CP_T_LO_D) return A.cp_tab[0] * T;
    if(T >= CP_T_HI_D) return A.H_tab[n - 1] + A.cp_tab[n - 1] * (T - CP_T_HI_D);
    const double x = (T - CP_T_LO_D) / CP_DT_D;
    int i = (int)x; if(i > n - 2) i = n - 2;
    const double f = x - i;
    return A.H_tab[i] + CP_DT_D * f * (A.cp_tab[i] + 0.5 * f * (A.cp_tab[i + 1] - A.cp_tab[i]));
}
static __device__ double mca_cp(const McaConst& A, double T){
    if(!A.cp_dyn) return A.cp_mix;
    const double ch = mca_cp_h2(A, T);
    if(A.cp_gas) return (A.r_h2 * ch + A.r_he * A.cp_he + A.r_ch4 * A.cp_ch4) / (A.r_h2 + A.r_he + A.r_ch4);
    return A.cp_mix + (A.r_h2 / A.r_mix) * (ch - A.cp_h2);
}
static __device__ double mca_enth(const McaConst& A, double T){
    if(!A.cp_dyn) return A.cp_mix * T;
    const double hh = mca_enth_h2(A, T);
    if(A.cp_gas) return (A.r_h2 * hh + (A.r_he * A.cp_he + A.r_ch4 * A.cp_ch4) * T) / (A.r_h2 + A.r_he + A.r_ch4);
    return (A.cp_mix - (A.r_h2 / A.r_mix) * A.cp_h2) * T + (A.r_h2 / A.r_mix) * hh;
}
static __device__ __noinline__ double mca_enth_inv(const McaConst& A, double h, double T0){
    if(!A.cp_dyn) return h / A.cp_mix;
    double T = (T0 > 0.0) ? T0 : h / A.cp_mix;
    for(int it = 0; it < 30; it++){
        const double f = mca_enth(A, T) - h, c = mca_cp(A, T);
        const double dT = f / c;
        T -= dT; if(T < 1.0) T = 1.0;
        if(fabs(dT) < 1.0e-10 * T) break;
    }
    return T;
}

// ATPhys.h:49-53 (the saturation pressure) and ConvectiveAdjustment.h:437-453 without the phase
// split; lg = log(T), the same value for every gas at one T, formed once by the caller
__device__ __forceinline__ double mca_qsat(const McaGas& s, double T, double lg, double pr){
    const double E = (T >= s.t_0) ? exp(s.C + (-s.L0 / T + s.del_alf * lg + s.del_bet * T) / (1e-3 * s.R))
                                  : exp(s.C_i + (-s.L0_i / T + s.del_alf_i * lg + s.del_bet_i * T) / (1e-3 * s.R));
    const double q = s.ep * E / pr;
    return isfinite(q) ? q : 0.0;
}
__device__ __forceinline__ double mca_lat(const McaGas& s, double T){ return T >= s.t_0 ? s.lv : s.ls; }

static __device__ __noinline__ double mca_fof(const McaConst& A, double TT, double hL, const double* qt, double pr, double z){
    double f = mca_enth(A, TT) + A.grav * z - hL;
    const double lg = log(TT);
    for(int g = 0; g < MCA_NG; g++) f -= mca_lat(A.G[g], TT) * mca_mx(0.0, qt[g] - mca_qsat(A.G[g], TT, lg, pr));
    return f;
}

// :455-488, the equilibrium of (hL, qt) at (p, z): Illinois regula falsi on the energy balance
static __device__ __noinline__ bool mca_equil(const McaConst& A, double hL, const double* qt, double pr, double z, double& T, double* cond){
    const double cp = A.cp_mix, tol_T = 1.0e-10;
    const double T_lo = A.cp_dyn ? mca_enth_inv(A, hL - A.grav * z, 0.0) : (hL - A.grav * z) / cp;
    if(!(T_lo > 0.0) || !(pr > 0.0)) return false;
    bool any = false;
    const double lg_lo = log(T_lo);
    for(int g = 0; g < MCA_NG; g++) if(qt[g] > mca_qsat(A.G[g], T_lo, lg_lo, pr)){ any = true; break; }
    if(!any){ T = T_lo; for(int g = 0; g < MCA_NG; g++) cond[g] = 0.0; return true; }
    double span = 0.0;
    for(int g = 0; g < MCA_NG; g++) span += mca_mx(A.G[g].lv, A.G[g].ls) * mca_mx(0.0, qt[g]);
    double a = T_lo, b = A.cp_dyn ? mca_enth_inv(A, mca_enth(A, T_lo) + span, T_lo) + 1.0e-9 : T_lo + span / cp + 1.0e-9;
    double fa = mca_fof(A, a, hL, qt, pr, z), fb = mca_fof(A, b, hL, qt, pr, z);
    int side = 0;
    for(int it = 0; it < 60 && b - a > tol_T; it++){
        double c = (fb - fa != 0.0) ? b - fb * (b - a) / (fb - fa) : 0.5 * (a + b);
        if(!(c > a && c < b)) c = 0.5 * (a + b);
        const double fc = mca_fof(A, c, hL, qt, pr, z);
        if(fc < 0.0){ a = c; fa = fc; if(side == -1) fb *= 0.5; side = -1; }
        else        { b = c; fb = fc; if(side == +1) fa *= 0.5; side = +1; }
        if(fabs(fc) <= cp * tol_T){ a = b = c; break; }
    }
    T = b;
    const double lg_b = log(T);
    for(int g = 0; g < MCA_NG; g++) cond[g] = mca_mx(0.0, qt[g] - mca_qsat(A.G[g], T, lg_b, pr));
    return true;
}

// One column's state in its warp's slice of shared memory (levels 0..im-1, i0..i1 used).
struct McaCol {
    double *T, *p, *z, *rho, *w, *hL, *qr, *Teq;   // im each
    double *qt, *ceq;                              // im * MCA_NG each
    double *par;                                   // two parcel results: T, condensate[4], solved
    unsigned char *touched, *eq_ok, *mod, *U;      // im each: mixed ever, equilibrium cached,
                                                   // mixed in this sweep, the pair test of the sweep's start
};
constexpr int MCA_PAR = 6;                         // doubles per parcel slot
// Bytes of one warp's slice for a column of im levels; a block's slices share at most MCA_SMEM_MAX.
constexpr size_t MCA_SMEM_MAX = 227 * 1024;
__host__ __device__ inline size_t mca_warp_bytes(int im){
    return (size_t)(16 * im + 2 * MCA_PAR) * sizeof(double) + (((size_t)4 * im + 7) / 8) * 8;
}
__device__ inline McaCol mca_col(char* base, int im){
    McaCol C;
    double* d = reinterpret_cast<double*>(base);
    C.T = d; C.p = d + im; C.z = d + 2 * im; C.rho = d + 3 * im; C.w = d + 4 * im; C.hL = d + 5 * im;
    C.qr = d + 6 * im; C.Teq = d + 7 * im; C.qt = d + 8 * im; C.ceq = d + 12 * im; C.par = d + 16 * im;
    unsigned char* f = reinterpret_cast<unsigned char*>(d + 16 * im + 2 * MCA_PAR);
    C.touched = f; C.eq_ok = f + im; C.mod = f + 2 * im; C.U = f + 3 * im;
    return C;
}

__device__ __forceinline__ double mca_trE(const McaConst& A, const McaCol& C, int i){ double e = 0.0; e += A.L_tr * C.qr[i]; return e; }

// :613-624, Ledoux virtual temperature with condensate loading; NH4SH is a condensed tracer
static __device__ double mca_tv(const McaConst& A, const McaCol& C, double TT, const double* v_, const double* cnd, int i_tr){
    double f = 1.0;
    for(int g = 0; g < MCA_NG; g++){ f += v_[g] * (1.0 / A.G[g].ep - 1.0); f -= cnd[g]; }
    f -= C.qr[i_tr];
    return TT * f;
}

// The equilibrium of cell a's state (hL, qt, NH4SH) at level b's pressure and height: the parcel
// of a pair test (a below b), or a cell's own (a = b).
__device__ __forceinline__ bool mca_solve_at(const McaConst& A, const McaCol& C, int a, int b, double& T, double* c){
    return mca_equil(A, C.hL[a] + mca_trE(A, C, a), &C.qt[a * MCA_NG], C.p[b], C.z[b], T, c);
}

// :627-644, the test of the pair (a, b = a+1) once both equilibria are known: the parcel (cell a at
// b's level: Tp, pc) against cell b's cached equilibrium.
static __device__ __noinline__ bool mca_decide(const McaConst& A, const McaCol& C, double Tp, const double* pc, int a, int b){
    const double tol_K = 1.0e-7;
    double pv[MCA_NG], ec[MCA_NG], ev[MCA_NG];
    const double Tb = C.Teq[b];
    for(int g = 0; g < MCA_NG; g++) ec[g] = C.ceq[b * MCA_NG + g];
    for(int g = 0; g < MCA_NG; g++){ pv[g] = C.qt[a * MCA_NG + g] - pc[g]; ev[g] = C.qt[b * MCA_NG + g] - ec[g]; }
    const double dTv = mca_tv(A, C, Tp, pv, pc, a) - mca_tv(A, C, Tb, ev, ec, b);
    return dTv > tol_K;
}

// The whole test of the pair (a, b) on one lane: the parcel, b's equilibrium if not cached (written
// by this lane only: each cell is the upper cell of one pair), the decision.
static __device__ __noinline__ bool mca_unstable(const McaConst& A, McaCol& C, int a, int b){
    double Tp, pc[MCA_NG];
    if(!mca_solve_at(A, C, a, b, Tp, pc)) return false;
    if(!C.eq_ok[b]){
        if(!mca_solve_at(A, C, b, b, C.Teq[b], &C.ceq[b * MCA_NG])) return false;
        C.eq_ok[b] = 1;
    }
    return mca_decide(A, C, Tp, pc, a, b);
}

// One round of equilibria across the warp, task t on lane t mod 32, every solve through one call
// site so that the lanes run it together. Tasks 0 .. nset-1 settle the segment cells lo .. lo+nset-1
// at their own levels (:645-661: T, the cached equilibrium, touched); the parcel tasks (cell ca
// lifted to level lb, result in parcel slot s) and the own-equilibrium task (cell own, if not
// cached) follow. Returns false on the lanes whose settle failed.
__device__ __forceinline__ bool mca_round(const McaConst& A, McaCol& C, int lane, int lo, int nset,
                                          int ca0, int lb0, int ca1, int lb1, int own){
    const int ntask = nset + 3;
    bool sok = true;
    for(int t = lane; t < ntask; t += 32){
        int ca, lb, slot = -1;
        if(t < nset){ ca = lb = lo + t; }
        else if(t == nset){ if(ca0 < 0) continue; ca = ca0; lb = lb0; slot = 0; }
        else if(t == nset + 1){ if(ca1 < 0) continue; ca = ca1; lb = lb1; slot = 1; }
        else { if(own < 0 || C.eq_ok[own]) continue; ca = lb = own; }
        double* To = slot < 0 ? &C.Teq[lb] : &C.par[slot * MCA_PAR];
        double* co = slot < 0 ? &C.ceq[lb * MCA_NG] : &C.par[slot * MCA_PAR + 1];
        const bool ok = mca_solve_at(A, C, ca, lb, *To, co);
        if(slot >= 0) C.par[slot * MCA_PAR + 5] = ok ? 1.0 : 0.0;
        else if(ok){ C.eq_ok[lb] = 1; if(t < nset){ C.T[lb] = C.Teq[lb]; C.touched[lb] = 1; } }
        else if(t < nset) sok = false;
    }
    return sok;
}
// The decision of a pair whose parcel is in slot s and whose upper cell's equilibrium is cached.
__device__ __forceinline__ bool mca_slot_unstable(const McaConst& A, const McaCol& C, int s, int a, int b){
    return C.par[s * MCA_PAR + 5] != 0.0 && C.eq_ok[b] && mca_decide(A, C, C.par[s * MCA_PAR], &C.par[s * MCA_PAR + 1], a, b);
}

// One warp per (j, k) column (blockDim = (32, W)), k over all km stored meridians as the reference
// loops; the warp's slice of dynamic shared memory holds the column. The arguments stay in the
// constant bank (__grid_constant__): the out-of-line helpers take the constants by reference, which
// otherwise copies the whole argument block to every thread's stack and reads it from there. Six
// resident blocks per SM (80 registers, the sweep's bookkeeping partly spilled to L1) measured 7 %
// faster than four at 128 registers.
template <typename S>
__global__ void __launch_bounds__(128, 6) mca_warp_kernel(const __grid_constant__ McaArgs<S> a){
    extern __shared__ __align__(16) char mca_smem[];
    const Grid& g = a.g;
    const McaConst& A = a.c;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x;
    const long col = (long)blockIdx.x * blockDim.y + threadIdx.y;
    if(col >= (long)g.jm * g.km) return;                     // a whole warp
    const int j = (int)(col / g.km), k = (int)(col % g.km);
    const int im = g.im, i0 = 1, i1 = im - 2;
    if(i1 - i0 < 1) return;
    McaCol C = mca_col(mca_smem + threadIdx.y * mca_warp_bytes(im), im);
    const size_t pl = (size_t)g.jm * g.kp, o0 = gidx(g, 0, j, k);

    bool ok = true;
    for(int i = i0 + lane; i <= i1; i += 32){
        const size_t o = o0 + (size_t)i * pl;
        C.T[i] = t_ld(a.t, a.tlo, o) * A.t_ref;
        C.p[i] = (double)a.ps[o];
        C.z[i] = (double)((float)i * A.hz) * 1.0e3;
        double rr = A.r_mix;                                // rho_at, cUranusModel.h:526-531
        if(A.local_rho){ const double r_ = (double)a.rho[o]; rr = (r_ > 0.0 && isfinite(r_)) ? r_ : A.r_mix; }
        C.rho[i] = rr;
        if(!(C.T[i] > 0.0) || !(C.p[i] > 0.0) || !(C.rho[i] > 0.0) || !isfinite(C.T[i] + C.p[i] + C.rho[i])) ok = false;
    }
    if(!__all_sync(FULL, ok)) return;
    __syncwarp();
    for(int i = i0 + lane; i <= i1; i += 32){
        const size_t o = o0 + (size_t)i * pl;
        const double lo = (i > i0) ? 0.5 * (C.z[i - 1] + C.z[i]) : C.z[i0];
        const double hi = (i < i1) ? 0.5 * (C.z[i] + C.z[i + 1]) : C.z[i1];
        C.w[i] = C.rho[i] * (hi - lo);
        if(!(C.w[i] > 0.0)) ok = false;
        double h = mca_enth(A, C.T[i]) + A.grav * C.z[i];
        for(int q = 0; q < MCA_NG; q++){
            const int x = i * MCA_NG + q;
            const double qv = mca_mx(0.0, (double)a.sp[q][0][o]) / C.rho[i];
            const double qc = mca_mx(0.0, (double)a.sp[q][1][o]) / C.rho[i];
            const double qi = mca_mx(0.0, (double)a.sp[q][2][o]) / C.rho[i];
            C.qt[x] = qv + qc + qi;
            h -= A.G[q].lv * qc + A.G[q].ls * qi;
        }
        C.qr[i] = (double)a.nh4sh[o] / C.rho[i];
        h -= A.L_tr * C.qr[i];
        C.hL[i] = h;
    }
    for(int i = lane; i < im; i += 32){ C.touched[i] = 0; C.eq_ok[i] = 0; }
    if(!__all_sync(FULL, ok)) return;
    __syncwarp();

    int passes = 0;
    bool changed = true, fail = false;
    long layers = 0;
    while(changed && passes < 64 && !fail){
        changed = false; passes++;
        // every pair's test at the start of the sweep, one pair per lane
        for(int i = i0 + lane; i < i1; i += 32) C.U[i] = mca_unstable(A, C, i, i + 1) ? 1 : 0;
        for(int i = lane; i < im; i += 32) C.mod[i] = 0;
        __syncwarp();
        int i = i0;
        while(i < i1 && !fail){
            bool uns;
            if(!C.mod[i] && !C.mod[i + 1]) uns = C.U[i] != 0;
            else {
                // re-test: the parcel (lane 0) and cell i+1's own equilibrium (lane 1) in one round
                mca_round(A, C, lane, i, 0, i, i + 1, -1, -1, i + 1);
                __syncwarp();
                int u = 0;
                if(lane == 0) u = mca_slot_unstable(A, C, 0, i, i + 1) ? 1 : 0;
                u = __shfl_sync(FULL, u, 0);
                uns = u != 0;
                __syncwarp();
            }
            if(!uns){ i++; continue; }
            int lo = i, hi = i + 1;
            for(;;){
                // the segment's mass-weighted means, summed in the reference's order
                double m_h = 0.0, m_q[MCA_NG], m_r = 0.0;
                if(lane == 0){
                    double sw = 0.0, sh = 0.0, sq[MCA_NG] = {0.0, 0.0, 0.0, 0.0}, sr = 0.0;
                    for(int q = lo; q <= hi; q++){
                        sw += C.w[q]; sh += C.w[q] * C.hL[q];
                        for(int s = 0; s < MCA_NG; s++) sq[s] += C.w[q] * C.qt[q * MCA_NG + s];
                        sr += C.w[q] * C.qr[q];
                    }
                    m_h = sh / sw;
                    for(int s = 0; s < MCA_NG; s++) m_q[s] = sq[s] / sw;
                    m_r = sr / sw;
                }
                m_h = __shfl_sync(FULL, m_h, 0);
                for(int s = 0; s < MCA_NG; s++) m_q[s] = __shfl_sync(FULL, lane == 0 ? m_q[s] : 0.0, 0);
                m_r = __shfl_sync(FULL, m_r, 0);
                for(int q = lo + lane; q <= hi; q += 32){
                    C.hL[q] = m_h;
                    for(int s = 0; s < MCA_NG; s++) C.qt[q * MCA_NG + s] = m_q[s];
                    C.qr[q] = m_r;
                    C.mod[q] = 1;
                }
                __syncwarp();
                // one round: the segment's settles and the two growth tests' solves (cell lo-1
                // lifted to level lo, the mixed cell hi lifted to level hi+1, cell hi+1's own),
                // none of which depends on another; the decisions follow from the results
                const bool below = lo > i0, above = hi < i1;
                const bool sok = mca_round(A, C, lane, lo, hi - lo + 1, below ? lo - 1 : -1, lo,
                                           above ? hi : -1, hi + 1, above ? hi + 1 : -1);
                fail = !__all_sync(FULL, sok);
                __syncwarp();
                if(fail) break;
                int gr = 0;
                if(lane == 0 && below) gr = mca_slot_unstable(A, C, 0, lo - 1, lo) ? 1 : 0;
                if(lane == 1 && above) gr = mca_slot_unstable(A, C, 1, hi, hi + 1) ? 2 : 0;
                gr = __reduce_or_sync(FULL, (unsigned)gr);
                __syncwarp();
                if(gr & 1) lo--;
                if(gr & 2) hi++;
                if(!gr) break;
            }
            layers += hi - lo + 1;
            changed = true;
            i = hi;
        }
    }
    if(fail || layers == 0) return;                        // nothing written: the column keeps its state
    for(int q = i0 + lane; q <= i1; q += 32){
        if(!C.touched[q]) continue;
        const size_t o = o0 + (size_t)q * pl;
        t_st(a.t, a.tlo, o, C.T[q] / A.t_ref);
        for(int s = 0; s < MCA_NG; s++){
            const int x = q * MCA_NG + s;
            const double ce = C.ceq[x];
            const double qv = C.qt[x] - ce;
            const bool liq = C.T[q] >= A.G[s].t_0;
            a.sp[s][0][o] = (S)(qv * C.rho[q]);
            a.sp[s][1][o] = (S)((liq ? ce : 0.0) * C.rho[q]);
            a.sp[s][2][o] = (S)((liq ? 0.0 : ce) * C.rho[q]);
        }
        a.nh4sh[o] = (S)(C.qr[q] * C.rho[q]);
    }
}

// CpH2.h:66-75: the running integral of the cp table, in the table's order (one thread).
static __global__ void mca_H_kernel(const double* cp, double* H){
    if(threadIdx.x != 0 || blockIdx.x != 0) return;
    H[0] = cp[0] * CP_T_LO_D;
    for(int i = 1; i < CP_TABLE_N; i++) H[i] = H[i - 1] + 0.5 * CP_DT_D * (cp[i] + cp[i - 1]);
}

}  // namespace aturan
