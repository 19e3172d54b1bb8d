// FP64 instantiation of the aturan_b200 kernels: the parity path.
//
// Compiled with --fmad=false: the reference's build never contracts a*b+c into an FMA, and
// with contraction off every +, -, *, / and sqrt here rounds exactly as the CPU's does (CUDA's
// FP64 division and square root are IEEE round-to-nearest). Together with the reference's
// operand order kept in every expression, the RHS, the RK4 update, the hydrostatic integral and
// both pressure solvers reproduce the CPU's results bit for bit; the saturation adjustment
// differs only where CUDA's exp/log round differently from the host libm's.
#include "rk4.cuh"
#include "satadj.cuh"
#include "pressure.cuh"
#include "mca.cuh"
#include "launch.h"
#include "launch_impl.cuh"

namespace aturan {
ATURAN_DEFINE_LAUNCHERS(double, double)

__global__ void scale_copy_f64_kernel(const double* in, double* out, size_t n, double coeff){
    for(size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        out[t] = coeff * in[t];
}
void launch_scale_copy_f64(const double* in, double* out, size_t n, double coeff, cudaStream_t st){
    scale_copy_f64_kernel<<<148 * 8, 256, 0, st>>>(in, out, n, coeff);
}

void launch_mca_H(const double* cp_tab, double* H, cudaStream_t st){
    mca_H_kernel<<<1, 32, 0, st>>>(cp_tab, H);
}

int launch_filter_f64(const Grid& g, double* x, bool ai, bool aj, bool ak, double strength, int phi_periodic, cudaStream_t st){
    return launch_filter<double>(g, x, nullptr, ai, aj, ak, strength, phi_periodic, st);
}

void launch_pdyn_bcs(Grid g, double* P, cudaStream_t st){
    pdyn_bc_r_kernel<<<dim3((g.km + 127) / 128, g.jm), 128, 0, st>>>(g, P);
    pdyn_bc_t_kernel<<<dim3((g.km + 127) / 128, g.im), 128, 0, st>>>(g, P);
    pdyn_bc_p_kernel<<<(g.im * g.jm + 255) / 256, 256, 0, st>>>(g, P);
}

void launch_rb_colour(Grid g, double* P, const double* src, const RBW* w, int colour, double omega, cudaStream_t st){
    const int half = g.km / 2;
    rb_colour_kernel<<<dim3((half + 127) / 128, g.jm - 2, g.im - 2), 128, 0, st>>>(g, P, src, w, colour, omega);
}
}  // namespace aturan
