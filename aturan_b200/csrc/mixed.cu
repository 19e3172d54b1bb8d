// FP32 instantiation of the aturan_b200 kernels: the mixed-precision path.
//
// State, n-copies, stage buffers, accumulator and forcing are stored and updated in FP32 and the
// stencils are FP32 arithmetic (FMA contraction allowed). The pressure family (p_dyn, p_hydro,
// p_baro, p_b0, p_bfollow) stays FP64: their gradients enter the momentum equations as
// differences of O(10) values and are formed in FP64 before rounding to FP32. The saturation
// adjustment computes in FP64 whatever the storage (satadj.cuh).
#include "launch.h"
#include "launch_impl.cuh"

namespace aturan {
ATURAN_DEFINE_LAUNCHERS(float, float)

__global__ void f64_to_f32_kernel(const double* in, float* out, size_t n){
    for(size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        out[t] = (float)in[t];
}
__global__ void f32_to_f64_kernel(const float* in, double* out, size_t n){
    for(size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        out[t] = (double)in[t];
}
__global__ void scale_copy_f32_kernel(const float* in, float* out, size_t n, double coeff){
    for(size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        out[t] = (float)(coeff * (double)in[t]);
}
void launch_scale_copy_f32(const float* in, float* out, size_t n, double coeff, cudaStream_t st){
    scale_copy_f32_kernel<<<148 * 8, 256, 0, st>>>(in, out, n, coeff);
}

void launch_f64_to_f32(const double* in, float* out, size_t n, cudaStream_t st){
    f64_to_f32_kernel<<<148 * 8, 256, 0, st>>>(in, out, n);
}
void launch_f32_to_f64(const float* in, double* out, size_t n, cudaStream_t st){
    f32_to_f64_kernel<<<148 * 8, 256, 0, st>>>(in, out, n);
}
}  // namespace aturan
