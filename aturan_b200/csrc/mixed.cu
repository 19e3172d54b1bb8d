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

// Contiguous [im][jm][km] FP64 <-> padded [im][jm][kp] field of type T (the layout change and,
// for FP32 fields, the conversion in one pass): one thread per element of a row's first km.
template <typename T>
__global__ void pack_in_kernel(const double* in, T* out, int km, int kp, size_t rows){
    const size_t r = blockIdx.y + (size_t)blockIdx.z * gridDim.y;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if(r >= rows || k >= km) return;
    out[r * kp + k] = (T)in[r * km + k];
}
template <typename T>
__global__ void pack_out_kernel(const T* in, double* out, int km, int kp, size_t rows){
    const size_t r = blockIdx.y + (size_t)blockIdx.z * gridDim.y;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if(r >= rows || k >= km) return;
    out[r * km + k] = (double)in[r * kp + k];
}
static dim3 pack_grid(int km, size_t rows){
    const unsigned y = (unsigned)(rows < 65535 ? rows : 65535);
    return dim3((km + 127) / 128, y, (unsigned)((rows + y - 1) / y));
}
void launch_pack_in_f64(const double* in, double* out, int km, int kp, size_t rows, cudaStream_t st){
    pack_in_kernel<double><<<pack_grid(km, rows), 128, 0, st>>>(in, out, km, kp, rows);
}
void launch_pack_in_f32(const double* in, float* out, int km, int kp, size_t rows, cudaStream_t st){
    pack_in_kernel<float><<<pack_grid(km, rows), 128, 0, st>>>(in, out, km, kp, rows);
}
void launch_pack_out_f64(const double* in, double* out, int km, int kp, size_t rows, cudaStream_t st){
    pack_out_kernel<double><<<pack_grid(km, rows), 128, 0, st>>>(in, out, km, kp, rows);
}
void launch_pack_out_f32(const float* in, double* out, int km, int kp, size_t rows, cudaStream_t st){
    pack_out_kernel<float><<<pack_grid(km, rows), 128, 0, st>>>(in, out, km, kp, rows);
}

// The temperature pair (common.cuh): FP64 in, hi = (float)x and lo = (float)(x - hi) out, and back.
__global__ void pack_in_pair_kernel(const double* in, float* hi, float* lo, int km, int kp, size_t rows){
    const size_t r = blockIdx.y + (size_t)blockIdx.z * gridDim.y;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if(r >= rows || k >= km) return;
    t_st(hi, lo, r * kp + k, in[r * km + k]);
}
__global__ void pack_out_pair_kernel(const float* hi, const float* lo, double* out, int km, int kp, size_t rows){
    const size_t r = blockIdx.y + (size_t)blockIdx.z * gridDim.y;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if(r >= rows || k >= km) return;
    out[r * km + k] = t_ld(hi, lo, r * kp + k);
}
void launch_pack_in_pair(const double* in, float* hi, float* lo, int km, int kp, size_t rows, cudaStream_t st){
    pack_in_pair_kernel<<<pack_grid(km, rows), 128, 0, st>>>(in, hi, lo, km, kp, rows);
}
void launch_pack_out_pair(const float* hi, const float* lo, double* out, int km, int kp, size_t rows, cudaStream_t st){
    pack_out_pair_kernel<<<pack_grid(km, rows), 128, 0, st>>>(hi, lo, out, km, kp, rows);
}
__global__ void scale_copy_pair_kernel(const float* hi, const float* lo, float* ohi, float* olo, size_t n, double coeff){
    for(size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        t_st(ohi, olo, t, coeff * t_ld(hi, lo, t));
}
void launch_scale_copy_pair(const float* hi, const float* lo, float* ohi, float* olo, size_t n, double coeff, cudaStream_t st){
    scale_copy_pair_kernel<<<148 * 8, 256, 0, st>>>(hi, lo, ohi, olo, n, coeff);
}

void launch_f64_to_f32(const double* in, float* out, size_t n, cudaStream_t st){
    f64_to_f32_kernel<<<148 * 8, 256, 0, st>>>(in, out, n);
}
void launch_f32_to_f64(const float* in, double* out, size_t n, cudaStream_t st){
    f32_to_f64_kernel<<<148 * 8, 256, 0, st>>>(in, out, n);
}
}  // namespace aturan
