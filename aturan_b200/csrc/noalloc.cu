// The buoyancy reference level for callers that cannot allocate device memory.
//
// Who cannot allocate: a host application that hands this library device buffers it owns and
// forbids any other allocation on the device -- a framework whose memory pool owns the whole GPU,
// or a solver plugin run under a fixed memory budget. Such a caller cannot create an aturan_ctx
// (which allocates the model state) but can still ask for this reduction on buffers it already
// holds.
//
// The reduction needs scratch memory for its per-block partial sums and the sin(theta) weights.
// Here that scratch is one file-scope __device__ array of fixed size, part of the library image:
// every GPU that loads the library holds STATIC_SCRATCH_DOUBLES doubles (288 KiB) until the
// process exits, whether or not the entry point is called. Its device address is fetched once per
// device with cudaGetSymbolAddress on the first call made on that device (with the device
// current); make that first call before any stream capture begins.
//
// The array is shared by all calls on a device and keeps the last call's contents. Each call
// overwrites every slot it reads before reading it (the weights by a kernel on the caller's stream,
// then the partial sums), so nothing has to start at zero; two calls whose kernels overlap on the
// GPU (different streams, no ordering between them) race on it and must not be issued.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <string>

#include "aturan_b200.h"
#include "common.cuh"
#include "rk4.cuh"

namespace aturan {
namespace {

constexpr int STATIC_NBLK = 32;                          // partial-sum blocks per level (as aturan_rk4_step)
constexpr int STATIC_MAX_IM = ATURAN_STATIC_MAX_IM;
constexpr int STATIC_MAX_JM = ATURAN_STATIC_MAX_JM;
constexpr size_t STATIC_SCRATCH_DOUBLES = (size_t)STATIC_MAX_JM + 2 * (size_t)STATIC_MAX_IM * STATIC_NBLK;

// [0, MAX_JM): sin(theta_j) weights; then part_sum[MAX_IM * NBLK], part_w[MAX_IM * NBLK]
__device__ __align__(256) double g_static_scratch[STATIC_SCRATCH_DOUBLES];

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mutex;
double* g_scratch_addr[MAX_DEVICES];                    // device address of g_static_scratch, per device

thread_local std::string g_err;

// sin(theta_j) into w[0..jm): one warp; lane 0 forms theta by the running sum of
// lib/Array_1D.cpp:50-60 (as aturan_ctx_create does on the host), then every lane takes sin of its
// share. CUDA's sin may round differently from the host's in the last bit.
__global__ void static_weights_kernel(double* w, int jm, double the0, double dthe){
    if(threadIdx.x == 0){
        double th = the0;
        for(int j = 0; j < jm; j++){ if(j > 0) th += dthe; w[j] = th; }
    }
    __syncwarp();
    for(int j = threadIdx.x; j < jm; j += 32) w[j] = sin(w[j]);
}

int fail(int code, const std::string& msg){
    g_err = msg;
    return code;
}

}  // namespace

const char* static_last_error(){ return g_err.c_str(); }

}  // namespace aturan

using namespace aturan;

extern "C" int aturan_buoy_ref_level_static(const aturan_params* p, const double* t, const double* p_stat,
                                            double* ref_out, void* stream){
    if(!p || !t || !p_stat || !ref_out) return fail(ATURAN_E_INVALID, "null argument");
    if(p->abi_version != ATURAN_ABI_VERSION) return fail(ATURAN_E_INVALID, "abi_version mismatch");
    if(p->im < 3 || p->jm < 3 || p->km < 3) return fail(ATURAN_E_INVALID, "grid too small");
    if(p->im > STATIC_MAX_IM || p->jm > STATIC_MAX_JM)
        return fail(ATURAN_E_INVALID, "grid exceeds the static scratch: im <= " + std::to_string(STATIC_MAX_IM) +
                    " and jm <= " + std::to_string(STATIC_MAX_JM) + " required (got im = " +
                    std::to_string(p->im) + ", jm = " + std::to_string(p->jm) + ")");
    // the reduction indexes a level's cells by a 32-bit int
    if((long long)p->jm * p->km > (long long)ATURAN_STATIC_MAX_LEVEL_CELLS)
        return fail(ATURAN_E_INVALID, "grid exceeds the static entry point's level size: jm * km <= " +
                    std::to_string((long long)ATURAN_STATIC_MAX_LEVEL_CELLS) + " required (got " +
                    std::to_string((long long)p->jm * p->km) + ")");
    int dev = 0;
    if(cudaGetDevice(&dev) != cudaSuccess){ cudaGetLastError(); return fail(ATURAN_E_CUDA, "no CUDA device"); }
    if(dev < 0 || dev >= MAX_DEVICES) return fail(ATURAN_E_CUDA, "device index out of range");
    double* scratch;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if(!g_scratch_addr[dev]){
            void* addr = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&addr, g_static_scratch);
            if(e != cudaSuccess){
                cudaGetLastError();
                return fail(ATURAN_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            }
            g_scratch_addr[dev] = reinterpret_cast<double*>(addr);
        }
        scratch = g_scratch_addr[dev];
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);

    // sin(theta_j) (RungeKutta_Uran_Turb.cpp:25) formed on the device into the static array, in
    // stream order before the reduction that reads it: no host buffer is involved
    static_weights_kernel<<<1, 32, 0, st>>>(scratch, p->jm, p->the0, p->dthe);

    Grid g;
    g.im = p->im; g.jm = p->jm; g.km = p->km; g.kp = p->km;   // the caller's contiguous [i][j][k]
    g.fstride = (size_t)g.im * g.jm * g.kp;
    HydroConst h{};
    h.g = p->g; h.rR = p->r_mix * p->R_mix; h.t_ref = p->t_ref;
    double* part_sum = scratch + STATIC_MAX_JM;
    double* part_w = part_sum + (size_t)STATIC_MAX_IM * STATIC_NBLK;
    buoy_partial_kernel<double><<<dim3(STATIC_NBLK, g.im), 256, 0, st>>>(g, t, p_stat, scratch, h, part_sum, part_w, STATIC_NBLK);
    buoy_finish_kernel<<<(g.im + 63) / 64, 64, 0, st>>>(g.im, STATIC_NBLK, part_sum, part_w, ref_out);
    const cudaError_t e = cudaGetLastError();
    if(e != cudaSuccess) return fail(ATURAN_E_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return ATURAN_OK;
}
