// The buoyancy reference level for callers that cannot allocate device memory.
//
// Who cannot allocate: a host application that hands this library device buffers it owns and
// forbids any other allocation on the device (a framework whose memory pool owns the whole GPU,
// a solver plugin with a fixed memory budget), and code that runs while a CUDA stream is being
// captured into a graph, where cudaMalloc is not permitted. Such a caller cannot create an
// aturan_ctx (which allocates the model state) but can still ask for this reduction on buffers it
// already holds.
//
// The reduction needs scratch memory for its per-block partial sums and the sin(theta) weights.
// Here that scratch is one file-scope __device__ array of fixed size, part of the library image:
// every GPU that loads the library holds STATIC_SCRATCH_DOUBLES doubles (288 KiB) until the
// process exits, whether or not the entry point is called. Its device address is fetched once per
// device with cudaGetSymbolAddress on the first call made on that device (with the device
// current); make that first call before any stream capture begins.
//
// The array is shared by all calls on a device and keeps the last call's contents. Each call
// overwrites every slot it reads before reading it, so nothing has to start at zero; two calls
// whose kernels overlap on the GPU (different streams, no ordering between them) race on it and
// must not be issued.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

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

    // sin(theta_j) on the host, as aturan_ctx_create builds it (the.z by the running sum of
    // lib/Array_1D.cpp:50-60, RungeKutta_Uran_Turb.cpp:25), copied into the static array.
    static thread_local std::vector<double> wsin;
    wsin.assign(p->jm, 0.0);
    double th = p->the0;
    for(int j = 0; j < p->jm; j++){ if(j > 0) th += p->dthe; wsin[j] = std::sin(th); }
    cudaError_t e = cudaMemcpyAsync(scratch, wsin.data(), sizeof(double) * p->jm, cudaMemcpyHostToDevice, st);
    if(e != cudaSuccess){ cudaGetLastError(); return fail(ATURAN_E_CUDA, std::string("weights: ") + cudaGetErrorString(e)); }

    Grid g;
    g.im = p->im; g.jm = p->jm; g.km = p->km; g.kp = p->km;   // the caller's contiguous [i][j][k]
    g.fstride = (size_t)g.im * g.jm * g.kp;
    HydroConst h{};
    h.g = p->g; h.rR = p->r_mix * p->R_mix; h.t_ref = p->t_ref;
    double* part_sum = scratch + STATIC_MAX_JM;
    double* part_w = part_sum + (size_t)STATIC_MAX_IM * STATIC_NBLK;
    buoy_partial_kernel<double><<<dim3(STATIC_NBLK, g.im), 256, 0, st>>>(g, t, p_stat, scratch, h, part_sum, part_w, STATIC_NBLK);
    buoy_finish_kernel<<<(g.im + 63) / 64, 64, 0, st>>>(g.im, STATIC_NBLK, part_sum, part_w, ref_out);
    e = cudaGetLastError();
    if(e != cudaSuccess) return fail(ATURAN_E_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return ATURAN_OK;
}
