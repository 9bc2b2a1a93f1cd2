// pearl_noalloc.cu — one accepted step without any device allocation.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cudaTypedefs.h>

#include "pearl_host.hpp"

using namespace pearl_gpu;

// ============================================================ no-allocation entry point
// pearl_gpu_advance_noalloc runs the same persistent kernel as pearl_gpu_advance
// for callers that must not allocate device memory themselves or through this
// library: programs whose device memory belongs to another allocator (a
// framework's caching pool, a fixed per-process budget) and latency-critical
// loops that cannot afford cudaMalloc/cudaFree, which may synchronise the
// device.  The caller passes the state planes in device memory; every scratch
// buffer (the trial state, the implicit-solve vectors, the reduction partials
// and the control block) is carved from one fixed array compiled into this
// library, which each GPU that loads the library keeps until the process exits.
namespace {

constexpr long long kNoAllocMaxCells = 262144;  // 512 x 512 cells
constexpr int kNoAllocMaxBlocks = 4096;         // bound of the cooperative grid
constexpr int kNoAllocPlanes = 17;  // trial phi(3) c mu + K chi icpt diag x r z p0 p1 Ap wE wN
constexpr size_t kNoAllocCtlDoubles = (sizeof(Ctl) + 255) / 256 * 32;
constexpr size_t kNoAllocDoubles =
    kNoAllocPlanes * (size_t)kNoAllocMaxCells + (size_t)2 * kNoAllocMaxBlocks * kMaxRed + kNoAllocCtlDoubles;
constexpr int kNoAllocMaxDevices = 64;

std::mutex g_noalloc_mutex;
double* g_noalloc_device_ptr[kNoAllocMaxDevices] = {};
CUcontext g_noalloc_device_ctx[kNoAllocMaxDevices] = {};

}  // namespace

// 17 planes of 262144 doubles + partials + control block: about 36 MB per GPU.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

namespace {

// The CUDA context current on the calling thread (driver entry point, so the
// library links no driver stub); null when it cannot be queried.
CUcontext current_context() {
    static PFN_cuCtxGetCurrent_v4000 get = nullptr;
    if (!get) {
        cudaDriverEntryPointQueryResult q;
        void* fn = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return nullptr;
        get = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(fn);
    }
    CUcontext c = nullptr;
    return get(&c) == CUDA_SUCCESS ? c : nullptr;
}

// Device address of g_noalloc_scratch on the current device, looked up on the
// first call per device.  The host-side name is only a stand-in for the device
// symbol, so the address must come from cudaGetSymbolAddress with that device
// current.  The address belongs to the device's context: when that context
// is replaced (cudaDeviceReset, or another library resetting the primary
// context), the address is looked up again instead of reusing a dead one.
int noalloc_scratch(int device, double** out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (device < 0 || device >= kNoAllocMaxDevices) return PEARL_ERR_NO_DEVICE;
    const CUcontext cur = current_context();
    if (!g_noalloc_device_ptr[device] || cur != g_noalloc_device_ctx[device]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return PEARL_ERR_CUDA;
        g_noalloc_device_ptr[device] = static_cast<double*>(p);
        // cudaGetSymbolAddress made the device's context current if none was
        g_noalloc_device_ctx[device] = cur ? cur : current_context();
    }
    *out = g_noalloc_device_ptr[device];
    return PEARL_OK;
}

}  // namespace

extern "C" int pearl_gpu_advance_noalloc(const pearl_params* params, int nx, int ny, double* d_phi,
                                         double* d_carbon, double* d_mu, pearl_scalars* scalars,
                                         double stop_time, pearl_step_info* out, void* stream) {
    if (!params || !d_phi || !d_carbon || !d_mu || !scalars || nx < 3 || ny < 2 || !valid_params(params))
        return PEARL_ERR_INVALID_ARGUMENT;
    if ((long long)nx * ny > kNoAllocMaxCells) return PEARL_ERR_TOO_LARGE;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return PEARL_ERR_NO_DEVICE;
    double* scratch = nullptr;
    int rc = noalloc_scratch(device, &scratch);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // Parameters and buffer table on the stack; nothing is allocated.
    pearl_gpu_ctx ctx;
    ctx.device = device;
    ctx.nx = nx;
    ctx.ny = ny;
    ctx.pitch = nx;  // the caller's planes are dense rows of nx doubles
    ctx.params = *params;
    fill_dev_params(&ctx);
    const size_t pe = (size_t)nx * ny;
    DevBufs& B = ctx.B;
    for (int a = 0; a < 3; ++a) B.phi[0][a] = d_phi + (size_t)a * pe;
    B.c[0] = d_carbon;
    B.mu[0] = d_mu;
    double* q = scratch;
    for (int a = 0; a < 3; ++a, q += pe) B.phi[1][a] = q;
    B.c[1] = q; q += pe;
    B.mu[1] = q; q += pe;
    B.K = q; q += pe;
    B.chi = q; q += pe;
    B.icpt = q; q += pe;
    B.diag = q; q += pe;
    B.x = q; q += pe;
    B.r = q; q += pe;
    B.z = q; q += pe;
    B.p[0] = q; q += pe;
    B.p[1] = q; q += pe;
    B.Ap = q; q += pe;
    B.wE = q; q += pe;
    B.wN = q;
    B.part = scratch + kNoAllocPlanes * (size_t)kNoAllocMaxCells;
    B.ctl = reinterpret_cast<Ctl*>(B.part + (size_t)2 * kNoAllocMaxBlocks * kMaxRed);

    int sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, g8::pearl_kernel, tile_geometry(8).threads, 0) !=
            cudaSuccess ||
        per_sm < 1)
        return PEARL_ERR_CUDA;
    const int grid = std::max(1, std::min(std::min(per_sm * sms, ctx.P.ntiles), kNoAllocMaxBlocks));

    // The scratch keeps the previous call's contents: reset the control block
    // (status, barrier counter, cached energies) before the launch.
    Ctl h;
    std::memset(&h, 0, sizeof h);
    h.S = *scalars;
    h.cur = 0;
    h.energy_valid = 0;
    if (cudaMemcpyAsync(B.ctl, &h, sizeof h, cudaMemcpyHostToDevice, st) != cudaSuccess) return PEARL_ERR_CUDA;

    KArgs a{};
    a.P = ctx.P;
    a.B = B;
    a.mode = kModeRun;
    a.L.max_steps = 1;
    a.L.config_max_steps = 0x7fffffffffffffffLL;
    a.L.stop_time = stop_time;
    a.L.end_time = INFINITY;
    a.L.output_eps = 0;
    void* kargs[] = {&a};
    if (cudaLaunchCooperativeKernel((const void*)g8::pearl_kernel, dim3(grid), dim3(tile_geometry(8).threads), kargs, 0,
                                    st) !=
        cudaSuccess)
        return PEARL_ERR_CUDA;
    if (cudaMemcpyAsync(&h, B.ctl, sizeof h, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return PEARL_ERR_CUDA;
    if (h.status != PEARL_OK) return h.status;
    if (h.steps != 1) return PEARL_ERR_INVALID_ADVANCE_TIME;
    // The accepted state sits in the scratch set; copy it into the caller's planes.
    if (h.cur == 1) {
        if (cudaMemcpyAsync(d_phi, B.phi[1][0], 3 * pe * sizeof(double), cudaMemcpyDeviceToDevice, st) !=
                cudaSuccess ||
            cudaMemcpyAsync(d_carbon, B.c[1], pe * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(d_mu, B.mu[1], pe * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return PEARL_ERR_CUDA;
    }
    *scalars = h.S;
    if (out) *out = h.last;
    return PEARL_OK;
}
