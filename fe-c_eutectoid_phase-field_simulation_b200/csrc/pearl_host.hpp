// pearl_host.hpp — host-side context of one device-resident domain and the
// helpers the host files share (pearl_ctx.cu defines them).
#pragma once

#include <cuda_runtime.h>

#include <nvtx3/nvToolsExt.h>

#include <string>

#include "pearl_kernels.cuh"

// NVTX range for a host-side call (launches, transfers): named spans on a
// profiler timeline; inert when no tool is attached.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

struct pearl_gpu_ctx {
    CUtensorMap maps[pearl_gpu::kMapCount];
    int warps = 8;  // block shape of the context's kernels: 8 or 16 warps (pearl_gpu::tile_geometry)
    bool use_tma = false;     // tensor maps built and shared memory granted (batches reuse the maps)
    bool stage_tma = false;   // this context's launches stage through TMA (see the size rule at create)
    int device = 0;
    int nx = 0, ny = 0, pitch = 0;
    cudaStream_t stream = nullptr;
    pearl_params params{};
    pearl_gpu::DevParams P{};
    pearl_gpu::DevBufs B{};
    double* slab = nullptr;
    float* slab32 = nullptr;  // FP32 planes of the mixed solve (allocated on first use)
    pearl_gpu::Ctl* d_ctl = nullptr;
    pearl_gpu::Ctl* h_ctl = nullptr;  // pinned
    double* d_stage = nullptr;  // dense device staging of one host state (5 n doubles)
    size_t stage_elems = 0;
    int grid = 0;
    long long launches = 0;
    double last_ms = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int adj_grid = 0;  // cooperative grid of the adjoint kernel (0 until first use)
    double* adj_slab = nullptr;  // the adjoint's checkpoints, tape and planes, kept for later calls
    size_t adj_slab_elems = 0;
    pearl_step_info* d_hist = nullptr;  // per-step history ring (pearl_gpu_set_history)
    void* d_fill = nullptr;             // filling commands of pearl_gpu_fill (PEARL_FILL_MAX_OPS)
    long long hist_cap = 0, hist_count = 0;
    std::string error;
};

namespace pearl_gpu {

constexpr int kDefaultWarpsXLog2 = 0;

const char* why_text(int why);
int fail(pearl_gpu_ctx* ctx, int status, const std::string& msg);
int cuda_fail(pearl_gpu_ctx* ctx, cudaError_t e, const char* what);
bool valid_params(const pearl_params* p);
double host_psi(const pearl_params* p, int a, double mu);
// Tile of (32 << wx) x (2 warps >> wx) cells: 2^wx warps side by side in x.
void set_tile_shape(pearl_gpu_ctx* ctx, int wx_log2);
// The persistent step kernel of a block shape; solve32: the kernel with the
// mixed form's FP32 inner solve.
const void* step_kernel(int warps, bool solve32 = false);
// Gives the context the kernels of another block shape (tile counts and TMA
// boxes follow); its own launch grid is kept.
void set_geometry(pearl_gpu_ctx* ctx, int warps);
void fill_dev_params(pearl_gpu_ctx* ctx);
int pull_ctl(pearl_gpu_ctx* ctx);
int push_ctl(pearl_gpu_ctx* ctx);
// Launch the persistent kernel in args.mode; on return h_ctl holds the device
// control block.  Maps the device status to the reference's messages.
int launch(pearl_gpu_ctx* ctx, KArgs& args);
size_t plane_elems(const pearl_gpu_ctx* ctx);
bool build_tensor_maps(pearl_gpu_ctx* ctx);

}  // namespace pearl_gpu

#define PG_CUDA(ctx, call)                                  \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
    } while (0)
