// pearl_kernels.cuh — launch arguments and kernel declarations shared by the
// device translation unit (pearl_fp64.cu: phases and kernels) and the host-side
// files (pearl_ctx.cu, pearl_batch.cu, pearl_adjoint_host.cu, pearl_noalloc.cu).
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>

#include "pearl_device.cuh"
#include "pearl_gpu.h"

namespace pearl_gpu {

enum Mode : int {
    kModeRun = 0,
    kModePropose = 1,
    kModeMix = 2,
    kModeDiffusion = 3,
    kModeEnergy = 4,
    kModeValid = 5,
    kModeSnapshot = 6,
    kModeMaybeShift = 7,
    kModeSmooth = 8,
    kModeMixSums = 9,
    kModeInitComposition = 10,
};

struct KArgs {
    CUtensorMap maps[kMapCount];  // 2-D TMA descriptors of the staged planes (valid when use_tma)
    int use_tma;
    DevParams P;
    DevBufs B;
    int mode;
    double dt;  // diagnostic modes
    pearl_run_limits L;
    double shift_trigger, shift_target, shift_c_gamma;
    int smooth_max_steps, smooth_min_steps;
    double smooth_energy_rtol, smooth_max_phase_change;
    double init_mu;
    // run-mode recording for the adjoint (all may be null): forced accepted-dt
    // sequence, log of accepted dt, and a tape slot per accepted step holding
    // the new state (phi x3, c, mu) and the diffusion solution u, tape_slot
    // doubles apart.
    const double* forced_dt;
    double* dt_log;
    double* tape;
    size_t tape_slot;
    // per-step history ring (null = off): step k of the launch goes to
    // hist[(hist_next + k) % hist_cap]
    pearl_step_info* hist;
    long long hist_cap, hist_next;
};

// One instance of a batch: its tensor maps, parameters and buffers.
struct alignas(64) BatchInstance {
    CUtensorMap maps[kMapCount];
    DevParams P;
    DevBufs B;  // B.ctl: the instance's control block; B.part: unused
};

struct BatchArgs {
    const BatchInstance* inst;
    const int* order;  // instance ids grouped by block group
    const int* first;  // group g owns order[first[g] .. first[g+1])
    const int* block_group;   // [grid] group of each block
    const int* group_block0;  // [groups + 1] group g owns blocks group_block0[g] .. group_block0[g+1]-1
    Ctl* group_ctl;           // [groups] barrier words and error status
    double* group_part;       // [grid][2][kMaxRed]: group g's slots start at block group_block0[g]
    int use_tma;
    pearl_run_limits L;
};

// Adjoint work planes and launch arguments (pearl_adjoint.cuh).
struct AdjBufs {
    double* bphi[3];  // adjoint of phi: of the step's output on entry, of its input on exit
    double* bc;       // adjoint of carbon
    double* bmu;      // adjoint of mu
    double *chi, *K, *ub, *lam, *r, *z, *p[2], *Ap, *diag;
    double* Fb[3];  // adjoint of the propose forces
    double* Ql[3];  // cell-local part of the phi adjoint
};

struct AdjArgs {
    DevParams P;
    DevBufs B;  // barrier words, status and reduction partials of the context
    AdjBufs J;
    int mode;            // 0: objective and adjoint seed; 1: one checkpoint segment backwards
    const double* ckpt;  // mode 1: state at the segment start (5 planes); mode 0: final state
    const double* tape;  // mode 1: slot j = state after step j of the segment + u_j
    size_t slot;         // doubles per tape slot
    const double* dts;   // accepted dt of the segment's steps
    int len;             // steps in the segment
    const double* target;  // mode 0: target alpha plane
    double obs_per_sigma;  // d obs / d sigma = 16/(pi^2 eps)
    double two_eps;        // d (2 eps sigma) / d sigma
    double* acc;           // [0] objective, [1..3] gradient (M, sigma, D_gamma), [4] adjoint CG iterations
};

// The kernels of each block shape (tile_geometry): g8 for 256-thread blocks,
// two per SM; g16 for 512-thread blocks, one per SM.
#define PEARL_DECLARE_KERNELS(WARPS, MIN_BLOCKS)                                                                \
    __global__ void __launch_bounds__(32 * (WARPS), MIN_BLOCKS) pearl_kernel(const __grid_constant__ KArgs args); \
    __global__ void __launch_bounds__(32 * (WARPS), MIN_BLOCKS)                                                 \
        pearl_kernel_mixed(const __grid_constant__ KArgs args);                                               \
    __global__ void __launch_bounds__(32 * (WARPS), MIN_BLOCKS)                                                 \
        pearl_batch_kernel(const __grid_constant__ BatchArgs args);                                           \
    __global__ void __launch_bounds__(32 * (WARPS), MIN_BLOCKS)                                                 \
        pearl_batch_kernel_mixed(const __grid_constant__ BatchArgs args);                                     \
    __global__ void __launch_bounds__(32 * (WARPS), MIN_BLOCKS)                                                 \
        pearl_adjoint_kernel(const __grid_constant__ AdjArgs args);                                           \
    __global__ void division_selftest_kernel(const double* a, const double* b, const double* rb, long long n,  \
                                             unsigned long long* mismatches, int use_exact);                  \
    __global__ void wait_limit_selftest_kernel(Ctl* ctl);
namespace g8 {
PEARL_DECLARE_KERNELS(8, 2)
}
namespace g16 {
PEARL_DECLARE_KERNELS(16, 1)
}
#undef PEARL_DECLARE_KERNELS
static_assert(tile_geometry(8).min_blocks == 2 && tile_geometry(16).min_blocks == 1, "kernel launch bounds");

}  // namespace pearl_gpu
