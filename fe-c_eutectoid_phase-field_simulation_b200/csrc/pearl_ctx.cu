// pearl_ctx.cu — host side of one device-resident domain: context creation,
// parameters, host transfers (the host's layout is reshaped on the device),
// launches of the persistent kernel and the single-domain C ABI of
// include/pearl_gpu.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "pearl_host.hpp"

using namespace pearl_gpu;

namespace pearl_gpu {

const char* why_text(int why) {
    switch (why) {
        case PEARL_WHY_PHASE_INCREMENT: return "phase increment";
        case PEARL_WHY_LINEAR_CLOSURE: return "linear/closure";
        case PEARL_WHY_BOUNDS: return "composition/phase bounds";
        case PEARL_WHY_MASS: return "mass conservation";
        case PEARL_WHY_ENERGY: return "free-energy increase";
        default: return "";
    }
}

int fail(pearl_gpu_ctx* ctx, int status, const std::string& msg) {
    if (ctx) ctx->error = msg;
    return status;
}

int cuda_fail(pearl_gpu_ctx* ctx, cudaError_t e, const char* what) {
    return fail(ctx, PEARL_ERR_CUDA, std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}


bool valid_params(const pearl_params* p) {
    for (int i = 0; i < 3; ++i) {
        // Parabola::validate (pearl_serial.cpp:76-79)
        if (!std::isfinite(p->A[i]) || !std::isfinite(p->B[i]) || !std::isfinite(p->C[i]) || !std::isfinite(p->D[i]) ||
            p->A[i] <= 0.0 || p->D[i] < 0.0)
            return false;
        if (!(p->tau[i] > 0) || !std::isfinite(p->tau[i])) return false;
    }
    // InterfaceParameters::validate / PhaseParameters::validate (:414-419, :522-529)
    if (!(p->epsilon > 0) || !(p->sigma > 0) || p->triple < 0 || !std::isfinite(p->epsilon) ||
        !std::isfinite(p->sigma) || !std::isfinite(p->triple))
        return false;
    if (!(p->Vm > 0) || !std::isfinite(p->Vm)) return false;
    if (!(p->dx > 0) || !(p->dy > 0) || !std::isfinite(p->dx + p->dy)) return false;
    if (p->cg_max < 0 || p->max_retries < 0) return false;
    return true;
}

double host_psi(const pearl_params* p, int a, double mu) {
    const double d = mu - p->B[a];
    return std::fma(-0.25 / p->A[a], d * d, p->C[a]);
}

// Tile of (32 << wx) x (2 warps >> wx) cells: 2^wx warps side by side in x.
void set_tile_shape(pearl_gpu_ctx* ctx, int wx_log2) {
    DevParams& P = ctx->P;
    P.warps_x_log2 = wx_log2;
    const int tile_w = 32 << wx_log2, tile_h = tile_geometry(ctx->warps).rows >> wx_log2;
    P.ntx = (ctx->nx + tile_w - 1) / tile_w;
    P.nty = (ctx->ny + tile_h - 1) / tile_h;
    P.ntiles = P.ntx * P.nty;
}

const void* step_kernel(int warps, bool solve32) {
    if (solve32) return warps == 16 ? (const void*)g16::pearl_kernel_mixed : (const void*)g8::pearl_kernel_mixed;
    return warps == 16 ? (const void*)g16::pearl_kernel : (const void*)g8::pearl_kernel;
}

void set_geometry(pearl_gpu_ctx* ctx, int warps) {
    if (ctx->warps == warps) return;
    ctx->warps = warps;
    set_tile_shape(ctx, ctx->P.warps_x_log2);
    if (ctx->use_tma && !build_tensor_maps(ctx)) ctx->use_tma = false;
}

void fill_dev_params(pearl_gpu_ctx* ctx) {
    const pearl_params* p = &ctx->params;
    DevParams& P = ctx->P;
    P.nx = ctx->nx;
    P.ny = ctx->ny;
    P.pitch = ctx->pitch;
    // Tile shape: warps side by side in x give longer contiguous row segments
    // (better DRAM locality); PEARL_GPU_TILE_WARPS_X = 1, 2, 4 or 8 overrides.
    int wx_log2 = kDefaultWarpsXLog2;
    if (const char* e = std::getenv("PEARL_GPU_TILE_WARPS_X")) {
        const int w = std::atoi(e);
        wx_log2 = w >= 8 ? 3 : w >= 4 ? 2 : w >= 2 ? 1 : 0;
    }
    set_tile_shape(ctx, wx_log2);
    P.dx = p->dx;
    P.dy = p->dy;
    P.dx2 = p->dx * p->dx;
    P.dy2 = p->dy * p->dy;
    P.Vm = p->Vm;
    P.eps = p->epsilon;
    const double pi = std::acos(-1.);
    P.obs = 16 * p->sigma / (pi * pi * p->epsilon);
    P.tr = p->triple / p->epsilon;
    P.two_eps_sigma = 2 * p->epsilon * p->sigma;
    P.eps_sigma = p->epsilon * p->sigma;
    double tmin = p->tau[0];
    for (int i = 0; i < 3; ++i) {
        P.tau[i] = p->tau[i];
        if (p->tau[i] < tmin) tmin = p->tau[i];
        P.A[i] = p->A[i];
        P.B[i] = p->B[i];
        P.C[i] = p->C[i];
        P.D[i] = p->D[i];
        P.chi_p[i] = 1.0 / (2.0 * p->A[i]);
        P.neg_q_A[i] = -0.25 / p->A[i];
        P.two_A[i] = 2.0 * p->A[i];
    }
    P.tau_min = tmin;
    P.mu_ref = p->mu_reference;
    // mixed-precision constants (P.mixed itself is set by pearl_gpu_set_precision)
    P.m_obs = (float)P.obs;
    P.m_tr = (float)P.tr;
    P.m_kx = (float)(P.two_eps_sigma / P.dx2);
    P.m_ky = (float)(P.two_eps_sigma / P.dy2);
    P.m_rVm = (float)(1.0 / p->Vm);
    for (int b = 0; b < 2; ++b) {
        const double mr = p->mu_reference;
        P.m_pa[b] = (float)(host_psi(p, b, mr) - host_psi(p, 2, mr));
        P.m_pb[b] = (float)(-(mr - p->B[b]) / (2.0 * p->A[b]) + (mr - p->B[2]) / (2.0 * p->A[2]));
        P.m_pc[b] = (float)(-0.25 / p->A[b] + 0.25 / p->A[2]);
    }
    for (int i = 0; i < 3; ++i) P.m_tau[i] = (float)p->tau[i];
    P.m_tau_min = (float)tmin;
    P.psi_t[0] = host_psi(p, 0, p->mu_reference) - host_psi(p, 2, p->mu_reference);
    P.psi_t[1] = host_psi(p, 1, p->mu_reference) - host_psi(p, 2, p->mu_reference);
    P.psi_t[2] = 0;
    P.dt_max = p->dt_max;
    P.dt_min = p->dt_min;
    P.max_phase_change = p->max_phase_change;
    P.cg_rtol = p->cg_rtol;
    P.cg_atol = p->cg_atol;
    P.closure_tol = p->closure_tol;
    P.energy_rtol = p->energy_rtol;
    P.energy_atol = p->energy_atol;
    const int gxgy = ctx->nx * ctx->ny;
    P.mass_scale = gxgy * p->dx * p->dy * 1e-6;
    P.energy_scale = p->sigma * std::max(ctx->nx * p->dx, ctx->ny * p->dy);
    P.cg_max = p->cg_max;
    P.max_retries = p->max_retries;
    P.check_energy = p->check_energy;
    P.phase_only = p->phase_only;
    // reciprocals of the constant divisors (RN(1/b), host IEEE division)
    P.r_Vm = 1.0 / P.Vm;
    P.r_dx = 1.0 / P.dx;
    P.r_dy = 1.0 / P.dy;
    P.r_dx2 = 1.0 / P.dx2;
    P.r_dy2 = 1.0 / P.dy2;
    P.r_3 = 1.0 / 3.0;
    for (int i = 0; i < 3; ++i) P.r_two_A[i] = 1.0 / P.two_A[i];
    const double divisors[] = {P.Vm, P.dx, P.dy, P.dx2, P.dy2, 3.0, P.two_A[0], P.two_A[1], P.two_A[2]};
    const double recips[] = {P.r_Vm, P.r_dx, P.r_dy, P.r_dx2, P.r_dy2, P.r_3, P.r_two_A[0], P.r_two_A[1], P.r_two_A[2]};
    P.exact_div = 1;
    for (int i = 0; i < 9; ++i)
        if (std::fpclassify(divisors[i]) != FP_NORMAL || std::fpclassify(recips[i]) != FP_NORMAL) P.exact_div = 0;
}

int pull_ctl(pearl_gpu_ctx* ctx) {
    PG_CUDA(ctx, cudaMemcpyAsync(ctx->h_ctl, ctx->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, ctx->stream));
    PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return PEARL_OK;
}

int push_ctl(pearl_gpu_ctx* ctx) {
    PG_CUDA(ctx, cudaMemcpyAsync(ctx->d_ctl, ctx->h_ctl, sizeof(Ctl), cudaMemcpyHostToDevice, ctx->stream));
    return PEARL_OK;
}

// Launch the persistent kernel in `mode`; on return h_ctl holds the device
// control block.  Maps the device status to the reference's messages.
int launch(pearl_gpu_ctx* ctx, KArgs& args) {
    static const char* const kNames[] = {"pearl_gpu run",       "pearl_gpu propose",  "pearl_gpu mixture",
                                         "pearl_gpu diffusion", "pearl_gpu energy",   "pearl_gpu valid_state",
                                         "pearl_gpu snapshot",  "pearl_gpu shift",    "pearl_gpu smooth",
                                         "pearl_gpu mixture sums", "pearl_gpu init composition"};
    const NvtxRange range(args.mode >= 0 && args.mode <= kModeInitComposition ? kNames[args.mode] : "pearl_gpu");
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    ctx->h_ctl->status = 0;
    ctx->h_ctl->why = 0;
    ctx->h_ctl->bar_count = 0;
    int rc = push_ctl(ctx);
    if (rc) return rc;
    args.P = ctx->P;
    args.B = ctx->B;
    void* kargs[] = {&args};
    PG_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    const bool tma = ctx->use_tma && ctx->stage_tma;
    args.use_tma = tma ? 1 : 0;
    if (tma) std::memcpy(args.maps, ctx->maps, sizeof ctx->maps);
    const TileGeometry g = tile_geometry(ctx->warps);
    // the mixed-solve kernel holds only the run mode
    const bool solve32 = ctx->P.mixed_cg != 0 && args.mode == kModeRun;
    PG_CUDA(ctx, cudaLaunchCooperativeKernel(step_kernel(ctx->warps, solve32), dim3(ctx->grid),
                                             dim3(g.threads), kargs,
                                             tma ? g.tma_smem_bytes : 0, ctx->stream));
    ctx->launches++;
    PG_CUDA(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
    rc = pull_ctl(ctx);
    if (rc) return rc;
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    ctx->last_ms = ms;
    const int st = ctx->h_ctl->status;
    if (st == PEARL_OK) return PEARL_OK;
    ctx->h_ctl->energy_valid = 0;
    switch (st) {
        case PEARL_ERR_INVALID_ADVANCE_TIME: return fail(ctx, st, "invalid advance time");
        case PEARL_ERR_REJECTED_BELOW_DT_MIN:
            return fail(ctx, st, std::string("step rejected below dt_min: ") + why_text(ctx->h_ctl->why));
        case PEARL_ERR_RETRY_LIMIT: return fail(ctx, st, std::string("step retry limit: ") + why_text(ctx->h_ctl->why));
        case PEARL_ERR_MIXTURE: return fail(ctx, st, "Invalid mixture coefficients");
        case PEARL_ERR_SIMPLEX: return fail(ctx, st, "Simplex projection failed");
        case PEARL_ERR_MAX_STEPS: return fail(ctx, st, "configured max_steps reached before end_time");
        case PEARL_ERR_UNSAFE_SHIFT: return fail(ctx, st, "unsafe shift: removed strip contains gamma");
        case PEARL_ERR_NONFINITE_CARBON: return fail(ctx, st, "Nonfinite total carbon");
        case PEARL_ERR_SMOOTHING:
            return fail(ctx, st, ctx->h_ctl->why == 1 ? "nonfinite smoothing force"
                                                      : "sharp smoothing could not find an energy-decreasing step");
        case PEARL_ERR_DEVICE_WAIT:
            // a grid barrier gave up waiting: reset the barrier words before any further launch
            ctx->h_ctl->bar_count = 0;
            push_ctl(ctx);
            return fail(ctx, st, "device grid barrier wait exceeded its limit");
        default: return fail(ctx, st, "invalid argument");
    }
}

size_t plane_elems(const pearl_gpu_ctx* ctx) { return (size_t)ctx->pitch * ctx->ny; }

// 2-D TMA descriptors for the planes the stencil phases stage through shared
// memory: box (kBoxW x box_h of the context's block shape) float64, dims (nx, ny), row stride pitch*8 bytes,
// zero fill outside.  Returns false when the driver cannot encode them; the
// kernels then read the planes directly.
bool build_tensor_maps(pearl_gpu_ctx* ctx) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        cudaDriverEntryPointQueryResult q;
        void* fn = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return false;
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    const DevBufs& B = ctx->B;
    double* planes[kMapCount] = {};
    for (int s = 0; s < 2; ++s) {
        for (int a = 0; a < 3; ++a) planes[kMapState + 5 * s + a] = B.phi[s][a];
        planes[kMapState + 5 * s + 3] = B.c[s];
        planes[kMapState + 5 * s + 4] = B.mu[s];
    }
    planes[kMapK] = B.K;
    planes[kMapChi] = B.chi;
    planes[kMapIcpt] = B.icpt;
    planes[kMapX] = B.x;
    planes[kMapZ] = B.z;
    planes[kMapP0] = B.p[0];
    planes[kMapP1] = B.p[1];
    planes[kMapWE] = B.wE;
    planes[kMapWN] = B.wN;
    planes[kMapR] = B.r;
    planes[kMapAp] = B.Ap;
    planes[kMapDiag] = B.diag;
    planes[kMapXc] = B.x;
    planes[kMapP0c] = B.p[0];
    planes[kMapP1c] = B.p[1];
    planes[kMapRc] = B.r;
    planes[kMapApc] = B.Ap;
    planes[kMapDiagc] = B.diag;
    for (int m = 0; m < kMap32WE; ++m) {
        const cuuint64_t dims[2] = {(cuuint64_t)ctx->nx, (cuuint64_t)ctx->ny};
        const cuuint64_t strides[1] = {(cuuint64_t)ctx->pitch * sizeof(double)};
        const bool tile_only = m >= kMapXc;
        const TileGeometry g = tile_geometry(ctx->warps);
        const cuuint32_t box[2] = {(cuuint32_t)(tile_only ? kTileX : kBoxW), (cuuint32_t)(tile_only ? g.rows : g.box_h)};
        const cuuint32_t estr[2] = {1, 1};
        // 128-byte L2 promotion: with 256-byte promotion the last box of a ragged
        // row also pulls the row's padding from HBM (a 256-instance sweep of
        // widths 32..192 ran 0.6 % slower; the 2048x4096 step is the same either way)
        if (encode(&ctx->maps[m], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, planes[m], dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    }
    // FP32 planes of the mixed solve, once pearl_gpu_set_precision has made them
    if (B.wE32) {
        float* planes32[6] = {B.wE32, B.wN32, B.z32, B.chi32, B.p32[0], B.p32[1]};
        const TileGeometry g = tile_geometry(ctx->warps);
        for (int m = kMap32WE; m < kMapCount; ++m) {
            const cuuint64_t dims[2] = {(cuuint64_t)ctx->nx, (cuuint64_t)ctx->ny};
            const cuuint64_t strides[1] = {(cuuint64_t)ctx->pitch * sizeof(float)};
            const cuuint32_t box[2] = {(cuuint32_t)kBoxW32, (cuuint32_t)g.box_h};
            const cuuint32_t estr[2] = {1, 1};
            if (encode(&ctx->maps[m], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, planes32[m - kMap32WE], dims, strides, box,
                       estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                       CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
                return false;
        }
    }
    return true;
}

int ensure_stage(pearl_gpu_ctx* ctx) {
    if (!ctx->d_stage) PG_CUDA(ctx, cudaMalloc(&ctx->d_stage, ctx->stage_elems * sizeof(double)));
    return PEARL_OK;
}

// Host fields in the reference's gathered layout (phi (y,x,a) interleaved,
// carbon and mu dense) travel as they are into a dense device staging buffer
// [phi 3n | carbon n | mu n]; these kernels move them to and from the padded
// SoA planes of one state set, so the host does no per-element work.
__global__ void unpack_state_kernel(const double* __restrict__ st, long long n, int nx, int pitch,
                                    double* p0, double* p1, double* p2, double* c, double* mu) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long y = i / nx, x = i - y * nx;
        const size_t d = (size_t)y * pitch + x;
        if (p0) {
            p0[d] = st[3 * i];
            p1[d] = st[3 * i + 1];
            p2[d] = st[3 * i + 2];
        }
        if (c) c[d] = st[3 * n + i];
        if (mu) mu[d] = st[4 * n + i];
    }
}

__global__ void pack_state_kernel(double* __restrict__ st, long long n, int nx, int pitch, const double* p0,
                                  const double* p1, const double* p2, const double* c, const double* mu) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long y = i / nx, x = i - y * nx;
        const size_t d = (size_t)y * pitch + x;
        if (p0) {
            st[3 * i] = p0[d];
            st[3 * i + 1] = p1[d];
            st[3 * i + 2] = p2[d];
        }
        if (c) st[3 * n + i] = c[d];
        if (mu) st[4 * n + i] = mu[d];
    }
}

int stage_grid(const pearl_gpu_ctx* ctx) {
    const long long n = (long long)ctx->nx * ctx->ny;
    return (int)std::max(1LL, std::min<long long>((n + 255) / 256, 148LL * 16));
}

int upload_set(pearl_gpu_ctx* ctx, int set, const double* phi, const double* carbon, const double* mu) {
    const NvtxRange range("pearl_gpu upload");
    if (int rc = ensure_stage(ctx)) return rc;
    const size_t n = (size_t)ctx->nx * ctx->ny;
    double* st = ctx->d_stage;
    if (phi) PG_CUDA(ctx, cudaMemcpyAsync(st, phi, 3 * n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    if (carbon)
        PG_CUDA(ctx, cudaMemcpyAsync(st + 3 * n, carbon, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    if (mu) PG_CUDA(ctx, cudaMemcpyAsync(st + 4 * n, mu, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    unpack_state_kernel<<<stage_grid(ctx), 256, 0, ctx->stream>>>(
        st, (long long)n, ctx->nx, ctx->pitch, phi ? ctx->B.phi[set][0] : nullptr, ctx->B.phi[set][1],
        ctx->B.phi[set][2], carbon ? ctx->B.c[set] : nullptr, mu ? ctx->B.mu[set] : nullptr);
    ctx->launches++;
    PG_CUDA(ctx, cudaGetLastError());
    PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return PEARL_OK;
}

int download_set(pearl_gpu_ctx* ctx, int set, double* phi, double* carbon, double* mu) {
    const NvtxRange range("pearl_gpu download");
    if (int rc = ensure_stage(ctx)) return rc;
    const size_t n = (size_t)ctx->nx * ctx->ny;
    double* st = ctx->d_stage;
    pack_state_kernel<<<stage_grid(ctx), 256, 0, ctx->stream>>>(
        st, (long long)n, ctx->nx, ctx->pitch, phi ? ctx->B.phi[set][0] : nullptr, ctx->B.phi[set][1],
        ctx->B.phi[set][2], carbon ? ctx->B.c[set] : nullptr, mu ? ctx->B.mu[set] : nullptr);
    ctx->launches++;
    PG_CUDA(ctx, cudaGetLastError());
    if (phi) PG_CUDA(ctx, cudaMemcpyAsync(phi, st, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (carbon)
        PG_CUDA(ctx, cudaMemcpyAsync(carbon, st + 3 * n, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (mu) PG_CUDA(ctx, cudaMemcpyAsync(mu, st + 4 * n, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return PEARL_OK;
}

}  // namespace pearl_gpu

// ------------------------------------------------------------------ filling commands
// One filling command on the device: its parameters plus the cosine and sine
// of its angles, taken on the host with the reference's expressions
// (angle*pi/180, std::cos, std::sin), so every cell sees the same directions
// as the reference.
struct DevFillOp {
    int method;
    double p[PEARL_FILL_MAX_PARAMS];
    double ux[3], uy[3];
};

// filling_centered_lamellar_phase (pearl_serial.cpp:1378-1388)
__device__ __forceinline__ int fill_centered_lamellar(double along, double period, double fraction, int ferrite,
                                                      int cementite) {
    double pos = fmod(along, period);
    if (pos < 0.0) pos += period;
    const double width = fraction * period;
    const double start = 0.5 * (period - width), end = 0.5 * (period + width);
    return pos >= start && pos < end ? cementite : ferrite;
}

// filling_phase_at (pearl_serial.cpp:1393-1514) of cell (gx, gy): the label of
// the last command that paints the cell, gamma (2) where none does.  Every
// comparison and product follows the reference's expressions and order.
__device__ int fill_label(const DevFillOp* ops, int nops, int gx, int gy) {
    const double pi = 3.14159265358979323846;
    int label = 2;
    for (int k = 0; k < nops; ++k) {
        const DevFillOp& o = ops[k];
        const double* p = o.p;
        if (o.method == PEARL_FILL_CUBE) {
            const int sel = (int)p[0];
            if (sel != 2 && gx >= p[1] && gx <= p[4] && gy >= p[2] && gy <= p[5]) label = sel;
        } else if (o.method == PEARL_FILL_CYLINDER) {
            const double dx = gx - p[1], dy = gy - p[2];
            const int sel = (int)p[0];
            if (sel != 2 && dx * dx + dy * dy <= p[5] * p[5]) label = sel;
        } else if (o.method == PEARL_FILL_CENTER_BOX_2D) {
            const bool inside = gx >= p[0] && gx < p[1] && gy >= p[2] && gy < p[3];
            label = (int)(inside ? p[4] : p[5]);
        } else if (o.method == PEARL_FILL_Y_JUNCTION_2D || o.method == PEARL_FILL_Y_JUNCTION_LAMELLAE_2D) {
            const bool lam = o.method == PEARL_FILL_Y_JUNCTION_LAMELLAE_2D;
            const int ferrite = (int)p[lam ? 13 : 11];
            label = (int)p[lam ? 15 : 12];
            if (!(gx >= p[0] && gx < p[1] && gy >= p[2] && gy < p[3])) continue;
            const double dx = gx - p[4], dy = gy - p[5];
            for (int arm = 0; arm < 3; ++arm) {
                const double along = dx * o.ux[arm] + dy * o.uy[arm];
                const double across = -dx * o.uy[arm] + dy * o.ux[arm];
                if (along >= 0.0 && along <= p[9] && fabs(across) <= p[10]) {
                    int sel = ferrite;
                    if (lam) {
                        const double period = p[11] + p[12];
                        double pos = fmod(along, period);
                        if (pos < 0.0) pos += period;
                        if (!(pos < p[11])) sel = (int)p[14];
                    }
                    label = sel;
                    break;  // the first arm that contains the cell wins
                }
            }
        } else if (o.method == PEARL_FILL_ADHERED_PEARLITE_ARM_2D) {
            const double dx = gx - p[0], dy = gy - p[1];
            const double along = dx * o.ux[0] + dy * o.uy[0];
            const double across = -dx * o.uy[0] + dy * o.ux[0];
            const double arm_length = p[3];
            const int pairs = (int)p[4];
            const double period = arm_length / (double)pairs;
            const double ferrite_width = (1.0 - p[5]) * period, cementite_width = p[5] * period;
            const double peak = p[6], contact = p[7], bridge = p[8];
            const int ferrite = (int)p[9], cementite = (int)p[10];
            int sel = -1;
            if (along >= 0.0 && along <= arm_length) {
                int pair = along >= arm_length ? pairs - 1 : (int)floor(along / period);
                pair = max(0, min(pairs - 1, pair));
                const double pair_start = (double)pair * period;
                const double local = along - pair_start;
                int segment;
                double seg_start, seg_len;
                if (local < ferrite_width) {
                    segment = 2 * pair;
                    seg_start = pair_start;
                    seg_len = ferrite_width;
                    sel = ferrite;
                } else {
                    segment = 2 * pair + 1;
                    seg_start = pair_start + ferrite_width;
                    seg_len = cementite_width;
                    sel = cementite;
                }
                double frac = (along - seg_start) / seg_len;
                if (frac < 0.0)
                    frac = 0.0;
                else if (frac > 1.0)
                    frac = 1.0;
                const double h0 = segment == 0 ? 0.0 : contact;
                const double h1 = segment == 2 * pairs - 1 ? 0.0 : contact;
                const double mean_end = 0.5 * (h0 + h1);
                double half = (1.0 - frac) * h0 + frac * h1 + (peak - mean_end) * sin(pi * frac);
                if (half > peak) half = peak;
                if (fabs(across) > half) sel = -1;
            }
            if (bridge > 0.0) {
                const double r2 = bridge * bridge;
                const double d_start = along * along + across * across;
                const double d_end = (along - arm_length) * (along - arm_length) + across * across;
                if (d_start <= r2) sel = ferrite;
                if (d_end <= r2) sel = cementite;
            }
            if (sel >= 0) label = sel;
        } else if (o.method == PEARL_FILL_PEARLITE_ELLIPSE_2D) {
            const double dx = gx - p[0], dy = gy - p[1];
            const double along = dx * o.ux[0] + dy * o.uy[0];
            const double across = -dx * o.uy[0] + dy * o.ux[0];
            const double start = p[3], period = p[5], length = p[4] * period;
            const double semi_major = 0.5 * length, semi_minor = p[6] * semi_major;
            const double centre = start + semi_major;
            const double na = (along - centre) / semi_major;
            const double nc = across / semi_minor;
            const double bridge = p[8];
            const int ferrite = (int)p[9], cementite = (int)p[10];
            int sel = -1;
            if (na * na + nc * nc <= 1.0) sel = fill_centered_lamellar(along - start, period, p[7], ferrite, cementite);
            if (bridge > 0.0) {
                const double ds = (along - start) * (along - start) + across * across;
                const double de = (along - (start + length)) * (along - (start + length)) + across * across;
                if (ds <= bridge * bridge || de <= bridge * bridge) sel = ferrite;
            }
            if (sel >= 0) label = sel;
        }
    }
    return label;
}

// One-hot phase fractions of every cell's label into the padded planes.
__global__ void fill_kernel(const DevFillOp* ops, int nops, int nx, int ny, int pitch, double* pa, double* pt,
                            double* pg) {
    const long long n = (long long)nx * ny;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx), y = (int)(i / nx);
        const int label = fill_label(ops, nops, x, y);
        const size_t j = (size_t)y * pitch + x;
        pa[j] = label == 0 ? 1.0 : 0.0;
        pt[j] = label == 1 ? 1.0 : 0.0;
        pg[j] = label == 2 ? 1.0 : 0.0;
    }
}

// FP64 throughput probe: eight independent FMA chains per thread, so the FP64
// pipe, not the dependency latency, bounds the loop.
__global__ void fp64_fma_chains_kernel(double* out, int iters, double a, double b) {
    double x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6,
           x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
        x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
        x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}

extern "C" {

const char* pearl_gpu_status_string(int status) {
    switch (status) {
        case PEARL_OK: return "ok";
        case PEARL_ERR_INVALID_ARGUMENT: return "invalid argument";
        case PEARL_ERR_CUDA: return "CUDA error";
        case PEARL_ERR_INVALID_ADVANCE_TIME: return "invalid advance time";
        case PEARL_ERR_REJECTED_BELOW_DT_MIN: return "step rejected below dt_min";
        case PEARL_ERR_RETRY_LIMIT: return "step retry limit";
        case PEARL_ERR_MIXTURE: return "Invalid mixture coefficients";
        case PEARL_ERR_SIMPLEX: return "Simplex projection failed";
        case PEARL_ERR_MAX_STEPS: return "configured max_steps reached before end_time";
        case PEARL_ERR_DEVICE_WAIT: return "device wait limit exceeded";
        case PEARL_ERR_UNSAFE_SHIFT: return "unsafe shift: removed strip contains gamma";
        case PEARL_ERR_NONFINITE_CARBON: return "Nonfinite total carbon";
        case PEARL_ERR_NO_DEVICE: return "no CUDA device";
        case PEARL_ERR_TOO_LARGE: return "domain exceeds the no-allocation scratch limit of 262144 cells";
        case PEARL_ERR_SMOOTHING: return "sharp smoothing failed";
        default: return "unknown status";
    }
}

const char* pearl_gpu_last_error(const pearl_gpu_ctx* ctx) { return ctx ? ctx->error.c_str() : "null context"; }

int pearl_gpu_create(const pearl_params* params, int nx, int ny, int device, pearl_gpu_ctx** out) {
    if (!out) return PEARL_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (!params || nx < 3 || ny < 2 || !valid_params(params)) return PEARL_ERR_INVALID_ARGUMENT;
    if ((long long)nx * ny > 2000000000LL) return PEARL_ERR_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0) return PEARL_ERR_NO_DEVICE;
    pearl_gpu_ctx* ctx = new pearl_gpu_ctx();
    ctx->device = device;
    ctx->nx = nx;
    ctx->ny = ny;
    ctx->pitch = (nx + 31) / 32 * 32;
    ctx->params = *params;
    auto bail = [&](int rc) {
        pearl_gpu_destroy(ctx);
        return rc;
    };
    if (cudaSetDevice(device) != cudaSuccess) return bail(PEARL_ERR_CUDA);
    int coop = 0, sms = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (!coop) return bail(PEARL_ERR_NO_DEVICE);
    // Block shape: 16 warps (512 threads, one block per SM, 32x32 tiles) when the
    // domain gives every SM at least four such tiles, 8 warps (two 256-thread
    // blocks per SM, 32x16 tiles) for smaller domains, which need the finer
    // split; PEARL_GPU_TILE_WARPS = 8 or 16 overrides.
    {
        const long long tiles16 = (long long)((nx + 31) / 32) * ((ny + 31) / 32);
        ctx->warps = tiles16 >= 4LL * sms ? 16 : 8;
        if (const char* e = std::getenv("PEARL_GPU_TILE_WARPS")) ctx->warps = std::atoi(e) == 16 ? 16 : 8;
    }
    fill_dev_params(ctx);
    // TMA staging of the stencil phases needs the 32x16 tile; PEARL_GPU_TMA=0 turns it off.
    const char* tma_env = std::getenv("PEARL_GPU_TMA");
    ctx->use_tma = ctx->P.warps_x_log2 == 0 && !(tma_env && std::atoi(tma_env) == 0);
    const TileGeometry geom = tile_geometry(ctx->warps);
    // both the FP64 kernel and the mixed-solve kernel of the block shape get the
    // stage buffers; the grid fits the residency of both
    for (bool solve32 : {false, true})
        if (ctx->use_tma && cudaFuncSetAttribute(step_kernel(ctx->warps, solve32),
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)geom.tma_smem_bytes) != cudaSuccess)
            ctx->use_tma = false;
    int per_sm = 1 << 30;
    for (bool solve32 : {false, true}) {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, step_kernel(ctx->warps, solve32), geom.threads,
                                                          ctx->use_tma ? geom.tma_smem_bytes : 0) != cudaSuccess ||
            n < 1)
            return bail(PEARL_ERR_CUDA);
        per_sm = std::min(per_sm, n);
    }
    ctx->grid = std::max(1, std::min(per_sm * sms, ctx->P.ntiles));
    // PEARL_GPU_GRID caps the block count (the grid-size sweeps of small domains)
    if (const char* e = std::getenv("PEARL_GPU_GRID"))
        if (std::atoi(e) > 0) ctx->grid = std::min(ctx->grid, std::atoi(e));
    // TMA staging pays once a block has a few tiles per pass to pipeline; with
    // fewer, the pipeline's fill and proxy fences cost more than plain loads
    // (1965 MHz, one GPU: 768x1024, 5.2 tiles a block, 0.258 staged against
    // 0.234 ms/step plain; 1024x1024, 6.9 tiles, 0.300 against 0.304;
    // 1024x2048, 13.8 tiles, 0.497 against 0.601; 256x512 0.0947 against
    // 0.0733).  PEARL_GPU_TMA=1 stages whatever the size, =0 never.
    ctx->stage_tma = ctx->use_tma && ((tma_env && std::atoi(tma_env) != 0) || ctx->P.ntiles >= 6LL * ctx->grid);
    // state: 2 x (3 phi + c + mu); work: K chi icpt diag x r z p0 p1 Ap  -> 20 planes
    const size_t pe = plane_elems(ctx);
    const int nplanes = 22;
    const size_t part = (size_t)2 * ctx->grid * kMaxRed;
    if (cudaMalloc(&ctx->slab, (nplanes * pe + part) * sizeof(double)) != cudaSuccess) return bail(PEARL_ERR_CUDA);
    if (cudaMemset(ctx->slab, 0, (nplanes * pe + part) * sizeof(double)) != cudaSuccess) return bail(PEARL_ERR_CUDA);
    double* q = ctx->slab;
    for (int s = 0; s < 2; ++s) {
        for (int a = 0; a < 3; ++a, q += pe) ctx->B.phi[s][a] = q;
        ctx->B.c[s] = q;
        q += pe;
        ctx->B.mu[s] = q;
        q += pe;
    }
    ctx->B.K = q; q += pe;
    ctx->B.chi = q; q += pe;
    ctx->B.icpt = q; q += pe;
    ctx->B.diag = q; q += pe;
    ctx->B.x = q; q += pe;
    ctx->B.r = q; q += pe;
    ctx->B.z = q; q += pe;
    ctx->B.p[0] = q; q += pe;
    ctx->B.p[1] = q; q += pe;
    ctx->B.Ap = q; q += pe;
    ctx->B.wE = q; q += pe;
    ctx->B.wN = q; q += pe;
    ctx->B.part = q;
    if (cudaMalloc(&ctx->d_ctl, sizeof(Ctl)) != cudaSuccess) return bail(PEARL_ERR_CUDA);
    if (cudaMallocHost(&ctx->h_ctl, sizeof(Ctl)) != cudaSuccess) return bail(PEARL_ERR_CUDA);
    std::memset(ctx->h_ctl, 0, sizeof(Ctl));
    ctx->B.ctl = ctx->d_ctl;
    if (ctx->use_tma && !build_tensor_maps(ctx)) ctx->use_tma = false;
    ctx->stage_elems = 5 * (size_t)nx * ny;  // device staging is allocated at the first host transfer
    if (cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess)
        return bail(PEARL_ERR_CUDA);
    if (cudaMemcpy(ctx->d_ctl, ctx->h_ctl, sizeof(Ctl), cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(PEARL_ERR_CUDA);
    *out = ctx;
    return PEARL_OK;
}

void pearl_gpu_destroy(pearl_gpu_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->slab) cudaFree(ctx->slab);
    if (ctx->d_ctl) cudaFree(ctx->d_ctl);
    if (ctx->h_ctl) cudaFreeHost(ctx->h_ctl);
    if (ctx->d_stage) cudaFree(ctx->d_stage);
    if (ctx->d_fill) cudaFree(ctx->d_fill);
    if (ctx->slab32) cudaFree(ctx->slab32);
    if (ctx->adj_slab) cudaFree(ctx->adj_slab);
    if (ctx->d_hist) cudaFree(ctx->d_hist);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    delete ctx;
}

int pearl_gpu_set_stream(pearl_gpu_ctx* ctx, void* stream) {
    if (!ctx) return PEARL_ERR_INVALID_ARGUMENT;
    ctx->stream = (cudaStream_t)stream;
    return PEARL_OK;
}

int pearl_gpu_set_precision(pearl_gpu_ctx* ctx, int precision) {
    if (!ctx) return PEARL_ERR_INVALID_ARGUMENT;
    if (precision < PEARL_PRECISION_FP64 || precision > PEARL_PRECISION_MIXED_SOLVE)
        return fail(ctx, PEARL_ERR_INVALID_ARGUMENT, "invalid precision");
    const bool solve32 = precision == PEARL_PRECISION_MIXED || precision == PEARL_PRECISION_MIXED_SOLVE;
    if (solve32 && !ctx->slab32) {
        // FP32 planes of the inner solve: wE wN chi diag r z p0 p1 Ap
        PG_CUDA(ctx, cudaSetDevice(ctx->device));
        const size_t pe = plane_elems(ctx);
        PG_CUDA(ctx, cudaMalloc(&ctx->slab32, 9 * pe * sizeof(float)));
        PG_CUDA(ctx, cudaMemset(ctx->slab32, 0, 9 * pe * sizeof(float)));
        float* q = ctx->slab32;
        float** planes[9] = {&ctx->B.wE32, &ctx->B.wN32, &ctx->B.chi32, &ctx->B.diag32, &ctx->B.r32,
                             &ctx->B.z32,  &ctx->B.p32[0], &ctx->B.p32[1], &ctx->B.Ap32};
        for (float** pl : planes) {
            *pl = q;
            q += pe;
        }
        // APPLY32 stages its FP32 planes through TMA like the FP64 passes
        if (ctx->use_tma && !build_tensor_maps(ctx)) ctx->use_tma = false;
    }
    ctx->P.mixed = precision == PEARL_PRECISION_MIXED || precision == PEARL_PRECISION_MIXED_PROPOSE;
    ctx->P.mixed_cg = solve32 ? 1 : 0;
    // an FP32 round stops once its residual has fallen by this factor
    // (PEARL_GPU_INNER_RTOL overrides)
    ctx->P.inner_rtol = 1e-6;
    if (const char* e = std::getenv("PEARL_GPU_INNER_RTOL")) ctx->P.inner_rtol = std::atof(e);
    return PEARL_OK;
}

int pearl_gpu_set_params(pearl_gpu_ctx* ctx, const pearl_params* params) {
    if (!ctx || !params || !valid_params(params)) return fail(ctx, PEARL_ERR_INVALID_ARGUMENT, "invalid parameters");
    ctx->params = *params;
    fill_dev_params(ctx);
    ctx->h_ctl->energy_valid = 0;
    return push_ctl(ctx);
}

int pearl_gpu_upload(pearl_gpu_ctx* ctx, const double* phi, const double* carbon, const double* mu,
                     const pearl_scalars* scalars) {
    if (!ctx) return PEARL_ERR_INVALID_ARGUMENT;
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    int rc = upload_set(ctx, ctx->h_ctl->cur, phi, carbon, mu);
    if (rc) return rc;
    if (scalars) ctx->h_ctl->S = *scalars;
    ctx->h_ctl->energy_valid = 0;
    rc = push_ctl(ctx);
    if (rc) return rc;
    PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return PEARL_OK;
}

int pearl_gpu_download(pearl_gpu_ctx* ctx, double* phi, double* carbon, double* mu, pearl_scalars* scalars) {
    if (!ctx) return PEARL_ERR_INVALID_ARGUMENT;
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    int rc = download_set(ctx, ctx->h_ctl->cur, phi, carbon, mu);
    if (rc) return rc;
    if (scalars) *scalars = ctx->h_ctl->S;
    return PEARL_OK;
}

int pearl_gpu_get_scalars(pearl_gpu_ctx* ctx, pearl_scalars* scalars) {
    if (!ctx || !scalars) return PEARL_ERR_INVALID_ARGUMENT;
    *scalars = ctx->h_ctl->S;
    return PEARL_OK;
}

int pearl_gpu_set_scalars(pearl_gpu_ctx* ctx, const pearl_scalars* scalars) {
    if (!ctx || !scalars) return PEARL_ERR_INVALID_ARGUMENT;
    ctx->h_ctl->S = *scalars;
    int rc = push_ctl(ctx);
    if (rc) return rc;
    PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return PEARL_OK;
}

int pearl_gpu_run(pearl_gpu_ctx* ctx, const pearl_run_limits* limits, pearl_run_report* report) {
    if (!ctx || !limits || limits->max_steps < 1) return fail(ctx, PEARL_ERR_INVALID_ARGUMENT, "invalid run limits");
    KArgs a{};
    a.mode = kModeRun;
    a.L = *limits;
    if (ctx->d_hist) {
        a.hist = ctx->d_hist;
        a.hist_cap = ctx->hist_cap;
        a.hist_next = ctx->hist_count % ctx->hist_cap;
    }
    int rc = launch(ctx, a);
    if (ctx->d_hist) ctx->hist_count += ctx->h_ctl->steps;
    if (report) {
        report->steps = ctx->h_ctl->steps;
        report->cg_total = ctx->h_ctl->cg_total;
        report->cg_peak = ctx->h_ctl->cg_peak;
        report->reached_stop = ctx->h_ctl->reached_stop;
        report->last = ctx->h_ctl->last;
    }
    return rc;
}

int pearl_gpu_run_replay(pearl_gpu_ctx* ctx, const double* accepted_dt, long long n, pearl_run_report* report) {
    if (!ctx || !accepted_dt || n < 1) return fail(ctx, PEARL_ERR_INVALID_ARGUMENT, "invalid replay");
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    double* d_dt = nullptr;
    PG_CUDA(ctx, cudaMalloc(&d_dt, sizeof(double) * (size_t)n));
    int rc = PEARL_OK;
    if (cudaMemcpyAsync(d_dt, accepted_dt, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, ctx->stream) !=
        cudaSuccess)
        rc = fail(ctx, PEARL_ERR_CUDA, "replay dt upload");
    if (rc == PEARL_OK) {
        KArgs a{};
        a.mode = kModeRun;
        a.L = pearl_run_limits{n, 0x7fffffffffffffffLL, 1e300, 1e300, 0};
        a.forced_dt = d_dt;
        if (ctx->d_hist) {
            a.hist = ctx->d_hist;
            a.hist_cap = ctx->hist_cap;
            a.hist_next = ctx->hist_count % ctx->hist_cap;
        }
        rc = launch(ctx, a);
        if (ctx->d_hist) ctx->hist_count += ctx->h_ctl->steps;
        if (report) {
            report->steps = ctx->h_ctl->steps;
            report->cg_total = ctx->h_ctl->cg_total;
            report->cg_peak = ctx->h_ctl->cg_peak;
            report->reached_stop = ctx->h_ctl->reached_stop;
            report->last = ctx->h_ctl->last;
        }
    }
    cudaStreamSynchronize(ctx->stream);
    cudaFree(d_dt);
    return rc;
}

int pearl_gpu_set_history(pearl_gpu_ctx* ctx, long long capacity) {
    if (!ctx || capacity < 0) return fail(ctx, PEARL_ERR_INVALID_ARGUMENT, "invalid history capacity");
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->d_hist) cudaFree(ctx->d_hist);
    ctx->d_hist = nullptr;
    ctx->hist_cap = 0;
    ctx->hist_count = 0;
    if (capacity == 0) return PEARL_OK;
    PG_CUDA(ctx, cudaMalloc(&ctx->d_hist, sizeof(pearl_step_info) * (size_t)capacity));
    ctx->hist_cap = capacity;
    return PEARL_OK;
}

int pearl_gpu_get_history(pearl_gpu_ctx* ctx, pearl_step_info* out, long long max_entries, long long* returned,
                          long long* recorded) {
    if (!ctx || max_entries < 0 || (max_entries > 0 && !out)) return PEARL_ERR_INVALID_ARGUMENT;
    const long long held = std::min(ctx->hist_count, ctx->hist_cap);
    const long long n = std::min(held, max_entries);
    // the last n entries, oldest first: at most two contiguous pieces of the ring
    if (n > 0) {
        const long long first = (ctx->hist_count - n) % ctx->hist_cap;
        const long long head = std::min(n, ctx->hist_cap - first);
        PG_CUDA(ctx, cudaMemcpyAsync(out, ctx->d_hist + first, sizeof(pearl_step_info) * (size_t)head,
                                     cudaMemcpyDeviceToHost, ctx->stream));
        if (n > head)
            PG_CUDA(ctx, cudaMemcpyAsync(out + head, ctx->d_hist, sizeof(pearl_step_info) * (size_t)(n - head),
                                         cudaMemcpyDeviceToHost, ctx->stream));
    }
    PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (returned) *returned = n;
    if (recorded) *recorded = ctx->hist_count;
    return PEARL_OK;
}

int pearl_gpu_advance(pearl_gpu_ctx* ctx, double stop_time, pearl_step_info* out) {
    if (!ctx) return PEARL_ERR_INVALID_ARGUMENT;
    pearl_run_limits L;
    L.max_steps = 1;
    L.config_max_steps = 0x7fffffffffffffffLL;
    L.stop_time = stop_time;
    L.end_time = INFINITY;
    L.output_eps = 0;
    pearl_run_report rep;
    int rc = pearl_gpu_run(ctx, &L, &rep);
    if (rc == PEARL_OK && rep.steps != 1) return fail(ctx, PEARL_ERR_INVALID_ADVANCE_TIME, "invalid advance time");
    if (out) *out = rep.last;
    return rc;
}

int pearl_gpu_maybe_shift(pearl_gpu_ctx* ctx, double trigger, double target, double c_gamma, int* rows) {
    if (!ctx) return PEARL_ERR_INVALID_ARGUMENT;
    KArgs a{};
    a.mode = kModeMaybeShift;
    a.shift_trigger = trigger;
    a.shift_target = target;
    a.shift_c_gamma = c_gamma;
    int rc = launch(ctx, a);
    if (rows) *rows = rc == PEARL_OK ? ctx->h_ctl->iout[0] : 0;
    return rc;
}

int pearl_gpu_snapshot(pearl_gpu_ctx* ctx, pearl_diag* out) {
    if (!ctx || !out) return PEARL_ERR_INVALID_ARGUMENT;
    KArgs a{};
    a.mode = kModeSnapshot;
    int rc = launch(ctx, a);
    if (rc) return rc;
    if (ctx->h_ctl->iout[0]) return fail(ctx, PEARL_ERR_MIXTURE, "Invalid mixture coefficients");
    const Ctl* h = ctx->h_ctl;
    out->c_min = h->out[0];
    out->c_max = h->out[1];
    out->mu_min = h->out[2];
    out->mu_max = h->out[3];
    out->phi_sum_error = h->out[4];
    out->mass = h->out[5];
    out->energy = h->out[6];
    out->ledger = out->mass + h->S.carbon_removed - h->S.carbon_added - h->S.initial_carbon;
    return PEARL_OK;
}

int pearl_gpu_smooth_interface(pearl_gpu_ctx* ctx, int max_steps, int min_steps, double energy_rtol,
                               double max_phase_change, pearl_smooth_report* out) {
    if (!ctx) return PEARL_ERR_INVALID_ARGUMENT;
    // smooth_interface_only's control check (pearl_serial.cpp:874-876)
    if (max_steps < 1 || min_steps < 0 || min_steps > max_steps || !(energy_rtol > 0) || !(max_phase_change > 0) ||
        max_phase_change > .2)
        return fail(ctx, PEARL_ERR_INVALID_ARGUMENT, "invalid sharp-smoothing controls");
    KArgs a{};
    a.mode = kModeSmooth;
    a.smooth_max_steps = max_steps;
    a.smooth_min_steps = min_steps;
    a.smooth_energy_rtol = energy_rtol;
    a.smooth_max_phase_change = max_phase_change;
    int rc = launch(ctx, a);
    if (rc) return rc;
    if (out) {
        const double* r = ctx->h_ctl->out;
        out->steps = (int)r[0];
        out->converged = (int)r[1];
        out->energy_initial = r[2];
        out->energy_final = r[3];
        out->final_relative_energy_change = r[4];
        out->final_max_phase_change = r[5];
        for (int k = 0; k < 3; ++k) {
            out->phase_fraction_before[k] = r[6 + k];
            out->phase_fraction_after[k] = r[9 + k];
        }
    }
    return PEARL_OK;
}

int pearl_gpu_mixture_sums(pearl_gpu_ctx* ctx, double* sum_c_intercept, double* sum_chi) {
    if (!ctx) return PEARL_ERR_INVALID_ARGUMENT;
    KArgs a{};
    a.mode = kModeMixSums;
    int rc = launch(ctx, a);
    if (rc) return rc;
    if (ctx->h_ctl->iout[0]) return fail(ctx, PEARL_ERR_MIXTURE, "Invalid mixture coefficients");
    if (sum_c_intercept) *sum_c_intercept = ctx->h_ctl->out[0];
    if (sum_chi) *sum_chi = ctx->h_ctl->out[1];
    return PEARL_OK;
}

int pearl_gpu_fill(pearl_gpu_ctx* ctx, const pearl_fill_op* ops, int nops) {
    if (!ctx) return PEARL_ERR_INVALID_ARGUMENT;
    if (nops < 0 || nops > PEARL_FILL_MAX_OPS || (nops > 0 && !ops))
        return fail(ctx, PEARL_ERR_INVALID_ARGUMENT, "invalid filling command list");
    // parameter counts of validate_filling_operations (pearl_serial.cpp:1299-1343)
    static const int kCount[8] = {0, 7, 6, 6, 13, 16, 11, 11};
    const double pi = 3.14159265358979323846;
    std::vector<DevFillOp> h((size_t)std::max(nops, 1));
    for (int k = 0; k < nops; ++k) {
        const pearl_fill_op& o = ops[k];
        if (o.method < PEARL_FILL_CUBE || o.method > PEARL_FILL_PEARLITE_ELLIPSE_2D || o.nparams != kCount[o.method])
            return fail(ctx, PEARL_ERR_INVALID_ARGUMENT, "unsupported filling method or parameter count");
        DevFillOp& d = h[(size_t)k];
        std::memset(&d, 0, sizeof d);
        d.method = o.method;
        for (int j = 0; j < o.nparams; ++j) d.p[j] = o.p[j];
        // the arms' directions, as filling_phase_at forms them (:1421-1422, :1441-1442, :1491-1492)
        if (o.method == PEARL_FILL_Y_JUNCTION_2D || o.method == PEARL_FILL_Y_JUNCTION_LAMELLAE_2D) {
            for (int arm = 0; arm < 3; ++arm) {
                const double ang = o.p[6 + arm] * pi / 180.0;
                d.ux[arm] = std::cos(ang);
                d.uy[arm] = std::sin(ang);
            }
        } else if (o.method == PEARL_FILL_ADHERED_PEARLITE_ARM_2D || o.method == PEARL_FILL_PEARLITE_ELLIPSE_2D) {
            const double ang = o.p[2] * pi / 180.0;
            d.ux[0] = std::cos(ang);
            d.uy[0] = std::sin(ang);
        }
    }
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    if (!ctx->d_fill) PG_CUDA(ctx, cudaMalloc(&ctx->d_fill, sizeof(DevFillOp) * PEARL_FILL_MAX_OPS));
    if (nops > 0)
        PG_CUDA(ctx, cudaMemcpyAsync(ctx->d_fill, h.data(), sizeof(DevFillOp) * nops, cudaMemcpyHostToDevice,
                                     ctx->stream));
    const int cur = ctx->h_ctl->cur;
    fill_kernel<<<stage_grid(ctx), 256, 0, ctx->stream>>>(static_cast<const DevFillOp*>(ctx->d_fill), nops, ctx->nx,
                                                          ctx->ny, ctx->pitch, ctx->B.phi[cur][0], ctx->B.phi[cur][1],
                                                          ctx->B.phi[cur][2]);
    ctx->launches++;
    PG_CUDA(ctx, cudaGetLastError());
    ctx->h_ctl->energy_valid = 0;
    int rc = push_ctl(ctx);
    if (rc) return rc;
    PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return PEARL_OK;
}

int pearl_gpu_init_composition(pearl_gpu_ctx* ctx, double mu, double* total_carbon) {
    if (!ctx) return PEARL_ERR_INVALID_ARGUMENT;
    KArgs a{};
    a.mode = kModeInitComposition;
    a.init_mu = mu;
    int rc = launch(ctx, a);
    if (rc) return rc;
    if (ctx->h_ctl->iout[0]) return fail(ctx, PEARL_ERR_MIXTURE, "Invalid mixture coefficients");
    if (total_carbon) *total_carbon = ctx->h_ctl->out[0];
    return PEARL_OK;
}

int pearl_gpu_propose_phi(pearl_gpu_ctx* ctx, double dt, double* max_change) {
    if (!ctx) return PEARL_ERR_INVALID_ARGUMENT;
    KArgs a{};
    a.mode = kModePropose;
    a.dt = dt;
    int rc = launch(ctx, a);
    if (rc) return rc;
    if (ctx->h_ctl->iout[1]) return fail(ctx, PEARL_ERR_SIMPLEX, "Simplex projection failed");
    if (max_change) *max_change = ctx->h_ctl->out[0];
    return PEARL_OK;
}

int pearl_gpu_upload_trial_phi(pearl_gpu_ctx* ctx, const double* phi) {
    if (!ctx || !phi) return PEARL_ERR_INVALID_ARGUMENT;
    int rc = upload_set(ctx, ctx->h_ctl->cur ^ 1, phi, nullptr, nullptr);
    if (rc) return rc;
    KArgs a{};
    a.mode = kModeMix;
    rc = launch(ctx, a);
    if (rc) return rc;
    if (ctx->h_ctl->iout[0]) return fail(ctx, PEARL_ERR_MIXTURE, "Invalid mixture coefficients");
    return PEARL_OK;
}

int pearl_gpu_implicit_diffusion(pearl_gpu_ctx* ctx, double dt, int* ok, int* iterations, double* residual,
                                 double* closure) {
    if (!ctx) return PEARL_ERR_INVALID_ARGUMENT;
    KArgs a{};
    a.mode = kModeDiffusion;
    a.dt = dt;
    int rc = launch(ctx, a);
    if (rc) return rc;
    if (ok) *ok = ctx->h_ctl->iout[0];
    if (iterations) *iterations = ctx->h_ctl->iout[1];
    if (residual) *residual = ctx->h_ctl->out[0];
    if (closure) *closure = ctx->h_ctl->out[1];
    return PEARL_OK;
}

int pearl_gpu_download_trial(pearl_gpu_ctx* ctx, double* phi, double* carbon, double* mu) {
    if (!ctx) return PEARL_ERR_INVALID_ARGUMENT;
    return download_set(ctx, ctx->h_ctl->cur ^ 1, phi, carbon, mu);
}

int pearl_gpu_energy_mass(pearl_gpu_ctx* ctx, double* energy, double* mass) {
    if (!ctx) return PEARL_ERR_INVALID_ARGUMENT;
    KArgs a{};
    a.mode = kModeEnergy;
    int rc = launch(ctx, a);
    if (rc) return rc;
    if (ctx->h_ctl->iout[0]) return fail(ctx, PEARL_ERR_MIXTURE, "Invalid mixture coefficients");
    if (energy) *energy = ctx->h_ctl->out[0];
    if (mass) *mass = ctx->h_ctl->out[1];
    return PEARL_OK;
}

int pearl_gpu_valid_state(pearl_gpu_ctx* ctx, int* valid) {
    if (!ctx || !valid) return PEARL_ERR_INVALID_ARGUMENT;
    KArgs a{};
    a.mode = kModeValid;
    int rc = launch(ctx, a);
    if (rc) return rc;
    *valid = ctx->h_ctl->iout[1] ? 0 : 1;
    return PEARL_OK;
}

int pearl_gpu_selftest_division(int device, const double* a, const double* b, long long n,
                                unsigned long long* mismatches) {
    if (!a || !b || n < 0 || !mismatches) return PEARL_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(device) != cudaSuccess) return PEARL_ERR_NO_DEVICE;
    std::vector<double> rb((size_t)n);
    for (long long i = 0; i < n; ++i) rb[(size_t)i] = 1.0 / b[i];
    double *da = nullptr, *db = nullptr, *drb = nullptr;
    unsigned long long* dm = nullptr;
    const size_t bytes = (size_t)n * sizeof(double);
    int rc = PEARL_OK;
    if (cudaMalloc(&da, bytes) != cudaSuccess || cudaMalloc(&db, bytes) != cudaSuccess ||
        cudaMalloc(&drb, bytes) != cudaSuccess || cudaMalloc(&dm, sizeof(unsigned long long)) != cudaSuccess)
        rc = PEARL_ERR_CUDA;
    if (rc == PEARL_OK && (cudaMemcpy(da, a, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
                           cudaMemcpy(db, b, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
                           cudaMemcpy(drb, rb.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
                           cudaMemset(dm, 0, sizeof(unsigned long long)) != cudaSuccess))
        rc = PEARL_ERR_CUDA;
    if (rc == PEARL_OK) {
        g8::division_selftest_kernel<<<1184, 256>>>(da, db, drb, n, dm, 1);
        if (cudaDeviceSynchronize() != cudaSuccess ||
            cudaMemcpy(mismatches, dm, sizeof(unsigned long long), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = PEARL_ERR_CUDA;
    }
    cudaFree(da);
    cudaFree(db);
    cudaFree(drb);
    cudaFree(dm);
    return rc;
}

int pearl_gpu_selftest_fp64_peak(int device, double* tflops) {
    if (!tflops) return PEARL_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(device) != cudaSuccess) return PEARL_ERR_NO_DEVICE;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms < 1)
        return PEARL_ERR_CUDA;
    const int blocks = sms * 8, threads = 256, iters = 1 << 14;
    double* out = nullptr;
    if (cudaMalloc(&out, sizeof(double) * blocks * threads) != cudaSuccess) return PEARL_ERR_CUDA;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = PEARL_OK;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) rc = PEARL_ERR_CUDA;
    double best = 0;
    if (rc == PEARL_OK) {
        fp64_fma_chains_kernel<<<blocks, threads>>>(out, 16, 0.999999, 1e-7);  // warm-up
        for (int rep = 0; rep < 3 && rc == PEARL_OK; ++rep) {
            float ms = 0;
            cudaEventRecord(e0);
            fp64_fma_chains_kernel<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
            cudaEventRecord(e1);
            if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess ||
                !(ms > 0))
                rc = PEARL_ERR_CUDA;
            else
                best = std::max(best, 2.0 * 8.0 * iters * (double)blocks * threads / (ms * 1e-3) / 1e12);
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(out);
    if (rc == PEARL_OK && cudaGetLastError() != cudaSuccess) rc = PEARL_ERR_CUDA;
    *tflops = best;
    return rc;
}

int pearl_gpu_selftest_wait_limit(pearl_gpu_ctx* ctx, int* status, double* waited_ms) {
    if (!ctx || !status) return PEARL_ERR_INVALID_ARGUMENT;
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    ctx->h_ctl->status = 0;
    ctx->h_ctl->why = 0;
    ctx->h_ctl->bar_count = 0;
    int rc = push_ctl(ctx);
    if (rc) return rc;
    Ctl* ctl = ctx->d_ctl;
    void* kargs[] = {&ctl};
    PG_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    PG_CUDA(ctx, cudaLaunchCooperativeKernel((const void*)g8::wait_limit_selftest_kernel, dim3(ctx->grid),
                                             dim3(tile_geometry(8).threads), kargs, 0, ctx->stream));
    ctx->launches++;
    PG_CUDA(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
    rc = pull_ctl(ctx);
    if (rc) return rc;
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    if (waited_ms) *waited_ms = ms;
    *status = ctx->h_ctl->status;
    // leave the barrier words and status as a fresh context has them
    ctx->h_ctl->status = 0;
    ctx->h_ctl->why = 0;
    ctx->h_ctl->bar_count = 0;
    rc = push_ctl(ctx);
    if (rc) return rc;
    PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return PEARL_OK;
}

int pearl_gpu_phase_times(const pearl_gpu_ctx* ctx, double* ms, long long* counts) {
    if (!ctx) return PEARL_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < 16; ++k) {
        if (ms) ms[k] = k < kTagCount ? ctx->h_ctl->phase_ns[k] * 1e-6 : 0.0;
        if (counts) counts[k] = k < kTagCount ? (long long)ctx->h_ctl->phase_count[k] : 0;
    }
    return PEARL_OK;
}

int pearl_gpu_geometry(const pearl_gpu_ctx* ctx, int* warps, int* warps_x_log2, int* grid_blocks) {
    if (!ctx) return PEARL_ERR_INVALID_ARGUMENT;
    if (warps) *warps = ctx->warps;
    if (warps_x_log2) *warps_x_log2 = ctx->P.warps_x_log2;
    if (grid_blocks) *grid_blocks = ctx->grid;
    return PEARL_OK;
}

int pearl_gpu_stats(const pearl_gpu_ctx* ctx, long long* launches, int* grid_blocks, double* last_ms) {
    if (!ctx) return PEARL_ERR_INVALID_ARGUMENT;
    if (launches) *launches = ctx->launches;
    if (grid_blocks) *grid_blocks = ctx->grid;
    if (last_ms) *last_ms = ctx->last_ms;
    return PEARL_OK;
}

}  // extern "C"

