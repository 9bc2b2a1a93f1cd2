// pearl_adjoint_host.cu — host side of the adjoint gradient: checkpointed
// forward, recomputation with tape and the reverse sweep (the device side is
// pearl_adjoint.cuh).
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

// ============================================================ adjoint
namespace {

// The adjoint kernel runs in 256-thread blocks, two per SM, for every context.
constexpr int kAdjThreads = tile_geometry(8).threads;

int launch_adjoint(pearl_gpu_ctx* ctx, AdjArgs& args) {
    const NvtxRange range(args.mode == 0 ? "pearl_gpu adjoint seed" : "pearl_gpu adjoint segment");
    if (!ctx->adj_grid) {
        int per_sm = 0, sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
        PG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, g8::pearl_adjoint_kernel, kAdjThreads, 0));
        if (per_sm < 1) return fail(ctx, PEARL_ERR_CUDA, "adjoint kernel cannot be resident");
        const long long cells = (long long)ctx->nx * ctx->ny;
        const long long want = (cells + kAdjThreads - 1) / kAdjThreads;
        // the reduction partials of the context are sized for ctx->grid blocks
        ctx->adj_grid = (int)std::max(1LL, std::min<long long>({want, (long long)per_sm * sms, (long long)ctx->grid}));
    }
    ctx->h_ctl->status = 0;
    ctx->h_ctl->why = 0;
    ctx->h_ctl->bar_count = 0;
    int rc = push_ctl(ctx);
    if (rc) return rc;
    args.P = ctx->P;
    args.B = ctx->B;
    void* kargs[] = {&args};
    PG_CUDA(ctx, cudaLaunchCooperativeKernel((const void*)g8::pearl_adjoint_kernel, dim3(ctx->adj_grid), dim3(kAdjThreads),
                                             kargs, 0, ctx->stream));
    ctx->launches++;
    rc = pull_ctl(ctx);
    if (rc) return rc;
    if (ctx->h_ctl->status == PEARL_ERR_DEVICE_WAIT) {
        ctx->h_ctl->bar_count = 0;
        push_ctl(ctx);
        return fail(ctx, PEARL_ERR_DEVICE_WAIT, "device grid barrier wait exceeded its limit");
    }
    return PEARL_OK;
}

}  // namespace

extern "C" int pearl_gpu_adjoint_gradient(pearl_gpu_ctx* ctx, long long nsteps, int checkpoint_every,
                                          const double* target_alpha, pearl_adjoint_report* out) {
    if (!ctx || nsteps < 1 || checkpoint_every < 1 || !target_alpha || !out) return PEARL_ERR_INVALID_ARGUMENT;
    if (ctx->params.phase_only) return fail(ctx, PEARL_ERR_INVALID_ARGUMENT, "adjoint needs implicit diffusion");
    if (ctx->P.mixed || ctx->P.mixed_cg)
        return fail(ctx, PEARL_ERR_INVALID_ARGUMENT, "adjoint differentiates the FP64 step");
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    std::memset(out, 0, sizeof *out);
    const size_t pe = plane_elems(ctx);
    const long long K = checkpoint_every;
    const long long nseg = (nsteps + K - 1) / K;
    const long long seglen = std::min(K, nsteps);
    const size_t n_ckpt = (size_t)(nseg + 1) * 5 * pe, n_tape = (size_t)seglen * 6 * pe, n_adj = 23 * pe;
    // working memory is kept in the context and grown when a call needs more, so
    // repeated gradients of one domain allocate once (a fresh cudaMalloc of
    // hundreds of MB per call cost up to 0.35 s of host time)
    const size_t need = n_ckpt + n_tape + n_adj + (size_t)nsteps + 8;
    if (ctx->adj_slab_elems < need) {
        if (ctx->adj_slab) cudaFree(ctx->adj_slab);
        ctx->adj_slab = nullptr;
        ctx->adj_slab_elems = 0;
        PG_CUDA(ctx, cudaMalloc(&ctx->adj_slab, need * sizeof(double)));
        ctx->adj_slab_elems = need;
    }
    double* const slab = ctx->adj_slab;
    double* ckpt = slab;
    double* tape = ckpt + n_ckpt;
    double* adj = tape + n_tape;
    double* dts = adj + n_adj;
    double* acc = dts + nsteps;
    AdjBufs J{};
    {
        double* q = adj;
        for (int a = 0; a < 3; ++a, q += pe) J.bphi[a] = q;
        J.bc = q; q += pe;
        J.bmu = q; q += pe;
        J.chi = q; q += pe;
        J.K = q; q += pe;
        J.ub = q; q += pe;
        J.lam = q; q += pe;
        J.r = q; q += pe;
        J.z = q; q += pe;
        J.p[0] = q; q += pe;
        J.p[1] = q; q += pe;
        J.Ap = q; q += pe;
        J.diag = q; q += pe;
        for (int a = 0; a < 3; ++a, q += pe) J.Fb[a] = q;
        for (int a = 0; a < 3; ++a, q += pe) J.Ql[a] = q;
    }
    double* target = adj + 22 * pe;
    std::vector<pearl_scalars> seg_scalars(nseg);
    cudaEvent_t e[4];
    for (auto& ev : e) cudaEventCreate(&ev);
    auto state = [&](int set) { return ctx->B.phi[set][0]; };  // 5 contiguous planes
    const Ctl initial_ctl = *ctx->h_ctl;
    bool have_initial = false;
    auto body = [&]() -> int {
        PG_CUDA(ctx, cudaMemsetAsync(slab, 0, (n_ckpt + n_tape + n_adj + (size_t)nsteps + 8) * sizeof(double),
                                     ctx->stream));
        PG_CUDA(ctx, cudaMemcpy2DAsync(target, ctx->pitch * sizeof(double), target_alpha, ctx->nx * sizeof(double),
                                       ctx->nx * sizeof(double), ctx->ny, cudaMemcpyHostToDevice, ctx->stream));
        // forward with a checkpoint at the start of every segment
        PG_CUDA(ctx, cudaEventRecord(e[0], ctx->stream));
        for (long long seg = 0; seg < nseg; ++seg) {
            const long long k0 = seg * K, len = std::min(K, nsteps - k0);
            PG_CUDA(ctx, cudaMemcpyAsync(ckpt + (size_t)seg * 5 * pe, state(ctx->h_ctl->cur), 5 * pe * sizeof(double),
                                         cudaMemcpyDeviceToDevice, ctx->stream));
            have_initial = true;
            seg_scalars[seg] = ctx->h_ctl->S;
            KArgs a{};
            a.mode = kModeRun;
            a.L = pearl_run_limits{len, 0x7fffffffffffffffLL, 1e300, 1e300, 0};
            a.dt_log = dts + k0;
            if (seg == nseg - 1) {
                // the reverse sweep starts here: tape this segment now instead of recomputing it
                a.tape = tape;
                a.tape_slot = 6 * pe;
            }
            int rc = launch(ctx, a);
            if (rc) return rc;
            if (ctx->h_ctl->steps != len) return fail(ctx, PEARL_ERR_INVALID_ARGUMENT, "forward stopped early");
            out->cg_forward += ctx->h_ctl->cg_total;
        }
        PG_CUDA(ctx, cudaEventRecord(e[1], ctx->stream));
        const Ctl final_ctl = *ctx->h_ctl;
        PG_CUDA(ctx, cudaMemcpyAsync(ckpt + (size_t)nseg * 5 * pe, state(final_ctl.cur), 5 * pe * sizeof(double),
                                     cudaMemcpyDeviceToDevice, ctx->stream));
        AdjArgs g{};
        g.J = J;
        g.target = target;
        g.acc = acc;
        g.obs_per_sigma = 16.0 / (std::acos(-1.0) * std::acos(-1.0) * ctx->params.epsilon);
        g.two_eps = 2.0 * ctx->params.epsilon;
        g.mode = 0;
        g.ckpt = state(final_ctl.cur);
        int rc = launch_adjoint(ctx, g);
        if (rc) return rc;
        // reverse sweep: recompute each segment from its checkpoint, then run it backwards
        double recompute_ms = 0;
        for (long long seg = nseg - 1; seg >= 0; --seg) {
            const long long k0 = seg * K, len = std::min(K, nsteps - k0);
            if (seg < nseg - 1) {
                PG_CUDA(ctx, cudaMemcpyAsync(state(0), ckpt + (size_t)seg * 5 * pe, 5 * pe * sizeof(double),
                                             cudaMemcpyDeviceToDevice, ctx->stream));
                ctx->h_ctl->cur = 0;
                ctx->h_ctl->S = seg_scalars[seg];
                ctx->h_ctl->energy_valid = 0;
                KArgs a{};
                a.mode = kModeRun;
                a.L = pearl_run_limits{len, 0x7fffffffffffffffLL, 1e300, 1e300, 0};
                a.forced_dt = dts + k0;
                a.tape = tape;
                a.tape_slot = 6 * pe;
                rc = launch(ctx, a);
                if (rc) return rc;
                recompute_ms += ctx->last_ms;
                if (ctx->h_ctl->steps != len)
                    return fail(ctx, PEARL_ERR_INVALID_ARGUMENT, "recomputation stopped early");
            }
            g.mode = 1;
            g.ckpt = ckpt + (size_t)seg * 5 * pe;
            g.tape = tape;
            g.slot = 6 * pe;
            g.dts = dts + k0;
            g.len = (int)len;
            rc = launch_adjoint(ctx, g);
            if (rc) return rc;
        }
        PG_CUDA(ctx, cudaEventRecord(e[2], ctx->stream));
        // leave the forward's final state in the context
        PG_CUDA(ctx, cudaMemcpyAsync(state(0), ckpt + (size_t)nseg * 5 * pe, 5 * pe * sizeof(double),
                                     cudaMemcpyDeviceToDevice, ctx->stream));
        *ctx->h_ctl = final_ctl;
        ctx->h_ctl->cur = 0;
        ctx->h_ctl->energy_valid = 0;
        rc = push_ctl(ctx);
        if (rc) return rc;
        double h_acc[8];
        PG_CUDA(ctx, cudaMemcpyAsync(h_acc, acc, sizeof h_acc, cudaMemcpyDeviceToHost, ctx->stream));
        PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        float f_ms = 0, b_ms = 0;
        cudaEventElapsedTime(&f_ms, e[0], e[1]);
        cudaEventElapsedTime(&b_ms, e[1], e[2]);
        out->objective = h_acc[0];
        out->grad[0] = h_acc[1];
        out->grad[1] = h_acc[2];
        out->grad[2] = h_acc[3];
        out->cg_adjoint = (long long)h_acc[4];
        out->steps = nsteps;
        out->checkpoints = (int)nseg;
        out->forward_ms = f_ms;
        out->recompute_ms = recompute_ms;
        out->adjoint_ms = b_ms - recompute_ms;
        return PEARL_OK;
    };
    const int rc = body();
    if (rc && have_initial) {
        // a failed gradient leaves the context in its initial state
        cudaMemcpyAsync(state(0), ckpt, 5 * pe * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
        *ctx->h_ctl = initial_ctl;
        ctx->h_ctl->cur = 0;
        ctx->h_ctl->energy_valid = 0;
        ctx->h_ctl->bar_count = 0;
        push_ctl(ctx);
    }
    cudaStreamSynchronize(ctx->stream);
    for (auto& ev : e) cudaEventDestroy(ev);
    return rc;
}

