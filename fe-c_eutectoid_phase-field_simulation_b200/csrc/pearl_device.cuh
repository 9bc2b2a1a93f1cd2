// pearl_device.cuh — device-side building blocks of the FP64 hot path.
//
// Pointwise thermodynamics and kinetics follow pearl_serial.cpp with the same
// floating-point operation order; the translation unit is compiled with
// -fmad=false, so a multiply followed by an add is never fused unless the
// reference itself calls std::fma.  Per-cell results are therefore bitwise
// equal to the reference's; only global sums (CG dot products, carbon mass,
// energy) differ, because they are reduced as a fixed-order tree instead of a
// sequential row-major loop.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "pearl_gpu.h"

namespace pearl_gpu {

constexpr int kTileX = 32;  // one warp spans 32 consecutive x cells (256 B of a row)
constexpr int kMaxRed = 6;  // values per grid reduction

// Device copy of pearl_params plus host-precomputed constants.  Each constant
// is evaluated on the host with the reference's own expression, so its bits
// equal what the reference recomputes per cell.
struct DevParams {
    int nx, ny, pitch, ntx, nty, ntiles;
    int warps_x_log2;  // tile = (32 << warps_x_log2) x (2 << (3 - warps_x_log2)) cells
    double dx, dy, dx2, dy2;
    double Vm, eps, obs, tr, two_eps_sigma, eps_sigma;
    double tau[3], tau_min;
    double A[3], B[3], C[3], D[3];
    double chi_p[3];     // Parabola::chi = 1/(2A)            (:85)
    double neg_q_A[3];   // -0.25/A of Parabola::psi           (:87)
    double two_A[3];     // 2.0*A of Parabola::c_at_mu         (:84)
    double psi_t[3];     // psi_a(mu_ref) - psi_gamma(mu_ref)  (:797)
    double mu_ref;
    double dt_max, dt_min, max_phase_change, cg_rtol, cg_atol, closure_tol, energy_rtol, energy_atol;
    double mass_scale;    // gx*gy*dx*dy*1e-6                  (:1152)
    double energy_scale;  // sigma*max(gx*dx, gy*dy)            (:1157)
    int cg_max, max_retries, check_energy, phase_only;
    // RN(1/b) of every constant divisor b, for div_by
    double r_Vm, r_dx, r_dy, r_dx2, r_dy2, r_3, r_two_A[3];
    int exact_div;  // 1 when every constant divisor and its reciprocal are normal numbers
    // Mixed precision (PROPOSE forces in FP32).  psi_b(mu) - psi_g(mu) is
    // expanded about mu_ref in delta = mu - mu_ref, which is formed in FP64:
    // m_pa[b] + delta*(m_pb[b] + delta*m_pc[b]), so FP32 never subtracts two
    // large free energies.
    int mixed;
    // Mixed precision of the implicit solve: FP32 inner Jacobi-PCG rounds on the
    // correction A d = r, accumulated into the FP64 unknown, each closed by an
    // FP64 residual of that unknown; an inner round stops once its residual has
    // fallen by inner_rtol (or to half the tolerance).  Needs the FP32 planes.
    int mixed_cg;
    double inner_rtol;
    float m_obs, m_tr, m_kx, m_ky, m_rVm;  // obs, tr, 2 eps sigma / dx^2, / dy^2, 1/Vm
    float m_pa[2], m_pb[2], m_pc[2];
    float m_tau[3], m_tau_min;
};

// a/b, correctly rounded, for a divisor b whose reciprocal rb = RN(1/b) was
// computed once on the host.  Residual correction with fused multiply-adds
// (Markstein, IBM J. Res. Dev. 34(1), 1990; Muller et al., Handbook of
// Floating-Point Arithmetic, ch. "Division"): q0 = a*rb, then twice
// q <- q + (a - q*b)*rb, where a - q*b is exact in one FMA.  After the first
// correction q is a faithful quotient, and Markstein's theorem makes the
// second one the correctly rounded a/b for normal operands and quotients, so
// the result equals IEEE division bitwise (checked on the device against
// '/' by pearl_gpu_selftest_division).  Zero and non-finite numerators keep
// the sign/special value of a*rb.  Falls back to '/' when the host found a
// divisor outside the normal range.
// The zero / non-finite test reads the bit patterns with integer operations,
// which leaves the FP64 pipe to the arithmetic: a == +-0 when its magnitude
// bits are all zero, q0 is Inf or NaN when its exponent field is all ones.
__device__ __forceinline__ double div_by(const DevParams& P, double a, double b, double rb) {
    if (!P.exact_div) return a / b;
    const double q0 = a * rb;
    double r = fma(-q0, b, a);
    double q = fma(r, rb, q0);
    r = fma(-q, b, a);
    q = fma(r, rb, q);
    const int ah = __double2hiint(a), al = __double2loint(a), qh = __double2hiint(q0);
    const bool special = (((ah & 0x7fffffff) | al) == 0) | ((qh & 0x7ff00000) == 0x7ff00000);
    return special ? q0 : q;
}

// div_by for the proposal's forces (positive divisors only): the same
// correctly rounded quotient for finite numerators and quotients, but without
// div_by's integer tests.  A zero numerator's sign is OR-ed into the result
// (the corrections turn -0 into +0, and a nonzero quotient already has the
// numerator's sign); a non-finite numerator gives NaN where IEEE division
// gives +-Inf.  Both are non-finite, and the proposal treats any non-finite
// force alike: the cell takes the reference's non-finite branch
// (pearl_serial.cpp:990-996), keeps its phi and reports an infinite change.
__device__ __forceinline__ double div_force(const DevParams& P, double a, double b, double rb) {
    if (!P.exact_div) return a / b;
    const double q0 = a * rb;
    double r = fma(-q0, b, a);
    double q = fma(r, rb, q0);
    r = fma(-q, b, a);
    q = fma(r, rb, q);
    return __hiloint2double(__double2hiint(q) | (__double2hiint(a) & (int)0x80000000), __double2loint(q));
}

// Device buffers: two state sets (current / trial, selected by Ctl::cur) and
// the work vectors of the implicit solve.  Every plane is ny rows of `pitch`
// doubles (pitch = nx rounded up to 32, so each row starts on 256 B).
struct DevBufs {
    double* phi[2][3];
    double* c[2];
    double* mu[2];
    double* K;     // transport K = sum phi_p D_p chi_p of trial phi
    double* chi;   // susceptibility of trial phi
    double* icpt;  // composition(mu_ref) of trial phi
    double* diag;  // Jacobi preconditioner
    double* x;     // mu - mu_ref (the CG unknown)
    double* r;
    double* z;
    double* p[2];  // search direction, double-buffered (read at neighbours while rewritten)
    double* Ap;
    double* wE;    // east-face weight .5*(K+K_east)/dx^2 of the current solve
    double* wN;    // north-face weight .5*(K+K_north)/dy^2, zero at the top wall
    double* part;  // [2][grid][kMaxRed] block partials
    struct Ctl* ctl;
    // FP32 planes of the mixed-precision solve (null until a context is put in a
    // mixed-solve precision): the solve's face weights, susceptibility and
    // Jacobi diagonal, and the inner CG's residual, preconditioned residual,
    // search direction (double-buffered) and A p.
    float* wE32;
    float* wN32;
    float* chi32;
    float* diag32;
    float* r32;
    float* z32;
    float* p32[2];
    float* Ap32;
};

// Device-resident control block: barrier words, the State scalars and the
// results of the last launch.  Host and device exchange it by value.
struct Ctl {
    unsigned long long bar_count;  // grid-barrier arrivals since the launch began (zeroed by the host)
    unsigned pad0[30];             // the polled counter has its 128-byte line to itself
    int status, why, cur, energy_valid;
    pearl_scalars S;
    double e0, mass0;
    pearl_step_info last;
    long long steps, cg_total;
    int cg_peak, reached_stop;
    double out[16];
    int iout[4];
    // per-phase device time of the last launch, measured by block 0 between
    // consecutive grid barriers (phase compute + reduction + barrier wait)
    unsigned long long phase_ns[16];
    unsigned long long phase_count[16];
};

enum PhaseTag : int {
    kTagPropose = 0, kTagSetup, kTagApply, kTagUpdate, kTagTrueRes, kTagReset, kTagFinal, kTagEnergy,
    kTagFinalPhaseOnly, kTagMix, kTagShift, kTagSnapshot, kTagSmooth, kTagInit, kTagAdjoint,
    kTagApply32, kTagCount
};
// The FP32 inner update and residual passes of the mixed solve are clocked as
// kTagUpdate and kTagTrueRes; only the FP32 apply has a tag of its own.

// ---------------------------------------------------------------- thermodynamics
// Parabola::psi (pearl_serial.cpp:86-89)
__device__ __forceinline__ double psi(const DevParams& P, int a, double mu) {
    const double d = mu - P.B[a];
    return fma(P.neg_q_A[a], d * d, P.C[a]);
}

// mixture (pearl_serial.cpp:125-138): returns false where the reference throws.
__device__ __forceinline__ bool mixture(const DevParams& P, double p0, double p1, double p2, double& chi,
                                        double& cint, double& K) {
    const double triple = 2.0 * p0 * p1 * p2;
    const double h0 = p0 * p0 * (3.0 - 2.0 * p0) + triple;
    const double h1 = p1 * p1 * (3.0 - 2.0 * p1) + triple;
    const double h2 = p2 * p2 * (3.0 - 2.0 * p2) + triple;
    double s = 0.0, ci = 0.0, k = 0.0;
    s += h0 * P.chi_p[0];
    ci -= h0 * P.chi_p[0] * P.B[0];
    k += p0 * P.D[0] * P.chi_p[0];
    s += h1 * P.chi_p[1];
    ci -= h1 * P.chi_p[1] * P.B[1];
    k += p1 * P.D[1] * P.chi_p[1];
    s += h2 * P.chi_p[2];
    ci -= h2 * P.chi_p[2] * P.B[2];
    k += p2 * P.D[2] * P.chi_p[2];
    chi = s;
    cint = ci;
    K = k;
    return (s > 0.0) && isfinite(s) && isfinite(ci) && isfinite(k) && !(k < 0.0);
}

// project_simplex (pearl_serial.cpp:491-509).  Inputs are finite here (the
// caller checks first, :990-996).  Returns false where the reference throws.
// The thresholds (sum-1)/1, /2, /3 are formed exactly: x/1 = x, x/2 = x*0.5,
// and /3 through div_by.
__device__ __forceinline__ bool project_simplex(const DevParams& P, double& z0, double& z1, double& z2) {
    double s0 = z0, s1 = z1, s2 = z2, t;
    if (s0 < s1) { t = s0; s0 = s1; s1 = t; }
    if (s1 < s2) { t = s1; s1 = s2; s2 = t; }
    if (s0 < s1) { t = s0; s0 = s1; s1 = t; }
    double sum = 0.0, threshold = 0.0, cand;
    int active = 0;
    sum += s0;
    cand = sum - 1.0;
    if (s0 > cand) { active = 1; threshold = cand; }
    sum += s1;
    cand = (sum - 1.0) * 0.5;
    if (s1 > cand) { active = 2; threshold = cand; }
    sum += s2;
    cand = div_by(P, sum - 1.0, 3.0, P.r_3);
    if (s2 > cand) { active = 3; threshold = cand; }
    // std::max(0.0, v) == (0.0 < v ? v : 0.0)
    double v = z0 - threshold;
    z0 = (0.0 < v) ? v : 0.0;
    v = z1 - threshold;
    z1 = (0.0 < v) ? v : 0.0;
    v = z2 - threshold;
    z2 = (0.0 < v) ? v : 0.0;
    return active != 0;
}

// local_tau (pearl_serial.cpp:533-537)
__device__ __forceinline__ double local_tau(const DevParams& P, double p0, double p1, double p2) {
    const double w0 = p0 * p1, w1 = p0 * p2, w2 = p1 * p2;
    const double s = w0 + w1 + w2;
    return s > 1e-30 ? (w0 * P.tau[0] + w1 * P.tau[1] + w2 * P.tau[2]) / s : P.tau_min;
}

// ---------------------------------------------------------------- TMA tile staging
// A 32x16-cell tile plus a one-cell halo is staged per field as one 2-D TMA
// box.  The box starts two cells left of the tile so that its x coordinate
// stays a multiple of two doubles (16 bytes): columns 0..35 hold x0-2..x0+33,
// rows 0..17 hold y0-1..y0+16.  Out-of-range rows and columns arrive as zeros;
// the periodic x wrap is patched with plain loads and the y walls never read
// their ghost row (the zero-flux faces are skipped or weighted by zero).
constexpr int kBoxW = kTileX + 4;
// FP32 boxes start four cells left of the tile (a 4-byte element's x must be a
// multiple of four for a 16-byte aligned copy): columns 0..39 hold x0-4..x0+35.
constexpr int kBoxW32 = kTileX + 8;
constexpr int kMaxStageFields = 9;
constexpr int kMaxStages = 4;

// Block shape.  A block of `warps` warps covers a tile 32 cells wide and 2 x
// warps rows high (each warp two adjacent rows).  The device code is compiled
// for two shapes: 8 warps (256 threads, two blocks per SM: 32x16 tiles) and 16
// warps (512 threads, one block per SM: 32x32 tiles, 148 blocks in the grid
// barrier and 5% fewer halo bytes per tile), in namespaces g8 and g16.  The
// shared-memory budget of the pipeline is two stages of the widest phase (9
// fields); phases staging fewer fields run more stages in the same space (up to 4).
struct TileGeometry {
    int warps, threads, rows;  // warps per block, threads, tile height in cells
    int box_h;                 // staged box height: the tile plus one halo row above and below
    int field_stride;          // doubles per staged field (128 B aligned)
    size_t pipe_doubles;       // pipeline stage buffers
    size_t tma_smem_bytes;     // dynamic shared memory of a block with TMA staging
    int min_blocks;            // resident blocks per SM the kernels are compiled for
};
constexpr TileGeometry tile_geometry(int warps) {
    const int box_h = 2 * warps + 2;
    const int stride = (int)(((size_t)kBoxW * box_h * sizeof(double) + 127) / 128 * 128 / sizeof(double));
    const size_t pipe = (size_t)2 * kMaxStageFields * stride;
    return TileGeometry{warps, 32 * warps, 2 * warps, box_h, stride, pipe, 128 + pipe * sizeof(double),
                        warps >= 16 ? 1 : 2};
}

#ifndef PEARL_TILE_WARPS
#define PEARL_TILE_WARPS 8
#endif
#if PEARL_TILE_WARPS == 16
#define PEARL_GEOM_NS g16
#elif PEARL_TILE_WARPS == 8
#define PEARL_GEOM_NS g8
#else
#error "PEARL_TILE_WARPS must be 8 or 16"
#endif

// The block shape this translation unit's device code is compiled for.
namespace PEARL_GEOM_NS {
constexpr TileGeometry kGeom = tile_geometry(PEARL_TILE_WARPS);
constexpr int kTileY = kGeom.warps;
constexpr int kTileRows = kGeom.rows;
constexpr int kTileRowsLog2 = kTileRows == 32 ? 5 : 4;
static_assert((1 << kTileRowsLog2) == kTileRows, "tile height is a power of two");
constexpr int kThreads = kGeom.threads;
constexpr int kBoxH = kGeom.box_h;
constexpr uint32_t kBoxBytes = kBoxW * kBoxH * sizeof(double);
constexpr int kFieldStride = kGeom.field_stride;
constexpr size_t kPipeDoubles = kGeom.pipe_doubles;
// floats per staged FP32 field (128 B aligned)
constexpr int kFieldStride32 = (int)(((size_t)kBoxW32 * kBoxH * sizeof(float) + 127) / 128 * 128 / sizeof(float));
constexpr size_t kTmaSmemBytes = kGeom.tma_smem_bytes;
constexpr int kMinBlocks = kGeom.min_blocks;
}  // namespace PEARL_GEOM_NS

// Tensor-map slots: state set s fields 0..4 (phi_a, phi_t, phi_g, c, mu) at
// 5*s + f, then the work planes.
enum MapId : int {
    kMapState = 0,  // + 5*set + field
    kMapK = 10, kMapChi, kMapIcpt, kMapX, kMapZ, kMapP0, kMapP1, kMapWE, kMapWN, kMapR, kMapAp, kMapDiag,
    // tile-only boxes (kTileX x kTileRows, no halo) for the pointwise CG update
    kMapXc, kMapP0c, kMapP1c, kMapRc, kMapApc, kMapDiagc,
    // FP32 planes of the mixed solve's APPLY32 (encoded once the planes exist):
    // kBoxW32 x box_h boxes starting four cells left of the tile
    kMap32WE, kMap32WN, kMap32Z, kMap32Chi, kMap32P0, kMap32P1,
    kMapCount
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Generic-proxy writes (plain stores) made visible to later TMA (async-proxy) reads.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async;" ::: "memory"); }
// The executing thread's shared-memory writes ordered before later async-proxy accesses.
__device__ __forceinline__ void fence_proxy_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// ---------------------------------------------------------------- grid barrier
__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

constexpr unsigned long long kBarrierTimeoutNs = 4000000000ull;  // 4 s; a phase takes well under 0.1 s

// Grid barrier for a cooperative launch (all blocks are co-resident) on one
// monotonic 64-bit arrival counter: a block's arrival ticket names its
// barrier, which completes when the counter reaches the next multiple of the
// block count, so there is no reset and no second word on the critical path
// (one atomic and one polled load per block; against a count-and-generation
// pair this took 19 % off a 256x512 step and 1 % off a 2048x4096 one).  The
// wait is bounded: after kBarrierTimeoutNs the block records
// PEARL_ERR_DEVICE_WAIT and every caller returns without further device work;
// the host zeroes the counter before the next launch.  Ordering: block
// barrier, arrival with release (and acquire) semantics at GPU scope, polling
// with acquire loads, block barrier.
__device__ __forceinline__ unsigned long long atom_add_acq_rel_gpu(unsigned long long* p, unsigned long long v) {
    unsigned long long old;
    asm volatile("atom.acq_rel.gpu.global.add.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
    return old;
}
__device__ __forceinline__ unsigned long long ld_acquire_gpu(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ bool grid_barrier(Ctl* ctl, unsigned nblocks) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        // the k-th barrier of the launch completes when the counter reaches k * nblocks
        const unsigned long long n = nblocks;
        const unsigned long long target = (atom_add_acq_rel_gpu(&ctl->bar_count, 1ull) / n + 1) * n;
        const unsigned long long t0 = globaltimer_ns();
        unsigned spins = 0;
        while (ld_acquire_gpu(&ctl->bar_count) < target) {
            if ((++spins & 255u) == 0 && globaltimer_ns() - t0 > kBarrierTimeoutNs) {
                ok = 0;
                atomicCAS(&ctl->status, 0, (int)PEARL_ERR_DEVICE_WAIT);
                break;
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// ---------------------------------------------------------------- reductions
// Deterministic reductions: fixed shuffle trees inside a warp, warps combined
// in index order, blocks combined in index order by every block identically,
// so all blocks hold bitwise-equal results and take the same decisions.
enum RedOp : unsigned { kSum = 0, kMax = 1, kMin = 2 };

__device__ __forceinline__ double red_apply(unsigned op, double a, double b) {
    // fmax/fmin drop NaN like the reference's std::max(acc, v)/std::min(acc, v)
    return op == kSum ? a + b : (op == kMax ? fmax(a, b) : fmin(a, b));
}
__device__ __forceinline__ double red_identity(unsigned op) {
    return op == kSum ? 0.0 : (op == kMax ? -INFINITY : INFINITY);
}
__device__ __forceinline__ unsigned op_of(unsigned ops, int k) { return (ops >> (2 * k)) & 3u; }

namespace PEARL_GEOM_NS {  // the block's warps
template <int NV>
__device__ __forceinline__ void block_publish(const double (&v)[NV], unsigned ops, double* part_slot, int bid) {
    __shared__ double s_red[kThreads / 32][kMaxRed];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        const unsigned op = op_of(ops, k);
        double t = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t = red_apply(op, t, __shfl_down_sync(0xffffffffu, t, o));
        if (lane == 0) s_red[warp][k] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            const unsigned op = op_of(ops, k);
            double acc = s_red[0][k];
            for (int w = 1; w < kThreads / 32; ++w) acc = red_apply(op, acc, s_red[w][k]);
            part_slot[bid * kMaxRed + k] = acc;
        }
    }
}
}  // namespace PEARL_GEOM_NS

template <int NV>
__device__ __forceinline__ void grid_gather(double (&out)[NV], unsigned ops, const double* part_slot, int nblk) {
    __shared__ double s_out[kMaxRed];
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            const unsigned op = op_of(ops, k);
            double acc = red_identity(op);
            for (int b = lane; b < nblk; b += 32) acc = red_apply(op, acc, part_slot[b * kMaxRed + k]);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc = red_apply(op, acc, __shfl_down_sync(0xffffffffu, acc, o));
            if (lane == 0) s_out[k] = acc;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = s_out[k];
    __syncthreads();
}

}  // namespace pearl_gpu
