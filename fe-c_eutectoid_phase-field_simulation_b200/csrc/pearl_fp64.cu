// pearl_fp64.cu — FP64 hot path of Pearl on B200: one persistent cooperative
// kernel runs whole accepted time steps (pearl::advance, pearl_serial.cpp:1119)
// including the retry loop and the Jacobi-PCG solve, with every decision
// (dt, acceptance, CG termination) taken on the device.
//
// Phases of one attempt (each is a sweep over the block's tiles followed by a
// deterministic grid reduction and a bounded grid barrier):
//   PROPOSE  propose_phi (:961-1002) + mixture of the trial phi (:1013-1020)
//   SETUP    implicit_diffusion set-up: apply(mu_offset), r, z, diag (:1021-1046)
//   APPLY    p = z + beta p ; A p ; <p,Ap>                          (:1067-1079)
//   UPDATE   x += alpha p ; r -= alpha Ap ; z = r/diag ; <r,z>,<r,r> (:1071-1078)
//   FINAL    true residual r = rhs - A x (:1051-1055) fused with the conservative
//            carbon update, closure, mu, valid_state, total_carbon and
//            reduced_energy of the trial state (:1082-1093, :1096-1116, :784-821)
//   RESET    z = r/diag ; <r,z> when the true residual misses     (:1060-1064)
//
// Thread mapping: a warp covers 32 consecutive x of two adjacent rows; the
// kTileY warps of a block stack 2 x kTileY rows.  This file is compiled once
// per block shape (PEARL_TILE_WARPS = 8: 32x16 tiles, two 256-thread blocks
// per SM; 16: 32x32 tiles, one 512-thread block per SM), into namespaces g8
// and g16.  The two cells of a thread share their vertical neighbour loads.
// Each phase's input fields are staged per tile by 2-D TMA copies into shared
// memory through an mbarrier pipeline (`sweep`).
//
// This file also holds the batched kernel (block groups running independent
// instances), the self-test kernels, and, through pearl_adjoint.cuh, the
// reverse-step kernel; the host side lives in pearl_ctx.cu, pearl_batch.cu,
// pearl_adjoint_host.cu and pearl_noalloc.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include <cudaTypedefs.h>

#include "pearl_kernels.cuh"

namespace pearl_gpu {
namespace PEARL_GEOM_NS {  // compiled once per block shape (PEARL_TILE_WARPS = 8, 16)



// One domain as seen by one block: its parameters, buffers and tensor maps,
// the block's index in the group of blocks that shares the domain, the
// group's barrier words and error status, and its reduction partials.  A
// single-domain launch is one group spanning the whole grid; a batched launch
// gives every group of blocks its own instances.
struct Dom {
    const DevParams& P;
    const DevBufs& B;
    const CUtensorMap* maps;
    int use_tma;
    int bid, nblk;
    Ctl* bar;      // barrier words and status of this block group
    double* part;  // [2][nblk][kMaxRed] partials of this block group
    double shift_trigger, shift_target, shift_c_gamma;
    int smooth_max_steps, smooth_min_steps;
    double smooth_energy_rtol, smooth_max_phase_change;
};

// The two cells (x, y0) and (x, y0+1) of one thread in tile t.
struct Pair {
    int x, y0;
    bool v0, v1;                   // cell valid (inside the domain)
    size_t i0, i1;                 // centres
    size_t iw0, ie0, iw1, ie1;     // x neighbours (periodic)
    size_t is0, in1;               // y neighbours outside the pair (zero-flux ghost = the cell itself)
};

__device__ __forceinline__ Pair pair_of(const DevParams& P, int t) {
    Pair c;
    const int bx = t % P.ntx, by = t / P.ntx;
    // the kTileY warps of a block are arranged 2^wx side by side in x and kTileY/2^wx in y
    const int warp = threadIdx.x >> 5;
    const int wx = warp & ((1 << P.warps_x_log2) - 1), wy = warp >> P.warps_x_log2;
    c.x = (bx << (5 + P.warps_x_log2)) + (wx << 5) + (threadIdx.x & 31);
    c.y0 = (by << (kTileRowsLog2 - P.warps_x_log2)) + 2 * wy;
    c.v0 = c.x < P.nx && c.y0 < P.ny;
    c.v1 = c.v0 && c.y0 + 1 < P.ny;
    const int xw = c.x == 0 ? P.nx - 1 : c.x - 1;
    const int xe = c.x == P.nx - 1 ? 0 : c.x + 1;
    const size_t row = (size_t)c.y0 * P.pitch;
    c.i0 = row + c.x;
    c.i1 = c.i0 + P.pitch;
    c.iw0 = row + xw;
    c.ie0 = row + xe;
    c.iw1 = c.iw0 + P.pitch;
    c.ie1 = c.ie0 + P.pitch;
    c.is0 = c.y0 > 0 ? c.i0 - P.pitch : c.i0;
    c.in1 = c.y0 + 2 < P.ny ? c.i1 + P.pitch : c.i1;
    return c;
}

// Five-point stencils of one field for both cells of a pair.  For the cell
// below, the north value is the upper cell; for the upper cell, the south value
// is the lower cell.  When the upper cell is outside the domain the lower cell
// is the top row and its north ghost is itself.
struct S2 {
    double c0, c1, w0, e0, w1, e1, s0, n1;
};
__device__ __forceinline__ S2 load_s2(const double* f, const Pair& c) {
    S2 s;
    s.c0 = f[c.i0];
    s.w0 = f[c.iw0];
    s.e0 = f[c.ie0];
    s.s0 = f[c.is0];
    if (c.v1) {
        s.c1 = f[c.i1];
        s.w1 = f[c.iw1];
        s.e1 = f[c.ie1];
        s.n1 = f[c.in1];
    } else {
        s.c1 = s.c0;
        s.w1 = s.e1 = s.n1 = 0;
    }
    return s;
}

// Face weights of implicit_diffusion's weights_at (pearl_serial.cpp:1022-1028)
struct Faces {
    double w0, w1, w2, w3;
};
// K is finite and nonnegative here (SET-UP runs only on a trial whose mixture
// passed its checks, pearl_serial.cpp:136), so div_force gives div_by's bits.
__device__ __forceinline__ double face_x(const DevParams& P, double k, double kn) {
    return div_force(P, .5 * (k + kn), P.dx2, P.r_dx2);
}
__device__ __forceinline__ double face_y(const DevParams& P, double k, double kn) {
    return div_force(P, .5 * (k + kn), P.dy2, P.r_dy2);
}
__device__ __forceinline__ Faces faces0(const DevParams& P, const S2& K, const Pair& c) {
    Faces f;
    f.w0 = face_x(P, K.c0, K.w0);
    f.w1 = face_x(P, K.c0, K.e0);
    f.w2 = face_y(P, K.c0, K.s0);
    f.w3 = face_y(P, K.c0, K.c1);
    if (c.y0 == 0) f.w2 = 0;
    if (c.y0 == P.ny - 1) f.w3 = 0;
    return f;
}
__device__ __forceinline__ Faces faces1(const DevParams& P, const S2& K, const Pair& c) {
    Faces f;
    f.w0 = face_x(P, K.c1, K.w1);
    f.w1 = face_x(P, K.c1, K.e1);
    f.w2 = face_y(P, K.c1, K.c0);
    f.w3 = face_y(P, K.c1, K.n1);
    if (c.y0 + 1 == P.ny - 1) f.w3 = 0;
    return f;
}

// apply (pearl_serial.cpp:1029-1035): chi*u + dt*sum_f w_f (u - u_f)
__device__ __forceinline__ double apply_at(double chi, double dt, const Faces& f, double u, double uw, double ue,
                                           double us, double un) {
    return chi * u + dt * (f.w0 * (u - uw) + f.w1 * (u - ue) + f.w2 * (u - us) + f.w3 * (u - un));
}
__device__ __forceinline__ double apply0(double chi, double dt, const Faces& f, const S2& u) {
    return apply_at(chi, dt, f, u.c0, u.w0, u.e0, u.s0, u.c1);
}
__device__ __forceinline__ double apply1(double chi, double dt, const Faces& f, const S2& u) {
    return apply_at(chi, dt, f, u.c1, u.w1, u.e1, u.c0, u.n1);
}
// conservative carbon change of the final update (pearl_serial.cpp:1085)
__device__ __forceinline__ double flux_at(double dt, const Faces& f, double u, double uw, double ue, double us,
                                          double un) {
    return dt * (f.w0 * (uw - u) + f.w1 * (ue - u) + f.w2 * (us - u) + f.w3 * (un - u));
}

// Per-cell reduced-energy density (pearl_serial.cpp:800-819) without the final
// dx*dy: cell terms, then the +x face, then the +y face unless at the top wall.
// chi/icpt are mixture(phi).susceptibility and composition(mu_ref, mixture(phi)).
struct Phi3 {
    double a, t, g;
};
#define DIVC(P, a, b, rb) (kForce ? div_force(P, a, b, rb) : div_by(P, a, b, rb))
// kForce: the final update's evaluation, whose divisions skip div_by's
// operand tests (div_force): the same value for a finite state, and a state
// that is not finite is rejected by valid_state before its energy is looked at.
template <bool kForce = false>
__device__ __forceinline__ double energy_cell(const DevParams& P, const Phi3& q, const Phi3& e, const Phi3& n,
                                              bool has_n, double carbon, double chi, double icpt) {
    const double triple = 2.0 * q.a * q.t * q.g;
    const double h0 = q.a * q.a * (3.0 - 2.0 * q.a) + triple;
    const double h1 = q.t * q.t * (3.0 - 2.0 * q.t) + triple;
    const double h2 = q.g * q.g * (3.0 - 2.0 * q.g) + triple;
    double chem = 0;
    chem += h0 * P.psi_t[0];
    chem += h1 * P.psi_t[1];
    chem += h2 * P.psi_t[2];
    if (!P.phase_only) {
        const double dc = carbon - icpt;
        chem += .5 * dc * dc / chi;
    }
    double t = DIVC(P, chem, P.Vm, P.r_Vm) + P.obs * (q.a * q.t + q.a * q.g + q.t * q.g) + P.tr * q.a * q.t * q.g;
    double z = DIVC(P, q.a * e.t - e.a * q.t, P.dx, P.r_dx);
    t += P.eps_sigma * z * z;
    z = DIVC(P, q.a * e.g - e.a * q.g, P.dx, P.r_dx);
    t += P.eps_sigma * z * z;
    z = DIVC(P, q.t * e.g - e.t * q.g, P.dx, P.r_dx);
    t += P.eps_sigma * z * z;
    if (has_n) {
        z = DIVC(P, q.a * n.t - n.a * q.t, P.dy, P.r_dy);
        t += P.eps_sigma * z * z;
        z = DIVC(P, q.a * n.g - n.a * q.g, P.dy, P.r_dy);
        t += P.eps_sigma * z * z;
        z = DIVC(P, q.t * n.g - n.t * q.g, P.dy, P.r_dy);
        t += P.eps_sigma * z * z;
    }
    return t;
}

// valid_state per cell (pearl_serial.cpp:1099-1114); true if the cell is bad.
// kForce: as energy_cell (a non-finite mu fails the test before its quotient).
template <bool kForce = false>
__device__ __forceinline__ bool bad_cell(const DevParams& P, const Phi3& q, double carbon, double mu) {
    bool good = true;
    double sum = 0;
    good = good && isfinite(q.a) && q.a >= -1e-12 && q.a <= 1 + 1e-12;
    sum += q.a;
    good = good && isfinite(q.t) && q.t >= -1e-12 && q.t <= 1 + 1e-12;
    sum += q.t;
    good = good && isfinite(q.g) && q.g >= -1e-12 && q.g <= 1 + 1e-12;
    sum += q.g;
    good = good && fabs(sum - 1) < 1e-10;
    good = good && isfinite(mu) && isfinite(carbon);
    if (!P.phase_only) {
        good = good && carbon >= -1e-10 && carbon <= 1 + 1e-10;
        const double qq[3] = {q.a, q.t, q.g};
#pragma unroll
        for (int a = 0; a < 3; ++a)
            if (qq[a] > .01) {
                const double ca = DIVC(P, mu - P.B[a], P.two_A[a], P.r_two_A[a]);
                good = good && ca >= -1e-10 && ca <= 1 + 1e-10;
            }
    }
    return !good;
}

#undef DIVC

__device__ __forceinline__ Phi3 load_phi(const double* const* ph, size_t i) { return Phi3{ph[0][i], ph[1][i], ph[2][i]}; }

// ------------------------------------------------------------------ grid reductions
struct PhaseClock {
    unsigned long long t_last;
    unsigned long long ns[kTagCount];
    unsigned cnt[kTagCount];
};

struct Red {
    const Dom& a;
    PhaseClock* clk;  // shared memory; used by thread 0 of block 0 only
    unsigned counter = 0;
    struct Pipe* pipe_ptr = nullptr;
    __device__ Red(const Dom& args, PhaseClock* c) : a(args), clk(c) {
        if (a.bid == 0 && threadIdx.x == 0) {
            clk->t_last = globaltimer_ns();
            for (int k = 0; k < kTagCount; ++k) {
                clk->ns[k] = 0;
                clk->cnt[k] = 0;
            }
        }
    }
    // publish the block partials, wait for the grid, combine; false on a device-wait timeout
    template <int NV>
    __device__ bool reduce(double (&v)[NV], unsigned ops, int tag) {
        // this thread's plane stores may be read by TMA (async proxy) after the barrier
        if (a.use_tma) fence_proxy_async();
        double* slot = a.part + (size_t)(counter & 1u) * a.nblk * kMaxRed;
        ++counter;
        block_publish<NV>(v, ops, slot, a.bid);
        if (!grid_barrier(a.bar, a.nblk)) return false;
        if (a.bid == 0 && threadIdx.x == 0) {
            const unsigned long long t = globaltimer_ns();
            clk->ns[tag] += t - clk->t_last;
            clk->cnt[tag] += 1;
            clk->t_last = t;
        }
        grid_gather<NV>(v, ops, slot, a.nblk);
        return true;
    }
    __device__ void flush() const {
        if (a.bid == 0 && threadIdx.x == 0)
            for (int k = 0; k < kTagCount; ++k) {
                a.B.ctl->phase_ns[k] = clk->ns[k];
                a.B.ctl->phase_count[k] = clk->cnt[k];
            }
    }
};

#define OPS2(a, b) ((unsigned)(a) | ((unsigned)(b) << 2))
#define OPS3(a, b, c) (OPS2(a, b) | ((unsigned)(c) << 4))
#define OPS4(a, b, c, d) (OPS3(a, b, c) | ((unsigned)(d) << 6))
#define OPS5(a, b, c, d, e) (OPS4(a, b, c, d) | ((unsigned)(e) << 8))

#define FOR_TILES(P) for (int t = a.bid; t < (P).ntiles; t += a.nblk)

// ------------------------------------------------------------------ stencil sources
// A phase body reads its input fields through a source that maps a field slot
// and a neighbour of one of the thread's two cells to a value.  GlobalSrc
// reads the planes directly; SmemSrc reads the tile staged by TMA.  The body,
// and therefore the arithmetic, is the same for both.
enum Dir : int { kC = 0, kW = 1, kE = 2, kS = 3, kN = 4 };

template <int NF, class T = double>
struct GlobalSrc {
    const T* f[NF];
    Pair c;
    __device__ __forceinline__ T v(int k, int cell, int dir) const {
        size_t i;
        if (cell == 0)
            i = dir == kC ? c.i0 : dir == kW ? c.iw0 : dir == kE ? c.ie0 : dir == kS ? c.is0 : (c.v1 ? c.i1 : c.i0);
        else
            i = dir == kC ? c.i1 : dir == kW ? c.iw1 : dir == kE ? c.ie1 : dir == kS ? c.i0 : c.in1;
        return f[k < NF ? k : 0][i];
    }
};

// Staged box geometry per element type: FP64 boxes start two cells left of the
// tile (36 columns), FP32 boxes four (40 columns), so that the box's x
// coordinate is a multiple of 16 bytes either way.
template <class T>
struct StageGeom;
template <>
struct StageGeom<double> {
    static constexpr int kHaloX = 2, kW = kBoxW, kStride = kFieldStride;
};
template <>
struct StageGeom<float> {
    static constexpr int kHaloX = 4, kW = kBoxW32, kStride = kFieldStride32;
};

template <int NF, class T = double>
struct SmemSrc {
    const T* base;       // stage base: field k at base + k*StageGeom<T>::kStride
    int lx, ly0;         // box column of x, box row of the lower cell
    bool south, v1, north1;
    int w;               // box row length (StageGeom<T>::kW with halo, kTileX without)
    __device__ __forceinline__ T v(int k, int cell, int dir) const {
        int ly = ly0 + cell, x = lx;
        if (dir == kW) x -= 1;
        if (dir == kE) x += 1;
        if (dir == kS) ly = cell == 0 ? (south ? ly - 1 : ly) : ly - 1;
        if (dir == kN) ly = cell == 0 ? (v1 ? ly + 1 : ly) : (north1 ? ly + 1 : ly);
        return base[k * StageGeom<T>::kStride + ly * w + x];
    }
};

// Both cells' five-point stencils of slot k (see S2); the upper cell's own
// neighbours are only read when it is inside the domain.
template <class Src>
__device__ __forceinline__ S2 stencil2(const Src& s, int k, bool v1) {
    S2 r;
    r.c0 = s.v(k, 0, kC);
    r.w0 = s.v(k, 0, kW);
    r.e0 = s.v(k, 0, kE);
    r.s0 = s.v(k, 0, kS);
    r.c1 = s.v(k, 0, kN);  // upper cell, or the lower cell itself at the top wall
    if (v1) {
        r.w1 = s.v(k, 1, kW);
        r.e1 = s.v(k, 1, kE);
        r.n1 = s.v(k, 1, kN);
    } else {
        r.w1 = r.e1 = r.n1 = 0;
    }
    return r;
}

// Face weights of cell `cell` of the pair from the stored east/north faces of
// this solve: the west face is the west neighbour's east face and the south
// face the south neighbour's north face (IEEE addition is commutative, so
// these equal weights_at's recomputation bitwise); zero at the walls.
template <class Src>
__device__ __forceinline__ Faces faces_stored(const Src& src, int se, int sn, int cell, const Pair& c) {
    Faces f;
    f.w0 = src.v(se, cell, kW);
    f.w1 = src.v(se, cell, kC);
    f.w2 = cell == 0 ? (c.y0 == 0 ? 0.0 : src.v(sn, 0, kS)) : src.v(sn, 0, kC);
    f.w3 = src.v(sn, cell, kC);
    return f;
}

// ------------------------------------------------------------------ TMA pipeline
// Stage s of the pipeline has a "full" barrier (one arrival with the expected
// bytes, completed by the copies); the block barrier that ends each tile frees
// the stage, and thread 0 then refills it with the tile S-1 ahead.  (Freeing
// stages warp by warp through "empty" barriers, so that a warp could run ahead
// into staged tiles, measured 1.686 against 1.683 ms/step with 512-thread
// blocks on 2048x4096, five runs each on one GPU, and was dropped.)
constexpr size_t kPipeHeaderBytes = 128;  // full[4] mbarriers
static_assert(kMaxStages * sizeof(uint64_t) <= kPipeHeaderBytes, "pipeline header");
struct Pipe {
    uint64_t* bar;     // kMaxStages "full" mbarriers in shared memory
    double* stage;     // stage buffers (kPipeDoubles)
    uint32_t parity;   // bit s: next completion phase expected on barrier s
};

__device__ __forceinline__ Pipe make_pipe(unsigned char* dsmem) {
    return Pipe{reinterpret_cast<uint64_t*>(dsmem), reinterpret_cast<double*>(dsmem + kPipeHeaderBytes), 0u};
}
// Thread 0 initialises the barriers; the caller synchronises the block after.
__device__ __forceinline__ void init_pipe(const Pipe& pp) {
    for (int s = 0; s < kMaxStages; ++s) mbar_init(&pp.bar[s], 1);
    mbar_fence_init();
}

// Bounded waits on a pipeline barrier.  A wait gives up after limit_ns, or
// early once another block of the group has recorded a device-wait timeout in
// *abort_status (the launch is failing, so waiting out the full limit again
// would only lengthen the error path).  Drains of in-flight copies pass no
// abort_status: they must wait for the copies themselves.
__device__ __forceinline__ bool wait_aborted(const int* abort_status) {
    return abort_status && *(const volatile int*)abort_status == (int)PEARL_ERR_DEVICE_WAIT;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  unsigned long long limit_ns = kBarrierTimeoutNs,
                                                  const int* abort_status = nullptr) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    for (unsigned it = 1;; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 63u) == 0 && (globaltimer_ns() - t0 > limit_ns || wait_aborted(abort_status))) return false;
    }
}
// Sweep the block's tiles, calling body(src, pair) for every tile whose first
// cell is inside the domain.  With TMA, field slot k of tile t is staged from
// tensor map maps[k]; slots whose bit is set in `stencil` also get the
// periodic x wrap patched from `planes`.  Returns false after a bounded wait
// ran out (the status is recorded; in-flight copies are drained, bounded).
// `reverse` walks the block's tiles from its last to its first: consecutive
// passes that alternate direction begin where the previous pass ended, on
// tiles whose planes are still in L2.  The direction is fixed per phase, so
// a run's sums do not depend on how it is split into launches.
template <int NF, bool kTileOnly = false, class T = double, class Body>
__device__ bool sweep(const Dom& a, Pipe& pp, const int (&maps)[NF], const T* const (&planes)[NF],
                      unsigned stencil, bool reverse, Body&& body) {
    using G_ = StageGeom<T>;
    const DevParams& P = a.P;
    const int G = a.nblk;
    const int nb = a.bid < P.ntiles ? (P.ntiles - 1 - a.bid) / G + 1 : 0;
    const auto tile_of = [&](int k) { return a.bid + (reverse ? nb - 1 - k : k) * G; };
    if (!a.use_tma) {
        for (int k = 0; k < nb; ++k) {
            const Pair c = pair_of(P, tile_of(k));
            if (!c.v0) continue;
            GlobalSrc<NF, T> src;
#pragma unroll
            for (int f = 0; f < NF; ++f) src.f[f] = planes[f];
            src.c = c;
            body(src, c);
        }
        return true;
    }
    constexpr size_t kStageElems = kPipeDoubles * sizeof(double) / sizeof(T);
    constexpr int S = (int)(kStageElems / ((size_t)NF * G_::kStride)) < kMaxStages
                          ? (int)(kStageElems / ((size_t)NF * G_::kStride))
                          : kMaxStages;
    static_assert(S >= 2, "pipeline needs two stages");
    T* const stage = reinterpret_cast<T*>(pp.stage);
    const auto issue = [&](int k) {  // one thread
        const int t = tile_of(k);
        const int bx = t % P.ntx, by = t / P.ntx;
        const int s = k % S;
        T* dst = stage + (size_t)s * NF * G_::kStride;
        // tile-only boxes start at the tile (x multiple of 32 cells); halo boxes
        // kHaloX cells left, one row up
        mbar_arrive_expect_tx(&pp.bar[s], NF * (uint32_t)sizeof(T) *
                                              (kTileOnly ? kTileX * kTileRows : (uint32_t)G_::kW * kBoxH));
#pragma unroll
        for (int f = 0; f < NF; ++f)
            tma_load_2d(dst + f * G_::kStride, &a.maps[maps[f]], bx * kTileX - (kTileOnly ? 0 : G_::kHaloX),
                        by * kTileRows - (kTileOnly ? 0 : 1), &pp.bar[s]);
    };
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // plain stores of the earlier passes (ordered by the grid barrier) before the
    // async reads of this sweep, by every thread that may issue copies (lane 0 of
    // each warp), once per sweep: no value that a sweep stages and uses is changed
    // by a plain store of the same sweep (a field written in a pass is either not
    // staged in it, or read only at the cells that the reading block itself
    // writes, after reading them)
    if (lane == 0) fence_proxy_async();
    // S-1 tiles ahead: the stage of tile k+S-1 is the one freed by the barrier ending tile k-1
    if (threadIdx.x == 0)
        for (int k = 0; k < S - 1 && k < nb; ++k) issue(k);
    for (int k = 0; k < nb; ++k) {
        const int s = k % S;
        if (threadIdx.x == 0 && k + S - 1 < nb) issue(k + S - 1);
        if (!mbar_wait_bounded(&pp.bar[s], (pp.parity >> s) & 1u, kBarrierTimeoutNs, &a.bar->status)) {
            atomicCAS(&a.bar->status, 0, (int)PEARL_ERR_DEVICE_WAIT);
            // drain the copies that may still be in flight, this tile's included
            // when the wait was cut short by another block's timeout, bounded
            for (int j = k; j < nb && j < k + S; ++j)
                mbar_wait_bounded(&pp.bar[j % S], (pp.parity >> (j % S)) & 1u, kBarrierTimeoutNs / 16);
            return false;
        }
        pp.parity ^= 1u << s;
        const int t = tile_of(k);
        const int bx = t % P.ntx, by = t / P.ntx;
        T* st = stage + (size_t)s * NF * G_::kStride;
        const bool left = bx == 0, right = (bx + 1) * kTileX >= P.nx;
        if (left || right) {
            // periodic wrap: box column of x=-1 from x=nx-1, box column of x=nx from x=0
            for (int idx = threadIdx.x; idx < NF * 2 * kBoxH; idx += kThreads) {
                const int f = idx / (2 * kBoxH), side = (idx / kBoxH) & 1, r = idx % kBoxH;
                if (!((stencil >> f) & 1u) || (side == 0 && !left) || (side == 1 && !right)) continue;
                int y = by * kTileRows - 1 + r;
                y = y < 0 ? 0 : (y > P.ny - 1 ? P.ny - 1 : y);
                const int col = side == 0 ? G_::kHaloX - 1 : P.nx - (bx * kTileX - G_::kHaloX);
                st[f * G_::kStride + r * G_::kW + col] = planes[f][(size_t)y * P.pitch + (side == 0 ? P.nx - 1 : 0)];
            }
            fence_proxy_async_shared();  // the patch's plain writes before the stage's next async refill
            __syncthreads();
        }
        const Pair c = pair_of(P, t);
        if (c.v0) {
            SmemSrc<NF, T> src =
                kTileOnly ? SmemSrc<NF, T>{st, lane, 2 * warp, c.y0 > 0, c.v1, c.y0 + 2 < P.ny, kTileX}
                          : SmemSrc<NF, T>{st, lane + G_::kHaloX, 2 * warp + 1, c.y0 > 0, c.v1, c.y0 + 2 < P.ny, G_::kW};
            body(src, c);
        }
        __syncthreads();  // every warp is done with stage s: it is refilled next iteration
    }
    return true;
}

// ------------------------------------------------------------------ phases
// propose_phi for cell `k` of the pair (pearl_serial.cpp:966-1001); slots 0-2
// hold phi, slot 3 holds mu.
struct Proposal {
    double z0, z1, z2, change;
    bool simplex_bad;
};
template <class Src>
__device__ __forceinline__ Proposal propose_cell(const DevParams& P, const Src& src, int k, double dt, bool south,
                                                 bool north) {
    const double q0 = src.v(0, k, kC), q1 = src.v(1, k, kC), q2 = src.v(2, k, kC);
    const double mu = src.v(3, k, kC);
    const double psi0 = psi(P, 2, mu);
    const double ps[3] = {psi(P, 0, mu), psi(P, 1, mu), psi0};
    const double q[3] = {q0, q1, q2};
    const double dtr[3] = {2.0 * q1 * q2, 2.0 * q0 * q2, 2.0 * q0 * q1};
    double f[3];
#pragma unroll
    for (int aa = 0; aa < 3; ++aa) {
        const double qa1 = q[(aa + 1) % 3], qa2 = q[(aa + 2) % 3];
        f[aa] = P.obs * (qa1 + qa2) + P.tr * qa1 * qa2;
        // b = gamma contributes (psi_g - psi_g)*dh/Vm = +-0, which leaves every
        // finite force unchanged (a non-finite dh makes the other terms
        // non-finite too), so only alpha and theta are added.
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const double dh = dtr[aa] + (b == aa ? 6.0 * q[b] * (1.0 - q[b]) : 0.0);
            f[aa] += div_force(P, (ps[b] - psi0) * dh, P.Vm, P.r_Vm);
        }
    }
    // four faces in the reference's order: -x, +x, -y (not at y=0), +y (not at the top)
#pragma unroll
    for (int dir = 0; dir < 4; ++dir) {
        if ((dir == 2 && !south) || (dir == 3 && !north)) continue;
        const int d = dir == 0 ? kW : dir == 1 ? kE : dir == 2 ? kS : kN;
        const double n[3] = {src.v(0, k, d), src.v(1, k, d), src.v(2, k, d)};
        const double d2 = dir < 2 ? P.dx2 : P.dy2, rd2 = dir < 2 ? P.r_dx2 : P.r_dy2;
#pragma unroll
        for (int aa = 0; aa < 3; ++aa)
#pragma unroll
            for (int b = aa + 1; b < 3; ++b) {
                const double w = div_force(P, P.two_eps_sigma * (q[aa] * n[b] - n[aa] * q[b]), d2, rd2);
                f[aa] += w * n[b];
                f[b] -= w * n[aa];
            }
    }
    const double mean = div_force(P, f[0] + f[1] + f[2], 3.0, P.r_3);
    const double scale = dt / (local_tau(P, q0, q1, q2) * P.eps);
    Proposal o;
    o.z0 = q0 - scale * (f[0] - mean);
    o.z1 = q1 - scale * (f[1] - mean);
    o.z2 = q2 - scale * (f[2] - mean);
    o.simplex_bad = false;
    if (!(isfinite(o.z0) && isfinite(o.z1) && isfinite(o.z2))) {
        o.change = INFINITY;
        o.z0 = q0;
        o.z1 = q1;
        o.z2 = q2;
    } else {
        o.simplex_bad = !project_simplex(P, o.z0, o.z1, o.z2);
        o.change = fmax(fmax(fabs(o.z0 - q0), fabs(o.z1 - q1)), fabs(o.z2 - q2));
    }
    return o;
}

// propose_phi with the forces, local tau and increment in FP32 (mixed
// precision); the state stays FP64: z = q - (double)increment, and the
// projection and max |dphi| are FP64 as in propose_cell.
template <class Src>
__device__ __forceinline__ Proposal propose_cell_mixed(const DevParams& P, const Src& src, int k, double dt,
                                                       bool south, bool north) {
    const double q0 = src.v(0, k, kC), q1 = src.v(1, k, kC), q2 = src.v(2, k, kC);
    const float del = (float)(src.v(3, k, kC) - P.mu_ref);
    const float q[3] = {(float)q0, (float)q1, (float)q2};
    float dps[2];
#pragma unroll
    for (int b = 0; b < 2; ++b) dps[b] = __fmaf_rn(del, __fmaf_rn(del, P.m_pc[b], P.m_pb[b]), P.m_pa[b]);
    const float dtr[3] = {2.0f * q[1] * q[2], 2.0f * q[0] * q[2], 2.0f * q[0] * q[1]};
    float f[3];
#pragma unroll
    for (int aa = 0; aa < 3; ++aa) {
        const float qa1 = q[(aa + 1) % 3], qa2 = q[(aa + 2) % 3];
        f[aa] = P.m_obs * (qa1 + qa2) + P.m_tr * qa1 * qa2;
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const float dh = dtr[aa] + (b == aa ? 6.0f * q[b] * (1.0f - q[b]) : 0.0f);
            f[aa] += dps[b] * dh * P.m_rVm;
        }
    }
#pragma unroll
    for (int dir = 0; dir < 4; ++dir) {
        if ((dir == 2 && !south) || (dir == 3 && !north)) continue;
        const int d = dir == 0 ? kW : dir == 1 ? kE : dir == 2 ? kS : kN;
        const float n[3] = {(float)src.v(0, k, d), (float)src.v(1, k, d), (float)src.v(2, k, d)};
        const float kk = dir < 2 ? P.m_kx : P.m_ky;
#pragma unroll
        for (int aa = 0; aa < 3; ++aa)
#pragma unroll
            for (int b = aa + 1; b < 3; ++b) {
                const float w = kk * __fmaf_rn(q[aa], n[b], -n[aa] * q[b]);
                f[aa] = __fmaf_rn(w, n[b], f[aa]);
                f[b] = __fmaf_rn(-w, n[aa], f[b]);
            }
    }
    const float mean = (f[0] + f[1] + f[2]) * (1.0f / 3.0f);
    const float w0 = q[0] * q[1], w1 = q[0] * q[2], w2 = q[1] * q[2], ws = w0 + w1 + w2;
    const float tau = ws > 1e-30f ? (w0 * P.m_tau[0] + w1 * P.m_tau[1] + w2 * P.m_tau[2]) / ws : P.m_tau_min;
    const float scale = (float)(dt / ((double)tau * P.eps));
    Proposal o;
    o.z0 = q0 - (double)(scale * (f[0] - mean));
    o.z1 = q1 - (double)(scale * (f[1] - mean));
    o.z2 = q2 - (double)(scale * (f[2] - mean));
    o.simplex_bad = false;
    if (!(isfinite(o.z0) && isfinite(o.z1) && isfinite(o.z2))) {
        o.change = INFINITY;
        o.z0 = q0;
        o.z1 = q1;
        o.z2 = q2;
    } else {
        o.simplex_bad = !project_simplex(P, o.z0, o.z1, o.z2);
        o.change = fmax(fmax(fabs(o.z0 - q0), fabs(o.z1 - q1)), fabs(o.z2 - q2));
    }
    return o;
}

// PROPOSE: propose_phi from state `cur` into state `1-cur`, then the mixture of
// the trial phi (K, chi, icpt); in phase_only mode also the reconstructed
// trial carbon and the copied trial mu (pearl_serial.cpp:1134-1136).
// Reduction: {max |dphi| (inf if non-finite), mixture invalid, simplex failed}.
__device__ bool phase_propose(const Dom& a, Red& red, int cur, double dt, double& change, bool& mixbad,
                              bool& simplexbad) {
    const DevParams& P = a.P;
    const DevBufs& B = a.B;
    double* const* tp = B.phi[cur ^ 1];
    double vchange = 0, vmix = 0, vsimp = 0;
    const int maps[4] = {kMapState + 5 * cur, kMapState + 5 * cur + 1, kMapState + 5 * cur + 2,
                         kMapState + 5 * cur + 4};
    const double* const planes[4] = {B.phi[cur][0], B.phi[cur][1], B.phi[cur][2], B.mu[cur]};
    // the FP64 and the mixed-precision proposal are separate sweeps, so each
    // loop is register-allocated on its own
    const auto body = [&](auto mixed_tag, const auto& src, const Pair& c) {
#pragma unroll 1
        for (int k = 0; k < 2; ++k) {
            if (k == 1 && !c.v1) break;
            const int y = c.y0 + k;
            const size_t i = k ? c.i1 : c.i0;
            const Proposal o = decltype(mixed_tag)::value ? propose_cell_mixed(P, src, k, dt, y > 0, y < P.ny - 1)
                                                          : propose_cell(P, src, k, dt, y > 0, y < P.ny - 1);
            if (o.change == INFINITY)
                vchange = INFINITY;
            else
                vchange = fmax(vchange, o.change);
            if (o.simplex_bad) vsimp = 1;
            tp[0][i] = o.z0;
            tp[1][i] = o.z1;
            tp[2][i] = o.z2;
            double chi, cint, K;
            if (!mixture(P, o.z0, o.z1, o.z2, chi, cint, K)) vmix = 1;
            B.K[i] = K;
            B.chi[i] = chi;
            B.icpt[i] = fma(chi, P.mu_ref, cint);
            if (P.phase_only) {
                const double mu = src.v(3, k, kC);
                B.c[cur ^ 1][i] = fma(chi, mu, cint);
                B.mu[cur ^ 1][i] = mu;
            }
        }
    };
    const bool ok =
        P.mixed ? sweep<4>(a, *red.pipe_ptr, maps, planes, 0x7u, true,
                           [&](const auto& src, const Pair& c) { body(std::true_type{}, src, c); })
                : sweep<4>(a, *red.pipe_ptr, maps, planes, 0x7u, true,
                           [&](const auto& src, const Pair& c) { body(std::false_type{}, src, c); });
    if (!ok) return false;
    double v[3] = {vchange, vmix, vsimp};
    if (!red.reduce<3>(v, OPS3(kMax, kMax, kMax), kTagPropose)) return false;
    change = v[0];
    mixbad = v[1] != 0;
    simplexbad = v[2] != 0;
    return true;
}

// MIX: K, chi, icpt of the trial phi (used when the trial phi was uploaded).
__device__ bool phase_mix(const Dom& a, Red& red, int cur, bool& mixbad) {
    const DevParams& P = a.P;
    const DevBufs& B = a.B;
    double* const* tp = B.phi[cur ^ 1];
    double vmix = 0;
    FOR_TILES(P) {
        const Pair c = pair_of(P, t);
        for (int k = 0; k < 2; ++k) {
            if (!(k ? c.v1 : c.v0)) continue;
            const size_t i = k ? c.i1 : c.i0;
            double chi, cint, K;
            if (!mixture(P, tp[0][i], tp[1][i], tp[2][i], chi, cint, K)) vmix = 1;
            B.K[i] = K;
            B.chi[i] = chi;
            B.icpt[i] = fma(chi, P.mu_ref, cint);
        }
    }
    double v[1] = {vmix};
    if (!red.reduce<1>(v, kMax, kTagMix)) return false;
    mixbad = v[0] != 0;
    return true;
}

// SETUP: apply(mu_offset) and the initial residual (pearl_serial.cpp:1036-1046).
// Slots: K, mu (stencils), chi, icpt, c.  Reduction: {<rhs,rhs>, <r,z>, <r,r>}.
// kSolve32: the mixed form's set-up (FP32 copies for the inner solve); the FP64
// kernel is compiled without it.
template <bool kSolve32>
__device__ bool phase_setup(const Dom& a, Red& red, int cur, double dt, double& rhs2, double& rz, double& rr) {
    const DevParams& P = a.P;
    const DevBufs& B = a.B;
    double s0 = 0, s1 = 0, s2 = 0;
    const int maps[5] = {kMapK, kMapState + 5 * cur + 4, kMapChi, kMapIcpt, kMapState + 5 * cur + 3};
    const double* const planes[5] = {B.K, B.mu[cur], B.chi, B.icpt, B.c[cur]};
    const bool ok = sweep<5>(a, *red.pipe_ptr, maps, planes, 0x3u, false, [&](const auto& src, const Pair& c) {
        const S2 K = stencil2(src, 0, c.v1);
        S2 u = stencil2(src, 1, c.v1);
        u.c0 -= P.mu_ref; u.c1 -= P.mu_ref; u.w0 -= P.mu_ref; u.e0 -= P.mu_ref;
        u.w1 -= P.mu_ref; u.e1 -= P.mu_ref; u.s0 -= P.mu_ref; u.n1 -= P.mu_ref;
        // the cell's set-up values; the mixed solve keeps the residual and the
        // Jacobi step in FP32 (FP32 copies of the solve's coefficients too) and
        // sums <r,z> of those, <r,r> of the FP64 residual
        const auto store = [&](size_t i, double chi, const Faces& f, double u0, double rhs, double r, double diag) {
            B.wE[i] = f.w1;
            B.wN[i] = f.w3;
            B.x[i] = u0;
            if constexpr (kSolve32) {
                const float r32 = (float)r, d32 = (float)diag, z32 = __fdiv_rn(r32, d32);
                B.wE32[i] = (float)f.w1;
                B.wN32[i] = (float)f.w3;
                B.chi32[i] = (float)chi;
                B.diag32[i] = d32;
                B.r32[i] = r32;
                B.z32[i] = z32;
                s1 += (double)r32 * (double)z32;
            } else {
                const double z = r / diag;
                B.r[i] = r;
                B.z[i] = z;
                B.diag[i] = diag;
                s1 += r * z;
            }
            s0 += rhs * rhs;
            s2 += r * r;
        };
        {
            const double chi = src.v(2, 0, kC), ic = src.v(3, 0, kC), cold = src.v(4, 0, kC);
            const Faces f = faces0(P, K, c);
            const double Au = apply0(chi, dt, f, u);
            const double diag = chi + dt * (f.w0 + f.w1 + f.w2 + f.w3);
            const double rhs = cold - ic;
            store(c.i0, chi, f, u.c0, rhs, rhs - Au, diag);
        }
        if (c.v1) {
            const double chi = src.v(2, 1, kC), ic = src.v(3, 1, kC), cold = src.v(4, 1, kC);
            const Faces f = faces1(P, K, c);
            const double Au = apply1(chi, dt, f, u);
            const double diag = chi + dt * (f.w0 + f.w1 + f.w2 + f.w3);
            const double rhs = cold - ic;
            store(c.i1, chi, f, u.c1, rhs, rhs - Au, diag);
        }
    });
    if (!ok) return false;
    double v[3] = {s0, s1, s2};
    if (!red.reduce<3>(v, OPS3(kSum, kSum, kSum), kTagSetup)) return false;
    rhs2 = v[0];
    rz = v[1];
    rr = v[2];
    return true;
}

// APPLY: p_new = z (first) or z + beta*p_old, written to p[pout]; Ap; <p,Ap>.
// Slots: wE, wN, z (stencils), chi, p_old (stencil).
__device__ bool phase_apply(const Dom& a, Red& red, double dt, bool first, double beta, int pout, double& pAp) {
    const DevBufs& B = a.B;
    double* pn = B.p[pout];
    double s = 0;
    const auto body = [&](const auto& src, const Pair& c) {
        S2 p = stencil2(src, 2, c.v1);
        if (!first) {
            const S2 po = stencil2(src, 4, c.v1);
            p.c0 = p.c0 + beta * po.c0;
            p.c1 = p.c1 + beta * po.c1;
            p.w0 = p.w0 + beta * po.w0;
            p.e0 = p.e0 + beta * po.e0;
            p.w1 = p.w1 + beta * po.w1;
            p.e1 = p.e1 + beta * po.e1;
            p.s0 = p.s0 + beta * po.s0;
            p.n1 = p.n1 + beta * po.n1;
        }
        const double Ap0 = apply0(src.v(3, 0, kC), dt, faces_stored(src, 0, 1, 0, c), p);
        pn[c.i0] = p.c0;
        B.Ap[c.i0] = Ap0;
        s += p.c0 * Ap0;
        if (c.v1) {
            const double Ap1 = apply1(src.v(3, 1, kC), dt, faces_stored(src, 0, 1, 1, c), p);
            pn[c.i1] = p.c1;
            B.Ap[c.i1] = Ap1;
            s += p.c1 * Ap1;
        }
    };
    bool ok;
    if (first) {
        const int maps[4] = {kMapWE, kMapWN, kMapZ, kMapChi};
        const double* const planes[4] = {B.wE, B.wN, B.z, B.chi};
        ok = sweep<4>(a, *red.pipe_ptr, maps, planes, 0x7u, true, body);
    } else {
        const int maps[5] = {kMapWE, kMapWN, kMapZ, kMapChi, pout ? kMapP0 : kMapP1};
        const double* const planes[5] = {B.wE, B.wN, B.z, B.chi, B.p[pout ^ 1]};
        ok = sweep<5>(a, *red.pipe_ptr, maps, planes, 0x17u, true, body);
    }
    if (!ok) return false;
    double v[1] = {s};
    if (!red.reduce<1>(v, kSum, kTagApply)) return false;
    pAp = v[0];
    return true;
}

// UPDATE: x += alpha p; r -= alpha Ap; z = r/diag; {<r,z>, <r,r>}.
// Slots (no stencils): x, p, r, Ap, diag.
__device__ bool phase_update(const Dom& a, Red& red, double alpha, int pcur, double& rz, double& rr) {
    const DevBufs& B = a.B;
    double s0 = 0, s1 = 0;
    const int maps[5] = {kMapXc, pcur ? kMapP1c : kMapP0c, kMapRc, kMapApc, kMapDiagc};
    const double* const planes[5] = {B.x, B.p[pcur], B.r, B.Ap, B.diag};
    const bool ok = sweep<5, true>(a, *red.pipe_ptr, maps, planes, 0x0u, false, [&](const auto& src, const Pair& c) {
        {
            const double x = src.v(0, 0, kC) + alpha * src.v(1, 0, kC), r = src.v(2, 0, kC) - alpha * src.v(3, 0, kC);
            const double z = r / src.v(4, 0, kC);
            B.x[c.i0] = x;
            B.r[c.i0] = r;
            B.z[c.i0] = z;
            s0 += r * z;
            s1 += r * r;
        }
        if (c.v1) {
            const double x = src.v(0, 1, kC) + alpha * src.v(1, 1, kC), r = src.v(2, 1, kC) - alpha * src.v(3, 1, kC);
            const double z = r / src.v(4, 1, kC);
            B.x[c.i1] = x;
            B.r[c.i1] = r;
            B.z[c.i1] = z;
            s0 += r * z;
            s1 += r * r;
        }
    });
    if (!ok) return false;
    double v[2] = {s0, s1};
    if (!red.reduce<2>(v, OPS2(kSum, kSum), kTagUpdate)) return false;
    rz = v[0];
    rr = v[1];
    return true;
}

// RESET: z = r/diag; <r,z>  (pearl_serial.cpp:1060-1064)
__device__ bool phase_reset(const Dom& a, Red& red, double& rz) {
    const DevParams& P = a.P;
    const DevBufs& B = a.B;
    double s = 0;
    FOR_TILES(P) {
        const Pair c = pair_of(P, t);
        for (int k = 0; k < 2; ++k) {
            if (!(k ? c.v1 : c.v0)) continue;
            const size_t i = k ? c.i1 : c.i0;
            const double r = B.r[i];
            const double z = r / B.diag[i];
            B.z[i] = z;
            s += r * z;
        }
    }
    double v[1] = {s};
    if (!red.reduce<1>(v, kSum, kTagReset)) return false;
    rz = v[0];
    return true;
}

// ------------------------------------------------------------------ mixed-precision solve
// The implicit system A u = rhs of the mixed form is solved by rounds of FP32
// Jacobi-PCG on the correction A d = r of the current FP64 unknown x, whose
// steps are accumulated into x in FP64; each round is closed by the FP64
// residual of x (a plain residual pass, or the final update when the round's
// own residual is already within the tolerance).  The operator, the
// preconditioner and the inner vectors are FP32 planes written by SETUP.
// APPLY32 stages its FP32 planes through the TMA pipeline (FP32 boxes); the
// pointwise UPDATE32 reads 16-byte groups directly.

struct F2 {
    float c0, c1, w0, e0, w1, e1, s0, n1;
};

// chi p + dt sum_f w_f (p - p_f) in FP32, with fused multiply-adds
__device__ __forceinline__ float apply32_at(float chi, float dt, float w0, float w1, float w2, float w3, float p,
                                            float pw, float pe, float ps, float pn) {
    float acc = w0 * (p - pw);
    acc = __fmaf_rn(w1, p - pe, acc);
    acc = __fmaf_rn(w2, p - ps, acc);
    acc = __fmaf_rn(w3, p - pn, acc);
    return __fmaf_rn(dt, acc, chi * p);
}

// Both cells' five-point FP32 stencils of slot k (the FP32 counterpart of
// stencil2, the same neighbour conventions).
template <class Src>
__device__ __forceinline__ F2 stencil2f(const Src& s, int k, bool v1) {
    F2 r;
    r.c0 = s.v(k, 0, kC);
    r.w0 = s.v(k, 0, kW);
    r.e0 = s.v(k, 0, kE);
    r.s0 = s.v(k, 0, kS);
    r.c1 = s.v(k, 0, kN);  // upper cell, or the lower cell itself at the top wall
    if (v1) {
        r.w1 = s.v(k, 1, kW);
        r.e1 = s.v(k, 1, kE);
        r.n1 = s.v(k, 1, kN);
    } else {
        r.w1 = r.e1 = r.n1 = 0.f;
    }
    return r;
}

// APPLY32: p = z (first) or z + beta p_old into p32[pout]; A p; <p,Ap> in FP64.
// The FP32 planes are staged through TMA like the FP64 passes' (FP32 boxes,
// kBoxW32 wide), or read from global memory when staging is off.
__device__ bool phase_apply32(const Dom& a, Red& red, double dt, bool first, double beta, int pout, double& pAp) {
    const DevBufs& B = a.B;
    float* __restrict__ pn = B.p32[pout];
    float* __restrict__ apo = B.Ap32;
    const float dtf = (float)dt, bf = (float)beta;
    double s = 0;
    const auto body = [&](const auto& src, const Pair& c) {
        F2 p = stencil2f(src, 2, c.v1);
        if (!first) {
            const F2 q = stencil2f(src, 4, c.v1);
            p.c0 = __fmaf_rn(bf, q.c0, p.c0);
            p.c1 = __fmaf_rn(bf, q.c1, p.c1);
            p.w0 = __fmaf_rn(bf, q.w0, p.w0);
            p.e0 = __fmaf_rn(bf, q.e0, p.e0);
            p.w1 = __fmaf_rn(bf, q.w1, p.w1);
            p.e1 = __fmaf_rn(bf, q.e1, p.e1);
            p.s0 = __fmaf_rn(bf, q.s0, p.s0);
            p.n1 = __fmaf_rn(bf, q.n1, p.n1);
        }
        // faces: west = the west neighbour's east face, south = the south neighbour's north face
        const float a0 = src.v(0, 0, kW), a1 = src.v(0, 0, kC), a2 = c.y0 == 0 ? 0.f : src.v(1, 0, kS),
                    a3 = src.v(1, 0, kC), x0 = src.v(3, 0, kC);
        float b0 = 0.f, b1 = 0.f, b3 = 0.f, x1 = 0.f;
        if (c.v1) {
            b0 = src.v(0, 1, kW);
            b1 = src.v(0, 1, kC);
            b3 = src.v(1, 1, kC);
            x1 = src.v(3, 1, kC);
        }
        const float ap0 = apply32_at(x0, dtf, a0, a1, a2, a3, p.c0, p.w0, p.e0, p.s0, p.c1);
        pn[c.i0] = p.c0;
        apo[c.i0] = ap0;
        s += (double)p.c0 * (double)ap0;
        if (c.v1) {
            const float ap1 = apply32_at(x1, dtf, b0, b1, a3, b3, p.c1, p.w1, p.e1, p.c0, p.n1);
            pn[c.i1] = p.c1;
            apo[c.i1] = ap1;
            s += (double)p.c1 * (double)ap1;
        }
    };
    // a first iteration stages no old direction (a single five-field sweep for
    // both cases has fewer spills but measured 1 % slower on the mixed step)
    bool ok;
    if (first) {
        const int maps[4] = {kMap32WE, kMap32WN, kMap32Z, kMap32Chi};
        const float* const planes[4] = {B.wE32, B.wN32, B.z32, B.chi32};
        ok = sweep<4, false, float>(a, *red.pipe_ptr, maps, planes, 0x7u, true, body);
    } else {
        const int maps[5] = {kMap32WE, kMap32WN, kMap32Z, kMap32Chi, pout ? kMap32P0 : kMap32P1};
        const float* const planes[5] = {B.wE32, B.wN32, B.z32, B.chi32, B.p32[pout ^ 1]};
        ok = sweep<5, false, float>(a, *red.pipe_ptr, maps, planes, 0x17u, true, body);
    }
    if (!ok) return false;
    double v[1] = {s};
    if (!red.reduce<1>(v, kSum, kTagApply32)) return false;
    pAp = v[0];
    return true;
}

// UPDATE32: x += alpha p (FP64); r -= alpha Ap; z = r/diag; {<r,z>, <r,r>} in FP64.
// Pointwise, so it runs over groups of four consecutive cells of a row: one
// 16-byte load per FP32 plane and two per FP64 plane a group (rows start on
// 128 bytes and the pitch is a multiple of 32 cells), which keeps enough bytes
// in flight without a staging pipeline.  Group g belongs to thread g mod
// (blocks x threads) of the block group, a fixed assignment, so the sums are
// deterministic; cells of the row padding (x >= nx) keep their values and add
// nothing.
__device__ bool phase_update32(const Dom& a, Red& red, double alpha, int pcur, double& rz, double& rr) {
    const DevParams& P = a.P;
    const DevBufs& B = a.B;
    const float* __restrict__ p = B.p32[pcur];
    const float* __restrict__ ap = B.Ap32;
    const float* __restrict__ dg = B.diag32;
    float* __restrict__ r32 = B.r32;
    float* __restrict__ z32 = B.z32;
    double* __restrict__ x = B.x;
    const float af = (float)alpha;
    double s0 = 0, s1 = 0;
    const int gpr = P.pitch / 4;
    const long long ng = (long long)gpr * P.ny;
    for (long long g = (long long)a.bid * kThreads + threadIdx.x; g < ng; g += (long long)a.nblk * kThreads) {
        const int y = (int)(g / gpr), x0 = (int)(g % gpr) * 4;
        if (x0 >= P.nx) continue;
        const size_t i = (size_t)y * P.pitch + x0;
        const float4 pv = *reinterpret_cast<const float4*>(p + i);
        const float4 av = *reinterpret_cast<const float4*>(ap + i);
        const float4 dv = *reinterpret_cast<const float4*>(dg + i);
        float4 rv = *reinterpret_cast<const float4*>(r32 + i);
        double2 xa = *reinterpret_cast<const double2*>(x + i), xb = *reinterpret_cast<const double2*>(x + i + 2);
        float4 zv = *reinterpret_cast<const float4*>(z32 + i);
        const float pp[4] = {pv.x, pv.y, pv.z, pv.w}, aa[4] = {av.x, av.y, av.z, av.w};
        const float dd[4] = {dv.x, dv.y, dv.z, dv.w};
        float rr4[4] = {rv.x, rv.y, rv.z, rv.w}, zz[4] = {zv.x, zv.y, zv.z, zv.w};
        double xx[4] = {xa.x, xa.y, xb.x, xb.y};
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            if (x0 + c >= P.nx) break;
            const float r = __fmaf_rn(-af, aa[c], rr4[c]), z = __fdiv_rn(r, dd[c]);
            xx[c] = xx[c] + alpha * (double)pp[c];
            rr4[c] = r;
            zz[c] = z;
            s0 += (double)r * (double)z;
            s1 += (double)r * (double)r;
        }
        *reinterpret_cast<float4*>(r32 + i) = make_float4(rr4[0], rr4[1], rr4[2], rr4[3]);
        *reinterpret_cast<float4*>(z32 + i) = make_float4(zz[0], zz[1], zz[2], zz[3]);
        *reinterpret_cast<double2*>(x + i) = make_double2(xx[0], xx[1]);
        *reinterpret_cast<double2*>(x + i + 2) = make_double2(xx[2], xx[3]);
    }
    double v[2] = {s0, s1};
    if (!red.reduce<2>(v, OPS2(kSum, kSum), kTagUpdate)) return false;
    rz = v[0];
    rr = v[1];
    return true;
}

// RESID32: the FP64 residual r = rhs - A x of the accumulated unknown (as the
// final update's), handed to the next FP32 round: r32 = r, z32 = r32/diag.
// Slots: wE, wN, x (stencils), chi, c, icpt.  Reduction {<r,r> FP64, <r32,z32>}.
__device__ bool phase_resid32(const Dom& a, Red& red, int cur, double dt, double& rr, double& rz) {
    const DevBufs& B = a.B;
    double s0 = 0, s1 = 0;
    const int maps[6] = {kMapWE, kMapWN, kMapX, kMapChi, kMapState + 5 * cur + 3, kMapIcpt};
    const double* const planes[6] = {B.wE, B.wN, B.x, B.chi, B.c[cur], B.icpt};
    const bool ok = sweep<6>(a, *red.pipe_ptr, maps, planes, 0x7u, true, [&](const auto& src, const Pair& c) {
#pragma unroll 1
        for (int k = 0; k < 2; ++k) {
            if (k == 1 && !c.v1) break;
            const size_t i = k ? c.i1 : c.i0;
            const Faces f = faces_stored(src, 0, 1, k, c);
            const double u = src.v(2, k, kC);
            const double r = (src.v(4, k, kC) - src.v(5, k, kC)) -
                             apply_at(src.v(3, k, kC), dt, f, u, src.v(2, k, kW), src.v(2, k, kE), src.v(2, k, kS),
                                      src.v(2, k, kN));
            const float r32 = (float)r, z32 = __fdiv_rn(r32, B.diag32[i]);
            B.r32[i] = r32;
            B.z32[i] = z32;
            s0 += r * r;
            s1 += (double)r32 * (double)z32;
        }
    });
    if (!ok) return false;
    double v[2] = {s0, s1};
    if (!red.reduce<2>(v, OPS2(kSum, kSum), kTagTrueRes)) return false;
    rr = v[0];
    rz = v[1];
    return true;
}

// RESET32: after a final update whose true residual missed, that residual
// (written by FINAL in FP64) starts the next FP32 round.  Reduction {<r32,z32>}.
__device__ bool phase_reset32(const Dom& a, Red& red, double& rz) {
    const DevParams& P = a.P;
    const DevBufs& B = a.B;
    double s = 0;
    FOR_TILES(P) {
        const Pair c = pair_of(P, t);
        for (int k = 0; k < 2; ++k) {
            if (!(k ? c.v1 : c.v0)) continue;
            const size_t i = k ? c.i1 : c.i0;
            const float r32 = (float)B.r[i], z32 = __fdiv_rn(r32, B.diag32[i]);
            B.r32[i] = r32;
            B.z32[i] = z32;
            s += (double)r32 * (double)z32;
        }
    }
    double v[1] = {s};
    if (!red.reduce<1>(v, kSum, kTagReset)) return false;
    rz = v[0];
    return true;
}

// FINAL: the true residual check of the converged solve (pearl_serial.cpp:1051-1055)
// fused with the carbon update, closure and mu (:1082-1093), valid_state,
// total_carbon and reduced_energy of the trial state.  Everything after the
// residual is speculative: the caller uses it only when the residual passes,
// and otherwise restarts CG from the r written here.  The two cells of a
// thread are processed one after the other (this phase carries the most live
// values).  Slots: wE, wN, x, phi_a, phi_t, phi_g (stencils), c, chi, icpt.
// Reduction: {closure max, bad max, carbon sum, energy sum, <r,r>}.
__device__ bool phase_final(const Dom& a, Red& red, int cur, double dt, double& closure, bool& bad,
                            double& mass, double& energy, double& rr) {
    const DevParams& P = a.P;
    const DevBufs& B = a.B;
    const int tr = cur ^ 1;
    double vclos = 0, vbad = 0, vmass = 0, ven = 0, vrr = 0;
    const int maps[9] = {kMapWE, kMapWN, kMapX, kMapState + 5 * tr, kMapState + 5 * tr + 1, kMapState + 5 * tr + 2,
                         kMapState + 5 * cur + 3, kMapChi, kMapIcpt};
    const double* const planes[9] = {B.wE, B.wN, B.x, B.phi[tr][0], B.phi[tr][1], B.phi[tr][2], B.c[cur], B.chi,
                                     B.icpt};
    const bool ok = sweep<9>(a, *red.pipe_ptr, maps, planes, 0x3Fu, true, [&](const auto& src, const Pair& c) {
#pragma unroll 1
        for (int k = 0; k < 2; ++k) {
            if (k == 1 && !c.v1) break;
            const int y = c.y0 + k;
            const size_t i = k ? c.i1 : c.i0;
            const bool has_n = y < P.ny - 1;
            const Faces f = faces_stored(src, 0, 1, k, c);
            const double u = src.v(2, k, kC);
            const double uw = src.v(2, k, kW), ue = src.v(2, k, kE), us = src.v(2, k, kS), un = src.v(2, k, kN);
            const double cold = src.v(6, k, kC);
            const double chi = src.v(7, k, kC), icpt = src.v(8, k, kC);
            const double r = (cold - icpt) - apply_at(chi, dt, f, u, uw, ue, us, un);
            B.r[i] = r;
            vrr += r * r;
            const double cn = cold + flux_at(dt, f, u, uw, ue, us, un);
            vclos = fmax(vclos, fabs(cn - (icpt + chi * u)));
            const double mun = P.mu_ref + (cn - icpt) / chi;
            B.c[tr][i] = cn;
            B.mu[tr][i] = mun;
            const Phi3 q{src.v(3, k, kC), src.v(4, k, kC), src.v(5, k, kC)};
            const Phi3 e{src.v(3, k, kE), src.v(4, k, kE), src.v(5, k, kE)};
            const Phi3 n = has_n ? Phi3{src.v(3, k, kN), src.v(4, k, kN), src.v(5, k, kN)} : Phi3{0, 0, 0};
            if (bad_cell<true>(P, q, cn, mun)) vbad = 1;
            vmass += cn;
            ven += energy_cell<true>(P, q, e, n, has_n, cn, chi, icpt);
        }
    });
    if (!ok) return false;
    double v[5] = {vclos, vbad, vmass, ven, vrr};
    if (!red.reduce<5>(v, OPS5(kMax, kMax, kSum, kSum, kSum), kTagFinal)) return false;
    closure = v[0];
    bad = v[1] != 0;
    mass = v[2] * P.dx * P.dy;
    energy = v[3] * P.dx * P.dy;
    rr = v[4];
    return true;
}

// Energy and validity of state set `s` whose mixture is recomputed from phi
// (ENERGY) or taken from the trial mixture buffers (phase-only FINAL).
// Accumulates in the same order as phase_final, so equal states give equal sums.
template <bool kFromBuffers>
__device__ void energy_sweep(const Dom& a, int s, double& ven, double& vmass, double& vmix, double& vbad) {
    const DevParams& P = a.P;
    const DevBufs& B = a.B;
    const double* const* ph = B.phi[s];
    FOR_TILES(P) {
        const Pair c = pair_of(P, t);
        if (!c.v0) continue;
        for (int k = 0; k < 2; ++k) {
            if (k == 1 && !c.v1) break;
            const size_t i = k ? c.i1 : c.i0;
            const size_t ie = k ? c.ie1 : c.ie0;
            const int y = c.y0 + k;
            const bool has_n = y < P.ny - 1;
            const size_t in = k ? c.in1 : c.i1;
            const Phi3 q = load_phi(ph, i), e = load_phi(ph, ie);
            const Phi3 n = has_n ? load_phi(ph, in) : Phi3{0, 0, 0};
            double chi = 1, icpt = 0;
            if (kFromBuffers) {
                chi = B.chi[i];
                icpt = B.icpt[i];
            } else if (!P.phase_only) {
                double cint, K;
                if (!mixture(P, q.a, q.t, q.g, chi, cint, K)) vmix = 1;
                icpt = fma(chi, P.mu_ref, cint);
            }
            const double cc = B.c[s][i];
            ven += energy_cell(P, q, e, n, has_n, cc, chi, icpt);
            vmass += cc;
            if (bad_cell(P, q, cc, B.mu[s][i])) vbad = 1;
        }
    }
}

// PHASE_ONLY FINAL: valid_state and reduced_energy of the trial state whose
// carbon and mu were written by PROPOSE.  Reduction: {bad max, energy sum}.
__device__ bool phase_final_phase_only(const Dom& a, Red& red, int cur, bool& bad, double& energy) {
    double ven = 0, vmass = 0, vmix = 0, vbad = 0;
    energy_sweep<true>(a, cur ^ 1, ven, vmass, vmix, vbad);
    double v[2] = {vbad, ven};
    if (!red.reduce<2>(v, OPS2(kMax, kSum), kTagFinalPhaseOnly)) return false;
    bad = v[0] != 0;
    energy = v[1] * a.P.dx * a.P.dy;
    return true;
}

// ENERGY: reduced_energy and total_carbon of state `s` (the e0, mass0 of
// advance, pearl_serial.cpp:1122-1123), plus mixture validity and
// valid_state.  Reduction: {energy sum, carbon sum, mixture invalid, bad}.
__device__ bool phase_energy(const Dom& a, Red& red, int s, double& energy, double& mass, bool& mixbad,
                             bool& bad) {
    double ven = 0, vmass = 0, vmix = 0, vbad = 0;
    energy_sweep<false>(a, s, ven, vmass, vmix, vbad);
    double v[4] = {ven, vmass, vmix, vbad};
    if (!red.reduce<4>(v, OPS4(kSum, kSum, kMax, kMax), kTagEnergy)) return false;
    energy = v[0] * a.P.dx * a.P.dy;
    mass = v[1] * a.P.dx * a.P.dy;
    mixbad = v[2] != 0;
    bad = v[3] != 0;
    return true;
}

__device__ __forceinline__ void set_error(const Dom& a, int status, int why) {
    if (a.bid == 0 && threadIdx.x == 0) {
        if (atomicCAS(&a.bar->status, 0, status) == 0) a.bar->why = why;
    }
}

// Implicit diffusion: SETUP, Jacobi-PCG (pearl_serial.cpp:1047-1080) and FINAL.
// Returns false only on a device-wait timeout.
struct DiffusionOut {
    bool ok;
    int it;
    double residual, closure, mass, energy;
    bool bad;
};

constexpr int kMixedMaxRounds = 16;  // FP32 rounds of one mixed solve before the attempt is rejected

// The mixed form's implicit diffusion: SETUP (FP64 residual, FP32 copies), FP32
// rounds, each closed by an FP64 residual, and FINAL once a residual is within
// the tolerance (pearl_serial.cpp:1010-1094 with the linear iteration
// replaced; the convergence test, the true-residual recheck, the conservative
// update and closure are the reference's).  One pass per loop turn, as in the
// FP64 solve: rr holds the residual estimate of the last pass (FP64 after
// SETUP, RESID32 and FINAL, FP32 after an inner update); o.it counts FP32
// iterations.
__device__ bool diffusion_mixed(const Dom& a, Red& red, int cur, double dt, DiffusionOut& o) {
    const DevParams& P = a.P;
    double rhs2, rz, rr;
    if (!phase_setup<true>(a, red, cur, dt, rhs2, rz, rr)) return false;
    const double tolerance = P.cg_atol + P.cg_rtol * sqrt(rhs2);
    double target = fmax(sqrt(rr) * P.inner_rtol, 0.5 * tolerance);  // this round's stop
    bool first = true;
    double beta = 0;
    int pbuf = 0, rounds = 1, it = 0;
    while (true) {
        o.it = it;
        o.residual = sqrt(rr);
        if (!isfinite(o.residual)) return true;
        if (o.residual <= tolerance) {
            // true residual and, speculatively, the update (pearl_serial.cpp:1051-1093)
            if (!phase_final(a, red, cur, dt, o.closure, o.bad, o.mass, o.energy, rr)) return false;
            o.residual = sqrt(rr);
            if (o.residual <= tolerance * 1.05) {
                o.ok = true;
                break;
            }
            o.closure = 0;
            o.bad = false;
            o.mass = 0;
            o.energy = 0;
            if (!phase_reset32(a, red, rz)) return false;
        } else if (!first && o.residual <= target) {
            // the round reached its stop: the FP64 residual of the accumulated unknown
            if (!phase_resid32(a, red, cur, dt, rr, rz)) return false;
        } else {
            if (it >= P.cg_max) return true;
            const int pout = pbuf ^ 1;
            double pAp;
            if (!phase_apply32(a, red, dt, first, beta, pout, pAp)) return false;
            pbuf = pout;
            if (!(pAp > 0) || !isfinite(pAp) || !isfinite(rz)) return true;
            double rz_next;
            if (!phase_update32(a, red, rz / pAp, pbuf, rz_next, rr)) return false;
            ++it;
            beta = rz_next / rz;
            rz = rz_next;
            first = false;
            continue;
        }
        // a new round from the FP64 residual just formed
        if (++rounds > kMixedMaxRounds) return true;
        target = fmax(sqrt(rr) * P.inner_rtol, 0.5 * tolerance);
        first = true;
    }
    o.ok = o.closure <= P.closure_tol;
    return true;
}

// kSolve32: the kernel of the mixed solve (diffusion_mixed); the FP64 kernels
// are compiled without it, so its registers do not weigh on their phases.
template <bool kSolve32>
__device__ bool diffusion(const Dom& a, Red& red, int cur, double dt, DiffusionOut& o) {
    const DevParams& P = a.P;
    o.ok = false;
    o.it = 0;
    o.residual = 0;
    o.closure = 0;
    o.bad = false;
    o.mass = 0;
    o.energy = 0;
    if constexpr (kSolve32) {
        return diffusion_mixed(a, red, cur, dt, o);
    }
    double rhs2, rz, rr;
    if (!phase_setup<false>(a, red, cur, dt, rhs2, rz, rr)) return false;
    const double tolerance = P.cg_atol + P.cg_rtol * sqrt(rhs2);
    bool first = true;
    double beta = 0;
    int pbuf = 0;  // p[pbuf] holds the current search direction
    for (int iteration = 0; iteration <= P.cg_max; ++iteration) {
        o.it = iteration;
        o.residual = sqrt(rr);
        if (!isfinite(o.residual)) return true;
        if (o.residual <= tolerance) {
            // true residual (pearl_serial.cpp:1051-1055) in the same pass as the final update
            if (!phase_final(a, red, cur, dt, o.closure, o.bad, o.mass, o.energy, rr)) return false;
            o.residual = sqrt(rr);
            if (o.residual <= tolerance * 1.05) {
                o.ok = true;
                break;
            }
            o.closure = 0;
            o.bad = false;
            o.mass = 0;
            o.energy = 0;
            if (!phase_reset(a, red, rz)) return false;
            first = true;
            continue;
        }
        if (iteration == P.cg_max) break;
        const int pout = pbuf ^ 1;
        double pAp;
        if (!phase_apply(a, red, dt, first, beta, pout, pAp)) return false;
        pbuf = pout;
        if (!(pAp > 0) || !isfinite(pAp) || !isfinite(rz)) return true;
        const double alpha = rz / pAp;
        double rz_next;
        if (!phase_update(a, red, alpha, pbuf, rz_next, rr)) return false;
        beta = rz_next / rz;
        rz = rz_next;
        first = false;
    }
    if (!o.ok) return true;
    o.ok = o.closure <= P.closure_tol;
    return true;
}

// One pearl::advance (pearl_serial.cpp:1119-1174) on the device.  All blocks
// execute it with identical scalars.  Returns false when the step ended with
// an error status (recorded in ctl) or a device-wait timeout.
struct StepState {
    pearl_scalars S;
    int cur;
    bool cache_valid;
    double e0, mass0;
};

template <bool kSolve32>
__device__ bool advance(const Dom& a, Red& red, StepState& st, double stop_time, pearl_step_info& info) {
    const DevParams& P = a.P;
    double dt = st.S.dt;
    if (P.dt_max < dt) dt = P.dt_max;
    if (stop_time - st.S.time < dt) dt = stop_time - st.S.time;
    if (!(dt > 0) || !isfinite(dt)) {
        set_error(a, PEARL_ERR_INVALID_ADVANCE_TIME, 0);
        return false;
    }
    if (!st.cache_valid) {
        double e, m;
        bool mixbad, bad;
        if (!phase_energy(a, red, st.cur, e, m, mixbad, bad)) return false;
        if (mixbad) {
            set_error(a, PEARL_ERR_MIXTURE, 0);
            return false;
        }
        st.e0 = P.check_energy ? e : 0;
        st.mass0 = P.phase_only ? 0 : m;
        st.cache_valid = true;
    }
    int why = PEARL_WHY_NONE;
    for (int attempt = 0; attempt <= P.max_retries; ++attempt) {
        pearl_step_info out;
        memset(&out, 0, sizeof out);
        out.retries = attempt;
        out.accepted_dt = dt;
        bool mixbad, simplexbad;
        if (!phase_propose(a, red, st.cur, dt, out.max_phase_change, mixbad, simplexbad)) return false;
        if (simplexbad) {
            set_error(a, PEARL_ERR_SIMPLEX, 0);
            return false;
        }
        bool good = isfinite(out.max_phase_change) && out.max_phase_change <= P.max_phase_change;
        why = PEARL_WHY_PHASE_INCREMENT;
        bool bad = false;
        double mass = 0, e1 = 0;
        if (good) {
            if (mixbad) {
                set_error(a, PEARL_ERR_MIXTURE, 0);
                return false;
            }
            if (P.phase_only) {
                if (!phase_final_phase_only(a, red, st.cur, bad, e1)) return false;
            } else {
                DiffusionOut d;
                if (!diffusion<kSolve32>(a, red, st.cur, dt, d)) return false;
                good = d.ok;
                out.cg_iterations = d.it;
                out.linear_residual = d.residual;
                out.closure = d.closure;
                why = PEARL_WHY_LINEAR_CLOSURE;
                bad = d.bad;
                mass = d.mass;
                e1 = d.energy;
            }
        }
        if (good) {
            good = !bad;
            why = PEARL_WHY_BOUNDS;
        }
        if (good && !P.phase_only) {
            good = fabs(mass - st.mass0) <= 1e-11 * fmax(fabs(st.mass0), P.mass_scale);
            why = PEARL_WHY_MASS;
        }
        if (good && P.check_energy) {
            out.energy_change = e1 - st.e0;
            const double tol = P.energy_atol + P.energy_rtol * fmax(fabs(st.e0), P.energy_scale);
            good = isfinite(e1) && e1 <= st.e0 + tol;
            why = PEARL_WHY_ENERGY;
        }
        if (good) {
            st.S.time = st.S.time + dt;
            st.S.step = st.S.step + 1;
            st.S.rejected = st.S.rejected + attempt;
            const double grown = dt * 1.1;
            st.S.dt = grown < P.dt_max ? grown : P.dt_max;
            st.cur ^= 1;
            st.e0 = P.check_energy ? e1 : 0;
            st.mass0 = P.phase_only ? 0 : mass;
            info = out;
            return true;
        }
        dt *= .5;
        if (dt < P.dt_min) {
            set_error(a, PEARL_ERR_REJECTED_BELOW_DT_MIN, why);
            return false;
        }
    }
    set_error(a, PEARL_ERR_RETRY_LIMIT, why);
    return false;
}

// Moving window on the device (maybe_shift + shift_rows, pearl_serial.cpp:2023-2071).
__device__ bool maybe_shift(const Dom& a, Red& red, StepState& st, int& rows_out) {
    const DevParams& P = a.P;
    const DevBufs& B = a.B;
    rows_out = 0;
    const int cur = st.cur;
    const double* g = B.phi[cur][2];
    double local = -1;
    FOR_TILES(P) {
        const Pair c = pair_of(P, t);
        for (int k = 0; k < 2; ++k) {
            const int y = c.y0 + k;
            if (!(k ? c.v1 : c.v0) || y == P.ny - 1) continue;
            const size_t i = k ? c.i1 : c.i0;
            const double av = 1 - 2 * g[i], bv = 1 - 2 * g[i + P.pitch];
            if (av >= 0 && bv < 0) local = fmax(local, ((y + 1) - .5 + av / (av - bv)) * P.dy);
        }
    }
    double v1[1] = {local};
    if (!red.reduce<1>(v1, kMax, kTagShift)) return false;
    const double front = v1[0];
    if (a.bid == 0 && threadIdx.x == 0) a.B.ctl->out[0] = front;
    if (front < a.shift_trigger) return true;
    const int rows = (int)floor((front - a.shift_target) / P.dy);
    double gmax = 0;
    FOR_TILES(P) {
        const Pair c = pair_of(P, t);
        for (int k = 0; k < 2; ++k) {
            if (!(k ? c.v1 : c.v0) || c.y0 + k >= rows) continue;
            gmax = fmax(gmax, g[k ? c.i1 : c.i0]);
        }
    }
    double v2[1] = {gmax};
    if (!red.reduce<1>(v2, kMax, kTagShift)) return false;
    if (v2[0] > 1e-6) {
        set_error(a, PEARL_ERR_UNSAFE_SHIFT, 0);
        return false;
    }
    if (rows <= 0 || rows >= P.ny || a.shift_c_gamma < 0 || a.shift_c_gamma > 1) {
        set_error(a, PEARL_ERR_INVALID_ARGUMENT, 0);
        return false;
    }
    const int nw = cur ^ 1;
    double removed = 0, vmix = 0, vnonfin = 0;
    FOR_TILES(P) {
        const Pair c = pair_of(P, t);
        for (int k = 0; k < 2; ++k) {
            if (!(k ? c.v1 : c.v0)) continue;
            const int y = c.y0 + k;
            const size_t i = k ? c.i1 : c.i0;
            if (y < rows) removed += B.c[cur][i] * P.dx * P.dy;
            double q0, q1, q2, cc;
            if (y + rows < P.ny) {
                const size_t j = i + (size_t)rows * P.pitch;
                q0 = B.phi[cur][0][j];
                q1 = B.phi[cur][1][j];
                q2 = B.phi[cur][2][j];
                cc = B.c[cur][j];
            } else {
                q0 = 0;
                q1 = 0;
                q2 = 1;
                cc = a.shift_c_gamma;
            }
            B.phi[nw][0][i] = q0;
            B.phi[nw][1][i] = q1;
            B.phi[nw][2][i] = q2;
            B.c[nw][i] = cc;
            double chi, cint, K;
            if (!mixture(P, q0, q1, q2, chi, cint, K)) vmix = 1;
            if (!isfinite(cc)) vnonfin = 1;
            B.mu[nw][i] = (cc - cint) / chi;  // close_mu / reconstruct_mu (:139-142, :789-792)
        }
    }
    double v3[3] = {removed, vmix, vnonfin};
    if (!red.reduce<3>(v3, OPS3(kSum, kMax, kMax), kTagShift)) return false;
    if (v3[1] != 0) {
        set_error(a, PEARL_ERR_MIXTURE, 0);
        return false;
    }
    if (v3[2] != 0) {
        set_error(a, PEARL_ERR_NONFINITE_CARBON, 0);
        return false;
    }
    const double added = rows * P.nx * a.shift_c_gamma * P.dx * P.dy;
    st.S.shift_distance += rows * P.dy;
    st.S.shifts++;
    st.S.carbon_added += added;
    st.S.carbon_removed += v3[0];
    st.cur = nw;
    st.cache_valid = false;
    rows_out = rows;
    return true;
}

// ------------------------------------------------------------------ initialisation
// Interface-only energy density of one cell (interface_energy_only,
// pearl_serial.cpp:822-842), without the final dx*dy.
__device__ __forceinline__ double interface_energy_cell(const DevParams& P, const Phi3& q, const Phi3& e,
                                                        const Phi3& n, bool has_n) {
    double t = P.obs * (q.a * q.t + q.a * q.g + q.t * q.g) + P.tr * q.a * q.t * q.g;
    double z = div_by(P, q.a * e.t - e.a * q.t, P.dx, P.r_dx);
    t += P.eps_sigma * z * z;
    z = div_by(P, q.a * e.g - e.a * q.g, P.dx, P.r_dx);
    t += P.eps_sigma * z * z;
    z = div_by(P, q.t * e.g - e.t * q.g, P.dx, P.r_dx);
    t += P.eps_sigma * z * z;
    if (has_n) {
        z = div_by(P, q.a * n.t - n.a * q.t, P.dy, P.r_dy);
        t += P.eps_sigma * z * z;
        z = div_by(P, q.a * n.g - n.a * q.g, P.dy, P.r_dy);
        t += P.eps_sigma * z * z;
        z = div_by(P, q.t * n.g - n.t * q.g, P.dy, P.r_dy);
        t += P.eps_sigma * z * z;
    }
    return t;
}

// Interface-only energy of state set `s` plus its phase-fraction sums.
// Reduction: {energy sum, sum phi_alpha, sum phi_theta, sum phi_gamma}.
__device__ bool phase_interface_energy(const Dom& a, Red& red, int s, double& energy, double* frac) {
    const DevParams& P = a.P;
    const double* const* ph = a.B.phi[s];
    double ven = 0, f0 = 0, f1 = 0, f2 = 0;
    FOR_TILES(P) {
        const Pair c = pair_of(P, t);
        if (!c.v0) continue;
        for (int k = 0; k < 2; ++k) {
            if (k == 1 && !c.v1) break;
            const size_t i = k ? c.i1 : c.i0;
            const bool has_n = c.y0 + k < P.ny - 1;
            const Phi3 q = load_phi(ph, i), e = load_phi(ph, k ? c.ie1 : c.ie0);
            const Phi3 n = has_n ? load_phi(ph, k ? c.in1 : c.i1) : Phi3{0, 0, 0};
            ven += interface_energy_cell(P, q, e, n, has_n);
            f0 += q.a;
            f1 += q.t;
            f2 += q.g;
        }
    }
    double v[4] = {ven, f0, f1, f2};
    if (!red.reduce<4>(v, OPS4(kSum, kSum, kSum, kSum), kTagSmooth)) return false;
    energy = v[0] * P.dx * P.dy;
    const double cells = (double)P.nx * P.ny;
    for (int k = 0; k < 3; ++k) frac[k] = v[1 + k] / cells;
    return true;
}

// Capillary force of smooth_interface_only (pearl_serial.cpp:892-917) written
// to the work planes x, r, z; reduction {max |force|}.
__device__ bool phase_smooth_force(const Dom& a, Red& red, int cur, double& force_max) {
    const DevParams& P = a.P;
    const DevBufs& B = a.B;
    const double* const* ph = B.phi[cur];
    double* fo[3] = {B.x, B.r, B.z};
    double vmax = 0;
    FOR_TILES(P) {
        const Pair c = pair_of(P, t);
        if (!c.v0) continue;
#pragma unroll 1
        for (int k = 0; k < 2; ++k) {
            if (k == 1 && !c.v1) break;
            const int y = c.y0 + k;
            const size_t i = k ? c.i1 : c.i0;
            const size_t iw = k ? c.iw1 : c.iw0, ie = k ? c.ie1 : c.ie0;
            const size_t is = k ? c.i0 : c.is0, in = k ? c.in1 : c.i1;
            const double q[3] = {ph[0][i], ph[1][i], ph[2][i]};
            double f[3];
#pragma unroll
            for (int aa = 0; aa < 3; ++aa) {
                const double qa1 = q[(aa + 1) % 3], qa2 = q[(aa + 2) % 3];
                f[aa] = P.obs * (qa1 + qa2) + P.tr * qa1 * qa2;
            }
#pragma unroll
            for (int dir = 0; dir < 4; ++dir) {
                if ((dir == 2 && y == 0) || (dir == 3 && y == P.ny - 1)) continue;
                const size_t j = dir == 0 ? iw : (dir == 1 ? ie : (dir == 2 ? is : in));
                const double n[3] = {ph[0][j], ph[1][j], ph[2][j]};
                const double d2 = dir < 2 ? P.dx2 : P.dy2, rd2 = dir < 2 ? P.r_dx2 : P.r_dy2;
#pragma unroll
                for (int aa = 0; aa < 3; ++aa)
#pragma unroll
                    for (int b = aa + 1; b < 3; ++b) {
                        const double w = div_by(P, P.two_eps_sigma * (q[aa] * n[b] - n[aa] * q[b]), d2, rd2);
                        f[aa] += w * n[b];
                        f[b] -= w * n[aa];
                    }
            }
            const double mean = div_by(P, f[0] + f[1] + f[2], 3.0, P.r_3);
#pragma unroll
            for (int aa = 0; aa < 3; ++aa) {
                const double v = f[aa] - mean;
                fo[aa][i] = v;
                vmax = fmax(vmax, fabs(v));
            }
        }
    }
    double v[1] = {vmax};
    if (!red.reduce<1>(v, kMax, kTagSmooth)) return false;
    force_max = v[0];
    return true;
}

// Backtracking trial of smooth_interface_only (pearl_serial.cpp:925-933):
// trial phi = project(phi - scale*force) into set cur^1.
// Reduction: {max |dphi|, simplex failed}.
__device__ bool phase_smooth_trial(const Dom& a, Red& red, int cur, double scale, double& change, bool& bad) {
    const DevParams& P = a.P;
    const DevBufs& B = a.B;
    const double* const* ph = B.phi[cur];
    double* const* tp = B.phi[cur ^ 1];
    double vch = 0, vbad = 0;
    FOR_TILES(P) {
        const Pair c = pair_of(P, t);
        for (int k = 0; k < 2; ++k) {
            if (!(k ? c.v1 : c.v0)) continue;
            const size_t i = k ? c.i1 : c.i0;
            const double q0 = ph[0][i], q1 = ph[1][i], q2 = ph[2][i];
            double z0 = q0 - scale * B.x[i], z1 = q1 - scale * B.r[i], z2 = q2 - scale * B.z[i];
            if (!(isfinite(z0) && isfinite(z1) && isfinite(z2)) || !project_simplex(P, z0, z1, z2)) vbad = 1;
            vch = fmax(vch, fabs(z0 - q0));
            vch = fmax(vch, fabs(z1 - q1));
            vch = fmax(vch, fabs(z2 - q2));
            tp[0][i] = z0;
            tp[1][i] = z1;
            tp[2][i] = z2;
        }
    }
    double v[2] = {vch, vbad};
    if (!red.reduce<2>(v, OPS2(kMax, kMax), kTagSmooth)) return false;
    change = v[0];
    bad = v[1] != 0;
    return true;
}

// smooth_interface_only (pearl_serial.cpp:869-958) on the phase fields of the
// current state.  Report layout in ctl->out: steps, converged, energy_initial,
// energy_final, final_relative_energy_change, final_max_phase_change,
// phase fractions before (3) and after (3).
__device__ bool smooth(const Dom& a, Red& red, StepState& st, double* rep) {
    const DevParams& P = a.P;
    const int max_steps = a.smooth_max_steps, min_steps = a.smooth_min_steps;
    const double energy_rtol = a.smooth_energy_rtol, max_change = a.smooth_max_phase_change;
    for (int k = 0; k < 12; ++k) rep[k] = 0;
    double frac[3];
    double e_init;
    if (!phase_interface_energy(a, red, st.cur, e_init, frac)) return false;
    for (int k = 0; k < 3; ++k) rep[6 + k] = frac[k];
    rep[2] = e_init;
    double previous = e_init;
    const double base_scale = .12 * fmin(P.dx2, P.dy2) / P.eps_sigma;
    int steps = 0;
    bool converged = false;
    double energy_final = 0, rel_final = 0, change_final = 0;
    for (int step = 1; step <= max_steps; ++step) {
        double force_max;
        if (!phase_smooth_force(a, red, st.cur, force_max)) return false;
        if (!isfinite(force_max)) {
            set_error(a, PEARL_ERR_SMOOTHING, 1);
            return false;
        }
        if (force_max == 0) {
            steps = step - 1;
            converged = true;
            rel_final = 0;
            change_final = 0;
            break;
        }
        double scale = fmin(base_scale, max_change / force_max);
        bool accepted = false;
        double new_energy = previous, actual_change = 0;
        for (int backtrack = 0; backtrack < 24 && !accepted; ++backtrack) {
            bool bad;
            if (!phase_smooth_trial(a, red, st.cur, scale, actual_change, bad)) return false;
            if (bad) {
                set_error(a, PEARL_ERR_SIMPLEX, 0);
                return false;
            }
            double f3[3];
            if (!phase_interface_energy(a, red, st.cur ^ 1, new_energy, f3)) return false;
            double big = 1.0;
            if (big < fabs(previous)) big = fabs(previous);
            if (big < fabs(e_init)) big = fabs(e_init);
            const double etol = 1e-14 * big;
            if (isfinite(new_energy) && new_energy <= previous + etol)
                accepted = true;
            else
                scale *= .5;
        }
        if (!accepted) {
            set_error(a, PEARL_ERR_SMOOTHING, 2);
            return false;
        }
        st.cur ^= 1;  // only the phase planes of the new set are meaningful here
        const double rel = fabs(previous - new_energy) / fmax(fabs(previous), 1e-300);
        steps = step;
        energy_final = new_energy;
        rel_final = rel;
        change_final = actual_change;
        previous = new_energy;
        if (step >= min_steps && rel < energy_rtol && actual_change < 1e-5) {
            converged = true;
            break;
        }
    }
    if (steps == 0) energy_final = e_init;
    double e_after;
    if (!phase_interface_energy(a, red, st.cur, e_after, frac)) return false;
    rep[0] = steps;
    rep[1] = converged ? 1 : 0;
    rep[3] = energy_final;
    rep[4] = rel_final;
    rep[5] = change_final;
    for (int k = 0; k < 3; ++k) rep[9 + k] = frac[k];
    st.cache_valid = false;
    return true;
}

// Sums of the mixture intercept and susceptibility (the mean_carbon solve of
// initialize, pearl_serial.cpp:1814-1822).  Reduction: {sum c0, sum chi, invalid}.
__device__ bool phase_mix_sums(const Dom& a, Red& red, int s, double& si, double& sc, bool& mixbad) {
    const DevParams& P = a.P;
    const double* const* ph = a.B.phi[s];
    double v0 = 0, v1 = 0, vb = 0;
    FOR_TILES(P) {
        const Pair c = pair_of(P, t);
        for (int k = 0; k < 2; ++k) {
            if (!(k ? c.v1 : c.v0)) continue;
            const size_t i = k ? c.i1 : c.i0;
            double chi, cint, K;
            if (!mixture(P, ph[0][i], ph[1][i], ph[2][i], chi, cint, K)) vb = 1;
            v0 += cint;
            v1 += chi;
        }
    }
    double v[3] = {v0, v1, vb};
    if (!red.reduce<3>(v, OPS3(kSum, kSum, kMax), kTagInit)) return false;
    si = v[0];
    sc = v[1];
    mixbad = v[2] != 0;
    return true;
}

// Uniform mu and the carbon it implies (initialize, pearl_serial.cpp:1823-1826).
// Reduction: {sum carbon, invalid}.
__device__ bool phase_init_composition(const Dom& a, Red& red, int s, double mu, double& mass, bool& mixbad) {
    const DevParams& P = a.P;
    const DevBufs& B = a.B;
    const double* const* ph = B.phi[s];
    double vm = 0, vb = 0;
    FOR_TILES(P) {
        const Pair c = pair_of(P, t);
        for (int k = 0; k < 2; ++k) {
            if (!(k ? c.v1 : c.v0)) continue;
            const size_t i = k ? c.i1 : c.i0;
            double chi, cint, K;
            if (!mixture(P, ph[0][i], ph[1][i], ph[2][i], chi, cint, K)) vb = 1;
            const double cc = fma(chi, mu, cint);
            B.mu[s][i] = mu;
            B.c[s][i] = cc;
            vm += cc;
        }
    }
    double v[2] = {vm, vb};
    if (!red.reduce<2>(v, OPS2(kSum, kMax), kTagInit)) return false;
    mass = v[0] * P.dx * P.dy;
    mixbad = v[1] != 0;
    return true;
}

// snapshot() reductions (pearl_serial.cpp:2266-2281) on state `s`.
__device__ bool snapshot(const Dom& a, Red& red, int s, double* out) {
    const DevParams& P = a.P;
    const DevBufs& B = a.B;
    const double* const* ph = B.phi[s];
    double minc = 1e300, maxc = -1e300, minmu = 1e300, maxmu = -1e300, sumerr = 0;
    FOR_TILES(P) {
        const Pair c = pair_of(P, t);
        for (int k = 0; k < 2; ++k) {
            if (!(k ? c.v1 : c.v0)) continue;
            const size_t i = k ? c.i1 : c.i0;
            const double cc = B.c[s][i], mu = B.mu[s][i];
            minc = fmin(minc, cc);
            maxc = fmax(maxc, cc);
            minmu = fmin(minmu, mu);
            maxmu = fmax(maxmu, mu);
            sumerr = fmax(sumerr, fabs(ph[0][i] + ph[1][i] + ph[2][i] - 1));
        }
    }
    double v[5] = {minc, maxc, minmu, maxmu, sumerr};
    if (!red.reduce<5>(v, OPS5(kMin, kMax, kMin, kMax, kMax), kTagSnapshot)) return false;
    for (int k = 0; k < 5; ++k) out[k] = v[k];
    return true;
}

// Copies the accepted state (set `cur`) and the diffusion solution u (the CG
// iterate x) into one tape slot, grid-stride over the padded planes.  No
// barrier is needed after it: the next step never writes set `cur`, and it
// rewrites x only in SETUP, which follows at least one grid barrier.
__device__ void record_tape(const Dom& a, int cur, double* slot) {
    const DevParams& P = a.P;
    const DevBufs& B = a.B;
    const size_t pe = (size_t)P.pitch * P.ny;
    const double* src[6] = {B.phi[cur][0], B.phi[cur][1], B.phi[cur][2], B.c[cur], B.mu[cur], B.x};
    for (size_t i = (size_t)a.bid * kThreads + threadIdx.x; i < pe; i += (size_t)a.nblk * kThreads)
#pragma unroll
        for (int f = 0; f < 6; ++f) slot[f * pe + i] = src[f][i];
}

// The persistent step kernel's body; kSolve32 selects the mixed form's inner
// solve (pearl_kernel_mixed), every other part is the same code.
template <bool kSolve32>
__device__ __forceinline__ void step_body(const KArgs& args) {
    const Dom a{args.P, args.B, args.maps, args.use_tma, (int)blockIdx.x, (int)gridDim.x, args.B.ctl, args.B.part,
                args.shift_trigger, args.shift_target, args.shift_c_gamma, args.smooth_max_steps,
                args.smooth_min_steps, args.smooth_energy_rtol, args.smooth_max_phase_change};
    Ctl* ctl = a.B.ctl;
    __shared__ PhaseClock clk;
    extern __shared__ __align__(128) unsigned char dsmem[];
    Pipe pipe = make_pipe(dsmem);
    if (a.use_tma) {
        if (threadIdx.x == 0) init_pipe(pipe);
        __syncthreads();
    }
    Red red(a, &clk);
    red.pipe_ptr = &pipe;
    StepState st;
    st.S = ctl->S;
    st.cur = ctl->cur;
    st.cache_valid = ctl->energy_valid != 0;
    st.e0 = ctl->e0;
    st.mass0 = ctl->mass0;
    const bool leader = blockIdx.x == 0 && threadIdx.x == 0;

    if (args.mode == kModeRun) {
        long long steps = 0, cg_total = 0;
        int cg_peak = 0, reached = 0;
        pearl_step_info last;
        memset(&last, 0, sizeof last);
        while (steps < args.L.max_steps) {
            if (!(st.S.time < args.L.end_time)) break;
            if (st.S.step >= args.L.config_max_steps) {
                set_error(a, PEARL_ERR_MAX_STEPS, 0);
                break;
            }
            pearl_step_info info;
            if (args.forced_dt) st.S.dt = args.forced_dt[steps];
            if (!advance<kSolve32>(a, red, st, args.L.stop_time, info)) break;
            if (args.dt_log && leader) args.dt_log[steps] = info.accepted_dt;
            if (args.hist && leader) args.hist[(args.hist_next + steps) % args.hist_cap] = info;
            if (args.tape) record_tape(a, st.cur, args.tape + args.tape_slot * steps);
            ++steps;
            cg_total += info.cg_iterations;
            cg_peak = info.cg_iterations > cg_peak ? info.cg_iterations : cg_peak;
            last = info;
            if (st.S.time >= args.L.stop_time - args.L.output_eps) {
                reached = 1;
                break;
            }
        }
        if (leader) {
            ctl->S = st.S;
            ctl->cur = st.cur;
            ctl->energy_valid = st.cache_valid ? 1 : 0;
            ctl->e0 = st.e0;
            ctl->mass0 = st.mass0;
            ctl->steps = steps;
            ctl->cg_total = cg_total;
            ctl->cg_peak = cg_peak;
            ctl->reached_stop = reached;
            ctl->last = last;
        }
        red.flush();
        return;
    }
    // the mixed-solve kernel runs only the run mode (the host launches every
    // other mode, none of which solves, in the FP64 kernel; a second solving
    // mode here would double the solve's code and its register pressure)
    if constexpr (kSolve32) return;
    if (args.mode == kModePropose) {
        double change;
        bool mixbad, simplexbad;
        if (!phase_propose(a, red, st.cur, args.dt, change, mixbad, simplexbad)) return;
        if (leader) {
            ctl->out[0] = change;
            ctl->iout[0] = mixbad;
            ctl->iout[1] = simplexbad;
        }
        red.flush();
        return;
    }
    if (args.mode == kModeMix) {
        bool mixbad;
        if (!phase_mix(a, red, st.cur, mixbad)) return;
        if (leader) ctl->iout[0] = mixbad;
        red.flush();
        return;
    }
    if (args.mode == kModeDiffusion) {
        DiffusionOut d;
        if (!diffusion<kSolve32>(a, red, st.cur, args.dt, d)) return;
        if (leader) {
            ctl->iout[0] = d.ok;
            ctl->iout[1] = d.it;
            ctl->out[0] = d.residual;
            ctl->out[1] = d.closure;
        }
        red.flush();
        return;
    }
    if (args.mode == kModeEnergy || args.mode == kModeValid) {
        double e, m;
        bool mixbad, bad;
        if (!phase_energy(a, red, st.cur, e, m, mixbad, bad)) return;
        if (leader) {
            ctl->out[0] = e;
            ctl->out[1] = m;
            ctl->iout[0] = mixbad;
            ctl->iout[1] = bad;
        }
        red.flush();
        return;
    }
    if (args.mode == kModeSnapshot) {
        double v[5];
        if (!snapshot(a, red, st.cur, v)) return;
        double e, m;
        bool mixbad, bad;
        if (!phase_energy(a, red, st.cur, e, m, mixbad, bad)) return;
        if (leader) {
            for (int k = 0; k < 5; ++k) ctl->out[k] = v[k];
            ctl->out[5] = m;
            ctl->out[6] = e;
            ctl->iout[0] = mixbad;
        }
        red.flush();
        return;
    }
    if (args.mode == kModeSmooth) {
        double rep[12];
        if (!smooth(a, red, st, rep)) return;
        if (leader) {
            for (int k = 0; k < 12; ++k) ctl->out[k] = rep[k];
            ctl->cur = st.cur;
            ctl->energy_valid = 0;
        }
        red.flush();
        return;
    }
    if (args.mode == kModeMixSums) {
        double si, sc;
        bool mixbad;
        if (!phase_mix_sums(a, red, st.cur, si, sc, mixbad)) return;
        if (leader) {
            ctl->out[0] = si;
            ctl->out[1] = sc;
            ctl->iout[0] = mixbad;
        }
        red.flush();
        return;
    }
    if (args.mode == kModeInitComposition) {
        double mass;
        bool mixbad;
        if (!phase_init_composition(a, red, st.cur, args.init_mu, mass, mixbad)) return;
        if (leader) {
            ctl->out[0] = mass;
            ctl->iout[0] = mixbad;
            ctl->energy_valid = 0;
        }
        red.flush();
        return;
    }
    if (args.mode == kModeMaybeShift) {
        int rows = 0;
        if (!maybe_shift(a, red, st, rows)) return;
        if (leader) {
            ctl->S = st.S;
            ctl->cur = st.cur;
            ctl->energy_valid = st.cache_valid ? 1 : 0;
            ctl->iout[0] = rows;
        }
        red.flush();
        return;
    }
}

__global__ void __launch_bounds__(kThreads, kMinBlocks) pearl_kernel(const __grid_constant__ KArgs args) {
    step_body<false>(args);
}
__global__ void __launch_bounds__(kThreads, kMinBlocks) pearl_kernel_mixed(const __grid_constant__ KArgs args) {
    step_body<true>(args);
}

// ------------------------------------------------------------------ batched instances
// A batch advances many independent instances (own grid size, parameters,
// dt, retries and CG count) in one cooperative launch.  The grid is split
// into groups of consecutive blocks (of equal or of per-instance sizes); each
// group runs the same `advance` device code on its own list of instances, one
// after another, with barriers and reductions local to the group.

template <bool kSolve32>
__device__ __forceinline__ void batch_body(const BatchArgs& args) {
    const int g = args.block_group[blockIdx.x];
    const int b0 = args.group_block0[g], nblk = args.group_block0[g + 1] - b0, bid = (int)blockIdx.x - b0;
    __shared__ PhaseClock clk;
    __shared__ DevParams sP;
    __shared__ DevBufs sB;
    extern __shared__ __align__(128) unsigned char dsmem[];
    Pipe pipe = make_pipe(dsmem);
    if (args.use_tma) {
        if (threadIdx.x == 0) init_pipe(pipe);
        __syncthreads();
    }
    Ctl* gctl = args.group_ctl + g;
    double* gpart = args.group_part + (size_t)b0 * 2 * kMaxRed;
    const bool leader = bid == 0 && threadIdx.x == 0;
    for (int j = args.first[g]; j < args.first[g + 1]; ++j) {
        const BatchInstance* I = args.inst + args.order[j];
        __syncthreads();
        if (threadIdx.x == 0) {
            sP = I->P;
            sB = I->B;
        }
        __syncthreads();
        const Dom a{sP, sB, I->maps, args.use_tma, bid, nblk, gctl, gpart, 0, 0, 0, 0, 0, 0, 0};
        Red red(a, &clk);
        red.pipe_ptr = &pipe;
        Ctl* ctl = sB.ctl;
        StepState st;
        st.S = ctl->S;
        st.cur = ctl->cur;
        st.cache_valid = ctl->energy_valid != 0;
        st.e0 = ctl->e0;
        st.mass0 = ctl->mass0;
        long long steps = 0, cg_total = 0;
        int cg_peak = 0, reached = 0;
        pearl_step_info last;
        memset(&last, 0, sizeof last);
        bool failed = false;
        while (steps < args.L.max_steps) {
            if (!(st.S.time < args.L.end_time)) break;
            if (st.S.step >= args.L.config_max_steps) {
                set_error(a, PEARL_ERR_MAX_STEPS, 0);
                failed = true;
                break;
            }
            pearl_step_info info;
            if (!advance<kSolve32>(a, red, st, args.L.stop_time, info)) {
                failed = true;
                break;
            }
            ++steps;
            cg_total += info.cg_iterations;
            cg_peak = info.cg_iterations > cg_peak ? info.cg_iterations : cg_peak;
            last = info;
            if (st.S.time >= args.L.stop_time - args.L.output_eps) {
                reached = 1;
                break;
            }
        }
        // a bounded wait that ran out leaves the group's barrier unusable: stop
        if (failed && *(volatile int*)&gctl->status == PEARL_ERR_DEVICE_WAIT) {
            if (leader) ctl->status = PEARL_ERR_DEVICE_WAIT;
            return;
        }
        if (leader) {
            ctl->S = st.S;
            ctl->cur = st.cur;
            ctl->energy_valid = st.cache_valid ? 1 : 0;
            ctl->e0 = st.e0;
            ctl->mass0 = st.mass0;
            ctl->steps = steps;
            ctl->cg_total = cg_total;
            ctl->cg_peak = cg_peak;
            ctl->reached_stop = reached;
            ctl->last = last;
            ctl->status = failed ? gctl->status : 0;
            ctl->why = failed ? gctl->why : 0;
            gctl->status = 0;
            gctl->why = 0;
        }
        red.flush();
    }
}

__global__ void __launch_bounds__(kThreads, kMinBlocks) pearl_batch_kernel(const __grid_constant__ BatchArgs args) {
    batch_body<false>(args);
}
__global__ void __launch_bounds__(kThreads, kMinBlocks)
    pearl_batch_kernel_mixed(const __grid_constant__ BatchArgs args) {
    batch_body<true>(args);
}

// Self-test of the exact constant-divisor division: counts elements where
// div_by(a, b, RN(1/b)) differs bitwise from the IEEE quotient a/b.
__global__ void division_selftest_kernel(const double* a, const double* b, const double* rb, long long n,
                                         unsigned long long* mismatches, int use_exact) {
    DevParams P;
    P.exact_div = use_exact;
    unsigned long long bad = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double q = div_by(P, a[i], b[i], rb[i]);
        const double ref = a[i] / b[i];
        if (__double_as_longlong(q) != __double_as_longlong(ref)) ++bad;
    }
    if (bad) atomicAdd(mismatches, bad);
}

// Self-test of the bounded grid-barrier wait: every block waits for one
// arrival more than the grid has, so no wait can complete; each gives up after
// kBarrierTimeoutNs and records PEARL_ERR_DEVICE_WAIT.
__global__ void wait_limit_selftest_kernel(Ctl* ctl) { grid_barrier(ctl, gridDim.x + 1u); }

#include "pearl_adjoint.cuh"

}  // namespace PEARL_GEOM_NS
}  // namespace pearl_gpu

