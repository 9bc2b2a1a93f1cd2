/*
 * pearl_gpu.h — C ABI of libpearl_gpu.so, the B200 (sm_100a) implementation of
 * the time-step hot path of the Pearl three-phase Fe-C pearlite phase-field
 * solver.
 *
 * The reference has no plugin or FFI layer: its hot path is the internal C++
 * call
 *     StepInfo pearl::advance(const Domain&, State&, const Thermo&,
 *                             const PhaseParameters&, const Controls&,
 *                             double mu_reference, double stop_time)
 * (pearl_serial.cpp:1119), called only from main's time loop
 * (pearl_serial.cpp:2296-2316).  This header is that boundary in C: plain
 * pointers and sizes, status codes instead of C++ exceptions, one device-
 * resident domain per context.  Each entry point names the reference
 * function or type it replaces.
 *
 * Conventions
 *  - Host arrays use the reference's gathered global layout
 *    (Domain::gather, pearl_serial.cpp:695-722): row-major (ny, nx), x fastest;
 *    phase fractions interleaved per cell as (alpha, theta, gamma).
 *    x (nx) is periodic, y (ny) has zero-flux walls.
 *  - The library owns all device memory; the caller owns host buffers.
 *  - Every call returns PEARL_OK (0) or a pearl_status code; the text of the
 *    last error, formatted like the reference's exception messages, is
 *    available from pearl_gpu_last_error().
 *  - A context is bound to one CUDA device and one stream; calls on the same
 *    context must not run concurrently from several host threads.
 */
#ifndef PEARL_GPU_H
#define PEARL_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define PEARL_GPU_ABI_VERSION 1

/* Physics and numerical controls of one run.
 * Replaces pearl::Thermo (pearl_serial.cpp:92), pearl::PhaseParameters
 * (:517-531), pearl::Controls (:767-773), the grid spacings of pearl::Domain
 * (:617) and the mu_reference argument of pearl::advance (:1119).
 * Thermodynamics are the run-temperature parabolas f_p(c) = A c^2 + B c + C,
 * phase index 0 alpha (ferrite), 1 theta (cementite), 2 gamma (austenite). */
typedef struct pearl_params {
    double A[3], B[3], C[3], D[3];
    double Vm, epsilon, sigma, triple;
    double tau[3]; /* tau_at, tau_ag, tau_tg */
    double dx, dy;
    double dt_max, dt_min, max_phase_change;
    double cg_rtol, cg_atol, closure_tol;
    double energy_rtol, energy_atol;
    int cg_max, max_retries, check_energy, phase_only;
    double mu_reference;
} pearl_params;

/* Scalar members of pearl::State (pearl_serial.cpp:758-764). */
typedef struct pearl_scalars {
    double time, dt, shift_distance, initial_carbon, carbon_added, carbon_removed;
    long long step, shifts, rejected;
} pearl_scalars;

/* pearl::StepInfo (pearl_serial.cpp:774-777). */
typedef struct pearl_step_info {
    double accepted_dt, max_phase_change, linear_residual, closure, energy_change;
    int cg_iterations, retries;
} pearl_step_info;

/* The contract of main's time loop (pearl_serial.cpp:2296-2316) for one call
 * of pearl_gpu_run: advance until an output time, the end time, a step budget
 * or an error, without returning to the host in between. */
typedef struct pearl_run_limits {
    long long max_steps;        /* accepted steps this call may take (>0) */
    long long config_max_steps; /* Config::max_steps: error once step >= this */
    double stop_time;           /* min(end_time, next_output) */
    double end_time;            /* loop runs while time < end_time */
    double output_eps;          /* 1e-12*max(end_time, output_dt): stop when time >= stop_time-eps */
} pearl_run_limits;

typedef struct pearl_run_report {
    long long steps;        /* accepted steps taken by this call */
    long long cg_total;     /* sum of StepInfo::cg_iterations */
    int cg_peak;            /* max StepInfo::cg_iterations */
    int reached_stop;       /* 1 if time >= stop_time - output_eps */
    pearl_step_info last;   /* StepInfo of the last accepted step */
} pearl_run_report;

/* Output-time reductions of main's snapshot() (pearl_serial.cpp:2266-2281). */
typedef struct pearl_diag {
    double c_min, c_max, mu_min, mu_max, phi_sum_error, mass, ledger, energy;
} pearl_diag;

typedef enum pearl_status {
    PEARL_OK = 0,
    PEARL_ERR_INVALID_ARGUMENT = 1,
    PEARL_ERR_CUDA = 2,
    PEARL_ERR_INVALID_ADVANCE_TIME = 3,   /* "invalid advance time" (:1121) */
    PEARL_ERR_REJECTED_BELOW_DT_MIN = 4,  /* "step rejected below dt_min: <why>" (:1171) */
    PEARL_ERR_RETRY_LIMIT = 5,            /* "step retry limit: <why>" (:1173) */
    PEARL_ERR_MIXTURE = 6,                /* "Invalid mixture coefficients" (:136) */
    PEARL_ERR_SIMPLEX = 7,                /* "Simplex projection failed" (:505) */
    PEARL_ERR_MAX_STEPS = 8,              /* "configured max_steps reached before end_time" (:2302) */
    PEARL_ERR_DEVICE_WAIT = 9,            /* a bounded device-side wait ran out (no reference counterpart) */
    PEARL_ERR_UNSAFE_SHIFT = 10,          /* "unsafe shift: removed strip contains gamma" (:2068) */
    PEARL_ERR_NONFINITE_CARBON = 11,      /* "Nonfinite total carbon" (:140) */
    PEARL_ERR_NO_DEVICE = 12,
    PEARL_ERR_TOO_LARGE = 13,             /* domain exceeds the no-allocation scratch (no reference counterpart) */
    PEARL_ERR_SMOOTHING = 14              /* "nonfinite smoothing force" (:920) or
                                             "sharp smoothing could not find an energy-decreasing step" (:940) */
} pearl_status;

/* Rejection reason <why> of the last attempt (pearl_serial.cpp:1133-1160). */
typedef enum pearl_why {
    PEARL_WHY_NONE = 0,
    PEARL_WHY_PHASE_INCREMENT = 1,  /* "phase increment" */
    PEARL_WHY_LINEAR_CLOSURE = 2,   /* "linear/closure" */
    PEARL_WHY_BOUNDS = 3,           /* "composition/phase bounds" */
    PEARL_WHY_MASS = 4,             /* "mass conservation" */
    PEARL_WHY_ENERGY = 5            /* "free-energy increase" */
} pearl_why;

/* pearl::SmoothReport (pearl_serial.cpp:844-853). */
typedef struct pearl_smooth_report {
    int steps, converged;
    double energy_initial, energy_final, final_relative_energy_change, final_max_phase_change;
    double phase_fraction_before[3], phase_fraction_after[3];
} pearl_smooth_report;

typedef struct pearl_gpu_ctx pearl_gpu_ctx;

/* Allocate one device-resident domain of nx*ny cells on `device`
 * (replaces pearl::Domain + pearl::State construction, pearl_serial.cpp:617, :763).
 * nx >= 3 and ny >= 2 as in Domain's constructor (:618). */
int pearl_gpu_create(const pearl_params* params, int nx, int ny, int device, pearl_gpu_ctx** out);
void pearl_gpu_destroy(pearl_gpu_ctx* ctx);

/* Run all work of this context on `stream` (a cudaStream_t; NULL = legacy default). */
int pearl_gpu_set_stream(pearl_gpu_ctx* ctx, void* stream);

/* Arithmetic of the step.  PEARL_PRECISION_FP64 (the default) is the
 * reference's arithmetic.  The mixed forms change two parts of it:
 *   - FP32 proposal: the propose_phi forces, local tau and phase increment in
 *     FP32 (the chemical-potential terms expanded about mu_reference with the
 *     offset formed in FP64); the projection and max |dphi| stay FP64;
 *   - FP32 inner solve: the implicit diffusion's linear system is solved by
 *     rounds of Jacobi-PCG in FP32 on the correction of the FP64 unknown,
 *     each round closed by its FP64 residual (iterative refinement); the
 *     convergence test on the FP64 residual, the true-residual recheck, the
 *     conservative carbon update and closure stay the reference's.
 * PEARL_PRECISION_MIXED has both, PEARL_PRECISION_MIXED_PROPOSE the first
 * only, PEARL_PRECISION_MIXED_SOLVE the second only.  The state, the mass and
 * energy reductions and every acceptance test stay FP64 in all of them.  A
 * form with the FP32 inner solve allocates its FP32 work planes (36 bytes per
 * cell) on first use.  No counterpart in the reference. */
enum {
    PEARL_PRECISION_FP64 = 0,
    PEARL_PRECISION_MIXED = 1,
    PEARL_PRECISION_MIXED_PROPOSE = 2,
    PEARL_PRECISION_MIXED_SOLVE = 3
};
int pearl_gpu_set_precision(pearl_gpu_ctx* ctx, int precision);

/* Replace the run parameters (same grid); invalidates cached step energies. */
int pearl_gpu_set_params(pearl_gpu_ctx* ctx, const pearl_params* params);

/* Host -> device state (Domain::load_global, pearl_serial.cpp:725-736).
 * phi_aos3[(y*nx+x)*3+a], carbon[y*nx+x], mu[y*nx+x]; scalars may be NULL. */
int pearl_gpu_upload(pearl_gpu_ctx* ctx, const double* phi_aos3, const double* carbon, const double* mu,
                     const pearl_scalars* scalars);
/* Device -> host state (Domain::gather, pearl_serial.cpp:695-722); any pointer may be NULL. */
int pearl_gpu_download(pearl_gpu_ctx* ctx, double* phi_aos3, double* carbon, double* mu, pearl_scalars* scalars);
int pearl_gpu_get_scalars(pearl_gpu_ctx* ctx, pearl_scalars* scalars);
int pearl_gpu_set_scalars(pearl_gpu_ctx* ctx, const pearl_scalars* scalars);

/* One accepted step: pearl::advance (pearl_serial.cpp:1119-1174).  On error
 * the state is unchanged and the status says why. */
int pearl_gpu_advance(pearl_gpu_ctx* ctx, double stop_time, pearl_step_info* out);

/* Many accepted steps in one device launch, deciding dt, retries and CG
 * termination on the GPU (main's loop body, pearl_serial.cpp:2296-2306). */
int pearl_gpu_run(pearl_gpu_ctx* ctx, const pearl_run_limits* limits, pearl_run_report* report);

/* Replays an accepted-dt sequence: n steps, step k attempted first with
 * accepted_dt[k] (host array) — the oracle replay of the reference
 * (advance with s.dt set to the accepted dt, pearl_serial.cpp:1120).  A step
 * whose forced dt is rejected retries with halved dt as usual, so a run that
 * cannot follow the sequence shows it in its time and rejection count. */
int pearl_gpu_run_replay(pearl_gpu_ctx* ctx, const double* accepted_dt, long long n, pearl_run_report* report);

/* Per-step history: with capacity > 0 the run loop records every accepted
 * step's pearl_step_info (accepted dt, retries, CG iterations, residual,
 * closure, ...) in a device ring of `capacity` entries, written inside the
 * persistent kernel (capacity 0 turns it off; each call restarts the count).
 * pearl_gpu_get_history copies the last min(recorded, capacity, max_entries)
 * entries, oldest first; *recorded receives the steps recorded since
 * pearl_gpu_set_history.  The reference keeps no such history
 * (VALIDATION.md:57-62); it is what replaying a run's dt sequence needs. */
int pearl_gpu_set_history(pearl_gpu_ctx* ctx, long long capacity);
int pearl_gpu_get_history(pearl_gpu_ctx* ctx, pearl_step_info* out, long long max_entries, long long* returned,
                          long long* recorded);

/* Moving window (maybe_shift + shift_rows, pearl_serial.cpp:2023-2071).
 * *rows receives the number of rows shifted (0 if the front is below trigger). */
int pearl_gpu_maybe_shift(pearl_gpu_ctx* ctx, double shift_trigger, double shift_target, double shift_gamma_carbon,
                          int* rows);

/* Output-time reductions of snapshot() (pearl_serial.cpp:2266-2281). */
int pearl_gpu_snapshot(pearl_gpu_ctx* ctx, pearl_diag* out);

/* ---- initialisation on the device (pearl::initialize, pearl_serial.cpp:1761-1837) ---- */
/* One filling command of the input file (parse_filling_operation,
 * pearl_serial.cpp:1197-1233): its method and its numeric parameters in input
 * order, already validated as validate_filling_operations (:1235-1349) does. */
enum {
    PEARL_FILL_CUBE = 1,                   /* FILLCUBE, 7 parameters */
    PEARL_FILL_CYLINDER = 2,               /* FILLCYLINDER, 6 */
    PEARL_FILL_CENTER_BOX_2D = 3,          /* FILLCENTERBOX2D, 6 */
    PEARL_FILL_Y_JUNCTION_2D = 4,          /* FILLYJUNCTION2D, 13 */
    PEARL_FILL_Y_JUNCTION_LAMELLAE_2D = 5, /* FILLYJUNCTIONLAMELLAE2D, 16 */
    PEARL_FILL_ADHERED_PEARLITE_ARM_2D = 6, /* FILLADHEREDPEARLITEARM2D, 11 */
    PEARL_FILL_PEARLITE_ELLIPSE_2D = 7     /* FILLPEARLITEELLIPSE2D, 11 */
};
#define PEARL_FILL_MAX_PARAMS 16
#define PEARL_FILL_MAX_OPS 256
typedef struct pearl_fill_op {
    int method; /* PEARL_FILL_* */
    int nparams;
    double p[PEARL_FILL_MAX_PARAMS];
} pearl_fill_op;
/* The "microsim" initial phases on the device: filling_phase_at
 * (pearl_serial.cpp:1393-1514) of every cell, the commands applied in input
 * order to a gamma background, written as one-hot phase fractions into the
 * context's current phase fields (carbon and mu are left as they are; the
 * step-energy carry is dropped).  The cosine and sine of every command's
 * angles are taken on the host with the reference's expressions; the cells'
 * arithmetic runs on the device in the reference's operation order.  Replaces
 * the host loop over cells of initialize (:1771-1772).  At most
 * PEARL_FILL_MAX_OPS commands; PEARL_ERR_INVALID_ARGUMENT for an unknown
 * method or a wrong parameter count. */
int pearl_gpu_fill(pearl_gpu_ctx* ctx, const pearl_fill_op* ops, int nops);
/* Capillarity-only smoothing of the current phase fields
 * (smooth_interface_only, pearl_serial.cpp:869-958). */
int pearl_gpu_smooth_interface(pearl_gpu_ctx* ctx, int max_steps, int min_steps, double energy_rtol,
                               double max_phase_change, pearl_smooth_report* out);
/* Sums over cells of mixture(phi).c_intercept and .susceptibility: the
 * mean_carbon chemical-potential solve (pearl_serial.cpp:1814-1822). */
int pearl_gpu_mixture_sums(pearl_gpu_ctx* ctx, double* sum_c_intercept, double* sum_chi);
/* mu = `mu` everywhere and carbon = composition(mu, mixture(phi))
 * (pearl_serial.cpp:1823-1826); *total_carbon receives total_carbon (:784-788). */
int pearl_gpu_init_composition(pearl_gpu_ctx* ctx, double mu, double* total_carbon);

/* ---- single hot-path functions, for per-function parity checks ---- */
/* propose_phi (pearl_serial.cpp:961-1002): writes the proposal into the trial buffer. */
int pearl_gpu_propose_phi(pearl_gpu_ctx* ctx, double dt, double* max_change);
/* Uploads phase fractions into the trial buffer (the trial.phi of implicit_diffusion). */
int pearl_gpu_upload_trial_phi(pearl_gpu_ctx* ctx, const double* phi_aos3);
/* implicit_diffusion (pearl_serial.cpp:1010-1094) on the trial phi; writes trial carbon and mu.
 * Always the reference's FP64 solve, whatever the context's precision (the
 * mixed forms' inner solve runs only inside pearl_gpu_advance / _run). */
int pearl_gpu_implicit_diffusion(pearl_gpu_ctx* ctx, double dt, int* ok, int* iterations, double* residual,
                                 double* closure);
int pearl_gpu_download_trial(pearl_gpu_ctx* ctx, double* phi_aos3, double* carbon, double* mu);
/* reduced_energy and total_carbon (pearl_serial.cpp:793-821, :784-788) of the current state. */
int pearl_gpu_energy_mass(pearl_gpu_ctx* ctx, double* energy, double* mass);
/* valid_state (pearl_serial.cpp:1096-1116) of the current state. */
int pearl_gpu_valid_state(pearl_gpu_ctx* ctx, int* valid);

/* ---- errors and accounting ---- */
const char* pearl_gpu_status_string(int status);
/* Message of the last failed call on this context (reference wording where one exists). */
const char* pearl_gpu_last_error(const pearl_gpu_ctx* ctx);
/* Device kernels launched by this context since creation; the grid size of the
 * persistent kernel; the device time of the last launch in milliseconds. */
int pearl_gpu_stats(const pearl_gpu_ctx* ctx, long long* kernel_launches, int* grid_blocks, double* last_kernel_ms);
/* Which block owns which cells, the only thing besides the reference's
 * arithmetic that a result depends on (the order of its global sums): warps
 * per block (8 or 16; a tile is 32 << warps_x_log2 cells wide and
 * 2*warps >> warps_x_log2 rows high), and the blocks of the persistent grid
 * (tile t belongs to block t mod grid_blocks).  No reference counterpart. */
int pearl_gpu_geometry(const pearl_gpu_ctx* ctx, int* warps, int* warps_x_log2, int* grid_blocks);
/* Device time of the last launch split by phase (16 slots, milliseconds and
 * phase counts): 0 propose, 1 diffusion set-up, 2 CG apply, 3 CG update,
 * 4 unused (the true-residual recheck runs inside slot 6), 5 CG restart,
 * 6 diffusion final (true residual, closure, mu, acceptance reductions),
 * 7 step-start energy, 8 phase-only final, 9 mixture, 10 moving window,
 * 11 snapshot, 12 interface smoothing, 13 initial composition.  Each slot
 * covers its sweep, reduction and grid barrier. */
int pearl_gpu_phase_times(const pearl_gpu_ctx* ctx, double* ms, long long* counts);

/* Self-test of the device's exact division by a precomputed reciprocal, which
 * the kernels use for every constant divisor of the reference's formulas
 * (Vm, dx, dy, dx*dx, dy*dy, 3, 2A): counts the n elements where it differs
 * bitwise from IEEE a[i]/b[i] on `device`.  No reference counterpart. */
int pearl_gpu_selftest_division(int device, const double* a, const double* b, long long n,
                                unsigned long long* mismatches);

/* FP64 throughput of `device`: independent FMA chains (8 per thread) in every
 * thread of a full grid, timed with CUDA events; *tflops receives the best of
 * three launches (an FMA counts two flops).  The roofline of the FP64-bound
 * phases (propose_phi, the final update with its energy).  No reference
 * counterpart. */
int pearl_gpu_selftest_fp64_peak(int device, double* tflops);

/* Self-test of the bounded device waits, on this context's grid and control
 * block: launches a grid barrier that waits for one block more than the grid
 * has, so every block must give up after the barrier's time limit (4 s).
 * *status receives the recorded status (PEARL_ERR_DEVICE_WAIT when the limit
 * works), *waited_ms (may be NULL) the device time; the context is left ready
 * for further calls.  No reference counterpart. */
int pearl_gpu_selftest_wait_limit(pearl_gpu_ctx* ctx, int* status, double* waited_ms);

/* One accepted step (as pearl_gpu_advance) for callers that cannot allocate
 * device memory: code whose GPU memory is owned by another allocator (a
 * framework's caching pool or a fixed memory budget) and latency-critical
 * loops that must avoid cudaMalloc/cudaFree, which can synchronise the device.
 * No counterpart in the reference.
 *
 * The caller owns the state in device memory as dense planes of nx*ny doubles
 * (row-major, x fastest): d_phi holds the alpha, theta and gamma planes back
 * to back, d_carbon and d_mu one plane each.  They are read as the current
 * state and overwritten with the accepted one; *scalars is read and updated.
 * Runs on the calling thread's current device and on `stream` (NULL = legacy
 * default stream) and returns after the step has finished.
 *
 * All scratch comes from one array compiled into the library (about 36 MB,
 * held by every GPU that loads the library until the process exits), so
 * nx*ny is limited to 262144 cells; larger domains return PEARL_ERR_TOO_LARGE.
 * The first call on each device looks up that array's device address; make
 * that first call before any stream capture.  The address is looked up again
 * when the device's CUDA context has changed since (after cudaDeviceReset),
 * so that call too must come before any capture.  All calls on a device share the
 * same scratch, so calls that overlap on the GPU (other streams or threads)
 * race and must be serialised by the caller. */
int pearl_gpu_advance_noalloc(const pearl_params* params, int nx, int ny, double* d_phi, double* d_carbon,
                              double* d_mu, pearl_scalars* scalars, double stop_time, pearl_step_info* out,
                              void* stream);

/* ---- adjoint: gradient of a final-state misfit ----
 * J = sum over cells of (phi_alpha - target_alpha)^2 after nsteps accepted
 * steps from the context's current state, and dJ/dtheta for
 * theta = (M, sigma, D_gamma): M is a common scale on every interface
 * mobility 1/tau (the forward runs at M = 1), sigma the interface energy,
 * D_gamma the austenite diffusivity.  Reverse mode: the forward stores a
 * checkpoint every `checkpoint_every` steps and the accepted dt of every
 * step, and records the last segment's states and diffusion solutions on a
 * tape; the reverse sweep recomputes every other segment from its
 * checkpoint with that dt sequence (recording it on the tape), then runs the
 * segment's adjoint steps backwards on the device, each adjoint linear solve
 * warm-started from the previous one.  The step is
 * differentiated as computed (propose_phi, pearl_serial.cpp:961-1002, with
 * the simplex projection on its active set; implicit_diffusion, :1010-1093,
 * with the linear system taken as solved exactly); acceptance decisions are
 * held fixed.  On success the context holds the forward's final state; on
 * error, its initial state.  Needs the FP64 step with implicit diffusion
 * (PEARL_ERR_INVALID_ARGUMENT in mixed precision or phase-only mode).  No
 * counterpart in the reference. */
typedef struct pearl_adjoint_report {
    double objective;
    double grad[3]; /* dJ/dM, dJ/dsigma, dJ/dD_gamma */
    long long steps, cg_forward, cg_adjoint;
    int checkpoints;
    double forward_ms, recompute_ms, adjoint_ms; /* device time of the three sweeps */
} pearl_adjoint_report;

/* target_alpha[y*nx+x] on the host.  The checkpoints, tape and adjoint
 * planes stay allocated in the context for later calls (grown when a call
 * needs more) and are freed by pearl_gpu_destroy. */
int pearl_gpu_adjoint_gradient(pearl_gpu_ctx* ctx, long long nsteps, int checkpoint_every,
                               const double* target_alpha, pearl_adjoint_report* out);

/* ---- batched instances: a parameter sweep in one persistent launch ----
 * n independent domains (each its own parameters and nx, ny) advance in one
 * cooperative launch.  The grid is split into groups of `group_blocks`
 * blocks, each group with its own grid barrier and reduction slots; the
 * instances are assigned to groups longest-first, and a group runs its
 * instances one after another.  With group_blocks = PEARL_BATCH_SIZED_GROUPS
 * the groups have per-instance sizes instead, chosen so that the slowest group
 * finishes soonest under a model of a pass's cost (powers of two up to the
 * grid, or an equal share of the grid per instance): small instances share
 * groups of a few blocks, large ones get many.  Every instance follows exactly the path of a
 * pearl_gpu_ctx (same kernels, same reduction order for the same group size),
 * so it is main's loop (pearl_serial.cpp:2296-2306) run once per instance.
 * No counterpart in the reference, which runs one case per process. */
typedef struct pearl_gpu_batch pearl_gpu_batch;
enum { PEARL_BATCH_SIZED_GROUPS = -1 };

/* group_blocks: blocks per group, or any value <= 0 (PEARL_BATCH_SIZED_GROUPS
 * among them) for groups sized per instance; pearl_gpu_batch_autotune can
 * choose instead. */
int pearl_gpu_batch_create(int n, const pearl_params* params, const int* nx, const int* ny, int device,
                           int group_blocks, pearl_gpu_batch** out);
void pearl_gpu_batch_destroy(pearl_gpu_batch* batch);
/* Host <-> device state of instance i, layouts as pearl_gpu_upload/download. */
int pearl_gpu_batch_upload(pearl_gpu_batch* batch, int i, const double* phi_aos3, const double* carbon,
                           const double* mu, const pearl_scalars* scalars);
int pearl_gpu_batch_download(pearl_gpu_batch* batch, int i, double* phi_aos3, double* carbon, double* mu,
                             pearl_scalars* scalars);
/* Up to limits->max_steps accepted steps of every instance under the same
 * limits, in one launch.  reports[i] and status[i] (pearl_status of instance
 * i; an instance that fails stops, the others go on) may be NULL.  Returns
 * PEARL_OK unless the launch itself failed. */
int pearl_gpu_batch_run(pearl_gpu_batch* batch, const pearl_run_limits* limits, pearl_run_report* reports,
                        int* status);
/* Times one launch of `steps` steps for each group size in {1,2,4,8,16}, for
 * per-instance group sizes (three weights of a pass's fixed cost against its
 * tiles), and each tile shape (32x16 cells with and without TMA staging, 64x8, 128x4),
 * restoring every instance's state after each trial, and keeps the fastest;
 * the choice is written to the out pointers (may be NULL; tile_warps_x = warps
 * side by side in x: 1, 2 or 4).  The tile shape changes which block owns
 * which cells, hence the order of the sums, not the arithmetic of a cell. */
int pearl_gpu_batch_autotune(pearl_gpu_batch* batch, int steps, int* group_blocks, int* use_tma,
                             int* tile_warps_x);
/* pearl_gpu_set_precision for every instance. */
int pearl_gpu_batch_set_precision(pearl_gpu_batch* batch, int precision);
/* Sets the configuration pearl_gpu_batch_autotune would choose: blocks per
 * group (or PEARL_BATCH_SIZED_GROUPS, with the fixed-cost weight the last
 * autotune chose, initially 4 tiles), TMA staging (used only with
 * tile_warps_x = 1) and the tile shape (tile_warps_x warps side by side in x:
 * 1, 2, 4 or 8). */
int pearl_gpu_batch_configure(pearl_gpu_batch* batch, int group_blocks, int use_tma, int tile_warps_x);
/* Host only (no GPU needed): the groups a batch launch of grid_blocks blocks
 * would use for instances of tiles[i] tiles each (32x16-cell tiles:
 * ceil(nx/32) * ceil(ny/16)), for group_blocks blocks per group or
 * PEARL_BATCH_SIZED_GROUPS, with a pass's fixed cost weighed as
 * pass_overhead_tiles tiles of one block.  Writes the group of every instance,
 * the size of every group (group_size needs room for grid_blocks entries), the
 * number of groups and the modelled longest group time in tiles (may be NULL). */
int pearl_gpu_batch_plan(int n, const long long* tiles, int grid_blocks, int group_blocks, double pass_overhead_tiles,
                         int* group_of_instance, int* group_size, int* ngroups, double* longest);
int pearl_gpu_batch_stats(const pearl_gpu_batch* batch, long long* kernel_launches, int* grid_blocks,
                          int* group_blocks, double* last_kernel_ms);
const char* pearl_gpu_batch_last_error(const pearl_gpu_batch* batch);

#ifdef __cplusplus
}
#endif
#endif /* PEARL_GPU_H */
