/*
 * pearl_oracle — CPU restatement of the Pearl time-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * bench's CPU-baseline leg may load this library, and only as the reference
 * results are compared against (or as the timed CPU port).  The product (libpearl_gpu.so, pearl_gpu)
 * never links or calls it.
 *
 * Every function restates the algorithm of the reference file
 * pearl_serial.cpp (cited as file:line) in plain C99, keeping the same
 * floating-point operation order, no FMA contraction except where the
 * reference calls std::fma, and the same sequential row-major reductions,
 * so that its results are bit-identical to the reference serial solver.
 * That identity is checked against the reference itself, compiled from its
 * own source by oracle/build_oracle.py into oracle/_ref/.
 *
 * Storage (the reference's gathered global layout, pearl_serial.cpp:695-722):
 *   phi[(y*nx + x)*3 + a]  a = 0 alpha (ferrite), 1 theta (cementite), 2 gamma
 *   carbon[y*nx + x], mu[y*nx + x]
 * x is periodic, y has zero-flux walls (pearl_serial.cpp:674-694).
 */
#ifndef PEARL_ORACLE_H
#define PEARL_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Same field order and meaning as pearl_params in include/pearl_gpu.h. */
typedef struct po_params {
    double A[3], B[3], C[3], D[3]; /* f_p(c) = A c^2 + B c + C; D diffusivity */
    double Vm, epsilon, sigma, triple;
    double tau[3]; /* tau_at, tau_ag, tau_tg */
    double dx, dy;
    double dt_max, dt_min, max_phase_change;
    double cg_rtol, cg_atol, closure_tol;
    double energy_rtol, energy_atol;
    int cg_max, max_retries, check_energy, phase_only;
    double mu_reference;
} po_params;

/* Same field order as pearl_scalars in include/pearl_gpu.h. */
typedef struct po_scalars {
    double time, dt, shift_distance, initial_carbon, carbon_added, carbon_removed;
    long long step, shifts, rejected;
} po_scalars;

/* pearl_serial.cpp:774-777 (StepInfo) */
typedef struct po_step_info {
    double accepted_dt, max_phase_change, linear_residual, closure, energy_change;
    int cg_iterations, retries;
} po_step_info;

/* pearl_serial.cpp:1004-1009 (DiffusionInfo) */
typedef struct po_diffusion_info {
    int ok, it;
    double residual, closure;
} po_diffusion_info;

/* Snapshot reductions, pearl_serial.cpp:2266-2281 */
typedef struct po_diag {
    double c_min, c_max, mu_min, mu_max, phi_sum_error, mass, ledger, energy;
} po_diag;

/* Status codes: same values as include/pearl_gpu.h. */
enum {
    PO_OK = 0,
    PO_ERR_INVALID_ARGUMENT = 1,
    PO_ERR_INVALID_ADVANCE_TIME = 3,
    PO_ERR_REJECTED_BELOW_DT_MIN = 4,
    PO_ERR_RETRY_LIMIT = 5,
    PO_ERR_MIXTURE = 6,
    PO_ERR_SIMPLEX = 7,
    PO_ERR_UNSAFE_SHIFT = 10,
    PO_ERR_NONFINITE_CARBON = 11
};
/* Rejection reasons, pearl_serial.cpp:1133-1160 */
enum {
    PO_WHY_NONE = 0,
    PO_WHY_PHASE_INCREMENT = 1,
    PO_WHY_LINEAR_CLOSURE = 2,
    PO_WHY_BOUNDS = 3,
    PO_WHY_MASS = 4,
    PO_WHY_ENERGY = 5
};

/* ---- summation order of the device kernels ----
 * The reference sums every global quantity sequentially in row-major order
 * (Domain::sum, pearl_serial.cpp:649-666; array_dot, :738-742; total_carbon,
 * :784-788; reduced_energy, :793-821).  libpearl_gpu sums the same per-cell
 * values in a fixed tree instead: the grid's blocks own tiles of 32 x 2*warps
 * cells (tile t: column t % ntx, row t / ntx; block b owns t = b, b+blocks,
 * ...), each thread accumulates its two cells (x, y0) and (x, y0+1) over its
 * block's tiles in the pass's walk order, warps reduce by shuffles
 * (offsets 16, 8, 4, 2, 1), a block adds its warps in index order, and 32
 * lanes add the block partials strided by 32 before a last shuffle tree.
 * Passes walk their tiles forwards (set-up, CG update, restart, step-start
 * energy) or backwards (CG apply, final update with its mass and energy), and
 * the energy of a cell is summed per cell first (cell terms, then its faces).
 * The device also carries the accepted trial's energy and carbon mass into
 * the next step instead of recomputing them.
 *
 * po_set_device_order(o) makes this oracle follow that order and that carry
 * (per-cell arithmetic is unchanged), so that, given the device's grid, it
 * reproduces the device's results bit for bit; po_set_device_order(NULL)
 * restores the reference's order.  o->threads > 1 runs the per-cell loops of
 * that mode on host threads (the results do not depend on it).  Test
 * infrastructure: it shows that the device differs from the reference only
 * in the order of its sums. */
typedef struct po_device_order {
    int warps;         /* warps per block: 8 (32x16 tiles) or 16 (32x32 tiles) */
    int warps_x_log2;  /* warps side by side in x: the tile is (32 << w) x (2*warps >> w) cells */
    int blocks;        /* blocks in the grid */
    int threads;       /* host threads for the per-cell loops */
} po_device_order;
void po_set_device_order(const po_device_order* order);
/* The device's tree sum of v[y*nx + x] over the domain; reverse = walk order. */
double po_device_sum(int nx, int ny, const double* v, int reverse);

/* ---- pointwise thermodynamics (pearl_serial.cpp:76-145) ---- */
double po_psi(const po_params* p, int phase, double mu);
void po_weights(const double phi[3], double h[3]);
void po_weight_derivatives(const double phi[3], double dh[3][3]);
int po_mixture(const po_params* p, const double phi[3], double* chi, double* c_intercept, double* transport);
int po_project_simplex(const double trial[3], double out[3]);
double po_local_tau(const double phi[3], const double tau[3]);

/* ---- hot path (pearl_serial.cpp:784-1174) ---- */
double po_total_carbon(const po_params* p, int nx, int ny, const double* carbon);
/* returns PO_OK or PO_ERR_MIXTURE; *energy receives the reduced energy */
int po_reduced_energy(const po_params* p, int nx, int ny, const double* phi, const double* carbon,
                      double* energy);
/* trial_phi receives the proposal; *change the global max |dphi| (inf if non-finite) */
int po_propose_phi(const po_params* p, int nx, int ny, const double* phi_old, const double* mu_old,
                   double* trial_phi, double dt, double* change);
int po_implicit_diffusion(const po_params* p, int nx, int ny, const double* carbon_old, const double* mu_old,
                          const double* trial_phi, double* trial_carbon, double* trial_mu, double dt,
                          po_diffusion_info* info);
/* implicit_diffusion that also returns the converged u = mu - mu_reference (u_out may be NULL). */
int po_implicit_diffusion_u(const po_params* p, int nx, int ny, const double* carbon_old, const double* mu_old,
                            const double* trial_phi, double* trial_carbon, double* trial_mu, double dt,
                            po_diffusion_info* info, double* u_out);
int po_valid_state(const po_params* p, int nx, int ny, const double* phi, const double* carbon,
                   const double* mu);
/* One accepted step.  Fields are updated in place on success.  *why receives the
 * rejection reason of the last attempt on error. */
int po_advance(const po_params* p, int nx, int ny, double* phi, double* carbon, double* mu,
               po_scalars* s, double stop_time, po_step_info* out, int* why);
/* Runs nsteps advances; forced_dt (nullable) replays an accepted-dt sequence by
 * setting s->dt before each step.  infos (nullable) receives per-step info.
 * Returns the first error; *steps_done the number of accepted steps. */
int po_advance_n(const po_params* p, int nx, int ny, double* phi, double* carbon, double* mu, po_scalars* s,
                 int nsteps, const double* forced_dt, double stop_time, po_step_info* infos, int* why,
                 int* steps_done);

/* ---- moving window and output reductions (pearl_serial.cpp:789-792, 2023-2071, 2266-2281) ---- */
int po_close_mu(const po_params* p, int nx, int ny, const double* phi, const double* carbon, double* mu);
double po_front_position(const po_params* p, int nx, int ny, const double* phi);
int po_shift_rows(const po_params* p, int nx, int ny, double* phi, double* carbon, double* mu, po_scalars* s,
                  int rows, double c_gamma);
/* *shifted = rows shifted (0 if none) */
int po_maybe_shift(const po_params* p, int nx, int ny, double* phi, double* carbon, double* mu, po_scalars* s,
                   double shift_trigger, double shift_target, double c_gamma, int* shifted);
int po_snapshot(const po_params* p, int nx, int ny, const double* phi, const double* carbon, const double* mu,
                const po_scalars* s, po_diag* out);

/* ---- capillarity-only preprocessing (pearl_serial.cpp:822-958) ---- */
double po_interface_energy_only(const po_params* p, int nx, int ny, const double* phi);
typedef struct po_smooth_report {
    int steps, converged;
    double energy_initial, energy_final, final_relative_energy_change, final_max_phase_change;
    double phase_fraction_before[3], phase_fraction_after[3];
} po_smooth_report;
int po_smooth_interface_only(const po_params* p, int nx, int ny, double* phi, int max_steps, int min_steps,
                             double energy_rtol, double max_phase_change, po_smooth_report* report);

/* ---- adjoint (no reference counterpart: the reference has no gradient) ----
 * Reverse-mode gradient of J = sum over cells of (phi_alpha - target)^2 after
 * nsteps accepted steps, with respect to theta = (mobility scale M, sigma,
 * D_gamma) at the given parameters.  M multiplies every interface mobility
 * 1/tau (the forward runs at M = 1).  The discrete step is differentiated as
 * computed: propose_phi (forces, local tau, simplex projection on its active
 * set) and implicit_diffusion with its linear system treated as solved
 * exactly.  The forward keeps a checkpoint every checkpoint_every steps; the
 * reverse sweep recomputes each segment from its checkpoint with the recorded
 * accepted dt sequence.  On return the fields hold the forward's final state. */
typedef struct po_adjoint_report {
    double objective;
    double grad[3]; /* dJ/dM, dJ/dsigma, dJ/dD_gamma */
    long long steps, cg_forward, cg_adjoint;
    int checkpoints;
} po_adjoint_report;
int po_adjoint_gradient(const po_params* p, int nx, int ny, double* phi, double* carbon, double* mu, po_scalars* s,
                        int nsteps, int checkpoint_every, const double* target_alpha, po_adjoint_report* out);
/* J only: nsteps accepted steps of the forward, then the misfit (fields updated in place). */
int po_adjoint_objective(const po_params* p, int nx, int ny, double* phi, double* carbon, double* mu,
                         po_scalars* s, int nsteps, const double* target_alpha, double* objective);

#ifdef __cplusplus
}
#endif
#endif
