/*
 * pearl_oracle.c — CPU restatement of the Pearl hot path (TEST INFRASTRUCTURE).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
 * this file, as the checker or as the timed CPU port; the product never does.
 * Each function restates the reference pearl_serial.cpp (cited file:line)
 * with the same operation order and sequential reductions.  It is compiled
 * with -ffp-contract=off so that, like the reference built for plain x86-64,
 * no multiply-add is fused except where the reference calls std::fma.
 */
#include "pearl_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* std::max / std::min argument semantics: max(a,b) = a<b ? b : a */
static inline double dmax(double a, double b) { return (a < b) ? b : a; }
static inline double dmin(double a, double b) { return (b < a) ? b : a; }

static inline int xm(int x, int nx) { return x == 0 ? nx - 1 : x - 1; }
static inline int xp(int x, int nx) { return x == nx - 1 ? 0 : x + 1; }
/* zero-flux ghost rows copy the edge row (pearl_serial.cpp:690-691) */
static inline int ym(int y) { return y == 0 ? 0 : y - 1; }
static inline int yp(int y, int ny) { return y == ny - 1 ? ny - 1 : y + 1; }
static inline size_t at(int x, int y, int nx) { return (size_t)y * (size_t)nx + (size_t)x; }

static double pi_value(void) { return acos(-1.0); }

/* Parabola::psi, pearl_serial.cpp:86-89 */
double po_psi(const po_params* p, int phase, double mu) {
    const double d = mu - p->B[phase];
    return fma(-0.25 / p->A[phase], d * d, p->C[phase]);
}

/* Parabola::chi, pearl_serial.cpp:85 */
static inline double chi_of(const po_params* p, int phase) { return 1.0 / (2.0 * p->A[phase]); }

/* weights, pearl_serial.cpp:102-107 */
void po_weights(const double phi[3], double h[3]) {
    const double triple = 2.0 * phi[0] * phi[1] * phi[2];
    for (int q = 0; q < 3; ++q) h[q] = phi[q] * phi[q] * (3.0 - 2.0 * phi[q]) + triple;
}

/* weight_derivatives, pearl_serial.cpp:109-116 */
void po_weight_derivatives(const double phi[3], double dh[3][3]) {
    const double dtriple[3] = {2.0 * phi[1] * phi[2], 2.0 * phi[0] * phi[2], 2.0 * phi[0] * phi[1]};
    for (int q = 0; q < 3; ++q)
        for (int a = 0; a < 3; ++a) dh[q][a] = dtriple[a] + (q == a ? 6.0 * phi[q] * (1.0 - phi[q]) : 0.0);
}

/* mixture, pearl_serial.cpp:125-138; returns PO_ERR_MIXTURE where the reference throws */
int po_mixture(const po_params* p, const double phi[3], double* chi, double* c_intercept, double* transport) {
    double h[3];
    po_weights(phi, h);
    double s = 0.0, ci = 0.0, k = 0.0;
    for (int q = 0; q < 3; ++q) {
        const double c = chi_of(p, q);
        s += h[q] * c;
        ci -= h[q] * c * p->B[q];
        k += phi[q] * p->D[q] * c;
    }
    *chi = s;
    *c_intercept = ci;
    *transport = k;
    if (!(s > 0.0) || !isfinite(s) || !isfinite(ci) || !isfinite(k) || k < 0.0) return PO_ERR_MIXTURE;
    return PO_OK;
}

/* project_simplex, pearl_serial.cpp:491-509 */
int po_project_simplex(const double trial[3], double out[3]) {
    for (int a = 0; a < 3; ++a)
        if (!isfinite(trial[a])) return PO_ERR_SIMPLEX;
    double s0 = trial[0], s1 = trial[1], s2 = trial[2], t;
    /* descending order; only the sorted values matter */
    if (s0 < s1) { t = s0; s0 = s1; s1 = t; }
    if (s1 < s2) { t = s1; s1 = s2; s2 = t; }
    if (s0 < s1) { t = s0; s0 = s1; s1 = t; }
    const double sorted[3] = {s0, s1, s2};
    double sum = 0.0, threshold = 0.0;
    int active = 0;
    for (int j = 0; j < 3; ++j) {
        sum += sorted[j];
        const double candidate = (sum - 1.0) / (j + 1);
        if (sorted[j] > candidate) {
            active = j + 1;
            threshold = candidate;
        }
    }
    if (active == 0) return PO_ERR_SIMPLEX;
    for (int a = 0; a < 3; ++a) out[a] = dmax(0.0, trial[a] - threshold);
    return PO_OK;
}

/* local_tau, pearl_serial.cpp:533-537 */
double po_local_tau(const double phi[3], const double tau[3]) {
    const double w0 = phi[0] * phi[1], w1 = phi[0] * phi[2], w2 = phi[1] * phi[2];
    const double s = w0 + w1 + w2;
    if (s > 1e-30) return (w0 * tau[0] + w1 * tau[1] + w2 * tau[2]) / s;
    double m = tau[0];
    if (tau[1] < m) m = tau[1];
    if (tau[2] < m) m = tau[2];
    return m;
}

static inline void load3(const double* phi, int x, int y, int nx, double v[3]) {
    const size_t i = at(x, y, nx) * 3;
    v[0] = phi[i];
    v[1] = phi[i + 1];
    v[2] = phi[i + 2];
}

/* total_carbon, pearl_serial.cpp:784-788 */
double po_total_carbon(const po_params* p, int nx, int ny, const double* carbon) {
    double v = 0;
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) v += carbon[at(x, y, nx)];
    return v * p->dx * p->dy;
}

/* reduced_energy, pearl_serial.cpp:793-821 */
int po_reduced_energy(const po_params* p, int nx, int ny, const double* phi, const double* carbon,
                      double* energy) {
    const double eps = p->epsilon, sigma = p->sigma;
    const double pi = pi_value();
    const double obstacle = 16 * sigma / (pi * pi * eps), triple = p->triple / eps;
    const double mu_r = p->mu_reference;
    const double psi[3] = {po_psi(p, 0, mu_r) - po_psi(p, 2, mu_r), po_psi(p, 1, mu_r) - po_psi(p, 2, mu_r), 0};
    double total = 0;
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            double q[3], h[3];
            load3(phi, x, y, nx, q);
            po_weights(q, h);
            double chem = 0;
            for (int a = 0; a < 3; ++a) chem += h[a] * psi[a];
            if (!p->phase_only) {
                double chi, ci, k;
                if (po_mixture(p, q, &chi, &ci, &k) != PO_OK) return PO_ERR_MIXTURE;
                const double dc = carbon[at(x, y, nx)] - fma(chi, mu_r, ci);
                chem += .5 * dc * dc / chi;
            }
            total += chem / p->Vm + obstacle * (q[0] * q[1] + q[0] * q[2] + q[1] * q[2]) + triple * q[0] * q[1] * q[2];
            for (int dir = 0; dir < 2; ++dir) {
                if (dir == 1 && y == ny - 1) continue;
                double nb[3];
                if (dir == 0)
                    load3(phi, xp(x, nx), y, nx, nb);
                else
                    load3(phi, x, y + 1, nx, nb);
                const double dist = dir == 0 ? p->dx : p->dy;
                for (int a = 0; a < 3; ++a)
                    for (int b = a + 1; b < 3; ++b) {
                        const double z = (q[a] * nb[b] - nb[a] * q[b]) / dist;
                        total += eps * sigma * z * z;
                    }
            }
        }
    *energy = total * p->dx * p->dy;
    return PO_OK;
}

/* propose_phi, pearl_serial.cpp:961-1002 */
int po_propose_phi(const po_params* p, int nx, int ny, const double* phi_old, const double* mu_old,
                   double* trial_phi, double dt, double* change_out) {
    const double eps = p->epsilon, sigma = p->sigma;
    const double pi = pi_value();
    const double obs = 16 * sigma / (pi * pi * eps), tr = p->triple / eps;
    double change = 0;
    static const int ox[4] = {-1, 1, 0, 0}, oy[4] = {0, 0, -1, 1};
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            double q[3], force[3] = {0, 0, 0}, dh[3][3];
            load3(phi_old, x, y, nx, q);
            const double mu = mu_old[at(x, y, nx)];
            const double psi0 = po_psi(p, 2, mu);
            po_weight_derivatives(q, dh);
            for (int a = 0; a < 3; ++a) {
                force[a] = obs * (q[(a + 1) % 3] + q[(a + 2) % 3]) + tr * q[(a + 1) % 3] * q[(a + 2) % 3];
                for (int b = 0; b < 3; ++b) force[a] += (po_psi(p, b, mu) - psi0) * dh[b][a] / p->Vm;
            }
            for (int dir = 0; dir < 4; ++dir) {
                if ((dir == 2 && y == 0) || (dir == 3 && y == ny - 1)) continue;
                int xx = x, yy = y;
                if (ox[dir] < 0) xx = xm(x, nx);
                if (ox[dir] > 0) xx = xp(x, nx);
                if (oy[dir] < 0) yy = ym(y);
                if (oy[dir] > 0) yy = yp(y, ny);
                double nb[3];
                load3(phi_old, xx, yy, nx, nb);
                const double dist = dir < 2 ? p->dx : p->dy;
                for (int a = 0; a < 3; ++a)
                    for (int b = a + 1; b < 3; ++b) {
                        const double w = 2 * eps * sigma * (q[a] * nb[b] - nb[a] * q[b]) / (dist * dist);
                        force[a] += w * nb[b];
                        force[b] -= w * nb[a];
                    }
            }
            const double mean = (force[0] + force[1] + force[2]) / 3,
                         scale = dt / (po_local_tau(q, p->tau) * eps);
            double z[3];
            for (int a = 0; a < 3; ++a) z[a] = q[a] - scale * (force[a] - mean);
            int finite = 1;
            for (int a = 0; a < 3; ++a) finite = finite && isfinite(z[a]);
            double* out = trial_phi + at(x, y, nx) * 3;
            if (!finite) {
                change = INFINITY;
                out[0] = q[0];
                out[1] = q[1];
                out[2] = q[2];
                continue;
            }
            double zp[3];
            if (po_project_simplex(z, zp) != PO_OK) return PO_ERR_SIMPLEX;
            for (int a = 0; a < 3; ++a) change = dmax(change, fabs(zp[a] - q[a]));
            out[0] = zp[0];
            out[1] = zp[1];
            out[2] = zp[2];
        }
    *change_out = change;
    return PO_OK;
}

/* weights_at, pearl_serial.cpp:1022-1028 */
static inline void face_weights(const po_params* p, const double* K, int x, int y, int nx, int ny, double w[4]) {
    const double k = K[at(x, y, nx)];
    const double dx2 = p->dx * p->dx, dy2 = p->dy * p->dy;
    w[0] = .5 * (k + K[at(xm(x, nx), y, nx)]) / dx2;
    w[1] = .5 * (k + K[at(xp(x, nx), y, nx)]) / dx2;
    w[2] = .5 * (k + K[at(x, ym(y), nx)]) / dy2;
    w[3] = .5 * (k + K[at(x, yp(y, ny), nx)]) / dy2;
    if (y == 0) w[2] = 0;
    if (y == ny - 1) w[3] = 0;
}

/* apply, pearl_serial.cpp:1029-1035 */
static void apply_op(const po_params* p, const double* K, const double* chi, double dt, int nx, int ny,
                     const double* in, double* out) {
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            double w[4];
            face_weights(p, K, x, y, nx, ny, w);
            const double c = in[at(x, y, nx)];
            out[at(x, y, nx)] = chi[at(x, y, nx)] * c +
                                dt * (w[0] * (c - in[at(xm(x, nx), y, nx)]) + w[1] * (c - in[at(xp(x, nx), y, nx)]) +
                                      w[2] * (c - in[at(x, ym(y), nx)]) + w[3] * (c - in[at(x, yp(y, ny), nx)]));
        }
}

/* array_dot, pearl_serial.cpp:738-742 */
static double dot(const double* a, const double* b, size_t n) {
    double s = 0;
    for (size_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

/* implicit_diffusion, pearl_serial.cpp:1010-1094.  u_out (may be NULL) receives
 * the converged solution u = mu - mu_reference of the linear system. */
int po_implicit_diffusion_u(const po_params* p, int nx, int ny, const double* carbon_old, const double* mu_old,
                            const double* trial_phi, double* trial_carbon, double* trial_mu, double dt,
                            po_diffusion_info* info, double* u_out) {
    const size_t n = (size_t)nx * (size_t)ny;
    const double mu_r = p->mu_reference;
    double* mem = (double*)malloc(sizeof(double) * n * 10);
    if (!mem) return PO_ERR_INVALID_ARGUMENT;
    double *chi = mem, *icpt = mem + n, *K = mem + 2 * n, *rhs = mem + 3 * n, *u = mem + 4 * n, *diag = mem + 5 * n;
    double *r = mem + 6 * n, *z = mem + 7 * n, *pd = mem + 8 * n, *Ap = mem + 9 * n;
    for (size_t i = 0; i < n; ++i) {
        double c, ci, k;
        if (po_mixture(p, trial_phi + 3 * i, &c, &ci, &k) != PO_OK) {
            free(mem);
            return PO_ERR_MIXTURE;
        }
        chi[i] = c;
        icpt[i] = fma(c, mu_r, ci);
        K[i] = k;
        rhs[i] = carbon_old[i] - icpt[i];
        u[i] = mu_old[i] - mu_r;
    }
    apply_op(p, K, chi, dt, nx, ny, u, Ap);
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            double w[4];
            face_weights(p, K, x, y, nx, ny, w);
            const size_t i = at(x, y, nx);
            diag[i] = chi[i] + dt * (w[0] + w[1] + w[2] + w[3]);
            r[i] = rhs[i] - Ap[i];
            z[i] = r[i] / diag[i];
            pd[i] = z[i];
        }
    const double tolerance = p->cg_atol + p->cg_rtol * sqrt(dot(rhs, rhs, n));
    double rz = dot(r, z, n);
    po_diffusion_info inf = {0, 0, 0.0, 0.0};
    for (int iteration = 0; iteration <= p->cg_max; ++iteration) {
        inf.it = iteration;
        inf.residual = sqrt(dot(r, r, n));
        if (!isfinite(inf.residual)) {
            *info = inf;
            free(mem);
            return PO_OK;
        }
        if (inf.residual <= tolerance) {
            apply_op(p, K, chi, dt, nx, ny, u, Ap);
            for (size_t i = 0; i < n; ++i) r[i] = rhs[i] - Ap[i];
            inf.residual = sqrt(dot(r, r, n));
            if (inf.residual <= tolerance * 1.05) {
                inf.ok = 1;
                break;
            }
            for (size_t i = 0; i < n; ++i) {
                z[i] = r[i] / diag[i];
                pd[i] = z[i];
            }
            rz = dot(r, z, n);
            continue;
        }
        if (iteration == p->cg_max) break;
        apply_op(p, K, chi, dt, nx, ny, pd, Ap);
        const double pAp = dot(pd, Ap, n);
        if (!(pAp > 0) || !isfinite(pAp) || !isfinite(rz)) {
            *info = inf;
            free(mem);
            return PO_OK;
        }
        const double alpha = rz / pAp;
        for (size_t i = 0; i < n; ++i) {
            u[i] += alpha * pd[i];
            r[i] -= alpha * Ap[i];
            z[i] = r[i] / diag[i];
        }
        const double rz_next = dot(r, z, n), beta = rz_next / rz;
        rz = rz_next;
        for (size_t i = 0; i < n; ++i) pd[i] = z[i] + beta * pd[i];
    }
    if (!inf.ok) {
        *info = inf;
        free(mem);
        return PO_OK;
    }
    double closure = 0;
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            double w[4];
            face_weights(p, K, x, y, nx, ny, w);
            const size_t i = at(x, y, nx);
            const double c = u[i];
            const double change = dt * (w[0] * (u[at(xm(x, nx), y, nx)] - c) + w[1] * (u[at(xp(x, nx), y, nx)] - c) +
                                        w[2] * (u[at(x, ym(y), nx)] - c) + w[3] * (u[at(x, yp(y, ny), nx)] - c));
            trial_carbon[i] = carbon_old[i] + change;
            closure = dmax(closure, fabs(trial_carbon[i] - (icpt[i] + chi[i] * c)));
            trial_mu[i] = mu_r + (trial_carbon[i] - icpt[i]) / chi[i];
        }
    inf.closure = closure;
    inf.ok = closure <= p->closure_tol;
    *info = inf;
    if (u_out) memcpy(u_out, u, sizeof(double) * n);
    free(mem);
    return PO_OK;
}

int po_implicit_diffusion(const po_params* p, int nx, int ny, const double* carbon_old, const double* mu_old,
                          const double* trial_phi, double* trial_carbon, double* trial_mu, double dt,
                          po_diffusion_info* info) {
    return po_implicit_diffusion_u(p, nx, ny, carbon_old, mu_old, trial_phi, trial_carbon, trial_mu, dt, info, NULL);
}

/* valid_state, pearl_serial.cpp:1096-1116 */
int po_valid_state(const po_params* p, int nx, int ny, const double* phi, const double* carbon,
                   const double* mu) {
    int good = 1;
    const size_t n = (size_t)nx * (size_t)ny;
    for (size_t i = 0; i < n; ++i) {
        double sum = 0;
        const double* q = phi + 3 * i;
        for (int a = 0; a < 3; ++a) {
            good = good && isfinite(q[a]) && q[a] >= -1e-12 && q[a] <= 1 + 1e-12;
            sum += q[a];
        }
        good = good && fabs(sum - 1) < 1e-10;
        good = good && isfinite(mu[i]) && isfinite(carbon[i]);
        if (!p->phase_only) {
            good = good && carbon[i] >= -1e-10 && carbon[i] <= 1 + 1e-10;
            for (int a = 0; a < 3; ++a)
                if (q[a] > .01) {
                    const double c = (mu[i] - p->B[a]) / (2.0 * p->A[a]);
                    good = good && c >= -1e-10 && c <= 1 + 1e-10;
                }
        }
    }
    return good;
}

/* advance, pearl_serial.cpp:1119-1174 */
int po_advance(const po_params* p, int nx, int ny, double* phi, double* carbon, double* mu, po_scalars* s,
               double stop_time, po_step_info* out_info, int* why_out) {
    double dt = s->dt;
    if (p->dt_max < dt) dt = p->dt_max;
    if (stop_time - s->time < dt) dt = stop_time - s->time;
    if (!(dt > 0) || !isfinite(dt)) return PO_ERR_INVALID_ADVANCE_TIME;
    const size_t n = (size_t)nx * (size_t)ny;
    double e0 = 0;
    if (p->check_energy) {
        int rc = po_reduced_energy(p, nx, ny, phi, carbon, &e0);
        if (rc) return rc;
    }
    const double mass0 = p->phase_only ? 0 : po_total_carbon(p, nx, ny, carbon);
    int why = PO_WHY_NONE;
    double* tphi = (double*)malloc(sizeof(double) * n * 5);
    if (!tphi) return PO_ERR_INVALID_ARGUMENT;
    double *tc = tphi + 3 * n, *tmu = tphi + 4 * n;
    const double gxgy = (double)(nx * ny);
    for (int attempt = 0; attempt <= p->max_retries; ++attempt) {
        memcpy(tphi, phi, sizeof(double) * 3 * n);
        memcpy(tc, carbon, sizeof(double) * n);
        memcpy(tmu, mu, sizeof(double) * n);
        po_step_info out;
        memset(&out, 0, sizeof out);
        out.retries = attempt;
        out.accepted_dt = dt;
        int rc = po_propose_phi(p, nx, ny, phi, mu, tphi, dt, &out.max_phase_change);
        if (rc) {
            free(tphi);
            return rc;
        }
        int good = isfinite(out.max_phase_change) && out.max_phase_change <= p->max_phase_change;
        why = PO_WHY_PHASE_INCREMENT;
        if (good) {
            if (p->phase_only) {
                for (size_t i = 0; i < n; ++i) {
                    double c, ci, k;
                    if (po_mixture(p, tphi + 3 * i, &c, &ci, &k) != PO_OK) {
                        free(tphi);
                        return PO_ERR_MIXTURE;
                    }
                    tc[i] = fma(c, tmu[i], ci);
                }
            } else {
                po_diffusion_info di;
                rc = po_implicit_diffusion(p, nx, ny, carbon, mu, tphi, tc, tmu, dt, &di);
                if (rc) {
                    free(tphi);
                    return rc;
                }
                good = di.ok;
                out.cg_iterations = di.it;
                out.linear_residual = di.residual;
                out.closure = di.closure;
                why = PO_WHY_LINEAR_CLOSURE;
            }
        }
        if (good) {
            good = po_valid_state(p, nx, ny, tphi, tc, tmu);
            why = PO_WHY_BOUNDS;
        }
        if (good && !p->phase_only) {
            const double m = po_total_carbon(p, nx, ny, tc);
            good = fabs(m - mass0) <= 1e-11 * dmax(fabs(mass0), gxgy * p->dx * p->dy * 1e-6);
            why = PO_WHY_MASS;
        }
        if (good && p->check_energy) {
            double e1;
            rc = po_reduced_energy(p, nx, ny, tphi, tc, &e1);
            if (rc) {
                free(tphi);
                return rc;
            }
            out.energy_change = e1 - e0;
            const double tol =
                p->energy_atol + p->energy_rtol * dmax(fabs(e0), p->sigma * dmax(nx * p->dx, ny * p->dy));
            good = isfinite(e1) && e1 <= e0 + tol;
            why = PO_WHY_ENERGY;
        }
        if (good) {
            memcpy(phi, tphi, sizeof(double) * 3 * n);
            memcpy(carbon, tc, sizeof(double) * n);
            memcpy(mu, tmu, sizeof(double) * n);
            s->time = s->time + dt;
            s->step = s->step + 1;
            s->rejected = s->rejected + attempt;
            s->dt = dmin(p->dt_max, dt * 1.1);
            if (out_info) *out_info = out;
            if (why_out) *why_out = PO_WHY_NONE;
            free(tphi);
            return PO_OK;
        }
        dt *= .5;
        if (dt < p->dt_min) {
            if (why_out) *why_out = why;
            free(tphi);
            return PO_ERR_REJECTED_BELOW_DT_MIN;
        }
    }
    if (why_out) *why_out = why;
    free(tphi);
    return PO_ERR_RETRY_LIMIT;
}

int po_advance_n(const po_params* p, int nx, int ny, double* phi, double* carbon, double* mu, po_scalars* s,
                 int nsteps, const double* forced_dt, double stop_time, po_step_info* infos, int* why,
                 int* steps_done) {
    int done = 0, rc = PO_OK;
    for (int k = 0; k < nsteps; ++k) {
        if (forced_dt) s->dt = forced_dt[k];
        rc = po_advance(p, nx, ny, phi, carbon, mu, s, stop_time, infos ? infos + k : NULL, why);
        if (rc) break;
        ++done;
    }
    if (steps_done) *steps_done = done;
    return rc;
}

/* close_mu, pearl_serial.cpp:789-792 (reconstruct_mu, :139-142) */
int po_close_mu(const po_params* p, int nx, int ny, const double* phi, const double* carbon, double* mu) {
    const size_t n = (size_t)nx * (size_t)ny;
    for (size_t i = 0; i < n; ++i) {
        double chi, ci, k;
        if (po_mixture(p, phi + 3 * i, &chi, &ci, &k) != PO_OK) return PO_ERR_MIXTURE;
        if (!isfinite(carbon[i])) return PO_ERR_NONFINITE_CARBON;
        mu[i] = (carbon[i] - ci) / chi;
    }
    return PO_OK;
}

/* front detection of maybe_shift, pearl_serial.cpp:2055-2062 */
double po_front_position(const po_params* p, int nx, int ny, const double* phi) {
    double local = -1;
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            if (y == ny - 1) continue;
            const double a = 1 - 2 * phi[at(x, y, nx) * 3 + 2], b = 1 - 2 * phi[at(x, y + 1, nx) * 3 + 2];
            if (a >= 0 && b < 0) local = dmax(local, ((y + 1) - .5 + a / (a - b)) * p->dy);
        }
    return local;
}

/* shift_rows, pearl_serial.cpp:2023-2052 */
int po_shift_rows(const po_params* p, int nx, int ny, double* phi, double* carbon, double* mu, po_scalars* s,
                  int rows, double c_gamma) {
    if (rows <= 0 || rows >= ny || c_gamma < 0 || c_gamma > 1) return PO_ERR_INVALID_ARGUMENT;
    double removed = 0, added = rows * nx * c_gamma * p->dx * p->dy;
    for (int y = 0; y < rows; ++y)
        for (int x = 0; x < nx; ++x) removed += carbon[at(x, y, nx)] * p->dx * p->dy;
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            const size_t i = at(x, y, nx);
            if (y + rows < ny) {
                const size_t j = at(x, y + rows, nx);
                carbon[i] = carbon[j];
                for (int a = 0; a < 3; ++a) phi[3 * i + a] = phi[3 * j + a];
            } else {
                carbon[i] = c_gamma;
                phi[3 * i] = 0;
                phi[3 * i + 1] = 0;
                phi[3 * i + 2] = 1;
            }
        }
    int rc = po_close_mu(p, nx, ny, phi, carbon, mu);
    if (rc) return rc;
    s->shift_distance += rows * p->dy;
    s->shifts++;
    s->carbon_added += added;
    s->carbon_removed += removed;
    return PO_OK;
}

/* maybe_shift, pearl_serial.cpp:2053-2071 */
int po_maybe_shift(const po_params* p, int nx, int ny, double* phi, double* carbon, double* mu, po_scalars* s,
                   double shift_trigger, double shift_target, double c_gamma, int* shifted) {
    *shifted = 0;
    const double front = po_front_position(p, nx, ny, phi);
    if (front < shift_trigger) return PO_OK;
    const int rows = (int)floor((front - shift_target) / p->dy);
    double gamma = 0;
    for (int y = 0; y < ny; ++y)
        if (y < rows)
            for (int x = 0; x < nx; ++x) gamma = dmax(gamma, phi[at(x, y, nx) * 3 + 2]);
    if (gamma > 1e-6) return PO_ERR_UNSAFE_SHIFT;
    int rc = po_shift_rows(p, nx, ny, phi, carbon, mu, s, rows, c_gamma);
    if (rc) return rc;
    *shifted = rows;
    return PO_OK;
}

/* snapshot reductions, pearl_serial.cpp:2266-2281 */
int po_snapshot(const po_params* p, int nx, int ny, const double* phi, const double* carbon, const double* mu,
                const po_scalars* s, po_diag* out) {
    double minc = 1e300, maxc = -1e300, minmu = 1e300, maxmu = -1e300, sumerr = 0;
    const size_t n = (size_t)nx * (size_t)ny;
    for (size_t i = 0; i < n; ++i) {
        minc = dmin(minc, carbon[i]);
        maxc = dmax(maxc, carbon[i]);
        minmu = dmin(minmu, mu[i]);
        maxmu = dmax(maxmu, mu[i]);
        const double* q = phi + 3 * i;
        sumerr = dmax(sumerr, fabs(q[0] + q[1] + q[2] - 1));
    }
    out->c_min = minc;
    out->c_max = maxc;
    out->mu_min = minmu;
    out->mu_max = maxmu;
    out->phi_sum_error = sumerr;
    out->mass = po_total_carbon(p, nx, ny, carbon);
    out->ledger = out->mass + s->carbon_removed - s->carbon_added - s->initial_carbon;
    return po_reduced_energy(p, nx, ny, phi, carbon, &out->energy);
}

/* interface_energy_only, pearl_serial.cpp:822-842 */
double po_interface_energy_only(const po_params* p, int nx, int ny, const double* phi) {
    const double eps = p->epsilon, sigma = p->sigma;
    const double pi = pi_value();
    const double obstacle = 16 * sigma / (pi * pi * eps), triple = p->triple / eps;
    double total = 0;
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            double q[3];
            load3(phi, x, y, nx, q);
            total += obstacle * (q[0] * q[1] + q[0] * q[2] + q[1] * q[2]) + triple * q[0] * q[1] * q[2];
            for (int dir = 0; dir < 2; ++dir) {
                if (dir == 1 && y == ny - 1) continue;
                double nb[3];
                if (dir == 0)
                    load3(phi, xp(x, nx), y, nx, nb);
                else
                    load3(phi, x, y + 1, nx, nb);
                const double dist = dir == 0 ? p->dx : p->dy;
                for (int a = 0; a < 3; ++a)
                    for (int b = a + 1; b < 3; ++b) {
                        const double z = (q[a] * nb[b] - nb[a] * q[b]) / dist;
                        total += eps * sigma * z * z;
                    }
            }
        }
    return total * p->dx * p->dy;
}

/* phase_fractions, pearl_serial.cpp:856-864 */
static void phase_fractions(int nx, int ny, const double* phi, double out[3]) {
    double local[3] = {0, 0, 0};
    const size_t n = (size_t)nx * (size_t)ny;
    for (size_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) local[a] += phi[3 * i + a];
    const double cells = (double)nx * ny;
    for (int a = 0; a < 3; ++a) out[a] = local[a] / cells;
}

/* smooth_interface_only, pearl_serial.cpp:869-958 */
int po_smooth_interface_only(const po_params* p, int nx, int ny, double* phi, int max_steps, int min_steps,
                             double energy_rtol, double max_phase_change, po_smooth_report* report) {
    if (max_steps < 1 || min_steps < 0 || min_steps > max_steps || !(energy_rtol > 0) || !(max_phase_change > 0) ||
        max_phase_change > .2)
        return PO_ERR_INVALID_ARGUMENT;
    po_smooth_report rep;
    memset(&rep, 0, sizeof rep);
    phase_fractions(nx, ny, phi, rep.phase_fraction_before);
    rep.energy_initial = po_interface_energy_only(p, nx, ny, phi);
    double previous = rep.energy_initial;
    const double eps = p->epsilon, sigma = p->sigma;
    const double pi = pi_value();
    const double obs = 16 * sigma / (pi * pi * eps), tr = p->triple / eps;
    const double base_scale = .12 * dmin(p->dx * p->dx, p->dy * p->dy) / (eps * sigma);
    const size_t n = (size_t)nx * (size_t)ny;
    double* force = (double*)malloc(sizeof(double) * 3 * n * 2);
    if (!force) return PO_ERR_INVALID_ARGUMENT;
    double* trial = force + 3 * n;
    static const int ox[4] = {-1, 1, 0, 0}, oy[4] = {0, 0, -1, 1};
    int rc = PO_OK;
    for (int step = 1; step <= max_steps; ++step) {
        double force_max = 0;
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                double q[3], f[3];
                load3(phi, x, y, nx, q);
                for (int a = 0; a < 3; ++a)
                    f[a] = obs * (q[(a + 1) % 3] + q[(a + 2) % 3]) + tr * q[(a + 1) % 3] * q[(a + 2) % 3];
                for (int dir = 0; dir < 4; ++dir) {
                    if ((dir == 2 && y == 0) || (dir == 3 && y == ny - 1)) continue;
                    int xx = x, yy = y;
                    if (ox[dir] < 0) xx = xm(x, nx);
                    if (ox[dir] > 0) xx = xp(x, nx);
                    if (oy[dir] < 0) yy = ym(y);
                    if (oy[dir] > 0) yy = yp(y, ny);
                    double nb[3];
                    load3(phi, xx, yy, nx, nb);
                    const double dist = dir < 2 ? p->dx : p->dy;
                    for (int a = 0; a < 3; ++a)
                        for (int b = a + 1; b < 3; ++b) {
                            const double w = 2 * eps * sigma * (q[a] * nb[b] - nb[a] * q[b]) / (dist * dist);
                            f[a] += w * nb[b];
                            f[b] -= w * nb[a];
                        }
                }
                const double mean = (f[0] + f[1] + f[2]) / 3;
                for (int a = 0; a < 3; ++a) {
                    force[at(x, y, nx) * 3 + a] = f[a] - mean;
                    force_max = dmax(force_max, fabs(force[at(x, y, nx) * 3 + a]));
                }
            }
        if (!isfinite(force_max)) {
            rc = PO_ERR_INVALID_ARGUMENT;
            break;
        }
        if (force_max == 0) {
            rep.steps = step - 1;
            rep.converged = 1;
            rep.final_relative_energy_change = 0;
            rep.final_max_phase_change = 0;
            break;
        }
        double scale = dmin(base_scale, max_phase_change / force_max);
        int accepted = 0;
        double new_energy = previous, actual_change = 0;
        for (int backtrack = 0; backtrack < 24 && !accepted; ++backtrack) {
            actual_change = 0;
            for (size_t i = 0; i < n; ++i) {
                double z[3], zp[3];
                for (int a = 0; a < 3; ++a) z[a] = phi[3 * i + a] - scale * force[3 * i + a];
                if (po_project_simplex(z, zp) != PO_OK) {
                    free(force);
                    return PO_ERR_SIMPLEX;
                }
                for (int a = 0; a < 3; ++a) actual_change = dmax(actual_change, fabs(zp[a] - phi[3 * i + a]));
                for (int a = 0; a < 3; ++a) trial[3 * i + a] = zp[a];
            }
            new_energy = po_interface_energy_only(p, nx, ny, trial);
            double big = 1.0;
            if (big < fabs(previous)) big = fabs(previous);
            if (big < fabs(rep.energy_initial)) big = fabs(rep.energy_initial);
            const double etol = 1e-14 * big;
            if (isfinite(new_energy) && new_energy <= previous + etol)
                accepted = 1;
            else
                scale *= .5;
        }
        if (!accepted) {
            rc = PO_ERR_INVALID_ARGUMENT;
            break;
        }
        memcpy(phi, trial, sizeof(double) * 3 * n);
        const double rel = fabs(previous - new_energy) / dmax(fabs(previous), 1e-300);
        rep.steps = step;
        rep.energy_final = new_energy;
        rep.final_relative_energy_change = rel;
        rep.final_max_phase_change = actual_change;
        previous = new_energy;
        if (step >= min_steps && rel < energy_rtol && actual_change < 1e-5) {
            rep.converged = 1;
            break;
        }
    }
    free(force);
    if (rc) return rc;
    if (rep.steps == 0) rep.energy_final = rep.energy_initial;
    phase_fractions(nx, ny, phi, rep.phase_fraction_after);
    if (report) *report = rep;
    return PO_OK;
}
