/*
 * pearl_oracle.c — CPU restatement of the Pearl hot path (TEST INFRASTRUCTURE).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
 * this file, as the reference results are compared against or as the timed
 * CPU port; the product never does.
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

/* ---- the device's summation order (pearl_oracle.h, po_set_device_order) ----
 * Off by default: every function below then sums in the reference's
 * sequential row-major order.  The per-cell loops that carry no sum run on
 * g_threads host threads in this mode; their results do not depend on it. */
static int g_dev = 0;
static po_device_order g_ord;
static int g_threads = 1;
#define DEV_PARALLEL_FOR _Pragma("omp parallel for num_threads(g_threads) if(g_dev && g_threads > 1) schedule(static)")

/* the device's step-energy carry: energy and carbon mass of the last accepted trial */
static struct {
    int valid;
    double e0, mass0;
} g_carry;

void po_set_device_order(const po_device_order* o) {
    g_carry.valid = 0;
    if (!o) {
        g_dev = 0;
        g_threads = 1;
        return;
    }
    g_ord = *o;
    if (g_ord.warps != 16) g_ord.warps = 8;
    if (g_ord.warps_x_log2 < 0 || (1 << g_ord.warps_x_log2) > g_ord.warps) g_ord.warps_x_log2 = 0;
    if (g_ord.blocks < 1) g_ord.blocks = 1;
    g_threads = o->threads > 1 ? o->threads : 1;
    g_dev = 1;
}

/* A warp's shuffle-down tree over its 32 lanes: at offsets 16, 8, 4, 2, 1
 * lane i adds lane i + o; the warp's value is lane 0's. */
static double lanes_tree(double a[32]) {
    for (int o = 16; o > 0; o >>= 1)
        for (int i = 0; i < o; ++i) a[i] = a[i] + a[i + o];
    return a[0];
}

double po_device_sum(int nx, int ny, const double* v, int reverse) {
    const int W = g_ord.warps, wx = g_dev ? g_ord.warps_x_log2 : 0, G = g_dev ? g_ord.blocks : 1;
    const int tile_w = 32 << wx, tile_h = (2 * W) >> wx;
    const int ntx = (nx + tile_w - 1) / tile_w, nty = (ny + tile_h - 1) / tile_h, ntiles = ntx * nty;
    double* part = (double*)malloc(sizeof(double) * (size_t)G);
    if (!part) return NAN;
#pragma omp parallel for num_threads(g_threads) if(g_threads > 1) schedule(dynamic, 4)
    for (int b = 0; b < G; ++b) {
        /* block b owns tiles b, b+G, ...; each thread keeps one running sum over them */
        const int nb = b < ntiles ? (ntiles - 1 - b) / G + 1 : 0;
        double block = 0;
        for (int w = 0; w < W; ++w) {
            const int wxi = w & ((1 << wx) - 1), wy = w >> wx;
            double lanes[32];
            for (int l = 0; l < 32; ++l) {
                double acc = 0;
                for (int k = 0; k < nb; ++k) {
                    const int t = b + (reverse ? nb - 1 - k : k) * G;
                    const int x = (t % ntx) * tile_w + (wxi << 5) + l, y0 = (t / ntx) * tile_h + 2 * wy;
                    if (x < nx && y0 < ny) {
                        acc += v[(size_t)y0 * (size_t)nx + (size_t)x];
                        if (y0 + 1 < ny) acc += v[(size_t)(y0 + 1) * (size_t)nx + (size_t)x];
                    }
                }
                lanes[l] = acc;
            }
            const double wv = lanes_tree(lanes);
            block = w == 0 ? wv : block + wv; /* warps in index order */
        }
        part[b] = block;
    }
    /* 32 lanes add the block partials strided by 32, then one more tree */
    double lanes[32];
    for (int l = 0; l < 32; ++l) {
        double acc = 0;
        for (int b = l; b < G; b += 32) acc += part[b];
        lanes[l] = acc;
    }
    free(part);
    return lanes_tree(lanes);
}

/* the device's dot product: per-cell products, then its tree */
static double device_dot(const double* a, const double* b, double* prod, int nx, int ny, int reverse) {
    const size_t n = (size_t)nx * (size_t)ny;
    DEV_PARALLEL_FOR
    for (long long i = 0; i < (long long)n; ++i) prod[i] = a[i] * b[i];
    return po_device_sum(nx, ny, prod, reverse);
}

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
    if (g_dev) return po_device_sum(nx, ny, carbon, 0) * p->dx * p->dy; /* step-start order */
    double v = 0;
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) v += carbon[at(x, y, nx)];
    return v * p->dx * p->dy;
}

/* reduced_energy's density per cell as the device sums it (pearl_serial.cpp:800-819):
 * the cell's chemical, obstacle and triple terms, then its +x and +y face terms
 * added to that cell's value.  cell[] receives nx*ny values; returns
 * PO_ERR_MIXTURE where the reference throws. */
static int energy_cells_device(const po_params* p, int nx, int ny, const double* phi, const double* carbon,
                               double* cell) {
    const double eps = p->epsilon, sigma = p->sigma;
    const double pi = pi_value();
    const double obstacle = 16 * sigma / (pi * pi * eps), triple = p->triple / eps;
    const double mu_r = p->mu_reference;
    const double psi[3] = {po_psi(p, 0, mu_r) - po_psi(p, 2, mu_r), po_psi(p, 1, mu_r) - po_psi(p, 2, mu_r), 0};
    int bad = 0;
#pragma omp parallel for num_threads(g_threads) if(g_threads > 1) schedule(static) reduction(|:bad)
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            double q[3], h[3];
            load3(phi, x, y, nx, q);
            po_weights(q, h);
            double chem = 0;
            for (int a = 0; a < 3; ++a) chem += h[a] * psi[a];
            if (!p->phase_only) {
                double chi, ci, k;
                if (po_mixture(p, q, &chi, &ci, &k) != PO_OK) bad = 1;
                const double dc = carbon[at(x, y, nx)] - fma(chi, mu_r, ci);
                chem += .5 * dc * dc / chi;
            }
            double t = chem / p->Vm + obstacle * (q[0] * q[1] + q[0] * q[2] + q[1] * q[2]) + triple * q[0] * q[1] * q[2];
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
                        t += eps * sigma * z * z;
                    }
            }
            cell[at(x, y, nx)] = t;
        }
    return bad ? PO_ERR_MIXTURE : PO_OK;
}

/* reduced_energy in the device's order: the step-start pass walks forwards,
 * the final update of a step backwards */
static int reduced_energy_device(const po_params* p, int nx, int ny, const double* phi, const double* carbon,
                                 int reverse, double* energy) {
    double* cell = (double*)malloc(sizeof(double) * (size_t)nx * (size_t)ny);
    if (!cell) return PO_ERR_INVALID_ARGUMENT;
    const int rc = energy_cells_device(p, nx, ny, phi, carbon, cell);
    if (rc == PO_OK) *energy = po_device_sum(nx, ny, cell, reverse) * p->dx * p->dy;
    free(cell);
    return rc;
}

/* reduced_energy, pearl_serial.cpp:793-821 */
int po_reduced_energy(const po_params* p, int nx, int ny, const double* phi, const double* carbon,
                      double* energy) {
    if (g_dev) return reduced_energy_device(p, nx, ny, phi, carbon, 0, energy);
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

/* propose_phi for the cell (x, y), pearl_serial.cpp:966-1001: writes the trial
 * phase fractions and *change = max |dphi| of the cell (INFINITY, with the old
 * fractions kept, where the proposal is not finite, :990-996). */
static int propose_cell(const po_params* p, int nx, int ny, const double* phi_old, const double* mu_old,
                        double* trial_phi, double dt, double obs, double tr, int x, int y, double* change) {
    static const int ox[4] = {-1, 1, 0, 0}, oy[4] = {0, 0, -1, 1};
    const double eps = p->epsilon, sigma = p->sigma;
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
    const double mean = (force[0] + force[1] + force[2]) / 3, scale = dt / (po_local_tau(q, p->tau) * eps);
    double z[3];
    for (int a = 0; a < 3; ++a) z[a] = q[a] - scale * (force[a] - mean);
    int finite = 1;
    for (int a = 0; a < 3; ++a) finite = finite && isfinite(z[a]);
    double* out = trial_phi + at(x, y, nx) * 3;
    if (!finite) {
        *change = INFINITY;
        out[0] = q[0];
        out[1] = q[1];
        out[2] = q[2];
        return PO_OK;
    }
    double zp[3];
    if (po_project_simplex(z, zp) != PO_OK) return PO_ERR_SIMPLEX;
    double c = 0;
    for (int a = 0; a < 3; ++a) c = dmax(c, fabs(zp[a] - q[a]));
    *change = c;
    out[0] = zp[0];
    out[1] = zp[1];
    out[2] = zp[2];
    return PO_OK;
}

/* propose_phi, pearl_serial.cpp:961-1002.  The global max |dphi| is the same
 * in any cell order; in the device's order the rows run on host threads. */
int po_propose_phi(const po_params* p, int nx, int ny, const double* phi_old, const double* mu_old,
                   double* trial_phi, double dt, double* change_out) {
    const double eps = p->epsilon, sigma = p->sigma;
    const double pi = pi_value();
    const double obs = 16 * sigma / (pi * pi * eps), tr = p->triple / eps;
    double change = 0;
    if (g_dev) {
        int bad = 0;
#pragma omp parallel for num_threads(g_threads) if(g_threads > 1) schedule(static) reduction(max:change) reduction(|:bad)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                double c;
                if (propose_cell(p, nx, ny, phi_old, mu_old, trial_phi, dt, obs, tr, x, y, &c) != PO_OK)
                    bad = 1;
                else
                    change = c > change ? c : change;
            }
        if (bad) return PO_ERR_SIMPLEX;
        *change_out = change;
        return PO_OK;
    }
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            double c;
            if (propose_cell(p, nx, ny, phi_old, mu_old, trial_phi, dt, obs, tr, x, y, &c) != PO_OK)
                return PO_ERR_SIMPLEX;
            change = dmax(change, c);
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
    DEV_PARALLEL_FOR
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
 * the converged solution u = mu - mu_reference of the linear system.
 *
 * In the device's order (po_set_device_order) every dot product is the
 * device's tree over the same per-cell products, walked as the device's pass
 * that forms it: the set-up sums (rhs.rhs, r.z, r.r), the CG update's (r.z,
 * r.r) and the restart's r.z forwards, the apply's p.Ap and the true residual's
 * r.r backwards; the residual tested at the head of an iteration is the r.r of
 * the pass that last wrote r, which is what the reference recomputes there. */
int po_implicit_diffusion_u(const po_params* p, int nx, int ny, const double* carbon_old, const double* mu_old,
                            const double* trial_phi, double* trial_carbon, double* trial_mu, double dt,
                            po_diffusion_info* info, double* u_out) {
    const size_t n = (size_t)nx * (size_t)ny;
    const long long nn = (long long)n;
    const double mu_r = p->mu_reference;
    double* mem = (double*)malloc(sizeof(double) * n * 11);
    if (!mem) return PO_ERR_INVALID_ARGUMENT;
    double *chi = mem, *icpt = mem + n, *K = mem + 2 * n, *rhs = mem + 3 * n, *u = mem + 4 * n, *diag = mem + 5 * n;
    double *r = mem + 6 * n, *z = mem + 7 * n, *pd = mem + 8 * n, *Ap = mem + 9 * n, *prod = mem + 10 * n;
#define PO_DOT(a, b, reverse) (g_dev ? device_dot(a, b, prod, nx, ny, reverse) : dot(a, b, n))
    int mixbad = 0;
#pragma omp parallel for num_threads(g_threads) if(g_dev && g_threads > 1) schedule(static) reduction(|:mixbad)
    for (long long i = 0; i < nn; ++i) {
        double c, ci, k;
        if (po_mixture(p, trial_phi + 3 * i, &c, &ci, &k) != PO_OK) mixbad = 1;
        chi[i] = c;
        icpt[i] = fma(c, mu_r, ci);
        K[i] = k;
        rhs[i] = carbon_old[i] - icpt[i];
        u[i] = mu_old[i] - mu_r;
    }
    if (mixbad) {
        free(mem);
        return PO_ERR_MIXTURE;
    }
    apply_op(p, K, chi, dt, nx, ny, u, Ap);
    DEV_PARALLEL_FOR
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
    const double tolerance = p->cg_atol + p->cg_rtol * sqrt(PO_DOT(rhs, rhs, 0));
    double rz = PO_DOT(r, z, 0);
    double rr = g_dev ? PO_DOT(r, r, 0) : 0; /* the device's r.r of the pass that last wrote r */
    po_diffusion_info inf = {0, 0, 0.0, 0.0};
    for (int iteration = 0; iteration <= p->cg_max; ++iteration) {
        inf.it = iteration;
        inf.residual = sqrt(g_dev ? rr : dot(r, r, n));
        if (!isfinite(inf.residual)) {
            *info = inf;
            free(mem);
            return PO_OK;
        }
        if (inf.residual <= tolerance) {
            apply_op(p, K, chi, dt, nx, ny, u, Ap);
            DEV_PARALLEL_FOR
            for (long long i = 0; i < nn; ++i) r[i] = rhs[i] - Ap[i];
            rr = PO_DOT(r, r, 1);
            inf.residual = sqrt(rr);
            if (inf.residual <= tolerance * 1.05) {
                inf.ok = 1;
                break;
            }
            DEV_PARALLEL_FOR
            for (long long i = 0; i < nn; ++i) {
                z[i] = r[i] / diag[i];
                pd[i] = z[i];
            }
            rz = PO_DOT(r, z, 0);
            continue;
        }
        if (iteration == p->cg_max) break;
        apply_op(p, K, chi, dt, nx, ny, pd, Ap);
        const double pAp = PO_DOT(pd, Ap, 1);
        if (!(pAp > 0) || !isfinite(pAp) || !isfinite(rz)) {
            *info = inf;
            free(mem);
            return PO_OK;
        }
        const double alpha = rz / pAp;
        DEV_PARALLEL_FOR
        for (long long i = 0; i < nn; ++i) {
            u[i] += alpha * pd[i];
            r[i] -= alpha * Ap[i];
            z[i] = r[i] / diag[i];
        }
        const double rz_next = PO_DOT(r, z, 0), beta = rz_next / rz;
        if (g_dev) rr = PO_DOT(r, r, 0);
        rz = rz_next;
        DEV_PARALLEL_FOR
        for (long long i = 0; i < nn; ++i) pd[i] = z[i] + beta * pd[i];
    }
#undef PO_DOT
    if (!inf.ok) {
        *info = inf;
        free(mem);
        return PO_OK;
    }
    double closure = 0;
#pragma omp parallel for num_threads(g_threads) if(g_dev && g_threads > 1) schedule(static) reduction(max:closure)
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
    const long long n = (long long)nx * (long long)ny;
#pragma omp parallel for num_threads(g_threads) if(g_dev && g_threads > 1) schedule(static) reduction(&&:good)
    for (long long i = 0; i < n; ++i) {
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
    double e0 = 0, mass0 = 0;
    if (g_dev && g_carry.valid) {
        /* the device carries the accepted trial's energy and mass into the next step */
        e0 = g_carry.e0;
        mass0 = g_carry.mass0;
    } else {
        if (p->check_energy) {
            int rc = po_reduced_energy(p, nx, ny, phi, carbon, &e0);
            if (rc) return rc;
        }
        mass0 = p->phase_only ? 0 : po_total_carbon(p, nx, ny, carbon);
    }
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
        /* in the device's order the trial's mass and energy are sums of its final
         * update, which walks backwards (phase-only: its energy pass, forwards) */
        double m = 0, e1 = 0;
        if (good && !p->phase_only) {
            m = g_dev ? po_device_sum(nx, ny, tc, 1) * p->dx * p->dy : po_total_carbon(p, nx, ny, tc);
            good = fabs(m - mass0) <= 1e-11 * dmax(fabs(mass0), gxgy * p->dx * p->dy * 1e-6);
            why = PO_WHY_MASS;
        }
        if (good && p->check_energy) {
            rc = g_dev ? reduced_energy_device(p, nx, ny, tphi, tc, !p->phase_only, &e1)
                       : po_reduced_energy(p, nx, ny, tphi, tc, &e1);
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
            if (g_dev) {
                g_carry.valid = 1;
                g_carry.e0 = p->check_energy ? e1 : 0;
                g_carry.mass0 = p->phase_only ? 0 : m;
            }
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
    g_carry.valid = 0; /* a run starts from the given fields: no carried energy */
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
