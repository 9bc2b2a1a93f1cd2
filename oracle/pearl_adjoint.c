/*
 * pearl_adjoint.c — CPU reference gradient of the Pearl time step.
 *
 * TEST INFRASTRUCTURE ONLY (same rules as pearl_oracle.c): what the device
 * adjoint is compared against, never part of the product.
 *
 * The reference has no adjoint.  This file differentiates the discrete step
 * of pearl_oracle.c (itself bit-identical to pearl_serial.cpp) by hand:
 *
 *   forward step k (accepted dt):
 *     phi' = P(z),  z_a = q_a - s (F_a - mean F),  s = dt M / (tau(q) eps)
 *            (propose_phi, pearl_serial.cpp:961-1002; P = project_simplex :491-509)
 *     A(phi') u = c - icpt(phi')                    (implicit_diffusion :1010-1080)
 *     c' = icpt(phi') + chi(phi') u,  mu' = mu_ref + u   (:1082-1093, exact solve)
 *
 *   reverse step k, given (phi'^, c'^, mu'^):
 *     u^ = mu'^ + chi c'^;   A lambda = u^   (A is symmetric)
 *     c^ = lambda;   chi^ = (c'^ - lambda)(u + mu_ref);   icpt^ = c'^ - lambda
 *     K^_i = sum over faces f=(i,j) of -dt (lambda_i - lambda_j)(u_i - u_j) / (2 h^2)
 *     phi'^ += dchi/dphi' chi^ + dicpt/dphi' ... + dK/dphi' K^
 *     z^ = Jacobian of P on its active set S applied to phi'^
 *     F^ = -s (z^ - mean z^),  s^ = -sum_a z^_a (F_a - mean F)
 *     q^, mu^ from the forces (obstacle, triple, chemical and gradient terms)
 *
 * With the linear system solved to cg_rtol the gradient is exact up to that
 * tolerance; the projection's Jacobian is taken on the active set of the
 * forward (the map is piecewise linear there).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "pearl_oracle.h"

static inline int xm(int x, int nx) { return x == 0 ? nx - 1 : x - 1; }
static inline int xp(int x, int nx) { return x == nx - 1 ? 0 : x + 1; }
static inline size_t at(int x, int y, int nx) { return (size_t)y * (size_t)nx + (size_t)x; }

/* neighbour (x,y) of direction dir (0 W, 1 E, 2 S, 3 N); 0 at a y wall */
static inline int neighbour(int x, int y, int nx, int ny, int dir, int* xx, int* yy) {
    *xx = x;
    *yy = y;
    if (dir == 0) *xx = xm(x, nx);
    if (dir == 1) *xx = xp(x, nx);
    if (dir == 2) {
        if (y == 0) return 0;
        *yy = y - 1;
    }
    if (dir == 3) {
        if (y == ny - 1) return 0;
        *yy = y + 1;
    }
    return 1;
}

/* Forces of propose_phi at one cell, in the same operation order as
 * po_propose_phi (pearl_serial.cpp:966-986). */
static void forces(const po_params* p, int nx, int ny, const double* phi, const double* mu, int x, int y,
                   double F[3]) {
    const double eps = p->epsilon, sigma = p->sigma, pi = acos(-1.0);
    const double obs = 16 * sigma / (pi * pi * eps), tr = p->triple / eps;
    const double* q = phi + at(x, y, nx) * 3;
    const double m = mu[at(x, y, nx)];
    const double psi0 = po_psi(p, 2, m);
    double dh[3][3];
    po_weight_derivatives(q, dh);
    for (int a = 0; a < 3; ++a) {
        F[a] = obs * (q[(a + 1) % 3] + q[(a + 2) % 3]) + tr * q[(a + 1) % 3] * q[(a + 2) % 3];
        for (int b = 0; b < 3; ++b) F[a] += (po_psi(p, b, m) - psi0) * dh[b][a] / p->Vm;
    }
    static const int order[4] = {0, 1, 2, 3};
    for (int k = 0; k < 4; ++k) {
        const int dir = order[k];
        int xx, yy;
        if (!neighbour(x, y, nx, ny, dir, &xx, &yy)) continue;
        const double* nb = phi + at(xx, yy, nx) * 3;
        const double dist = dir < 2 ? p->dx : p->dy;
        for (int a = 0; a < 3; ++a)
            for (int b = a + 1; b < 3; ++b) {
                const double w = 2 * eps * sigma * (q[a] * nb[b] - nb[a] * q[b]) / (dist * dist);
                F[a] += w * nb[b];
                F[b] -= w * nb[a];
            }
    }
}

/* Threshold of project_simplex (pearl_serial.cpp:491-509) for z. */
static double simplex_threshold(const double z[3]) {
    double s0 = z[0], s1 = z[1], s2 = z[2], t;
    if (s0 < s1) { t = s0; s0 = s1; s1 = t; }
    if (s1 < s2) { t = s1; s1 = s2; s2 = t; }
    if (s0 < s1) { t = s0; s0 = s1; s1 = t; }
    const double sorted[3] = {s0, s1, s2};
    double sum = 0.0, threshold = 0.0;
    for (int j = 0; j < 3; ++j) {
        sum += sorted[j];
        const double candidate = (sum - 1.0) / (j + 1);
        if (sorted[j] > candidate) threshold = candidate;
    }
    return threshold;
}

/* Reverse of propose_phi.  gbar = phi'^ (in), qbar = phi^ (out, overwritten),
 * mubar = mu^ (out, overwritten); grad[0] += M^, grad[1] += sigma^. */
static void propose_adjoint(const po_params* p, int nx, int ny, double dt, const double* phi, const double* mu,
                            const double* gbar, double* qbar, double* mubar, double* Fbar, double grad[3]) {
    const double eps = p->epsilon, sigma = p->sigma, pi = acos(-1.0);
    const double obs = 16 * sigma / (pi * pi * eps), tr = p->triple / eps;
    const size_t n = (size_t)nx * ny;
    memset(qbar, 0, sizeof(double) * 3 * n);
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            const size_t i = at(x, y, nx);
            const double* q = phi + 3 * i;
            const double m = mu[i];
            double F[3];
            forces(p, nx, ny, phi, mu, x, y, F);
            const double mean = (F[0] + F[1] + F[2]) / 3;
            const double tau = po_local_tau(q, p->tau);
            const double s = dt / (tau * eps);
            double z[3], g[3];
            for (int a = 0; a < 3; ++a) {
                g[a] = F[a] - mean;
                z[a] = q[a] - s * g[a];
            }
            const double th = simplex_threshold(z);
            int active[3], na = 0;
            double gsum = 0;
            for (int a = 0; a < 3; ++a) {
                active[a] = z[a] - th > 0;
                if (active[a]) {
                    ++na;
                    gsum += gbar[3 * i + a];
                }
            }
            double zb[3];
            for (int a = 0; a < 3; ++a) zb[a] = active[a] ? gbar[3 * i + a] - gsum / na : 0.0;
            /* z = q - s g */
            double* qb = qbar + 3 * i;
            for (int a = 0; a < 3; ++a) qb[a] += zb[a];
            const double sbar = -(zb[0] * g[0] + zb[1] * g[1] + zb[2] * g[2]);
            const double zmean = (zb[0] + zb[1] + zb[2]) / 3;
            double* Fb = Fbar + 3 * i;
            for (int a = 0; a < 3; ++a) Fb[a] = -s * (zb[a] - zmean);
            /* s = dt M / (tau eps): M^ (at M = 1) and tau^ */
            grad[0] += sbar * s;
            const double taubar = -sbar * s / tau;
            const double w0 = q[0] * q[1], w1 = q[0] * q[2], w2 = q[1] * q[2], W = w0 + w1 + w2;
            if (W > 1e-30) {
                const double wb0 = taubar * (p->tau[0] - tau) / W, wb1 = taubar * (p->tau[1] - tau) / W,
                             wb2 = taubar * (p->tau[2] - tau) / W;
                qb[0] += wb0 * q[1] + wb1 * q[2];
                qb[1] += wb0 * q[0] + wb2 * q[2];
                qb[2] += wb1 * q[0] + wb2 * q[1];
            }
            /* obstacle and triple terms */
            for (int a = 0; a < 3; ++a) {
                const int a1 = (a + 1) % 3, a2 = (a + 2) % 3;
                qb[a1] += Fb[a] * (obs + tr * q[a2]);
                qb[a2] += Fb[a] * (obs + tr * q[a1]);
                grad[1] += Fb[a] * (q[a1] + q[a2]) * obs / sigma;
            }
            /* chemical term: sum_b (psi_b(m) - psi_g(m)) dh[b][a] / Vm */
            double dh[3][3], dpsi[3], dpsi_dm[3];
            po_weight_derivatives(q, dh);
            const double psi_g = po_psi(p, 2, m), dpsig = -(m - p->B[2]) / (2 * p->A[2]);
            double dsum = 0;
            for (int b = 0; b < 3; ++b) {
                dpsi[b] = po_psi(p, b, m) - psi_g;
                dpsi_dm[b] = -(m - p->B[b]) / (2 * p->A[b]) - dpsig;
                dsum += dpsi[b];
            }
            double mb = 0;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) mb += Fb[a] * dpsi_dm[b] * dh[b][a] / p->Vm;
            mubar[i] = mb;
            /* d dh[b][a] / d q_c = d dtriple_a / d q_c + [a==b==c] (6 - 12 q_a) */
            for (int a = 0; a < 3; ++a)
                for (int c = 0; c < 3; ++c) {
                    double d = 0;
                    if (c != a) d = dsum * 2 * q[3 - a - c];
                    if (c == a) d = dpsi[a] * (6 - 12 * q[a]);
                    qb[c] += Fb[a] * d / p->Vm;
                }
        }
    /* gradient terms: scatter to the cell (q) and its neighbour (n) */
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            const size_t i = at(x, y, nx);
            const double* q = phi + 3 * i;
            const double* Fb = Fbar + 3 * i;
            for (int dir = 0; dir < 4; ++dir) {
                int xx, yy;
                if (!neighbour(x, y, nx, ny, dir, &xx, &yy)) continue;
                const size_t j = at(xx, yy, nx);
                const double* nb = phi + 3 * j;
                const double dist = dir < 2 ? p->dx : p->dy;
                const double kappa = 2 * eps * sigma / (dist * dist);
                for (int a = 0; a < 3; ++a)
                    for (int b = a + 1; b < 3; ++b) {
                        const double X = q[a] * nb[b] - nb[a] * q[b];
                        const double Y = Fb[a] * nb[b] - Fb[b] * nb[a];
                        qbar[3 * i + a] += kappa * nb[b] * Y;
                        qbar[3 * i + b] -= kappa * nb[a] * Y;
                        qbar[3 * j + a] += kappa * (-q[b] * Y - X * Fb[b]);
                        qbar[3 * j + b] += kappa * (q[a] * Y + X * Fb[a]);
                        grad[1] += kappa * X * Y / sigma;
                    }
            }
        }
}

static void face_w(const po_params* p, const double* K, int x, int y, int nx, int ny, double w[4]) {
    const double k = K[at(x, y, nx)];
    const double dx2 = p->dx * p->dx, dy2 = p->dy * p->dy;
    w[0] = .5 * (k + K[at(xm(x, nx), y, nx)]) / dx2;
    w[1] = .5 * (k + K[at(xp(x, nx), y, nx)]) / dx2;
    w[2] = y == 0 ? 0 : .5 * (k + K[at(x, y - 1, nx)]) / dy2;
    w[3] = y == ny - 1 ? 0 : .5 * (k + K[at(x, y + 1, nx)]) / dy2;
}

static void apply_A(const po_params* p, const double* K, const double* chi, double dt, int nx, int ny,
                    const double* in, double* out) {
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            double w[4];
            face_w(p, K, x, y, nx, ny, w);
            const double c = in[at(x, y, nx)];
            double s = w[0] * (c - in[at(xm(x, nx), y, nx)]) + w[1] * (c - in[at(xp(x, nx), y, nx)]);
            if (y > 0) s += w[2] * (c - in[at(x, y - 1, nx)]);
            if (y < ny - 1) s += w[3] * (c - in[at(x, y + 1, nx)]);
            out[at(x, y, nx)] = chi[at(x, y, nx)] * c + dt * s;
        }
}

/* Reverse of implicit_diffusion.  cbar: c'^ in, lambda out.  phibar += the
 * trial-phi adjoint.  grad[2] += D_gamma^.  Returns CG iterations or -1. */
static int diffusion_adjoint(const po_params* p, int nx, int ny, double dt, const double* tphi, const double* u,
                             double* cbar, const double* mubar_next, double* phibar, double* work,
                             double grad[3]) {
    const size_t n = (size_t)nx * ny;
    double *chi = work, *K = work + n, *ub = work + 2 * n, *lam = work + 3 * n, *r = work + 4 * n;
    double *z = work + 5 * n, *pd = work + 6 * n, *Ap = work + 7 * n, *diag = work + 8 * n;
    double chi_q[3];
    for (int q = 0; q < 3; ++q) chi_q[q] = 1.0 / (2.0 * p->A[q]);
    double ub2 = 0;
    for (size_t i = 0; i < n; ++i) {
        double c, ci, k;
        if (po_mixture(p, tphi + 3 * i, &c, &ci, &k) != PO_OK) return -1;
        chi[i] = c;
        K[i] = k;
        ub[i] = mubar_next[i] + c * cbar[i];
        ub2 += ub[i] * ub[i];
    }
    /* Jacobi-PCG for A lambda = u^ from lambda = 0 */
    int it = 0;
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            double w[4];
            face_w(p, K, x, y, nx, ny, w);
            const size_t i = at(x, y, nx);
            diag[i] = chi[i] + dt * (w[0] + w[1] + w[2] + w[3]);
            lam[i] = 0;
            r[i] = ub[i];
            z[i] = r[i] / diag[i];
            pd[i] = z[i];
        }
    const double tol = p->cg_rtol * sqrt(ub2);
    double rz = 0, rr = ub2;
    for (size_t i = 0; i < n; ++i) rz += r[i] * z[i];
    while (sqrt(rr) > tol && it < p->cg_max) {
        apply_A(p, K, chi, dt, nx, ny, pd, Ap);
        double pAp = 0;
        for (size_t i = 0; i < n; ++i) pAp += pd[i] * Ap[i];
        if (!(pAp > 0)) return -1;
        const double alpha = rz / pAp;
        double rzn = 0;
        rr = 0;
        for (size_t i = 0; i < n; ++i) {
            lam[i] += alpha * pd[i];
            r[i] -= alpha * Ap[i];
            z[i] = r[i] / diag[i];
            rzn += r[i] * z[i];
            rr += r[i] * r[i];
        }
        const double beta = rzn / rz;
        rz = rzn;
        for (size_t i = 0; i < n; ++i) pd[i] = z[i] + beta * pd[i];
        ++it;
    }
    if (sqrt(rr) > tol) return -1;
    const double mu_r = p->mu_reference;
    const double ih2x = 0.5 / (p->dx * p->dx), ih2y = 0.5 / (p->dy * p->dy);
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            const size_t i = at(x, y, nx);
            double Kb = 0;
            for (int dir = 0; dir < 4; ++dir) {
                int xx, yy;
                if (!neighbour(x, y, nx, ny, dir, &xx, &yy)) continue;
                const size_t j = at(xx, yy, nx);
                Kb += -dt * (lam[i] - lam[j]) * (u[i] - u[j]) * (dir < 2 ? ih2x : ih2y);
            }
            const double cb = cbar[i] - lam[i];
            const double* q = tphi + 3 * i;
            double dh[3][3], hb[3];
            po_weight_derivatives(q, dh);
            for (int k = 0; k < 3; ++k) hb[k] = chi_q[k] * cb * (u[i] + mu_r - p->B[k]);
            for (int a = 0; a < 3; ++a) {
                double s = Kb * p->D[a] * chi_q[a];
                for (int k = 0; k < 3; ++k) s += hb[k] * dh[k][a];
                phibar[3 * i + a] += s;
            }
            grad[2] += Kb * q[2] * chi_q[2];
            cbar[i] = lam[i];
        }
    return it;
}

int po_adjoint_objective(const po_params* p, int nx, int ny, double* phi, double* carbon, double* mu,
                         po_scalars* s, int nsteps, const double* target_alpha, double* objective) {
    int why = 0, done = 0;
    const int rc = po_advance_n(p, nx, ny, phi, carbon, mu, s, nsteps, NULL, 1e300, NULL, &why, &done);
    if (rc) return rc;
    const size_t n = (size_t)nx * ny;
    double J = 0;
    for (size_t i = 0; i < n; ++i) {
        const double d = phi[3 * i] - target_alpha[i];
        J += d * d;
    }
    *objective = J;
    return PO_OK;
}

int po_adjoint_gradient(const po_params* p, int nx, int ny, double* phi, double* carbon, double* mu, po_scalars* s,
                        int nsteps, int checkpoint_every, const double* target_alpha, po_adjoint_report* out) {
    if (!p || !phi || !carbon || !mu || !s || !target_alpha || !out || nsteps < 1 || checkpoint_every < 1 ||
        p->phase_only)
        return PO_ERR_INVALID_ARGUMENT;
    memset(out, 0, sizeof *out);
    const size_t n = (size_t)nx * ny, st = 5 * n;
    const int nseg = (nsteps + checkpoint_every - 1) / checkpoint_every;
    const int K = checkpoint_every;
    double* ckpt = (double*)malloc(sizeof(double) * st * (size_t)nseg);
    double* dts = (double*)malloc(sizeof(double) * (size_t)nsteps);
    double* tape = (double*)malloc(sizeof(double) * st * (size_t)(K + 1));
    double* utape = (double*)malloc(sizeof(double) * n * (size_t)K);
    double* adj = (double*)malloc(sizeof(double) * n * 5);
    double* tmp = (double*)malloc(sizeof(double) * n * 7);
    double* work = (double*)malloc(sizeof(double) * n * 9);
    int rc = PO_OK;
    if (!ckpt || !dts || !tape || !utape || !adj || !tmp || !work) {
        rc = PO_ERR_INVALID_ARGUMENT;
        goto done;
    }
    /* forward with checkpoints */
    for (int k = 0; k < nsteps; ++k) {
        if (k % K == 0) {
            double* c = ckpt + st * (size_t)(k / K);
            memcpy(c, phi, sizeof(double) * 3 * n);
            memcpy(c + 3 * n, carbon, sizeof(double) * n);
            memcpy(c + 4 * n, mu, sizeof(double) * n);
        }
        po_step_info info;
        int why = 0;
        rc = po_advance(p, nx, ny, phi, carbon, mu, s, 1e300, &info, &why);
        if (rc) goto done;
        dts[k] = info.accepted_dt;
        out->cg_forward += info.cg_iterations;
    }
    out->steps = nsteps;
    out->checkpoints = nseg;
    /* objective and the adjoint of the final state */
    {
        double J = 0;
        memset(adj, 0, sizeof(double) * 5 * n);
        for (size_t i = 0; i < n; ++i) {
            const double d = phi[3 * i] - target_alpha[i];
            J += d * d;
            adj[3 * i] = 2 * d;
        }
        out->objective = J;
    }
    for (int seg = nseg - 1; seg >= 0; --seg) {
        const int k0 = seg * K, len = (k0 + K <= nsteps) ? K : nsteps - k0;
        memcpy(tape, ckpt + st * (size_t)seg, sizeof(double) * st);
        for (int j = 0; j < len; ++j) {
            const double* sj = tape + st * (size_t)j;
            double* sn = tape + st * (size_t)(j + 1);
            double change;
            rc = po_propose_phi(p, nx, ny, sj, sj + 4 * n, sn, dts[k0 + j], &change);
            if (rc) goto done;
            po_diffusion_info di;
            rc = po_implicit_diffusion_u(p, nx, ny, sj + 3 * n, sj + 4 * n, sn, sn + 3 * n, sn + 4 * n, dts[k0 + j],
                                         &di, utape + n * (size_t)j);
            if (rc) goto done;
            if (!di.ok) {
                rc = PO_ERR_RETRY_LIMIT;
                goto done;
            }
        }
        for (int j = len - 1; j >= 0; --j) {
            const double* sj = tape + st * (size_t)j;
            const double* sn = tape + st * (size_t)(j + 1);
            double* phibar = adj;
            double* cbar = adj + 3 * n;
            double* mubar = adj + 4 * n;
            const int it = diffusion_adjoint(p, nx, ny, dts[k0 + j], sn, utape + n * (size_t)j, cbar, mubar, phibar,
                                             work, out->grad);
            if (it < 0) {
                rc = PO_ERR_RETRY_LIMIT;
                goto done;
            }
            out->cg_adjoint += it;
            double* qbar = tmp;
            double* mub = tmp + 3 * n;
            double* Fbar = tmp + 4 * n;
            propose_adjoint(p, nx, ny, dts[k0 + j], sj, sj + 4 * n, phibar, qbar, mub, Fbar, out->grad);
            memcpy(phibar, qbar, sizeof(double) * 3 * n);
            memcpy(mubar, mub, sizeof(double) * n);
        }
    }
done:
    free(ckpt);
    free(dts);
    free(tape);
    free(utape);
    free(adj);
    free(tmp);
    free(work);
    return rc;
}
