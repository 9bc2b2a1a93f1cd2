// Reverse-mode adjoint of the accepted time step, included by pearl_fp64.cu
// inside namespace pearl_gpu after the forward phases (it uses Dom, Red and
// the forward's thermodynamic helpers).  The reference has no gradient; the
// step map differentiated here is the forward of this library:
//
//   phi' = P(z),  z_a = q_a - s (F_a - mean F),  s = dt M / (tau(q) eps)
//                                            (propose_phi, pearl_serial.cpp:961-1002)
//   A(phi') u = c - icpt(phi'),  c' = icpt + chi u,  mu' = mu_ref + u
//                                            (implicit_diffusion, :1010-1093)
//
// with the linear system taken as solved exactly and the simplex projection P
// differentiated on its active set.  Parameters: the mobility scale M (a
// common factor on every 1/tau, 1 in the forward), sigma and D_gamma.
//
// Layout: every plane has the forward's pitch.  A tape slot holds the state
// after a step (phi x3, c, mu) and that step's solution u: 6 planes.


struct Cell {
    size_t i, n[4];  // centre and W, E, S, N neighbours
    bool has[4];     // S and N are absent at the y walls
};

__device__ __forceinline__ Cell cell_at(const DevParams& P, long long idx) {
    const int x = (int)(idx % P.nx), y = (int)(idx / P.nx);
    Cell c;
    const size_t row = (size_t)y * P.pitch;
    c.i = row + x;
    c.n[0] = row + (x == 0 ? P.nx - 1 : x - 1);
    c.n[1] = row + (x == P.nx - 1 ? 0 : x + 1);
    c.has[0] = c.has[1] = true;
    c.has[2] = y > 0;
    c.has[3] = y < P.ny - 1;
    c.n[2] = c.has[2] ? c.i - P.pitch : c.i;
    c.n[3] = c.has[3] ? c.i + P.pitch : c.i;
    return c;
}

#define FOR_CELLS(P)                                                                                     \
    for (long long idx_ = (long long)a.bid * kThreads + threadIdx.x; idx_ < (long long)(P).nx * (P).ny; \
         idx_ += (long long)a.nblk * kThreads)

// The forces of propose_cell for one cell, with the same arithmetic (so z and
// the projection's active set equal the forward's bitwise).
__device__ __forceinline__ void adj_forces(const DevParams& P, const double q[3], double mu, const double nb[4][3],
                                           const bool has[4], double f[3]) {
    const double psi0 = psi(P, 2, mu);
    const double ps[3] = {psi(P, 0, mu), psi(P, 1, mu), psi0};
    const double dtr[3] = {2.0 * q[1] * q[2], 2.0 * q[0] * q[2], 2.0 * q[0] * q[1]};
#pragma unroll
    for (int aa = 0; aa < 3; ++aa) {
        const double qa1 = q[(aa + 1) % 3], qa2 = q[(aa + 2) % 3];
        f[aa] = P.obs * (qa1 + qa2) + P.tr * qa1 * qa2;
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const double dh = dtr[aa] + (b == aa ? 6.0 * q[b] * (1.0 - q[b]) : 0.0);
            f[aa] += div_by(P, (ps[b] - psi0) * dh, P.Vm, P.r_Vm);
        }
    }
#pragma unroll
    for (int dir = 0; dir < 4; ++dir) {
        if (!has[dir]) continue;
        const double* n = nb[dir];
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
}

__device__ __forceinline__ void load3p(const double* base, size_t pe, size_t i, double v[3]) {
    v[0] = base[i];
    v[1] = base[pe + i];
    v[2] = base[2 * pe + i];
}

// mode 0: J = sum (phi_alpha - target)^2 of the final state; seed the adjoint.
__device__ bool adj_seed(const Dom& a, Red& red, const AdjArgs& g) {
    const DevParams& P = a.P;
    double s = 0;
    FOR_CELLS(P) {
        const Cell c = cell_at(P, idx_);
        const double d = g.ckpt[c.i] - g.target[c.i];
        s += d * d;
        g.J.bphi[0][c.i] = 2.0 * d;
        g.J.bphi[1][c.i] = 0;
        g.J.bphi[2][c.i] = 0;
        g.J.bc[c.i] = 0;
        g.J.bmu[c.i] = 0;
    }
    double v[1] = {s};
    if (!red.reduce<1>(v, kSum, kTagAdjoint)) return false;
    if (a.bid == 0 && threadIdx.x == 0) {
        g.acc[0] = v[0];
        g.acc[1] = g.acc[2] = g.acc[3] = g.acc[4] = 0;
    }
    return true;
}

__device__ __forceinline__ double adj_face(const DevParams& P, double k, double kn, int dir) {
    return 0.5 * (k + kn) / (dir < 2 ? P.dx2 : P.dy2);
}

// One reverse step.  s0: state before the step (5 planes); s1: tape slot of the step.
__device__ bool adj_step(const Dom& a, Red& red, const AdjArgs& g, const double* s0, const double* s1, double dt,
                         double (&grad)[3], long long& cg_its) {
    const DevParams& P = a.P;
    const AdjBufs& J = g.J;
    const size_t pe = (size_t)P.pitch * P.ny;
    const double* u = s1 + 5 * pe;
    // SET-UP (one pass): trial mixture, u^ = mu'^ + chi c'^, and the Jacobi-PCG
    // start for A lambda = u^ warm-started from the previous reverse step's
    // lambda (the adjoint carbon of consecutive steps differs little).  K at
    // the neighbours is recomputed from their trial phi, so no pass is needed
    // between writing K and reading it.
    double ub2 = 0, rz = 0, rr = 0;
    FOR_CELLS(P) {
        const Cell c = cell_at(P, idx_);
        double q[3];
        load3p(s1, pe, c.i, q);
        double chi, cint, k;
        mixture(P, q[0], q[1], q[2], chi, cint, k);
        const double ub = J.bmu[c.i] + chi * J.bc[c.i];
        const double l0 = J.lam[c.i];
        double ws = 0, al = 0;
#pragma unroll
        for (int d = 0; d < 4; ++d)
            if (c.has[d]) {
                double qn[3];
                load3p(s1, pe, c.n[d], qn);
                const double kn = qn[0] * P.D[0] * P.chi_p[0] + qn[1] * P.D[1] * P.chi_p[1] + qn[2] * P.D[2] * P.chi_p[2];
                const double w = adj_face(P, k, kn, d);
                ws += w;
                al += w * (l0 - J.lam[c.n[d]]);
            }
        const double diag = chi + dt * ws;
        const double r = ub - (chi * l0 + dt * al);
        const double z = r / diag;
        J.chi[c.i] = chi;
        J.K[c.i] = k;
        J.diag[c.i] = diag;
        J.r[c.i] = r;
        J.z[c.i] = z;
        ub2 += ub * ub;
        rz += r * z;
        rr += r * r;
    }
    double v3s[3] = {ub2, rz, rr};
    if (!red.reduce<3>(v3s, OPS3(kSum, kSum, kSum), kTagAdjoint)) return false;
    ub2 = v3s[0];
    rz = v3s[1];
    rr = v3s[2];
    const double tol = P.cg_rtol * sqrt(ub2);
    double v1[1];
    int it = 0, pb = 0;
    double beta = 0;
    bool first = true;
    while (sqrt(rr) > tol && it < P.cg_max) {
        // APPLY: p = z + beta p_old (recomputed at the neighbours), Ap, <p,Ap>
        const int po = pb ^ 1;
        double pap = 0;
        FOR_CELLS(P) {
            const Cell c = cell_at(P, idx_);
            const double pc = first ? J.z[c.i] : J.z[c.i] + beta * J.p[pb][c.i];
            const double k = J.K[c.i];
            double s = 0;
#pragma unroll
            for (int d = 0; d < 4; ++d)
                if (c.has[d]) {
                    const size_t j = c.n[d];
                    const double pn = first ? J.z[j] : J.z[j] + beta * J.p[pb][j];
                    s += adj_face(P, k, J.K[j], d) * (pc - pn);
                }
            const double ap = J.chi[c.i] * pc + dt * s;
            J.p[po][c.i] = pc;
            J.Ap[c.i] = ap;
            pap += pc * ap;
        }
        v1[0] = pap;
        if (!red.reduce<1>(v1, kSum, kTagAdjoint)) return false;
        pap = v1[0];
        pb = po;
        if (!(pap > 0) || !isfinite(pap)) break;
        const double alpha = rz / pap;
        double rzn = 0, rrn = 0;
        FOR_CELLS(P) {
            const Cell c = cell_at(P, idx_);
            J.lam[c.i] += alpha * J.p[pb][c.i];
            const double r = J.r[c.i] - alpha * J.Ap[c.i];
            const double z = r / J.diag[c.i];
            J.r[c.i] = r;
            J.z[c.i] = z;
            rzn += r * z;
            rrn += r * r;
        }
        double v2[2] = {rzn, rrn};
        if (!red.reduce<2>(v2, OPS2(kSum, kSum), kTagAdjoint)) return false;
        beta = v2[0] / rz;
        rz = v2[0];
        rr = v2[1];
        first = false;
        ++it;
    }
    cg_its += it;
    // P3: diffusion adjoint (c^ = lambda, trial-phi adjoint) fused with the
    // cell-local part of the propose adjoint at the state before the step.
    double gM = 0, gS = 0, gD = 0;
    FOR_CELLS(P) {
        const Cell c = cell_at(P, idx_);
        const size_t i = c.i;
        const double lam = J.lam[i], ui = u[i];
        double Kb = 0;
#pragma unroll
        for (int d = 0; d < 4; ++d)
            if (c.has[d]) {
                const size_t j = c.n[d];
                Kb -= dt * (lam - J.lam[j]) * (ui - u[j]) * (0.5 / (d < 2 ? P.dx2 : P.dy2));
            }
        const double cb = J.bc[i] - lam;
        double tq[3];
        load3p(s1, pe, i, tq);
        const double dtr[3] = {2.0 * tq[1] * tq[2], 2.0 * tq[0] * tq[2], 2.0 * tq[0] * tq[1]};
        double hb[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) hb[k] = P.chi_p[k] * cb * (ui + P.mu_ref - P.B[k]);
        double gb[3];
#pragma unroll
        for (int aa = 0; aa < 3; ++aa) {
            double s = Kb * P.D[aa] * P.chi_p[aa];
#pragma unroll
            for (int k = 0; k < 3; ++k) s += hb[k] * (dtr[aa] + (k == aa ? 6.0 * tq[k] * (1.0 - tq[k]) : 0.0));
            gb[aa] = J.bphi[aa][i] + s;
        }
        gD += Kb * tq[2] * P.chi_p[2];
        J.bc[i] = lam;
        // propose adjoint, cell-local part
        double q[3], nb[4][3];
        load3p(s0, pe, i, q);
#pragma unroll
        for (int d = 0; d < 4; ++d) load3p(s0, pe, c.n[d], nb[d]);
        const double m = s0[4 * pe + i];
        double f[3];
        adj_forces(P, q, m, nb, c.has, f);
        const double mean = div_by(P, f[0] + f[1] + f[2], 3.0, P.r_3);
        const double tau = local_tau(P, q[0], q[1], q[2]);
        const double sc = dt / (tau * P.eps);
        double gg[3], z[3];
#pragma unroll
        for (int aa = 0; aa < 3; ++aa) {
            gg[aa] = f[aa] - mean;
            z[aa] = q[aa] - sc * gg[aa];
        }
        double o0 = z[0], o1 = z[1], o2 = z[2];
        (void)project_simplex(P, o0, o1, o2);  // z is finite in an accepted step
        const bool act[3] = {o0 > 0.0, o1 > 0.0, o2 > 0.0};
        const int na = (int)act[0] + (int)act[1] + (int)act[2];
        double gs = 0;
#pragma unroll
        for (int aa = 0; aa < 3; ++aa)
            if (act[aa]) gs += gb[aa];
        double zb[3];
#pragma unroll
        for (int aa = 0; aa < 3; ++aa) zb[aa] = act[aa] ? gb[aa] - gs / na : 0.0;
        double qb[3] = {zb[0], zb[1], zb[2]};
        const double sbar = -(zb[0] * gg[0] + zb[1] * gg[1] + zb[2] * gg[2]);
        const double zm = (zb[0] + zb[1] + zb[2]) / 3.0;
        double Fb[3];
#pragma unroll
        for (int aa = 0; aa < 3; ++aa) Fb[aa] = -sc * (zb[aa] - zm);
        gM += sbar * sc;
        const double taub = -sbar * sc / tau;
        const double w0 = q[0] * q[1], w1 = q[0] * q[2], w2 = q[1] * q[2], W = w0 + w1 + w2;
        if (W > 1e-30) {
            const double wb0 = taub * (P.tau[0] - tau) / W, wb1 = taub * (P.tau[1] - tau) / W,
                         wb2 = taub * (P.tau[2] - tau) / W;
            qb[0] += wb0 * q[1] + wb1 * q[2];
            qb[1] += wb0 * q[0] + wb2 * q[2];
            qb[2] += wb1 * q[0] + wb2 * q[1];
        }
#pragma unroll
        for (int aa = 0; aa < 3; ++aa) {
            const int a1 = (aa + 1) % 3, a2 = (aa + 2) % 3;
            qb[a1] += Fb[aa] * (P.obs + P.tr * q[a2]);
            qb[a2] += Fb[aa] * (P.obs + P.tr * q[a1]);
            gS += Fb[aa] * (q[a1] + q[a2]) * g.obs_per_sigma;
        }
        // chemical term: sum_b (psi_b - psi_g) dh[b][a] / Vm
        const double psig = psi(P, 2, m), dpsig = -(m - P.B[2]) * P.chi_p[2];
        double dpsi[3], dpsim[3], dsum = 0;
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            dpsi[b] = psi(P, b, m) - psig;
            dpsim[b] = -(m - P.B[b]) * P.chi_p[b] - dpsig;
            dsum += dpsi[b];
        }
        const double dtq[3] = {2.0 * q[1] * q[2], 2.0 * q[0] * q[2], 2.0 * q[0] * q[1]};
        double mb = 0;
#pragma unroll
        for (int aa = 0; aa < 3; ++aa)
#pragma unroll
            for (int b = 0; b < 3; ++b)
                mb += Fb[aa] * dpsim[b] * (dtq[aa] + (b == aa ? 6.0 * q[b] * (1.0 - q[b]) : 0.0)) / P.Vm;
#pragma unroll
        for (int aa = 0; aa < 3; ++aa)
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
                const double d = cc != aa ? dsum * 2.0 * q[3 - aa - cc] : dpsi[aa] * (6.0 - 12.0 * q[aa]);
                qb[cc] += Fb[aa] * d / P.Vm;
            }
        J.bmu[i] = mb;
#pragma unroll
        for (int aa = 0; aa < 3; ++aa) {
            J.Fb[aa][i] = Fb[aa];
            J.Ql[aa][i] = qb[aa];
        }
    }
    double v3[3] = {gM, gS, gD};
    if (!red.reduce<3>(v3, OPS3(kSum, kSum, kSum), kTagAdjoint)) return false;
    grad[0] += v3[0];
    grad[1] += v3[1];
    grad[2] += v3[2];
    // P4: gradient-term couplings, gathered from the four neighbours
    double gS2 = 0;
    FOR_CELLS(P) {
        const Cell c = cell_at(P, idx_);
        const size_t i = c.i;
        double q[3], Fi[3], qb[3];
        load3p(s0, pe, i, q);
#pragma unroll
        for (int aa = 0; aa < 3; ++aa) {
            Fi[aa] = J.Fb[aa][i];
            qb[aa] = J.Ql[aa][i];
        }
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            if (!c.has[d]) continue;
            const size_t j = c.n[d];
            double n[3], Fj[3];
            load3p(s0, pe, j, n);
#pragma unroll
            for (int aa = 0; aa < 3; ++aa) Fj[aa] = J.Fb[aa][j];
            const double d2 = d < 2 ? P.dx2 : P.dy2;
            const double kappa = P.two_eps_sigma / d2;
#pragma unroll
            for (int aa = 0; aa < 3; ++aa)
#pragma unroll
                for (int b = aa + 1; b < 3; ++b) {
                    // this cell's own forces with neighbour n
                    const double X = q[aa] * n[b] - n[aa] * q[b];
                    const double Y = Fi[aa] * n[b] - Fi[b] * n[aa];
                    qb[aa] += kappa * n[b] * Y;
                    qb[b] -= kappa * n[aa] * Y;
                    gS2 += X * Y * (g.two_eps / d2);
                    // the neighbour's forces, in which this cell is the neighbour
                    const double Xj = n[aa] * q[b] - q[aa] * n[b];
                    const double Yj = Fj[aa] * q[b] - Fj[b] * q[aa];
                    qb[aa] += kappa * (-n[b] * Yj - Xj * Fj[b]);
                    qb[b] += kappa * (n[aa] * Yj + Xj * Fj[aa]);
                }
        }
#pragma unroll
        for (int aa = 0; aa < 3; ++aa) J.bphi[aa][i] = qb[aa];
    }
    v1[0] = gS2;
    if (!red.reduce<1>(v1, kSum, kTagAdjoint)) return false;
    grad[1] += v1[0];
    return true;
}

__global__ void __launch_bounds__(kThreads, kMinBlocks) pearl_adjoint_kernel(const __grid_constant__ AdjArgs args) {
    const Dom a{args.P, args.B, nullptr, 0, (int)blockIdx.x, (int)gridDim.x, args.B.ctl, args.B.part,
                0, 0, 0, 0, 0, 0, 0};
    __shared__ PhaseClock clk;
    Red red(a, &clk);
    const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
    if (args.mode == 0) {
        if (!adj_seed(a, red, args)) return;
        red.flush();
        return;
    }
    double grad[3] = {0, 0, 0};
    long long its = 0;
    for (int j = args.len - 1; j >= 0; --j) {
        const double* s0 = j == 0 ? args.ckpt : args.tape + args.slot * (size_t)(j - 1);
        const double* s1 = args.tape + args.slot * (size_t)j;
        if (!adj_step(a, red, args, s0, s1, args.dts[j], grad, its)) return;
    }
    if (leader) {
        args.acc[1] += grad[0];
        args.acc[2] += grad[1];
        args.acc[3] += grad[2];
        args.acc[4] += (double)its;
    }
    red.flush();
}
