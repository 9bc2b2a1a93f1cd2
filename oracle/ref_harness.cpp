// ref_harness.cpp — TEST INFRASTRUCTURE: exposes the UNMODIFIED reference
// solver (pearl_serial.cpp, compiled from where it lies by
// oracle/build_oracle.py) through a small C ABI, so that tests can check the C
// restatement (pearl_oracle.c) and the GPU path against the reference itself,
// and the bench can time the reference's own CPU path.
//
// The reference source is #included, not copied: the build passes its
// directory with -I.  Its main() is renamed so this file can be a library.
// The entry points reuse the data layouts of pearl_oracle.h.
#define main pearl_reference_cli_main
#include <pearl_serial.cpp>
#undef main

#include <cstring>
#include <string>

#include "pearl_oracle.h"

namespace {

struct Setup {
    pearl::Thermo thermo{};
    pearl::PhaseParameters phase{{0, 0, 0}, {0, 0, 0}, 0};
    pearl::Controls control;
};

Setup make_setup(const po_params* p) {
    Setup s;
    for (int i = 0; i < 3; ++i) s.thermo[i] = {p->A[i], p->B[i], p->C[i], p->D[i]};
    s.phase.interface = {p->epsilon, p->sigma, p->triple};
    s.phase.tau = {p->tau[0], p->tau[1], p->tau[2]};
    s.phase.Vm = p->Vm;
    s.control.dt_max = p->dt_max;
    s.control.dt_min = p->dt_min;
    s.control.max_phase_change = p->max_phase_change;
    s.control.cg_rtol = p->cg_rtol;
    s.control.cg_atol = p->cg_atol;
    s.control.closure_tol = p->closure_tol;
    s.control.energy_rtol = p->energy_rtol;
    s.control.energy_atol = p->energy_atol;
    s.control.cg_max = p->cg_max;
    s.control.max_retries = p->max_retries;
    s.control.check_energy = p->check_energy != 0;
    s.control.phase_only = p->phase_only != 0;
    return s;
}

void load_fields(const pearl::Domain& d, pearl::State& st, const double* phi, const double* carbon, const double* mu) {
    for (int y = 1; y <= d.ny; ++y)
        for (int x = 1; x <= d.nx; ++x) {
            const std::size_t i = static_cast<std::size_t>(y - 1) * d.nx + (x - 1);
            for (int c = 0; c < 3; ++c) st.phi(x, y, c) = phi[3 * i + c];
            if (carbon) st.carbon(x, y) = carbon[i];
            if (mu) st.mu(x, y) = mu[i];
        }
    d.halo(st.phi);
    d.halo(st.carbon);
    d.halo(st.mu);
}

void store_fields(const pearl::Domain& d, const pearl::State& st, double* phi, double* carbon, double* mu) {
    for (int y = 1; y <= d.ny; ++y)
        for (int x = 1; x <= d.nx; ++x) {
            const std::size_t i = static_cast<std::size_t>(y - 1) * d.nx + (x - 1);
            if (phi)
                for (int c = 0; c < 3; ++c) phi[3 * i + c] = st.phi(x, y, c);
            if (carbon) carbon[i] = st.carbon(x, y);
            if (mu) mu[i] = st.mu(x, y);
        }
}

void load_scalars(pearl::State& st, const po_scalars* s) {
    st.time = s->time;
    st.dt = s->dt;
    st.shift_distance = s->shift_distance;
    st.initial_carbon = s->initial_carbon;
    st.carbon_added = s->carbon_added;
    st.carbon_removed = s->carbon_removed;
    st.step = s->step;
    st.shifts = s->shifts;
    st.rejected = s->rejected;
}

void store_scalars(const pearl::State& st, po_scalars* s) {
    s->time = st.time;
    s->dt = st.dt;
    s->shift_distance = st.shift_distance;
    s->initial_carbon = st.initial_carbon;
    s->carbon_added = st.carbon_added;
    s->carbon_removed = st.carbon_removed;
    s->step = st.step;
    s->shifts = st.shifts;
    s->rejected = st.rejected;
}

void copy_error(const std::exception& e, char* err, int errlen) {
    if (err && errlen > 0) {
        std::strncpy(err, e.what(), static_cast<std::size_t>(errlen) - 1);
        err[errlen - 1] = 0;
    }
}

}  // namespace

extern "C" {

// Runs nsteps calls of pearl::advance (pearl_serial.cpp:1119).  forced_dt
// (nullable) sets State::dt before each call, which replays an accepted-dt
// sequence.  Returns 0, or 1 with the reference's exception text in err.
int ref_advance_n(const po_params* p, int nx, int ny, double* phi, double* carbon, double* mu, po_scalars* s,
                  int nsteps, const double* forced_dt, double stop_time, po_step_info* infos, int* steps_done,
                  char* err, int errlen) {
    int done = 0;
    try {
        Setup su = make_setup(p);
        pearl::Domain d(nx, ny, p->dx, p->dy);
        pearl::State st(d);
        load_fields(d, st, phi, carbon, mu);
        load_scalars(st, s);
        for (int k = 0; k < nsteps; ++k) {
            if (forced_dt) st.dt = forced_dt[k];
            pearl::StepInfo info = pearl::advance(d, st, su.thermo, su.phase, su.control, p->mu_reference, stop_time);
            if (infos) {
                infos[k].accepted_dt = info.accepted_dt;
                infos[k].max_phase_change = info.max_phase_change;
                infos[k].linear_residual = info.linear_residual;
                infos[k].closure = info.closure;
                infos[k].energy_change = info.energy_change;
                infos[k].cg_iterations = info.cg_iterations;
                infos[k].retries = info.retries;
            }
            ++done;
        }
        store_fields(d, st, phi, carbon, mu);
        store_scalars(st, s);
    } catch (const std::exception& e) {
        copy_error(e, err, errlen);
        if (steps_done) *steps_done = done;
        return 1;
    }
    if (steps_done) *steps_done = done;
    return 0;
}

// pearl::propose_phi (pearl_serial.cpp:961)
int ref_propose_phi(const po_params* p, int nx, int ny, const double* phi_old, const double* mu_old,
                    double* trial_phi, double dt, double* change, char* err, int errlen) {
    try {
        Setup su = make_setup(p);
        pearl::Domain d(nx, ny, p->dx, p->dy);
        pearl::State old(d);
        load_fields(d, old, phi_old, nullptr, mu_old);
        pearl::State trial = old;
        *change = pearl::propose_phi(d, old, trial, su.thermo, su.phase, dt);
        store_fields(d, trial, trial_phi, nullptr, nullptr);
    } catch (const std::exception& e) {
        copy_error(e, err, errlen);
        return 1;
    }
    return 0;
}

// pearl::implicit_diffusion (pearl_serial.cpp:1010)
int ref_implicit_diffusion(const po_params* p, int nx, int ny, const double* carbon_old, const double* mu_old,
                           const double* trial_phi, double* trial_carbon, double* trial_mu, double dt,
                           po_diffusion_info* info, char* err, int errlen) {
    try {
        Setup su = make_setup(p);
        pearl::Domain d(nx, ny, p->dx, p->dy);
        pearl::State old(d);
        load_fields(d, old, trial_phi, carbon_old, mu_old);
        pearl::State trial = old;
        pearl::DiffusionInfo di = pearl::implicit_diffusion(d, old, trial, su.thermo, dt, p->mu_reference, su.control);
        info->ok = di.ok;
        info->it = di.it;
        info->residual = di.residual;
        info->closure = di.closure;
        store_fields(d, trial, nullptr, trial_carbon, trial_mu);
    } catch (const std::exception& e) {
        copy_error(e, err, errlen);
        return 1;
    }
    return 0;
}

// pearl::reduced_energy and pearl::total_carbon (pearl_serial.cpp:793, :784)
int ref_energy_and_mass(const po_params* p, int nx, int ny, const double* phi, const double* carbon, double* energy,
                        double* mass, char* err, int errlen) {
    try {
        Setup su = make_setup(p);
        pearl::Domain d(nx, ny, p->dx, p->dy);
        pearl::State st(d);
        load_fields(d, st, phi, carbon, nullptr);
        *energy = pearl::reduced_energy(d, st, su.thermo, su.phase, p->mu_reference, su.control.phase_only);
        *mass = pearl::total_carbon(d, st);
    } catch (const std::exception& e) {
        copy_error(e, err, errlen);
        return 1;
    }
    return 0;
}

// pearl::valid_state (pearl_serial.cpp:1096)
int ref_valid_state(const po_params* p, int nx, int ny, const double* phi, const double* carbon, const double* mu) {
    Setup su = make_setup(p);
    pearl::Domain d(nx, ny, p->dx, p->dy);
    pearl::State st(d);
    load_fields(d, st, phi, carbon, mu);
    return pearl::valid_state(d, st, su.thermo, su.control.phase_only) ? 1 : 0;
}

// pearl::maybe_shift (pearl_serial.cpp:2053); the moving-window keys are passed explicitly.
int ref_maybe_shift(const po_params* p, int nx, int ny, double* phi, double* carbon, double* mu, po_scalars* s,
                    double shift_trigger, double shift_target, double c_gamma, int* shifted, char* err,
                    int errlen) {
    try {
        Setup su = make_setup(p);
        pearl::Domain d(nx, ny, p->dx, p->dy);
        pearl::State st(d);
        load_fields(d, st, phi, carbon, mu);
        load_scalars(st, s);
        pearl::Config config;
        config.moving_window = true;
        config.shift_trigger = shift_trigger;
        config.shift_target = shift_target;
        config.shift_gamma_carbon = c_gamma;
        config.thermo = su.thermo;
        const long long before = st.shifts;
        pearl::maybe_shift(d, st, config);
        *shifted = st.shifts != before ? 1 : 0;
        store_fields(d, st, phi, carbon, mu);
        store_scalars(st, s);
    } catch (const std::exception& e) {
        copy_error(e, err, errlen);
        return 1;
    }
    return 0;
}

// pearl::smooth_interface_only (pearl_serial.cpp:869)
int ref_smooth(const po_params* p, int nx, int ny, double* phi, int max_steps, int min_steps, double energy_rtol,
               double max_phase_change, po_smooth_report* report, char* err, int errlen) {
    try {
        Setup su = make_setup(p);
        pearl::Domain d(nx, ny, p->dx, p->dy);
        pearl::State st(d);
        load_fields(d, st, phi, nullptr, nullptr);
        pearl::SmoothReport r =
            pearl::smooth_interface_only(d, st, su.phase, max_steps, min_steps, energy_rtol, max_phase_change);
        report->steps = r.steps;
        report->converged = r.converged;
        report->energy_initial = r.energy_initial;
        report->energy_final = r.energy_final;
        report->final_relative_energy_change = r.final_relative_energy_change;
        report->final_max_phase_change = r.final_max_phase_change;
        for (int a = 0; a < 3; ++a) {
            report->phase_fraction_before[a] = r.phase_fraction_before[a];
            report->phase_fraction_after[a] = r.phase_fraction_after[a];
        }
        store_fields(d, st, phi, nullptr, nullptr);
    } catch (const std::exception& e) {
        copy_error(e, err, errlen);
        return 1;
    }
    return 0;
}

// Temperature laws (pearl_serial.cpp:203-218, :236-276): evaluated ABC for tests
// of the host configuration code.  law 0 = linear_gp, 1 = phase_diagram_fixed_curvature.
int ref_thermo_at_undercooling(int law, const double* ref_abcd /*12*/, const double* slopes /*9 or 7*/,
                               double undercooling, double* out_abcd /*12*/, char* err, int errlen) {
    try {
        pearl::Thermo ref{};
        for (int i = 0; i < 3; ++i)
            ref[i] = {ref_abcd[4 * i], ref_abcd[4 * i + 1], ref_abcd[4 * i + 2], ref_abcd[4 * i + 3]};
        pearl::Thermo out{};
        if (law == 0) {
            for (int i = 0; i < 3; ++i) {
                pearl::GrandPotentialPolynomial slope{slopes[3 * i], slopes[3 * i + 1], slopes[3 * i + 2]};
                out[i] = pearl::at_undercooling(ref[i], slope, undercooling);
            }
        } else {
            pearl::PhaseDiagramInput pd;
            pd.reference_composition = {slopes[0], slopes[1], slopes[2]};
            pd.composition_slope = {slopes[3], slopes[4], slopes[5], slopes[6]};
            out = pearl::at_phase_diagram_undercooling(ref, pd, undercooling);
        }
        for (int i = 0; i < 3; ++i) {
            out_abcd[4 * i] = out[i].free_energy_quadratic;
            out_abcd[4 * i + 1] = out[i].free_energy_linear;
            out_abcd[4 * i + 2] = out[i].free_energy_constant;
            out_abcd[4 * i + 3] = out[i].diffusivity;
        }
    } catch (const std::exception& e) {
        copy_error(e, err, errlen);
        return 1;
    }
    return 0;
}

}  // extern "C"
