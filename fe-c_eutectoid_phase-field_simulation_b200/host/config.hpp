// config.hpp — the plain-text input of the Pearl solver, parsed exactly as the
// reference does (read_config, pearl_serial.cpp:1600-1758): same keys,
// defaults, validation order and error messages, so an input that the
// reference accepts or rejects is accepted or rejected here the same way.
#pragma once

#include <array>
#include <map>
#include <string>
#include <vector>

#include "pearl_gpu.h"

namespace pearl_host {

// Parabola f(c) = A c^2 + B c + C with diffusivity D (pearl_serial.cpp:72-90).
struct Parabola {
    double A = 0, B = 0, C = 0, D = 0;
    void validate() const;
    double mu(double c) const;       // fma(2A, c, B)
    double c_at_mu(double mu) const; // (mu-B)/(2A)
    double chi() const;              // 1/(2A)
};
using Thermo = std::array<Parabola, 3>;

// Grand-potential coefficients in 80-bit precision (pearl_serial.cpp:190-193).
struct GrandPotential {
    long double q2 = 0, q1 = 0, q0 = 0;
};

struct PhaseDiagram {
    std::array<double, 3> reference_composition{};
    std::array<double, 4> composition_slope{};
};

struct FillOp {
    std::string method;
    std::vector<double> p;
};

struct Config {
    int nx = 0, ny = 0, theta_columns = 0, phase_a = 0, phase_b = 2;
    double dx = 0, dy = 0, end_time = 0, output_dt = 0, seed_height = 0, radius = 0;
    double initial_mu = 0, initial_carbon = 0;
    std::string composition_mode, initialization = "lamella", mode = "coupled";
    int smooth_steps = 100, smooth_min_steps = 100;
    double smooth_energy_rtol = 1e-10, smooth_max_phase_change = 0.02;
    Thermo thermo{}, reference_thermo{};
    std::array<GrandPotential, 3> temperature_slope{};
    std::string thermo_mode = "direct_at_temperature", temperature_law = "linear_gp";
    PhaseDiagram diagram;
    double T = 0, T_eutectoid = 0, undercooling = 0, max_undercooling = 0;
    double epsilon = 0, sigma = 0, triple = 0, Vm = 0;
    std::array<double, 3> tau{};
    // Controls (pearl_serial.cpp:767-773)
    double dt_max = 1e-3, dt_min = 1e-12, max_phase_change = .04, cg_rtol = 1e-11, cg_atol = 1e-14,
           closure_tol = 1e-10, energy_rtol = 1e-11, energy_atol = 1e-12;
    int cg_max = 2000, max_retries = 24;
    bool check_energy = true, phase_only = false;
    double dt = 0, shift_trigger = 0, shift_target = 0, shift_gamma_carbon = 0;
    long long max_steps = 100000000;
    bool moving_window = false;
    std::vector<FillOp> fill;
    std::map<std::string, std::string> raw;

    std::string physics_signature() const;
    pearl_params device_params(double mu_reference) const;
};

Config read_config(const std::string& path);

// Temperature laws (pearl_serial.cpp:195-276), evaluated once in long double.
Parabola at_undercooling(const Parabola& reference, const GrandPotential& slope, double undercooling);
Thermo at_phase_diagram_undercooling(const Thermo& reference, const PhaseDiagram& diagram, double undercooling);
GrandPotential to_grand_potential(const Parabola& p);

// FILL commands (pearl_serial.cpp:1181-1349); the cells are painted on the
// device (pearl_gpu_fill, filling_phase_at :1393-1514).
FillOp parse_fill(const std::string& method, const std::string& value, int line);
void validate_fill(const std::vector<FillOp>& ops, int nx, int ny);

// Obstacle profile used by the native initialisations (pearl_serial.cpp:563-569).
double profile(double distance, double epsilon);

}  // namespace pearl_host
