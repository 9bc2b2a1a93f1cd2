// config.cpp — input parsing, temperature laws and FILL geometry of the Pearl
// host driver.  Every rule, default and message follows the reference file
// pearl_serial.cpp at the cited lines; the code is this project's own.
#include "config.hpp"

#include <algorithm>
#include <cmath>
#include <fstream>
#include <iomanip>
#include <limits>
#include <set>
#include <sstream>
#include <stdexcept>

// Model identifier embedded in every checkpoint signature by the reference
// (pearl_serial.cpp:31-33).  It must be identical so that checkpoints written
// by either program pass the other's restart check.
#define PEARL_SOURCE_DIGEST "344eef3b2e1fdbd8a41d81378491b923f6d815d8ef917f8397729c5a57965580"

namespace pearl_host {

namespace {
constexpr double kNaN = std::numeric_limits<double>::quiet_NaN();

std::string trim(const std::string& s) {
    const auto a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return {};
    const auto b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}
}  // namespace

// ------------------------------------------------------------------ Parabola
void Parabola::validate() const {
    if (!std::isfinite(A) || !std::isfinite(B) || !std::isfinite(C) || !std::isfinite(D) || A <= 0.0 || D < 0.0)
        throw std::invalid_argument("Parabola requires finite A>0, B, C, D>=0");
}
double Parabola::mu(double c) const { return std::fma(2.0 * A, c, B); }
double Parabola::c_at_mu(double m) const { return (m - B) / (2.0 * A); }
double Parabola::chi() const { return 1.0 / (2.0 * A); }

// ------------------------------------------------------------------ temperature laws
GrandPotential to_grand_potential(const Parabola& p) {
    p.validate();
    const long double A = p.A, B = p.B, C = p.C;
    return {-1 / (4 * A), B / (2 * A), C - B * B / (4 * A)};
}

static Parabola from_grand_potential(const GrandPotential& g, double D) {
    if (!std::isfinite(g.q2) || !std::isfinite(g.q1) || !std::isfinite(g.q0) || g.q2 >= 0)
        throw std::invalid_argument("temperature law requires finite q2<0, q1, q0");
    const long double A = -1 / (4 * g.q2), B = -g.q1 / (2 * g.q2);
    Parabola p{static_cast<double>(A), static_cast<double>(B), static_cast<double>(g.q0 + B * B / (4 * A)), D};
    p.validate();
    return p;
}

Parabola at_undercooling(const Parabola& reference, const GrandPotential& slope, double undercooling) {
    if (!std::isfinite(undercooling) || undercooling < 0)
        throw std::invalid_argument("undercooling must be finite and nonnegative");
    if (!std::isfinite(slope.q2) || !std::isfinite(slope.q1) || !std::isfinite(slope.q0))
        throw std::invalid_argument("nonfinite temperature derivative");
    reference.validate();
    if (undercooling == 0) return reference;
    GrandPotential g = to_grand_potential(reference);
    const long double change = -static_cast<long double>(undercooling);
    g.q2 += change * slope.q2;
    g.q1 += change * slope.q1;
    g.q0 += change * slope.q0;
    return from_grand_potential(g, reference.D);
}

Thermo at_phase_diagram_undercooling(const Thermo& reference, const PhaseDiagram& diagram, double undercooling) {
    if (!std::isfinite(undercooling) || undercooling < 0)
        throw std::invalid_argument("undercooling must be finite and nonnegative");
    for (const auto& p : reference) p.validate();
    for (double c : diagram.reference_composition)
        if (!std::isfinite(c) || c < 0 || c > 1)
            throw std::invalid_argument("phase-diagram reference carbon must be in [0,1]");
    for (double s : diagram.composition_slope)
        if (!std::isfinite(s)) throw std::invalid_argument("phase-diagram slope must be finite dc/dT");
    const long double dT = -static_cast<long double>(undercooling);
    const long double gA = reference[2].A;
    const long double gcE = diagram.reference_composition[2];
    Thermo out = reference;
    for (int product = 0; product <= 1; ++product) {
        const long double pA = reference[product].A;
        const long double pcE = diagram.reference_composition[product];
        const long double pcc = dT * diagram.composition_slope[2 * product];
        const long double gcc = dT * diagram.composition_slope[2 * product + 1];
        const long double pc = pcE + pcc, gc = gcE + gcc;
        if (!std::isfinite(pc) || !std::isfinite(gc) || pc < 0 || pc > 1 || gc < 0 || gc > 1)
            throw std::invalid_argument("phase-diagram extrapolated carbon outside [0,1]");
        if (undercooling == 0) continue;
        out[product].B = static_cast<double>(reference[product].B + 2 * (gA * gcc - pA * pcc));
        out[product].C = static_cast<double>(reference[product].C + pA * pcc * (2 * pcE + pcc) -
                                             gA * gcc * (2 * gcE + gcc));
        out[product].validate();
    }
    return out;
}

double profile(double distance, double epsilon) {
    const double pi = std::acos(-1.0), half = pi * pi * epsilon / 8;
    if (distance <= -half) return 1;
    if (distance >= half) return 0;
    return 0.5 * (1 - std::sin(4 * distance / (pi * epsilon)));
}

// ------------------------------------------------------------------ FILL geometry
FillOp parse_fill(const std::string& method, const std::string& value, int line) {
    const auto malformed = [&]() {
        return std::invalid_argument("Invalid " + method + " filling parameters at input line " +
                                     std::to_string(line) +
                                     ": expected {finite_number,...}, optionally followed by ';'");
    };
    std::string list = trim(value);
    if (!list.empty() && list.back() == ';') {
        list.pop_back();
        list = trim(list);
    }
    if (list.size() < 3 || list.front() != '{' || list.back() != '}') throw malformed();
    list = list.substr(1, list.size() - 2);
    FillOp op{method, {}};
    std::size_t start = 0;
    while (true) {
        const std::size_t comma = list.find(',', start);
        const std::string item =
            trim(list.substr(start, comma == std::string::npos ? std::string::npos : comma - start));
        if (item.empty()) throw malformed();
        std::size_t used = 0;
        double v = 0;
        try {
            v = std::stod(item, &used);
        } catch (const std::exception&) {
            throw malformed();
        }
        if (used != item.size() || !std::isfinite(v)) throw malformed();
        op.p.push_back(v);
        if (comma == std::string::npos) break;
        start = comma + 1;
    }
    return op;
}

void validate_fill(const std::vector<FillOp>& ops, int nx, int ny) {
    if (nx <= 0 || ny <= 0) throw std::invalid_argument("Filling requires positive nx and ny");
    for (const auto& op : ops) {
        const auto& p = op.p;
        const auto fail = [&](const std::string& why) { throw std::invalid_argument(op.method + ": " + why); };
        const auto count = [&](std::size_t n) {
            if (p.size() != n) fail("expected " + std::to_string(n) + " parameters");
            for (double v : p)
                if (!std::isfinite(v)) fail("parameters must be finite");
        };
        const auto integer = [&](std::size_t i) {
            if (std::trunc(p[i]) != p[i] || p[i] < static_cast<double>(std::numeric_limits<int>::min()) ||
                p[i] > static_cast<double>(std::numeric_limits<int>::max()))
                fail("parameter " + std::to_string(i + 1) + " must be a representable integer");
        };
        const auto phase = [&](std::size_t i) {
            integer(i);
            if (p[i] < 0 || p[i] > 2) fail("phase IDs must be alpha=0, theta=1 or gamma=2; gamma grain clones are unsupported");
        };
        const auto distinct = [&](std::initializer_list<std::size_t> idx) {
            for (auto i : idx) phase(i);
            for (auto a = idx.begin(); a != idx.end(); ++a)
                for (auto b = a + 1; b != idx.end(); ++b)
                    if (p[*a] == p[*b]) fail("listed phase IDs must be distinct");
        };
        const auto half_open_box = [&]() {
            for (std::size_t i = 0; i < 4; ++i) integer(i);
            if (!(0 <= p[0] && p[0] < p[1] && p[1] <= nx && 0 <= p[2] && p[2] < p[3] && p[3] <= ny))
                fail("box must satisfy 0<=xlo<xhi<=nx and 0<=ylo<yhi<=ny");
        };
        const auto center = [&](std::size_t x, std::size_t y, bool integers) {
            if (integers) {
                integer(x);
                integer(y);
            }
            if (!(0 <= p[x] && p[x] < nx && 0 <= p[y] && p[y] < ny)) fail("center/junction must be inside the physical grid");
        };
        const auto positive = [&](std::size_t i) {
            if (!(p[i] > 0.0)) fail("parameter " + std::to_string(i + 1) + " must be positive");
        };
        const auto fraction = [&](std::size_t i) {
            if (!(p[i] > 0.0 && p[i] < 1.0)) fail("cementite fraction must be strictly between 0 and 1");
        };
        const auto nonnegative = [&](std::size_t i) {
            if (p[i] < 0.0) fail("parameter " + std::to_string(i + 1) + " must be nonnegative");
        };
        const auto angle = [&](std::size_t i) {
            if (!std::isfinite(p[i] * 3.14159265358979323846 / 180.0)) fail("angle conversion to radians overflows");
        };
        const auto squared = [&](std::size_t i) {
            const double s = p[i] * p[i];
            if (!std::isfinite(s) || (p[i] > 0.0 && s == 0.0)) fail("length squared overflows or underflows");
        };
        const auto resolved = [&](double v, const std::string& name) {
            if (!(v > 0.0) || !std::isfinite(v)) fail(name + " must remain finite and positive");
        };
        const std::string& m = op.method;
        if (m == "FILLCUBE") {
            count(7);
            phase(0);
            for (std::size_t i = 1; i < 7; ++i) integer(i);
            if (p[3] != 0 || p[6] != 0) fail("2D filling requires zlo=zhi=0");
            if (!(0 <= p[1] && p[1] <= p[4] && p[4] < nx && 0 <= p[2] && p[2] <= p[5] && p[5] < ny))
                fail("inclusive bounds must satisfy 0<=xlo<=xhi<nx and 0<=ylo<=yhi<ny");
        } else if (m == "FILLCENTERBOX2D") {
            count(6);
            half_open_box();
            distinct({4, 5});
        } else if (m == "FILLYJUNCTION2D" || m == "FILLYJUNCTIONLAMELLAE2D") {
            const bool lam = m == "FILLYJUNCTIONLAMELLAE2D";
            count(lam ? 16 : 13);
            half_open_box();
            center(4, 5, true);
            positive(9);
            positive(10);
            angle(6);
            angle(7);
            angle(8);
            if (lam) {
                positive(11);
                positive(12);
                distinct({13, 14, 15});
                resolved(p[11] + p[12], "lamellar period");
            } else {
                distinct({11, 12});
            }
        } else if (m == "FILLCYLINDER") {
            count(6);
            phase(0);
            center(1, 2, true);
            integer(3);
            integer(4);
            positive(5);
            if (p[3] != 0 || p[4] != 0) fail("2D cylinder cross-section requires zlo=zhi=0");
            squared(5);
        } else if (m == "FILLADHEREDPEARLITEARM2D") {
            count(11);
            center(0, 1, false);
            positive(3);
            integer(4);
            positive(4);
            if (p[4] > std::numeric_limits<int>::max() / 2) fail("pair_count is too large");
            fraction(5);
            positive(6);
            nonnegative(7);
            nonnegative(8);
            distinct({9, 10});
            if (p[7] > p[6]) fail("contact_half_width must not exceed peak_half_width");
            angle(2);
            squared(3);
            squared(6);
            squared(8);
            const double period = p[3] / p[4];
            resolved(period, "arm period");
            resolved((1.0 - p[5]) * period, "ferrite segment length");
            resolved(p[5] * period, "cementite segment length");
        } else if (m == "FILLPEARLITEELLIPSE2D") {
            count(11);
            center(0, 1, false);
            nonnegative(3);
            integer(4);
            positive(4);
            positive(5);
            positive(6);
            fraction(7);
            nonnegative(8);
            distinct({9, 10});
            angle(2);
            squared(8);
            const double length = p[4] * p[5];
            const double semi_major = 0.5 * length, semi_minor = p[6] * semi_major;
            resolved(length, "ellipse length");
            resolved(semi_major, "ellipse semimajor axis");
            resolved(semi_minor, "ellipse semiminor axis");
            resolved(p[7] * p[5], "cementite lamellar width");
            if (!std::isfinite((p[3] + length) * (p[3] + length))) fail("ellipse endpoint distance overflows");
        } else if (m == "FILLTHREEGRAINYJUNCTION2D" || m == "FILLYJUNCTIONPEARLITE2D") {
            fail("historical multi-grain initialization requires separate gamma grain fields; "
                 "Pearl has one gamma field and will not merge grain IDs silently");
        } else {
            fail("unsupported filling method in the 2D three-phase Pearl solver; see FILLING_METHODS.md");
        }
    }
}

// ------------------------------------------------------------------ signature
std::string Config::physics_signature() const {
    std::ostringstream o;
    o << std::setprecision(17) << "pearlite-v0.4-reference;source=" << PEARL_SOURCE_DIGEST
      << ";3ph;binary;equal-sigma;Jat=0;Xperiodic;Ynoflux;";
    o << nx << ';' << ny << ';' << dx << ';' << dy << ';' << Vm << ';' << epsilon << ';' << sigma << ';' << triple
      << ';';
    o << thermo_mode << ';' << T << ';' << T_eutectoid << ';' << undercooling << ';' << max_undercooling << ';';
    if (thermo_mode == "eutectoid_reference") {
        for (const auto& p : reference_thermo) o << p.A << ';' << p.B << ';' << p.C << ';';
        if (temperature_law == "linear_gp") {
            for (const auto& s : temperature_slope) o << s.q2 << ';' << s.q1 << ';' << s.q0 << ';';
        } else {
            o << "phase-diagram-fixed-curvature-v1;";
            for (double c : diagram.reference_composition) o << c << ';';
            for (double s : diagram.composition_slope) o << s << ';';
        }
    }
    for (const auto& p : thermo) o << p.A << ';' << p.B << ';' << p.C << ';' << p.D << ';';
    for (double t : tau) o << t << ';';
    o << mode << ';' << initialization << ';' << seed_height << ';' << theta_columns << ';' << radius << ';'
      << phase_a << ';' << phase_b << ';' << composition_mode << ';' << initial_mu << ';' << initial_carbon << ';';
    o << smooth_steps << ';' << smooth_min_steps << ';' << smooth_energy_rtol << ';' << smooth_max_phase_change
      << ';';
    o << moving_window << ';' << shift_trigger << ';' << shift_target << ';' << shift_gamma_carbon;
    if (initialization == "microsim") {
        o << ";filling-v1";
        for (const auto& op : fill) {
            o << ';' << op.method;
            for (double c : op.p) o << ';' << c;
        }
    }
    return o.str();
}

pearl_params Config::device_params(double mu_reference) const {
    pearl_params p{};
    for (int i = 0; i < 3; ++i) {
        p.A[i] = thermo[i].A;
        p.B[i] = thermo[i].B;
        p.C[i] = thermo[i].C;
        p.D[i] = thermo[i].D;
        p.tau[i] = tau[i];
    }
    p.Vm = Vm;
    p.epsilon = epsilon;
    p.sigma = sigma;
    p.triple = triple;
    p.dx = dx;
    p.dy = dy;
    p.dt_max = dt_max;
    p.dt_min = dt_min;
    p.max_phase_change = max_phase_change;
    p.cg_rtol = cg_rtol;
    p.cg_atol = cg_atol;
    p.closure_tol = closure_tol;
    p.energy_rtol = energy_rtol;
    p.energy_atol = energy_atol;
    p.cg_max = cg_max;
    p.max_retries = max_retries;
    p.check_energy = check_energy ? 1 : 0;
    p.phase_only = phase_only ? 1 : 0;
    p.mu_reference = mu_reference;
    return p;
}

// ------------------------------------------------------------------ read_config
Config read_config(const std::string& path) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error("cannot open input: " + path);
    Config c;
    std::string line;
    int ln = 0;
    while (std::getline(in, line)) {
        ++ln;
        line = trim(line.substr(0, line.find('#')));
        if (line.empty()) continue;
        const auto pos = line.find('=');
        if (pos == std::string::npos) throw std::runtime_error("missing = on line " + std::to_string(ln));
        const std::string key = trim(line.substr(0, pos)), val = trim(line.substr(pos + 1));
        if (key.rfind("FILL", 0) == 0) {
            c.fill.push_back(parse_fill(key, val, ln));
            continue;
        }
        if (key.empty() || val.empty() || c.raw.count(key)) throw std::runtime_error("empty/duplicate key: " + key);
        c.raw[key] = val;
    }
    std::set<std::string> used;
    const auto str = [&](const std::string& k, const std::string& def = "") {
        const auto it = c.raw.find(k);
        if (it == c.raw.end()) return def;
        used.insert(k);
        return it->second;
    };
    const auto number = [&](const std::string& k, double def = kNaN) {
        const std::string s = str(k);
        if (s.empty()) {
            if (!std::isfinite(def)) throw std::runtime_error("missing required key: " + k);
            return def;
        }
        std::size_t n = 0;
        const double v = std::stod(s, &n);  // an unparsable value throws std::invalid_argument("stod")
        if (n != s.size() || !std::isfinite(v)) throw std::runtime_error("invalid number: " + k);
        return v;
    };
    const auto integer = [&](const std::string& k, int def = -1) {
        const double a = number(k, def < 0 ? kNaN : def);
        if (a != std::floor(a) || std::abs(a) > 1e8) throw std::runtime_error("invalid integer: " + k);
        return static_cast<int>(a);
    };
    c.nx = integer("nx");
    c.ny = integer("ny");
    c.dx = number("dx");
    c.dy = number("dy", c.dx);
    c.epsilon = number("epsilon");
    c.sigma = number("sigma");
    c.triple = number("triple");
    c.Vm = number("Vm");
    c.tau[0] = number("tau_at");
    c.tau[1] = number("tau_ag");
    c.tau[2] = number("tau_tg");
    const std::array<std::string, 3> names{"alpha", "theta", "gamma"};
    c.thermo_mode = str("thermo_mode");
    if (c.thermo_mode == "eutectoid_reference") {
        c.T_eutectoid = number("T_eutectoid");
        c.undercooling = number("undercooling");
        c.max_undercooling = number("max_undercooling");
        c.temperature_law = str("temperature_law");
        if (c.temperature_law != "linear_gp" && c.temperature_law != "phase_diagram_fixed_curvature")
            throw std::runtime_error("temperature_law must be linear_gp or phase_diagram_fixed_curvature");
        c.T = c.T_eutectoid - c.undercooling;
        if (c.T_eutectoid <= 0 || c.T <= 0 || c.undercooling < 0 || c.max_undercooling < 0 ||
            c.undercooling > c.max_undercooling)
            throw std::runtime_error("temperature outside declared undercooling interval");
        for (int i = 0; i < 3; ++i) {
            const std::string& n = names[i];
            c.reference_thermo[i].A = number("Aeq_" + n);
            c.reference_thermo[i].B = number("Beq_" + n);
            c.reference_thermo[i].C = number("Ceq_" + n);
            c.reference_thermo[i].D = number("D_" + n);
            if (c.temperature_law == "linear_gp") {
                c.temperature_slope[i].q2 = number("dq2_dT_" + n);
                c.temperature_slope[i].q1 = number("dq1_dT_" + n);
                c.temperature_slope[i].q0 = number("dq0_dT_" + n);
                c.thermo[i] = at_undercooling(c.reference_thermo[i], c.temperature_slope[i], c.undercooling);
            }
        }
        if (c.temperature_law == "phase_diagram_fixed_curvature") {
            c.diagram.reference_composition = {number("ceq_alpha"), number("ceq_theta"), number("ceq_gamma")};
            c.diagram.composition_slope[0] = number("slope_alpha_on_alpha_gamma");
            c.diagram.composition_slope[1] = number("slope_gamma_on_alpha_gamma");
            c.diagram.composition_slope[2] = number("slope_theta_on_theta_gamma");
            c.diagram.composition_slope[3] = number("slope_gamma_on_theta_gamma");
            c.thermo = at_phase_diagram_undercooling(c.reference_thermo, c.diagram, c.undercooling);
        }
    } else if (c.thermo_mode == "direct_at_temperature") {
        c.T = number("temperature");
        if (c.T <= 0) throw std::runtime_error("temperature must be positive");
        for (int i = 0; i < 3; ++i) {
            const std::string& n = names[i];
            c.thermo[i].A = number("A_" + n);
            c.thermo[i].B = number("B_" + n);
            c.thermo[i].C = number("C_" + n);
            c.thermo[i].D = number("D_" + n);
            c.thermo[i].validate();
        }
    } else {
        throw std::runtime_error(
            "Set thermo_mode=eutectoid_reference or direct_at_temperature. "
            "Legacy inputs require an explicit mode and temperature; no temperature is guessed.");
    }
    c.dt = number("dt");
    c.dt_max = number("dt_max", c.dt);
    c.dt_min = number("dt_min", c.dt / 1048576.0);
    c.end_time = number("end_time");
    c.output_dt = number("output_dt");
    c.max_steps = integer("max_steps", 100000000);
    c.initialization = str("initialization", "lamella");
    c.mode = str("mode", "coupled");
    if (c.mode != "coupled" && c.mode != "phase_only") throw std::runtime_error("mode must be coupled or phase_only");
    c.phase_only = c.mode == "phase_only";
    c.seed_height = number("seed_height", c.ny * c.dy / 4);
    c.theta_columns = integer("theta_columns", c.nx / 2);
    c.radius = number("radius", std::min(c.nx * c.dx, c.ny * c.dy) / 4);
    c.phase_a = integer("phase_a", 0);
    c.phase_b = integer("phase_b", 2);
    if (c.initialization != "lamella" && c.initialization != "sharp_smooth" && c.initialization != "flat" &&
        c.initialization != "circle" && c.initialization != "microsim")
        throw std::runtime_error("unknown initialization");
    if (c.initialization == "microsim") {
        if (c.fill.empty()) throw std::runtime_error("initialization=microsim requires at least one FILL operation");
        validate_fill(c.fill, c.nx, c.ny);
    } else if (!c.fill.empty()) {
        throw std::runtime_error("FILL operations require initialization=microsim; no geometry is silently ignored");
    }
    c.smooth_steps = integer("smooth_steps", 100);
    c.smooth_min_steps = integer("smooth_min_steps", c.smooth_steps);
    c.smooth_energy_rtol = number("smooth_energy_rtol", 1e-10);
    c.smooth_max_phase_change = number("smooth_max_phase_change", 0.02);
    if (c.phase_a < 0 || c.phase_a > 2 || c.phase_b < 0 || c.phase_b > 2 || c.phase_a == c.phase_b)
        throw std::runtime_error("invalid phase pair");
    const int choices = static_cast<int>(c.raw.count("initial_mu") + c.raw.count("gamma_carbon") +
                                         c.raw.count("mean_carbon"));
    if (choices != 1) throw std::runtime_error("specify exactly one of initial_mu, gamma_carbon, mean_carbon");
    if (c.raw.count("initial_mu")) {
        c.composition_mode = "mu";
        c.initial_mu = number("initial_mu");
    }
    if (c.raw.count("gamma_carbon")) {
        c.composition_mode = "gamma";
        c.initial_carbon = number("gamma_carbon");
        c.initial_mu = c.thermo[2].mu(c.initial_carbon);
    }
    if (c.raw.count("mean_carbon")) {
        c.composition_mode = "mean";
        c.initial_carbon = number("mean_carbon");
    }
    c.max_phase_change = number("max_phase_change", .04);
    c.cg_rtol = number("cg_rtol", 1e-11);
    c.cg_atol = number("cg_atol", 1e-14);
    c.cg_max = integer("cg_max", 2000);
    c.closure_tol = number("closure_tol", 1e-10);
    c.energy_atol = number("energy_atol", 1e-13 * c.sigma * std::max(c.nx * c.dx, c.ny * c.dy));
    c.moving_window = integer("moving_window", 0) != 0;
    c.shift_trigger = number("shift_trigger", .65 * c.ny * c.dy);
    c.shift_target = number("shift_target", .35 * c.ny * c.dy);
    c.shift_gamma_carbon = number("shift_gamma_carbon", c.composition_mode == "gamma"
                                                            ? c.initial_carbon
                                                            : c.thermo[2].c_at_mu(c.initial_mu));
    for (const auto& kv : c.raw)
        if (!used.count(kv.first)) throw std::runtime_error("unknown key: " + kv.first);
    // PhaseParameters::validate (pearl_serial.cpp:414-419, :522-529)
    if (!(c.epsilon > 0) || !(c.sigma > 0) || c.triple < 0 || !std::isfinite(c.epsilon) || !std::isfinite(c.sigma) ||
        !std::isfinite(c.triple))
        throw std::invalid_argument("Invalid interface parameters");
    for (double t : c.tau)
        if (!(t > 0) || !std::isfinite(t)) throw std::invalid_argument("tau must be finite and positive");
    if (!(c.Vm > 0) || !std::isfinite(c.Vm)) throw std::invalid_argument("Invalid Vm");
    if (c.nx < 3 || c.ny < 2 || c.dx <= 0 || c.dy <= 0 || c.dt <= 0 || c.dt_min <= 0 || c.dt_max < c.dt ||
        c.dt_min > c.dt || c.end_time <= 0 || c.output_dt <= 0 || c.max_steps < 1)
        throw std::runtime_error("invalid geometry/time bounds");
    if (c.theta_columns < 1 || c.theta_columns >= c.nx || c.seed_height <= 0 || c.seed_height >= c.ny * c.dy)
        throw std::runtime_error("invalid seed geometry");
    if (c.max_phase_change <= 0 || c.max_phase_change > .2 || c.cg_rtol <= 0 || c.cg_atol <= 0 ||
        c.closure_tol <= 0 || c.energy_atol < 0)
        throw std::runtime_error("invalid numerical control");
    if (c.smooth_steps < 1 || c.smooth_min_steps < 0 || c.smooth_min_steps > c.smooth_steps ||
        c.smooth_energy_rtol <= 0 || c.smooth_max_phase_change <= 0 || c.smooth_max_phase_change > .2)
        throw std::runtime_error("invalid smoothing control");
    if (c.moving_window && (c.shift_target <= 0 || c.shift_trigger <= c.shift_target ||
                            c.shift_trigger >= c.ny * c.dy || c.shift_gamma_carbon < 0 || c.shift_gamma_carbon > 1))
        throw std::runtime_error("invalid moving window settings");
    return c;
}

}  // namespace pearl_host
