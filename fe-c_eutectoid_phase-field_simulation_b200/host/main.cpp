// main.cpp — the pearl_gpu executable, a drop-in for the reference's
// pearl_serial (main, pearl_serial.cpp:2184-2336): same command line, input
// file, output directory contents and error messages.  Initialisation,
// time stepping, the moving window and the output reductions run on one GPU
// through libpearl_gpu.so; the host parses the input, builds the initial
// geometry and writes the files.
//
//   pearl_gpu input.in NEW_OUTPUT_DIR [--restart frame.h5] [--px N --py N]
//             [--max-steps N] [--thermo-only]
//
// --px/--py are accepted for command-line compatibility and must be 1 (one
// device-resident domain).  PEARL_GPU_DEVICE selects the CUDA device (default 0).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <csignal>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "config.hpp"
#include "io.hpp"
#include "pearl_gpu.h"

using namespace pearl_host;
namespace fs = std::filesystem;

namespace {

volatile std::sig_atomic_t interrupted = 0;
void on_signal(int) { interrupted = 1; }

// Accepted steps per device launch between host checks of SIGINT/SIGTERM.
constexpr long long kStepsPerLaunch = 256;

struct Gpu {
    pearl_gpu_ctx* ctx = nullptr;
    ~Gpu() { pearl_gpu_destroy(ctx); }
    void check(int rc) const {
        if (rc != PEARL_OK) {
            const char* msg = ctx ? pearl_gpu_last_error(ctx) : "";
            throw std::runtime_error(msg && *msg ? msg : pearl_gpu_status_string(rc));
        }
    }
};

// Frame output on a background thread, so the device launches up to the next
// output time overlap the file writing.  One frame is in flight at a time:
// wait() joins it, rethrows its error, and only then emits its diagnostics and
// console lines, so files and lines appear in the reference's order (frame,
// then its log line) and a failed write logs nothing for that frame.
class FrameWriter {
  public:
    explicit FrameWriter(std::ofstream& log) : log_(log) {}
    // on an error elsewhere the frame in flight still completes and, if it was
    // written, its lines appear before the error message, as in the reference
    ~FrameWriter() {
        if (worker_.joinable()) worker_.join();
        if (pending_ && !error_) {
            log_ << log_line_;
            log_.flush();
            std::cout << out_line_;
        }
    }
    void wait() {
        if (worker_.joinable()) worker_.join();
        if (error_) {
            std::exception_ptr e = error_;
            error_ = nullptr;
            std::rethrow_exception(e);
        }
        if (pending_) {
            log_ << log_line_;
            log_.flush();
            std::cout << out_line_;
            pending_ = false;
        }
    }
    // st must stay untouched until the next wait()
    void submit(const HostState& st, const Config& config, double mu_reference, fs::path path, std::string log_line,
                std::string out_line) {
        wait();
        log_line_ = std::move(log_line);
        out_line_ = std::move(out_line);
        pending_ = true;
        worker_ = std::thread([this, &st, &config, mu_reference, path = std::move(path)]() {
            try {
                write_frame(st, config, mu_reference, path);
            } catch (...) {
                error_ = std::current_exception();
            }
        });
    }

  private:
    std::ofstream& log_;
    std::thread worker_;
    std::exception_ptr error_;
    std::string log_line_, out_line_;
    bool pending_ = false;
};

std::array<double, 3> cell_phi(const std::vector<double>& phi, size_t i) { return {phi[3 * i], phi[3 * i + 1], phi[3 * i + 2]}; }

// Host copies of the reference's serial reductions, used where the reference's
// exact sequential sums are reported (pearl_serial.cpp:822-842, :856-864).
double interface_energy_only(const Config& c, const std::vector<double>& phi) {
    const double eps = c.epsilon, sigma = c.sigma;
    const double obstacle = 16 * sigma / (std::acos(-1.) * std::acos(-1.) * eps), triple = c.triple / eps;
    double total = 0;
    for (int y = 0; y < c.ny; ++y)
        for (int x = 0; x < c.nx; ++x) {
            const auto p = cell_phi(phi, static_cast<size_t>(y) * c.nx + x);
            total += obstacle * (p[0] * p[1] + p[0] * p[2] + p[1] * p[2]) + triple * p[0] * p[1] * p[2];
            for (int dir = 0; dir < 2; ++dir) {
                if (dir == 1 && y == c.ny - 1) continue;
                const int xn = dir == 0 ? (x + 1) % c.nx : x, yn = dir == 0 ? y : y + 1;
                const auto n = cell_phi(phi, static_cast<size_t>(yn) * c.nx + xn);
                const double dist = dir == 0 ? c.dx : c.dy;
                for (int a = 0; a < 3; ++a)
                    for (int b = a + 1; b < 3; ++b) {
                        const double z = (p[a] * n[b] - n[a] * p[b]) / dist;
                        total += eps * sigma * z * z;
                    }
            }
        }
    return total * c.dx * c.dy;
}

std::array<double, 3> phase_fractions(const Config& c, const std::vector<double>& phi) {
    std::array<double, 3> local{0, 0, 0};
    const size_t cells = static_cast<size_t>(c.nx) * c.ny;
    for (size_t i = 0; i < cells; ++i)
        for (int a = 0; a < 3; ++a) local[a] += phi[3 * i + a];
    std::array<double, 3> out{};
    const double n = static_cast<double>(c.nx) * c.ny;
    for (int a = 0; a < 3; ++a) out[a] = local[a] / n;
    return out;
}

// The input's filling commands in the C ABI's form (method code + parameters).
std::vector<pearl_fill_op> device_fill_ops(const std::vector<FillOp>& fill) {
    static const std::pair<const char*, int> kMethods[] = {
        {"FILLCUBE", PEARL_FILL_CUBE},
        {"FILLCYLINDER", PEARL_FILL_CYLINDER},
        {"FILLCENTERBOX2D", PEARL_FILL_CENTER_BOX_2D},
        {"FILLYJUNCTION2D", PEARL_FILL_Y_JUNCTION_2D},
        {"FILLYJUNCTIONLAMELLAE2D", PEARL_FILL_Y_JUNCTION_LAMELLAE_2D},
        {"FILLADHEREDPEARLITEARM2D", PEARL_FILL_ADHERED_PEARLITE_ARM_2D},
        {"FILLPEARLITEELLIPSE2D", PEARL_FILL_PEARLITE_ELLIPSE_2D},
    };
    if (fill.size() > PEARL_FILL_MAX_OPS) throw std::invalid_argument("too many filling commands");
    std::vector<pearl_fill_op> ops;
    for (const auto& f : fill) {
        pearl_fill_op o{};
        for (const auto& m : kMethods)
            if (f.method == m.first) o.method = m.second;
        if (!o.method || f.p.size() > PEARL_FILL_MAX_PARAMS)
            throw std::invalid_argument("Unvalidated/unsupported filling method: " + f.method);
        o.nparams = static_cast<int>(f.p.size());
        for (size_t j = 0; j < f.p.size(); ++j) o.p[j] = f.p[j];
        ops.push_back(o);
    }
    return ops;
}

// Native initial geometry (pearl_serial.cpp:1764-1794).
std::vector<double> initial_geometry(const Config& c) {
    std::vector<double> phi(static_cast<size_t>(c.nx) * c.ny * 3, 0.0);
    const double width = c.theta_columns * c.dx, L = c.nx * c.dx, eps = c.epsilon;
    for (int y = 0; y < c.ny; ++y)
        for (int x = 0; x < c.nx; ++x) {
            const double xx = (x + 1 - .5) * c.dx, yy = (y + 1 - .5) * c.dy;
            std::array<double, 3> p{};
            if (c.initialization == "lamella") {
                const double dist = xx < width ? -std::min(xx, width - xx) : std::min(xx - width, L - xx);
                const double th = profile(dist, eps), product = profile(yy - c.seed_height, eps);
                p = {(1 - th) * product, th * product, 1 - product};
            } else if (c.initialization == "microsim") {
                p = {0, 0, 1};  // painted on the device by pearl_gpu_fill
            } else if (c.initialization == "sharp_smooth") {
                const bool product = yy < c.seed_height;
                if (!product)
                    p = {0, 0, 1};
                else if (x < c.theta_columns)
                    p = {0, 1, 0};
                else
                    p = {1, 0, 0};
            } else {
                const double dist = c.initialization == "flat"
                                        ? yy - c.seed_height
                                        : std::hypot(xx - .5 * L, yy - .5 * c.ny * c.dy) - c.radius;
                const double u = profile(dist, eps);
                p[c.phase_a] = u;
                p[c.phase_b] = 1 - u;
            }
            const size_t i = (static_cast<size_t>(y) * c.nx + x) * 3;
            phi[i] = p[0];
            phi[i + 1] = p[1];
            phi[i + 2] = p[2];
        }
    return phi;
}

}  // namespace

int main(int argc, char** argv) {
    int status = 0;
    try {
        if (argc < 3)
            throw std::invalid_argument(
                "Usage: pearl input.in NEW_OUTPUT_DIR [--restart frame.h5] [--px N --py N] [--max-steps N] "
                "[--thermo-only]");
        const std::string input = argv[1], output = argv[2];
        std::string restart;
        bool thermo_only = false;
        int px = 1, py = 1;
        long long stop_steps = -1;
        for (int k = 3; k < argc; ++k) {
            const std::string key = argv[k];
            if (key == "--thermo-only") {
                thermo_only = true;
                continue;
            }
            if (k + 1 == argc) throw std::invalid_argument("missing CLI value");
            const std::string val = argv[++k];
            if (key == "--restart")
                restart = val;
            else if (key == "--px")
                px = std::stoi(val);
            else if (key == "--py")
                py = std::stoi(val);
            else if (key == "--max-steps")
                stop_steps = std::stoll(val);
            else
                throw std::invalid_argument("unknown CLI flag: " + key);
        }
        if (thermo_only && !restart.empty()) throw std::invalid_argument("--thermo-only cannot be combined with --restart");
        Config config = read_config(input);
        if (stop_steps == 0 || stop_steps < -1) throw std::invalid_argument("max-steps must be positive");
        // Domain's checks (pearl_serial.cpp:618-619, :635-636)
        if (config.nx < 3 || config.ny < 2 || config.dx <= 0 || config.dy <= 0 || !std::isfinite(config.dx + config.dy) ||
            px < 1 || py < 1)
            throw std::invalid_argument("invalid grid");
        if (px != 1 || py != 1) throw std::invalid_argument("serial build requires px=py=1");
        bool outok = true;
        try {
            if (fs::exists(output)) throw std::runtime_error("output path already exists; refuse overwrite");
            fs::create_directories(output);
            fs::copy_file(input, fs::path(output) / "Input.in");
            write_thermodynamic_report(config, fs::path(output) / "thermodynamics.txt");
        } catch (...) {
            outok = false;
        }
        if (!outok) throw std::runtime_error("cannot create NEW output directory");
        if (thermo_only) {
            std::cout << "THERMO_ONLY: report written; no initialization or evolution performed\n";
            return 0;
        }
        const int device = std::getenv("PEARL_GPU_DEVICE") ? std::atoi(std::getenv("PEARL_GPU_DEVICE")) : 0;
        Gpu gpu;
        pearl_params params = config.device_params(config.initial_mu);
        const int rc_create = pearl_gpu_create(&params, config.nx, config.ny, device, &gpu.ctx);
        if (rc_create != PEARL_OK) throw std::runtime_error(pearl_gpu_status_string(rc_create));
        HostState st;
        st.nx = config.nx;
        st.ny = config.ny;
        const size_t cells = static_cast<size_t>(config.nx) * config.ny;
        pearl_smooth_report smooth{};
        double mu_reference = 0;
        if (restart.empty()) {
            // initialize (pearl_serial.cpp:1761-1837) with smoothing and composition on the device
            st.phi = initial_geometry(config);
            st.carbon.assign(cells, 0.0);
            st.mu.assign(cells, 0.0);
            gpu.check(pearl_gpu_upload(gpu.ctx, st.phi.data(), st.carbon.data(), st.mu.data(), nullptr));
            if (config.initialization == "microsim") {
                // filling_phase_at of every cell (pearl_serial.cpp:1771-1772) on the device
                const std::vector<pearl_fill_op> ops = device_fill_ops(config.fill);
                gpu.check(pearl_gpu_fill(gpu.ctx, ops.data(), static_cast<int>(ops.size())));
                gpu.check(pearl_gpu_download(gpu.ctx, st.phi.data(), nullptr, nullptr, nullptr));
            }
            if (config.initialization == "sharp_smooth" || config.initialization == "microsim") {
                write_initial_phases(config.nx, config.ny, config.dx, config.dy, st.phi,
                                     fs::path(output) / "init_sharp.h5", "init_sharp", 0);
                gpu.check(pearl_gpu_smooth_interface(gpu.ctx, config.smooth_steps, config.smooth_min_steps,
                                                     config.smooth_energy_rtol, config.smooth_max_phase_change,
                                                     &smooth));
                gpu.check(pearl_gpu_download(gpu.ctx, st.phi.data(), nullptr, nullptr, nullptr));
                write_initial_phases(config.nx, config.ny, config.dx, config.dy, st.phi,
                                     fs::path(output) / "init_smoothed.h5", "init_smoothed", smooth.steps);
            } else {
                const auto f = phase_fractions(config, st.phi);
                for (int a = 0; a < 3; ++a) smooth.phase_fraction_before[a] = smooth.phase_fraction_after[a] = f[a];
                smooth.energy_initial = interface_energy_only(config, st.phi);
                smooth.energy_final = smooth.energy_initial;
                smooth.converged = 1;
            }
            double mu = config.initial_mu;
            if (config.composition_mode == "mean") {
                // One-time solve of pearl_serial.cpp:1814-1822.  Its two sums cancel
                // strongly, so they are formed on the host in the reference's
                // sequential order, which makes mu_reference bitwise equal to it.
                if (config.initialization == "sharp_smooth" || config.initialization == "microsim") {
                    // st.phi already holds the smoothed fields
                } else {
                    gpu.check(pearl_gpu_download(gpu.ctx, st.phi.data(), nullptr, nullptr, nullptr));
                }
                double si = 0, sc = 0;
                for (size_t i = 0; i < cells; ++i) {
                    const auto p = cell_phi(st.phi, i);
                    const double triple = 2.0 * p[0] * p[1] * p[2];
                    double chi = 0.0, ci = 0.0;
                    for (int q = 0; q < 3; ++q) {
                        const double h = p[q] * p[q] * (3.0 - 2.0 * p[q]) + triple;
                        const double cq = config.thermo[q].chi();
                        chi += h * cq;
                        ci -= h * cq * config.thermo[q].B;
                    }
                    si += ci;
                    sc += chi;
                }
                mu = (config.nx * config.ny * config.initial_carbon - si) / sc;
            }
            double mass = 0;
            gpu.check(pearl_gpu_init_composition(gpu.ctx, mu, &mass));
            pearl_scalars s{};
            s.time = 0;
            s.step = 0;
            s.rejected = 0;
            s.dt = config.dt;
            s.initial_carbon = mass;
            gpu.check(pearl_gpu_set_scalars(gpu.ctx, &s));
            params = config.device_params(mu);
            gpu.check(pearl_gpu_set_params(gpu.ctx, &params));
            int valid = 0;
            gpu.check(pearl_gpu_valid_state(gpu.ctx, &valid));
            if (!valid) throw std::runtime_error("initial state out of model range");
            mu_reference = mu;
        } else {
            // read_checkpoint (pearl_serial.cpp:1970-2020)
            mu_reference = read_checkpoint_file(st, config, restart);
            params = config.device_params(mu_reference);
            gpu.check(pearl_gpu_set_params(gpu.ctx, &params));
            gpu.check(pearl_gpu_upload(gpu.ctx, st.phi.data(), st.carbon.data(), st.mu.data(), &st.s));
            int valid = 0;
            gpu.check(pearl_gpu_valid_state(gpu.ctx, &valid));
            if (!valid) throw std::runtime_error("invalid checkpoint state");
            double closure = 0;
            for (size_t i = 0; i < cells; ++i) {
                const auto p = cell_phi(st.phi, i);
                const double triple = 2.0 * p[0] * p[1] * p[2];
                double chi = 0.0, ci = 0.0;
                for (int q = 0; q < 3; ++q) {
                    const double h = p[q] * p[q] * (3.0 - 2.0 * p[q]) + triple;
                    const double cq = config.thermo[q].chi();
                    chi += h * cq;
                    ci -= h * cq * config.thermo[q].B;
                }
                closure = std::max(closure, std::abs(st.carbon[i] - std::fma(chi, st.mu[i], ci)));
            }
            if (closure > config.closure_tol) throw std::runtime_error("checkpoint closure failed");
            double v = 0;
            for (size_t i = 0; i < cells; ++i) v += st.carbon[i];
            const double ledger = v * config.dx * config.dy + st.s.carbon_removed - st.s.carbon_added -
                                  st.s.initial_carbon;
            if (!config.phase_only && std::abs(ledger) > 1e-10 * config.nx * config.ny * config.dx * config.dy)
                throw std::runtime_error("checkpoint mass ledger failed");
        }
        pearl_scalars S{};
        gpu.check(pearl_gpu_get_scalars(gpu.ctx, &S));
        if (restart.empty()) {
            std::ofstream initlog(fs::path(output) / "initialization_report.txt");
            initlog << std::setprecision(17);
            initlog << "initialization=" << config.initialization << "\n";
            initlog << "physical_time_after_preprocess=" << S.time << "\n";
            initlog << "solver_step_after_preprocess=" << S.step << "\n";
            initlog << "smooth_steps_completed=" << smooth.steps << "\n";
            initlog << "smooth_energy_converged=" << (smooth.converged ? 1 : 0) << "\n";
            initlog << "smooth_energy_initial=" << smooth.energy_initial << "\n";
            initlog << "smooth_energy_final=" << smooth.energy_final << "\n";
            initlog << "smooth_final_relative_energy_change=" << smooth.final_relative_energy_change << "\n";
            initlog << "smooth_final_max_phase_change=" << smooth.final_max_phase_change << "\n";
            initlog << "phase_fraction_before=" << smooth.phase_fraction_before[0] << ','
                    << smooth.phase_fraction_before[1] << ',' << smooth.phase_fraction_before[2] << "\n";
            initlog << "phase_fraction_after=" << smooth.phase_fraction_after[0] << ','
                    << smooth.phase_fraction_after[1] << ',' << smooth.phase_fraction_after[2] << "\n";
            initlog << "mu_reference=" << mu_reference << "\n";
            initlog << "NOTE=smoothing is capillarity-only preprocessing pseudo-time; carbon diffusion is disabled and "
                       "physical time is reset to zero before coupled evolution.\n";
        }
        if (S.time >= config.end_time) throw std::runtime_error("checkpoint time >= end_time");
        std::signal(SIGINT, on_signal);
        std::signal(SIGTERM, on_signal);
        const long long first_step = S.step;
        long long frames = 0;
        double next_output =
            (std::floor((S.time + 1e-12 * config.output_dt) / config.output_dt) + 1.0) * config.output_dt;
        pearl_step_info last{};
        long long cg_total = 0;
        int cg_peak = 0;
        const auto start = std::chrono::steady_clock::now();
        std::ofstream log(fs::path(output) / "diagnostics.csv");
        if (!log) throw std::runtime_error("cannot open diagnostics");
        log << "time,step,dt_next,mean_carbon,mass_ledger_error,reduced_energy,phi_sum_error,c_min,c_max,mu_min,"
               "mu_max,cg_last,cg_peak,closure_last,rejected,shift_distance,wall_s\n";
        std::cout << "resources: ranks=1 layout=" << px << "x" << py << " grid=" << config.nx << "x" << config.ny
                  << "\n";
        // Frames and checkpoints keep the reference's HDF5 object model but are
        // not HDF5 files (libhdf5 is not linked): say so once, before the first.
        std::cout << "NOTE: frame_*.h5 and checkpoint.h5 are written in the PEARL-H5-STUB container, not HDF5; "
                     "HDF5 tools (h5py, ParaView) cannot open them\n";
        st.phi.resize(3 * cells);
        st.carbon.resize(cells);
        st.mu.resize(cells);
        FrameWriter writer(log);
        const auto snapshot = [&]() {
            pearl_diag d{};
            gpu.check(pearl_gpu_snapshot(gpu.ctx, &d));
            const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
            writer.wait();  // the previous frame is written and st is free
            gpu.check(pearl_gpu_download(gpu.ctx, st.phi.data(), st.carbon.data(), st.mu.data(), &st.s));
            std::ostringstream fn;
            fn << "frame_" << std::setfill('0') << std::setw(6) << frames++ << ".h5";
            std::ostringstream line, out;
            line << std::setprecision(17) << st.s.time << ',' << st.s.step << ',' << st.s.dt << ','
                 << d.mass / (config.nx * config.ny * config.dx * config.dy) << ',' << d.ledger << ',' << d.energy << ','
                 << d.phi_sum_error << ',' << d.c_min << ',' << d.c_max << ',' << d.mu_min << ',' << d.mu_max << ','
                 << last.cg_iterations << ',' << cg_peak << ',' << last.closure << ',' << st.s.rejected << ','
                 << st.s.shift_distance << ',' << wall << '\n';
            out << "t=" << st.s.time << " step=" << st.s.step << " dt_next=" << st.s.dt << " mass_error=" << d.ledger
                << " CG=" << last.cg_iterations << " rejected=" << st.s.rejected << "\n";
            writer.submit(st, config, mu_reference, fs::path(output) / fn.str(), line.str(), out.str());
        };
        snapshot();
        bool stopped = false;
        double saved_time = S.time;
        const double eps = 1e-12 * std::max(config.end_time, config.output_dt);
        while (true) {
            gpu.check(pearl_gpu_get_scalars(gpu.ctx, &S));
            if (!(S.time < config.end_time)) break;
            const bool stop = interrupted || (stop_steps > 0 && S.step - first_step >= stop_steps);
            if (stop) {
                stopped = true;
                break;
            }
            if (S.step >= config.max_steps) throw std::runtime_error("configured max_steps reached before end_time");
            pearl_run_limits lim{};
            lim.max_steps = kStepsPerLaunch;
            if (stop_steps > 0) lim.max_steps = std::min(lim.max_steps, stop_steps - (S.step - first_step));
            lim.config_max_steps = config.max_steps;
            lim.stop_time = std::min(config.end_time, next_output);
            lim.end_time = config.end_time;
            lim.output_eps = eps;
            pearl_run_report rep{};
            gpu.check(pearl_gpu_run(gpu.ctx, &lim, &rep));
            cg_total += rep.cg_total;
            cg_peak = std::max(cg_peak, rep.cg_peak);
            if (rep.steps > 0) last = rep.last;
            gpu.check(pearl_gpu_get_scalars(gpu.ctx, &S));
            if (S.time >= next_output - eps || S.time >= config.end_time - eps) {
                // snap only the clock within rounding tolerance (pearl_serial.cpp:2309-2310)
                if (std::abs(S.time - next_output) <= eps) S.time = next_output;
                if (std::abs(S.time - config.end_time) <= eps) S.time = config.end_time;
                gpu.check(pearl_gpu_set_scalars(gpu.ctx, &S));
                if (config.moving_window) {
                    int rows = 0;
                    gpu.check(pearl_gpu_maybe_shift(gpu.ctx, config.shift_trigger, config.shift_target,
                                                    config.shift_gamma_carbon, &rows));
                }
                snapshot();
                gpu.check(pearl_gpu_get_scalars(gpu.ctx, &S));
                saved_time = S.time;
                next_output += config.output_dt;
            }
        }
        if (S.time != saved_time) snapshot();
        writer.wait();
        gpu.check(pearl_gpu_download(gpu.ctx, st.phi.data(), st.carbon.data(), st.mu.data(), &st.s));
        write_frame(st, config, mu_reference, fs::path(output) / "checkpoint.h5");
        std::ofstream fin(fs::path(output) / (stopped ? "STOPPED.txt" : "COMPLETED.txt"));
        fin << std::setprecision(17) << "status=" << (stopped ? "USER_STOPPED" : "HORIZON_COMPLETED")
            << "\ntime=" << st.s.time << "\nstep=" << st.s.step << "\nCG_total=" << cg_total
            << "\nrejected=" << st.s.rejected << "\nThis is a solver status, not certification of cooperative growth.\n";
    } catch (const std::exception& e) {
        std::cerr << "ERROR: " << e.what() << '\n';
        status = 1;
    }
    return status;
}
