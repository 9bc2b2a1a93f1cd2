// io.cpp — frames, checkpoints, XMF sidecars and text reports (see io.hpp).
#include "io.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <stdexcept>

namespace pearl_host {

namespace fs = std::filesystem;

void FieldFile::add(const std::string& name, int nx, int ny, std::vector<double> v) {
    datasets.push_back({name, ny, nx, std::move(v)});
}
void FieldFile::attr(const std::string& name, double v) { attributes.push_back({name, false, v, {}}); }
void FieldFile::attr(const std::string& name, const std::string& s) { attributes.push_back({name, true, 0, s}); }

const FieldFile::Dataset* FieldFile::dataset(const std::string& name) const {
    for (const auto& d : datasets)
        if (d.name == name) return &d;
    return nullptr;
}
double FieldFile::number(const std::string& name) const {
    for (const auto& a : attributes)
        if (a.name == name && !a.is_string) return a.value;
    throw std::runtime_error("HDF5 open/create failure");
}
std::string FieldFile::text(const std::string& name) const {
    for (const auto& a : attributes)
        if (a.name == name && a.is_string) return a.text;
    throw std::runtime_error("HDF5 open/create failure");
}

void FieldFile::write(const fs::path& path) const {
    if (fs::exists(path)) throw std::runtime_error("HDF5 open/create failure");
    FILE* f = std::fopen(path.c_str(), "wbx");
    if (!f) throw std::runtime_error("HDF5 open/create failure");
    bool ok = std::fprintf(f, "PEARL-H5-STUB 1\n") > 0;
    for (const auto& d : datasets) {
        ok = ok && std::fprintf(f, "D %s %d %d\n", d.name.c_str(), d.ny, d.nx) > 0;
        ok = ok && std::fwrite(d.data.data(), sizeof(double), d.data.size(), f) == d.data.size();
        ok = ok && std::fputc('\n', f) != EOF;
    }
    for (const auto& a : attributes) {
        if (a.is_string) {
            ok = ok && std::fprintf(f, "A %s s %zu\n", a.name.c_str(), a.text.size()) > 0;
            ok = ok && std::fwrite(a.text.data(), 1, a.text.size(), f) == a.text.size();
            ok = ok && std::fputc('\n', f) != EOF;
        } else {
            ok = ok && std::fprintf(f, "A %s d %a\n", a.name.c_str(), a.value) > 0;
        }
    }
    ok = ok && std::fprintf(f, "END\n") > 0;
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) throw std::runtime_error("HDF5: flush");
}

FieldFile FieldFile::read(const fs::path& path) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("HDF5 open/create failure");
    FieldFile out;
    char line[4096];
    bool ok = std::fgets(line, sizeof line, f) && std::strncmp(line, "PEARL-H5-STUB 1", 15) == 0;
    bool ended = false;
    while (ok && std::fgets(line, sizeof line, f)) {
        if (std::strncmp(line, "END", 3) == 0) {
            ended = true;
            break;
        }
        char name[2048], kind = 0, rest[2048];
        if (line[0] == 'D') {
            int ny = 0, nx = 0;
            if (std::sscanf(line, "D %2047s %d %d", name, &ny, &nx) != 3 || ny < 0 || nx < 0) {
                ok = false;
                break;
            }
            Dataset d{name, ny, nx, std::vector<double>(static_cast<size_t>(ny) * nx)};
            ok = std::fread(d.data.data(), sizeof(double), d.data.size(), f) == d.data.size();
            std::fgetc(f);
            out.datasets.push_back(std::move(d));
        } else if (line[0] == 'A' && std::sscanf(line, "A %2047s %c %2047s", name, &kind, rest) == 3) {
            Attribute a{name, kind == 's', 0, {}};
            if (kind == 'd') {
                a.value = std::strtod(rest, nullptr);
            } else {
                const size_t n = static_cast<size_t>(std::strtoull(rest, nullptr, 10));
                a.text.resize(n);
                ok = n == 0 || std::fread(&a.text[0], 1, n, f) == n;
                std::fgetc(f);
            }
            out.attributes.push_back(std::move(a));
        } else {
            ok = false;
        }
    }
    std::fclose(f);
    if (!ok || !ended) throw std::runtime_error("HDF5 open/create failure");
    return out;
}

namespace {

void write_xmf(const fs::path& h5, int nx, int ny, double dx, double dy, double time, double shift_distance,
               const char* grid_name, bool with_time, const std::vector<std::string>& names, bool atomic) {
    auto xmf = h5;
    xmf.replace_extension(".xmf");
    auto target = xmf;
    if (atomic) target += ".part";
    std::ofstream out(target);
    if (!out) throw std::runtime_error(atomic ? "cannot write XMF" : "initial XMF write failure");
    out << std::setprecision(17) << "<?xml version=\"1.0\"?>\n<Xdmf Version=\"3.0\"><Domain><Grid Name=\""
        << grid_name << "\" GridType=\"Uniform\">\n";
    if (with_time) out << "<Time Value=\"" << time << "\"/>\n";
    out << "<Topology TopologyType=\"2DCoRectMesh\" Dimensions=\"" << ny << " " << nx << "\"/>\n"
        << "<Geometry GeometryType=\"ORIGIN_DXDY\"><DataItem Dimensions=\"2\" Format=\"XML\">"
        << .5 * dy + shift_distance << " " << .5 * dx << "</DataItem><DataItem Dimensions=\"2\" Format=\"XML\">" << dy
        << " " << dx << "</DataItem></Geometry>\n";
    for (const auto& name : names)
        out << "<Attribute Name=\"" << name << "\" AttributeType=\"Scalar\" Center=\"Node\"><DataItem Dimensions=\""
            << ny << " " << nx << "\" NumberType=\"Float\" Precision=\"8\" Format=\"HDF\">"
            << h5.filename().string() << ":/" << name << "</DataItem></Attribute>\n";
    out << "</Grid></Domain></Xdmf>\n";
    out.close();
    if (!out) throw std::runtime_error(atomic ? "XMF write failure" : "initial XMF write failure");
    if (atomic) fs::rename(target, xmf);
}

std::vector<double> phase_plane(const std::vector<double>& phi, size_t cells, int a) {
    std::vector<double> v(cells);
    for (size_t i = 0; i < cells; ++i) v[i] = phi[3 * i + a];
    return v;
}

}  // namespace

void write_frame(const HostState& st, const Config& config, double mu_reference, const fs::path& path) {
    if (fs::exists(path)) throw std::runtime_error("refuse overwriting frame " + path.string());
    auto temp = path;
    temp += ".part";
    const size_t cells = static_cast<size_t>(st.nx) * st.ny;
    FieldFile f;
    const char* names[3] = {"alpha", "theta", "gamma"};
    for (int a = 0; a < 3; ++a) f.add(names[a], st.nx, st.ny, phase_plane(st.phi, cells, a));
    f.add("carbon", st.nx, st.ny, st.carbon);
    f.add("mu", st.nx, st.ny, st.mu);
    f.attr("physics_signature", config.physics_signature());
    f.attr("format", std::string("pearlite-v0.4-5fields"));
    f.attr("thermo_mode", config.thermo_mode);
    f.attr("temperature_K", config.T);
    if (config.thermo_mode == "eutectoid_reference") {
        f.attr("T_eutectoid_K", config.T_eutectoid);
        f.attr("undercooling_K", config.undercooling);
    }
    f.attr("time", st.s.time);
    f.attr("dt_next", st.s.dt);
    f.attr("step", static_cast<double>(st.s.step));
    f.attr("dx", config.dx);
    f.attr("dy", config.dy);
    f.attr("nx", config.nx);
    f.attr("ny", config.ny);
    f.attr("shift_distance", st.s.shift_distance);
    f.attr("shifts", static_cast<double>(st.s.shifts));
    f.attr("initial_carbon", st.s.initial_carbon);
    f.attr("carbon_added", st.s.carbon_added);
    f.attr("carbon_removed", st.s.carbon_removed);
    f.attr("mu_reference", mu_reference);
    f.attr("rejected_steps", static_cast<double>(st.s.rejected));
    f.write(temp);
    fs::rename(temp, path);
    write_xmf(path, st.nx, st.ny, config.dx, config.dy, st.s.time, st.s.shift_distance, "pearlite", true,
              {"alpha", "theta", "gamma", "carbon", "mu"}, true);
}

double read_checkpoint_file(HostState& st, const Config& config, const std::string& path) {
    FieldFile f = FieldFile::read(path);
    if (f.text("format") != "pearlite-v0.4-5fields" || f.text("physics_signature") != config.physics_signature())
        throw std::runtime_error("checkpoint physics signature mismatch");
    const auto get = [&](const char* name) {
        const auto* d = f.dataset(name);
        if (!d) throw std::runtime_error("HDF5 open/create failure");
        if (d->ny != config.ny || d->nx != config.nx) throw std::runtime_error("checkpoint dimensions mismatch");
        return d->data;
    };
    const auto a = get("alpha"), t = get("theta"), g = get("gamma");
    st.nx = config.nx;
    st.ny = config.ny;
    st.carbon = get("carbon");
    st.mu = get("mu");
    st.phi.resize(3 * st.carbon.size());
    for (size_t i = 0; i < st.carbon.size(); ++i) {
        st.phi[3 * i] = a[i];
        st.phi[3 * i + 1] = t[i];
        st.phi[3 * i + 2] = g[i];
    }
    const char* keys[10] = {"time", "dt_next", "step", "shift_distance", "shifts", "initial_carbon",
                            "carbon_added", "carbon_removed", "mu_reference", "rejected_steps"};
    double meta[10];
    for (int k = 0; k < 10; ++k) meta[k] = f.number(keys[k]);
    for (double v : meta)
        if (!std::isfinite(v)) throw std::runtime_error("nonfinite checkpoint metadata");
    if (meta[0] < 0 || meta[1] <= 0 || meta[2] < 0 || meta[2] != std::floor(meta[2]) || meta[2] > 9e15)
        throw std::runtime_error("bad checkpoint time/step");
    st.s.time = meta[0];
    st.s.dt = std::min(config.dt_max, meta[1]);
    st.s.step = static_cast<long long>(meta[2]);
    st.s.shift_distance = meta[3];
    st.s.shifts = static_cast<long long>(meta[4]);
    st.s.initial_carbon = meta[5];
    st.s.carbon_added = meta[6];
    st.s.carbon_removed = meta[7];
    st.s.rejected = static_cast<long long>(meta[9]);
    return meta[8];
}

void write_initial_phases(int nx, int ny, double dx, double dy, const std::vector<double>& phi, const fs::path& path,
                          const std::string& stage, int pseudo_step) {
    if (fs::exists(path)) throw std::runtime_error("initial snapshot exists");
    auto temp = path;
    temp += ".part";
    const size_t cells = static_cast<size_t>(nx) * ny;
    FieldFile f;
    const char* names[3] = {"alpha", "theta", "gamma"};
    for (int a = 0; a < 3; ++a) f.add(names[a], nx, ny, phase_plane(phi, cells, a));
    f.attr("format", std::string("pearlite-preprocessing-phases-only"));
    f.attr("stage", stage);
    f.attr("pseudo_step", pseudo_step);
    f.attr("dx", dx);
    f.attr("dy", dy);
    f.write(temp);
    fs::rename(temp, path);
    write_xmf(path, nx, ny, dx, dy, 0, 0, stage.c_str(), false, {"alpha", "theta", "gamma"}, false);
}

void write_thermodynamic_report(const Config& config, const fs::path& path) {
    std::ofstream out(path);
    if (!out) throw std::runtime_error("cannot write thermodynamics report");
    out << std::setprecision(17);
    out << "thermo_mode=" << config.thermo_mode << "\nrun_temperature_K=" << config.T << "\nVm_m3_per_mol="
        << config.Vm << "\n";
    out << "energy_convention=legacy v0.3 molar-code convention; chemical term Psi/Vm, c=atomic fraction\n";
    out << "unit_scope=this preserves the inherited conversion; it does not certify the material's physical molar "
           "volume\n";
    out << "thermal_history=isothermal at the run temperature; no finite-rate cooling segment\n";
    if (config.thermo_mode == "eutectoid_reference") {
        out << "T_eutectoid_K=" << config.T_eutectoid << "\nundercooling_K=" << config.undercooling
            << "\nmax_undercooling_K=" << config.max_undercooling << "\ntemperature_law=" << config.temperature_law
            << "\n";
        if (config.temperature_law == "phase_diagram_fixed_curvature") {
            const auto& d = config.diagram;
            out << "phase_diagram_slope_units=carbon mole fraction/K (dc_eq/dT)\n";
            out << "phase_diagram_curvature=fixed at supplied reference Aeq\n";
            out << "phase_diagram_gamma_reference=ABC held at reference values\n";
            out << "phase_diagram_reference_c_alpha_theta_gamma=" << d.reference_composition[0] << ','
                << d.reference_composition[1] << ',' << d.reference_composition[2] << "\n";
            out << "phase_diagram_slopes_alpha_ag_gamma_ag_theta_tg_gamma_tg=";
            for (int j = 0; j < 4; ++j) out << (j ? "," : "") << d.composition_slope[j];
            out << "\nphase_diagram_reference_residual=preserved, not retuned\n";
        }
    }
    const char* names[3] = {"alpha", "theta", "gamma"};
    for (int i = 0; i < 3; ++i) {
        const std::string n = names[i];
        if (config.thermo_mode == "eutectoid_reference") {
            const auto& p = config.reference_thermo[i];
            const auto& s = config.temperature_slope[i];
            out << "reference_" << n << "_ABC=" << p.A << ',' << p.B << ',' << p.C << "\n";
            if (config.temperature_law == "linear_gp")
                out << "dq_dT_" << n << "_q2_q1_q0=" << s.q2 << ',' << s.q1 << ',' << s.q0 << "\n";
        }
        const auto& p = config.thermo[i];
        const GrandPotential g = to_grand_potential(p);
        out << "effective_" << n << "_ABC=" << p.A << ',' << p.B << ',' << p.C << "\n";
        out << "effective_" << n << "_q2_q1_q0=" << g.q2 << ',' << g.q1 << ',' << g.q0 << "\n";
        out << "effective_" << n << "_chi=" << p.chi() << "\nD_" << n << "=" << p.D << "\n";
    }
    out << "initial_composition_mode=" << config.composition_mode << "\n";
    if (config.composition_mode != "mean")
        out << "initial_mu_at_run_temperature=" << config.initial_mu << "\n";
    else
        out << "initial_mu_at_run_temperature=solved after smoothing from specified mean_carbon\n";
    out << "initialization_note=one local mu field; tip samples at distinct positions need not be equal\n";
    out << "tau_at_ag_tg=" << config.tau[0] << ',' << config.tau[1] << ',' << config.tau[2] << "\n";
    out << "tau_note=explicit input, not recalibrated by changing temperature; physical applicability remains a "
           "separate check\n";
    out.close();
    if (!out) throw std::runtime_error("thermodynamics report write failed");
}

}  // namespace pearl_host
