// io.hpp — frames, checkpoints and reports of the Pearl host driver.
//
// The reference writes HDF5 through libhdf5 (pearl_serial.cpp:1843-2160).
// libhdf5 is not installed on the machines this project is built and run on,
// so frames and checkpoints are written in a self-describing container that
// keeps the reference's HDF5 object model exactly: the same five (ny, nx)
// float64 datasets and the same named attributes, in the same order:
//
//   PEARL-H5-STUB 1\n
//   D <name> <ny> <nx>\n<ny*nx little-endian float64>\n     one per dataset
//   A <name> d <C99 hex float>\n                             double attribute
//   A <name> s <nbytes>\n<bytes>\n                           string attribute
//   END\n
//
// It is the format of the HDF5 stand-in used to build the reference solver
// here, so checkpoints move between the two programs in both directions.
// XMF sidecars are byte-identical to the reference's apart from the data
// format they name.
#pragma once

#include <filesystem>
#include <map>
#include <string>
#include <vector>

#include "config.hpp"

namespace pearl_host {

struct FieldFile {
    struct Dataset {
        std::string name;
        int ny = 0, nx = 0;
        std::vector<double> data;
    };
    struct Attribute {
        std::string name;
        bool is_string = false;
        double value = 0;
        std::string text;
    };
    std::vector<Dataset> datasets;
    std::vector<Attribute> attributes;

    void add(const std::string& name, int nx, int ny, std::vector<double> v);
    void attr(const std::string& name, double v);
    void attr(const std::string& name, const std::string& s);
    const Dataset* dataset(const std::string& name) const;
    double number(const std::string& name) const;
    std::string text(const std::string& name) const;

    // Write to `path` exclusively (fails if it exists), as the reference's H5F_ACC_EXCL create.
    void write(const std::filesystem::path& path) const;
    static FieldFile read(const std::filesystem::path& path);
};

struct HostState {
    int nx = 0, ny = 0;
    std::vector<double> phi, carbon, mu;  // phi[(y*nx+x)*3+a]
    pearl_scalars s{};
};

// write_frame (pearl_serial.cpp:1914-1968): fields + 17 attributes, atomic
// .part rename, refuses to overwrite, then the XMF sidecar.
void write_frame(const HostState& st, const Config& config, double mu_reference, const std::filesystem::path& path);
// read_checkpoint (pearl_serial.cpp:1970-2020) without the device checks; returns mu_reference.
double read_checkpoint_file(HostState& st, const Config& config, const std::string& path);
// write_initial_phases (pearl_serial.cpp:2075-2115)
void write_initial_phases(int nx, int ny, double dx, double dy, const std::vector<double>& phi,
                          const std::filesystem::path& path, const std::string& stage, int pseudo_step);
// write_thermodynamic_report (pearl_serial.cpp:2118-2160)
void write_thermodynamic_report(const Config& config, const std::filesystem::path& path);

}  // namespace pearl_host
