// Shared front half of the coulombo and potentials binaries: options, atoms, grid, states.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <string>
#include <thread>
#include <vector>

#include "../host/io.hpp"
#include "cl_cpp.hpp"

namespace clapp {

struct Inputs {
    int orbitals = 20;
    int skip_lines = 0;
    int threads = 1;
    int mode = CL_MODE_FP64_PLAIN;
    double dielectric = 1.0;
    std::string output_dir;
    int raw[3], pad[3];
    double origin[3], step[3];
    int64_t n_atoms = 0;
    std::vector<int64_t> cells;
    std::vector<std::string> files, basenames;
    std::vector<double> coeff;  // [state][atom][orb]{re,im}
};

// --threads-per-node (coulombo.cpp:36-54): accepted as in the reference, used as the number
// of text-parser threads.  --precision and --method select the device form (default fp64 and
// rounds: the plain path, the reference's method).
inline void parse_common_options(const clio::ParseResults& pr, Inputs& in) {
    std::string value;
    if (pr.has_value("threads-per-node", value)) {
        in.threads = std::atoi(value.c_str());
        if (in.threads <= 0) clio::throwfr("invalid value for threads-per-node");
    } else {
        in.threads = std::max(1u, std::thread::hardware_concurrency());
    }
    bool fp32 = false, sublattice = false;
    if (pr.has_value("precision", value)) {
        if (value == "fp64")
            fp32 = false;
        else if (value == "fp32")
            fp32 = true;
        else
            clio::throwfr("invalid value for precision: %s", value.c_str());
    }
    if (pr.has_value("method", value)) {
        if (value == "rounds")
            sublattice = false;
        else if (value == "sublattice")
            sublattice = true;
        else
            clio::throwfr("invalid value for method: %s", value.c_str());
    }
    in.mode = sublattice ? (fp32 ? CL_MODE_FP32_SUBLATTICE : CL_MODE_FP64_SUBLATTICE)
                         : (fp32 ? CL_MODE_FP32_ROUNDS : CL_MODE_FP64_PLAIN);
}

// "Reading atom positions" (coulombo.cpp:56-74, FunctionCollection.cpp:14-20)
inline void read_atoms(const clio::ParseResults& pr, Inputs& in) {
    std::string value;
    if (pr.has_value("orbitals", value)) {
        in.orbitals = std::atoi(value.c_str());
        if (in.orbitals <= 0) clio::throwfr("invalid value for orbitals");
    }
    if (pr.has_value("skip-lines", value)) {
        in.skip_lines = std::atoi(value.c_str());
        if (in.skip_lines <= 0) clio::throwfr("invalid value for skip-lines");
    }
    std::vector<double> pos = clio::load_atoms(pr.get_value("atoms"));
    in.n_atoms = (int64_t)(pos.size() / 3);
    in.cells.resize((size_t)in.n_atoms);
    check(cl_detect_grid(pos.data(), in.n_atoms, in.raw, in.pad, in.origin, in.step, in.cells.data()));
    if (pr.has_value("dielectric", value)) in.dielectric = std::atof(value.c_str());
    if (pr.has_value("output-dir", in.output_dir) && !in.output_dir.empty()) in.output_dir += '/';
}

inline std::string basename_of(const std::string& arg) {
    auto s = arg.find_last_of('/');
    return s == std::string::npos ? arg : arg.substr(s + 1);
}

inline void read_state_file(Inputs& in, const std::string& path) {
    const size_t per = (size_t)in.n_atoms * in.orbitals * 2;
    const size_t off = in.coeff.size();
    in.coeff.resize(off + per);
    clio::load_state(path, in.n_atoms, in.orbitals, in.skip_lines, in.threads, in.coeff.data() + off);
}

// onsite / dielectric model of coulombo.cpp:157-177, checked before the calculator exists
struct KernelOptions {
    double onsite = 0.0;
    double tf_lattice = 0.0;
};
inline KernelOptions kernel_options(const clio::ParseResults& pr, const Inputs& in) {
    std::string value;
    double onsite = 0.0;
    if (pr.has_value("onsite", value)) onsite = std::atof(value.c_str());
    double tf = 0.0;
    if (pr.has_value("tf-lattice", value)) {
        double lattice = std::atof(value.c_str());
        if (!std::isgreater(lattice, 0.0)) clio::throwfr("--tf-lattice parameter must be positive");
        if (!std::isgreater(in.dielectric, 1.0)) clio::throwfr("dielectric constant must be >1 to use Thomas-Fermi model");
        tf = lattice;
    }
    return KernelOptions{onsite, tf};
}

}  // namespace clapp
