// potentials -- drop-in replacement for the reference's quasi-potential tool
// (potentials.cpp:30-207): V(r) of every state's own density at every atom, one
// "potential-<file>" per input with "%.12le" lines.
#include <cstdio>
#include <cstdlib>
#include <limits>
#include <string>
#include <vector>

#include "common.hpp"

namespace {

const char* kUsage =
    "Coulombo v2.0 (c) 2023 [Computer Physics Communications] Rozanski & Zielinski:\n"
    "Exploiting underlying crystal lattice for efficient computation of Coulomb matrix elements in multi-million "
    "atoms nanostructures\n"
    "(B200 implementation of the integral path)\n"
    "\nUSAGE:\n"
    " potentials [FLAGS/OPTIONS] data files ...\n"
    "\nOPTIONS:\n"
    "  --atoms=PATH           path to *.3d file with atoms' positions\n"
    "  --dielectric=VALUE     dielectric constant, default: 1\n"
    "  --onsite=ENERGY        energy for on-site contribution, default: 0 (eV)\n"
    "  --orbitals=N           number of (spin-)orbitals per atom, default: 20\n"
    "  --output-dir=DIR       directory for output files, default: current\n"
    "  --precision=fp64|fp32  fp64: all-FP64 path (default); fp32: FP32 transforms, FP64 sums\n"
    "  --method=rounds|sublattice  rounds: the 8-round convolution (default); sublattice: the\n"
    "                           exact per-residue-class decomposition where the structure allows\n"
    "  --skip-lines=N         number of lines to be skipped on top of each LCAO file, default: 0\n"
    "  --threads-per-node=N   number of host threads for reading inputs, default: all cores\n"
    "  --tf-lattice=VALUE     lattice constant (A) for Thomas-Fermi-Resta model,\n"
    "                           default: model not applied\n"
    "\n";

void run(const clio::ParseResults& pr) {
    clio::Timer timer;
    clapp::Inputs in;
    clapp::parse_common_options(pr, in);

    timer.start("Reading atom positions");
    clapp::read_atoms(pr, in);

    timer.start("Reading wavefunctions");
    const int input_count = (int)pr.args.size();
    if (input_count >= std::numeric_limits<short>::max()) clio::throwfr("too many input files");
    std::vector<std::string> names;
    for (const auto& arg : pr.args) {
        clapp::read_state_file(in, arg);
        names.push_back(clapp::basename_of(arg));
    }

    timer.start("Initializing calculator");
    const clapp::KernelOptions kopt = clapp::kernel_options(pr, in);
    clapp::Calculator calc(in.pad, in.step, in.mode);
    clapp::check(cl_set_kernel_coulomb(calc.get(), in.dielectric, kopt.onsite, kopt.tf_lattice));
    clapp::check(cl_set_states(calc.get(), input_count, 0, in.n_atoms, in.orbitals, in.coeff.data(),
                               in.cells.data()));

    timer.start("Computing all quasi-potentials");
    std::vector<double> pot((size_t)input_count * in.n_atoms);
    clapp::check(cl_potentials(calc.get(), pot.data()));
    for (int s = 0; s < input_count; ++s) {
        const std::string path = in.output_dir + "potential-" + names[s];
        FILE* f = std::fopen(path.c_str(), "w");
        if (!f) clio::throwfr("cannot open file %s for writing", path.c_str());
        for (int64_t a = 0; a < in.n_atoms; ++a) std::fprintf(f, "%.12le\n", pot[(size_t)s * in.n_atoms + a]);
        std::fclose(f);
    }
}

}  // namespace

int main(int argc, char** argv) {
    try {
        clio::Parser cmd;
        for (const char* v : {"atoms", "dielectric", "onsite", "orbitals", "method", "output-dir", "precision", "skip-lines",
                              "threads-per-node", "tf-lattice"})
            cmd.allow_value(v);
        clio::ParseResults pr = cmd.process(argc, argv);
        if (pr.args.empty()) {
            std::fputs(kUsage, stderr);
            return EXIT_FAILURE;
        }
        run(pr);
    } catch (std::exception& ex) {
        std::fprintf(stderr, "ERROR: %s\n", ex.what());
        return EXIT_FAILURE;
    }
    return 0;
}
