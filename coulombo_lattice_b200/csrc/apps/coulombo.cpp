// coulombo -- drop-in replacement for the reference's integral driver (coulombo.cpp:30-315):
// same options, inputs, phase lines, XXXX.txt outputs and "ERROR: <msg>" failures; the
// convolutions run on the GPU through libcoulombo_lattice.so.
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
    " coulombo [FLAGS/OPTIONS] data files ...\n"
    "\nOPTIONS:\n"
    "  --atoms=PATH           path to *.3d file with atoms' positions\n"
    "  --dielectric=VALUE     dielectric constant, default: 1\n"
    "  --integrals=LIST       comma-separated list of integrals to be computed\n"
    "                           (eg. \"eeee,hhhh,ehhe,eheh\"),\n"
    "                           default: all integrals are computed\n"
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
    std::string integrals = "****";
    pr.has_value("integrals", integrals);

    timer.start("Reading wavefunctions");
    const int input_count = (int)pr.args.size();
    if (input_count >= std::numeric_limits<short>::max()) clio::throwfr("too many input files");
    int holes = 0, electrons = 0;
    for (const auto& arg : pr.args) {
        const std::string base = clapp::basename_of(arg);
        if (!base.empty() && base[0] == 'h') {
            if (electrons) clio::throwfr("hole states must appear before electron states");
            ++holes;
        } else if (!base.empty() && base[0] == 'e') {
            ++electrons;
        } else {
            clio::throwfr("invalid state file name: %s", arg.c_str());
        }
        clapp::read_state_file(in, arg);
    }

    timer.start("Preparing plan");
    int64_t count = 0;
    clapp::check(cl_enumerate_integrals(integrals.c_str(), input_count, holes, &count, nullptr, 0));
    std::vector<int16_t> specs((size_t)count * 4);
    clapp::check(cl_enumerate_integrals(integrals.c_str(), input_count, holes, &count, specs.data(), count));

    timer.start("Initializing calculator");
    const clapp::KernelOptions kopt = clapp::kernel_options(pr, in);
    clapp::Calculator calc(in.pad, in.step, in.mode);
    clapp::check(cl_set_kernel_coulomb(calc.get(), in.dielectric, kopt.onsite, kopt.tf_lattice));

    // the coefficient upload overlaps the transforms (cl_compute_states)
    timer.start("Computing requested integrals");
    std::vector<double> values((size_t)count * 2, 0.0);
    clapp::check(cl_compute_states(calc.get(), input_count, holes, in.n_atoms, in.orbitals, in.coeff.data(),
                                   in.cells.data(), count, specs.data(), values.data()));

    timer.start("Exporting results");
    clio::write_integrals(in.output_dir, specs, values.data(), holes, electrons);
}

}  // namespace

int main(int argc, char** argv) {
    try {
        clio::Parser cmd;
        for (const char* v : {"atoms", "dielectric", "integrals", "onsite", "orbitals", "method", "output-dir", "precision",
                              "skip-lines", "threads-per-node", "tf-lattice"})
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
