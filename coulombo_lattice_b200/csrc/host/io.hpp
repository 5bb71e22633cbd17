// Text inputs and outputs of the drop-in binaries, plus the command-line parser and the
// phase timer.  Formats and messages follow the reference:
//   atoms file   FunctionCollection.cpp:38-54   "x y z [ignored...]" until the first line
//                                               without three numbers
//   state file   FunctionCollection.cpp:56-84   skip N header lines, then atoms*orbitals lines
//                                               "re im [ignored...]", else "file is truncated"
//   options      Parser.cpp:35-99                --name=value / --flag / -abc / positional
//   timer lines  Timer.cpp:11-77                 "<phase>... (x.xxx s)" on stderr
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <set>
#include <string>
#include <vector>

namespace clio {

// Reads the atom positions as [atom][3] doubles.
std::vector<double> load_atoms(const std::string& path);

// Reads n_atoms*n_orb complex coefficients ({re, im} interleaved) into dst after skipping
// skip_lines lines, using up to `threads` parser threads.
void load_state(const std::string& path, int64_t n_atoms, int n_orb, int skip_lines, int threads, double* dst);

struct ParseResults {
    std::set<std::string> flags;
    std::map<std::string, std::string> values;
    std::vector<std::string> args;
    bool has_value(const std::string& name, std::string& out) const;
    const std::string& get_value(const std::string& name) const;
};

class Parser {
public:
    Parser& allow_value(const std::string& name) {
        values_.insert(name);
        return *this;
    }
    Parser& allow_flag(const std::string& name) {
        flags_.insert(name);
        return *this;
    }
    ParseResults process(int argc, char** argv) const;

private:
    std::set<std::string> values_, flags_;
    std::map<char, std::string> short_;
};

// Phase timer: start(msg) closes the previous phase with "(x.xxx s)" and opens a new one.
class Timer {
public:
    ~Timer();
    void start(const char* msg);
    void stop();

private:
    bool open_ = false;
    double t0_ = 0;
};

// printf-style std::runtime_error, the reference's throwfr (throwf.hpp:14-35).
[[noreturn]] void throwfr(const char* fmt, ...) __attribute__((format(printf, 1, 2)));

// Writes the XXXX.txt files of coulombo.cpp:213-262.  specs are 1-based input indices,
// values {re, im}; holes are numbered in reverse in the files.  threads <= 0: all host threads.
void write_integrals(const std::string& out_prefix, const std::vector<int16_t>& specs, const double* values,
                     int n_holes, int n_electrons, int threads = 0);

}  // namespace clio
