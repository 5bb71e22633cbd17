// Thin C++ owner of a cl_ctx: every non-zero status becomes std::runtime_error carrying
// cl_last_error(), so the binaries keep the reference's "ERROR: <message>" behaviour.
#pragma once

#include <stdexcept>
#include <string>

#include "coulombo_lattice.h"

namespace clapp {

inline void check(int status) {
    if (status != CL_OK) throw std::runtime_error(cl_last_error());
}

class Calculator {
public:
    Calculator(const int dims[3], const double step[3], int mode) {
        check(cl_create(&ctx_, dims[0], dims[1], dims[2], step[0], step[1], step[2], mode));
    }
    ~Calculator() { cl_destroy(ctx_); }
    Calculator(const Calculator&) = delete;
    Calculator& operator=(const Calculator&) = delete;
    cl_ctx* get() const { return ctx_; }

private:
    cl_ctx* ctx_ = nullptr;
};

}  // namespace clapp
