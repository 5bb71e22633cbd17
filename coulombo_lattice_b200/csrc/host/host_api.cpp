// C ABI of the host-side helpers and the thread-local error channel.
#include <cstring>
#include <string>

#include <stdexcept>
#include <vector>

#include "coulombo_lattice.h"
#include "host_logic.hpp"
#include "io.hpp"
#include "status.hpp"

namespace cl {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }
const char* last_error() { return g_last_error.c_str(); }

void fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    int n = vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    throw Error(code, n > 0 ? std::string(buf) : std::string("error"));
}

}  // namespace cl

extern "C" {

const char* cl_last_error(void) { return cl::last_error(); }

int cl_round_up_235(int n, int c) {
    int r = -1;
    int st = cl::guarded([&] { r = cl::round_up_235(n, c); });
    return st == CL_OK ? r : -1;
}

int cl_detect_grid(const double* pos, int64_t n_atoms, int raw[3], int pad[3], double origin[3],
                   double step[3], int64_t* cells) {
    return cl::guarded([&] {
        if (!pos || !raw || !pad || !origin || !step) cl::fail(CL_ERR_ARGUMENT, "null argument");
        cl::Grid g = cl::detect_grid(pos, n_atoms, cells);
        for (int d = 0; d < 3; ++d) {
            raw[d] = g.raw[d];
            pad[d] = g.pad[d];
            origin[d] = g.origin[d];
            step[d] = g.step[d];
        }
    });
}

int cl_enumerate_integrals(const char* pattern, int n_inputs, int n_holes, int64_t* count,
                           int16_t* specs, int64_t capacity) {
    return cl::guarded([&] {
        if (!pattern || !count) cl::fail(CL_ERR_ARGUMENT, "null argument");
        cl::Pattern p(pattern, n_holes);
        auto list = cl::enumerate_integrals(p, n_inputs);
        *count = static_cast<int64_t>(list.size());
        if (specs) {
            if (capacity < *count) cl::fail(CL_ERR_ARGUMENT, "specs capacity %lld < %lld",
                                            (long long)capacity, (long long)*count);
            for (size_t i = 0; i < list.size(); ++i)
                for (int k = 0; k < 4; ++k) specs[4 * i + k] = list[i][k];
        }
    });
}

int cl_vertex_cover(int n_vertices, int64_t n_edges, const int32_t* edges, uint8_t* in_cover) {
    return cl::guarded([&] {
        if (n_vertices < 0 || n_edges < 0 || (n_edges && !edges) || !in_cover)
            cl::fail(CL_ERR_ARGUMENT, "invalid argument");
        std::vector<std::pair<int, int>> e;
        e.reserve(static_cast<size_t>(n_edges));
        for (int64_t i = 0; i < n_edges; ++i) {
            int a = edges[2 * i], b = edges[2 * i + 1];
            if (a < 0 || a >= n_vertices || b < 0 || b >= n_vertices)
                cl::fail(CL_ERR_ARGUMENT, "edge vertex out of range");
            e.push_back({a, b});
        }
        auto cover = cl::vertex_cover(n_vertices, e);
        std::memset(in_cover, 0, static_cast<size_t>(n_vertices));
        for (int v : cover) in_cover[v] = 1;
    });
}

int cl_plan(int n_inputs, int64_t n_int, const int16_t* spec, int32_t* steps) {
    return cl::guarded([&] {
        if (n_int < 0 || (n_int && (!spec || !steps))) cl::fail(CL_ERR_ARGUMENT, "invalid argument");
        std::vector<std::array<int16_t, 4>> specs(static_cast<size_t>(n_int));
        for (int64_t i = 0; i < n_int; ++i)
            for (int k = 0; k < 4; ++k) specs[i][k] = spec[4 * i + k];
        auto plan = cl::compute_plan(n_inputs, specs);
        for (size_t i = 0; i < plan.size(); ++i) {
            steps[5 * i + 0] = plan[i].id;
            steps[5 * i + 1] = plan[i].left.product;
            steps[5 * i + 2] = plan[i].left.conjugate;
            steps[5 * i + 3] = plan[i].right.product;
            steps[5 * i + 4] = plan[i].right.conjugate;
        }
    });
}

int cl_write_integrals(const char* out_prefix, int n_holes, int n_electrons, int64_t n_int, const int16_t* spec,
                       const double* values, int threads) {
    return cl::guarded([&] {
        if (!out_prefix || n_holes < 0 || n_electrons < 0 || n_int < 0 || (n_int && (!spec || !values)))
            cl::fail(CL_ERR_ARGUMENT, "invalid arguments");
        std::vector<int16_t> specs(spec, spec + 4 * n_int);
        try {
            clio::write_integrals(out_prefix, specs, values, n_holes, n_electrons, threads);
        } catch (const std::runtime_error& e) {
            cl::fail(CL_ERR_ARGUMENT, "%s", e.what());
        }
    });
}

}  // extern "C"
