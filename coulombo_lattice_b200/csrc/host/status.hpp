// Status codes and the thread-local error message behind cl_last_error().
#pragma once

#include <cstdarg>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "coulombo_lattice.h"

namespace cl {

// An error that carries one of the CL_ERR_* codes across the internal C++ layers; the C ABI
// wrappers catch it and turn it into a return code plus a message.
struct Error : std::runtime_error {
    int code;
    Error(int code, const std::string& msg) : std::runtime_error(msg), code(code) {}
};

[[noreturn]] void fail(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));

void set_last_error(const char* msg);
const char* last_error();

// Runs fn() and maps exceptions to status codes.
template <class F>
int guarded(F&& fn) {
    try {
        fn();
        set_last_error("");
        return CL_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return CL_ERR_MEMORY;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return CL_ERR_ARGUMENT;
    } catch (...) {
        set_last_error("unknown error");
        return CL_ERR_ARGUMENT;
    }
}

}  // namespace cl
