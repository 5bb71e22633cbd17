// Text inputs/outputs, option parser and phase timer of the drop-in binaries; see io.hpp.
#include "io.hpp"

#include <sys/time.h>

#include <algorithm>
#include <array>
#include <charconv>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <thread>
#include <unordered_map>

namespace clio {

void throwfr(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    int n = vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    throw std::runtime_error(n > 0 ? buf : "error");
}

namespace {

std::string read_file(const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throwfr("could not open file: %s", path.c_str());
    std::string data;
    if (std::fseek(f, 0, SEEK_END) == 0) {
        long sz = std::ftell(f);
        if (sz > 0) {
            data.resize((size_t)sz);
            std::fseek(f, 0, SEEK_SET);
            size_t got = std::fread(&data[0], 1, (size_t)sz, f);
            data.resize(got);
        }
    }
    std::fclose(f);
    return data;
}

// One number the way sscanf("%lf") reads it: skip blanks, optional sign, then a decimal
// or "inf"/"nan" literal.
bool parse_number(const char*& p, const char* end, double& v) {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\v' || *p == '\f')) ++p;
    if (p >= end) return false;
    bool neg = false;
    if (*p == '+' || *p == '-') {
        neg = (*p == '-');
        ++p;
        if (p >= end || *p == '+' || *p == '-') return false;
    }
    auto r = std::from_chars(p, end, v, std::chars_format::general);
    if (r.ec != std::errc() && r.ec != std::errc::result_out_of_range) return false;
    if (r.ptr == p) return false;
    p = r.ptr;
    if (neg) v = -v;
    return true;
}

}  // namespace

std::vector<double> load_atoms(const std::string& path) {
    std::string data = read_file(path);
    std::vector<double> out;
    const char* p = data.data();
    const char* end = p + data.size();
    while (p < end) {
        const char* nl = static_cast<const char*>(std::memchr(p, '\n', (size_t)(end - p)));
        const char* le = nl ? nl : end;
        const char* q = p;
        double x, y, z;
        if (!(parse_number(q, le, x) && parse_number(q, le, y) && parse_number(q, le, z))) break;
        out.push_back(x);
        out.push_back(y);
        out.push_back(z);
        if (!nl) break;
        p = nl + 1;
    }
    return out;
}

void load_state(const std::string& path, int64_t n_atoms, int n_orb, int skip_lines, int threads, double* dst) {
    std::string data = read_file(path);
    const char* base = data.data();
    const char* end = base + data.size();
    const char* p = base;
    for (int i = 0; i < skip_lines && p < end; ++i) {
        const char* nl = static_cast<const char*>(std::memchr(p, '\n', (size_t)(end - p)));
        p = nl ? nl + 1 : end;
    }
    const int64_t need = n_atoms * (int64_t)n_orb;
    // line starts, then parallel parsing of independent line ranges
    std::vector<const char*> starts;
    starts.reserve((size_t)need + 1);
    while ((int64_t)starts.size() < need && p < end) {
        starts.push_back(p);
        const char* nl = static_cast<const char*>(std::memchr(p, '\n', (size_t)(end - p)));
        p = nl ? nl + 1 : end;
    }
    if ((int64_t)starts.size() < need) throwfr("file is truncated: %s", path.c_str());
    starts.push_back(p);
    int nt = std::max(1, std::min(threads, 64));
    if (need < 100000) nt = 1;
    std::vector<int> bad(nt, 0);
    auto work = [&](int t) {
        const int64_t i0 = need * t / nt, i1 = need * (t + 1) / nt;
        for (int64_t i = i0; i < i1; ++i) {
            const char* q = starts[i];
            const char* le = static_cast<const char*>(std::memchr(q, '\n', (size_t)(end - q)));
            if (!le) le = end;
            double re, im;
            if (!(parse_number(q, le, re) && parse_number(q, le, im))) {
                bad[t] = 1;
                return;
            }
            dst[2 * i] = re;
            dst[2 * i + 1] = im;
        }
    };
    if (nt == 1) {
        work(0);
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < nt; ++t) pool.emplace_back(work, t);
        for (auto& th : pool) th.join();
    }
    for (int b : bad)
        if (b) throwfr("file is truncated: %s", path.c_str());
}

// ---------------------------------------------------------------------------------------
// Parser.cpp:35-99
// ---------------------------------------------------------------------------------------
bool ParseResults::has_value(const std::string& name, std::string& out) const {
    auto it = values.find(name);
    if (it == values.end()) return false;
    out = it->second;
    return true;
}

const std::string& ParseResults::get_value(const std::string& name) const {
    auto it = values.find(name);
    if (it == values.end()) throwfr("parameter '%s' not specified", name.c_str());
    return it->second;
}

ParseResults Parser::process(int argc, char** argv) const {
    ParseResults r;
    for (int i = 1; i < argc; ++i) {
        std::string s = argv[i];
        if (s.size() > 1 && s[0] == '-') {
            if (s[1] == '-') {
                auto eq = s.find('=', 2);
                if (eq != std::string::npos) {
                    std::string name = s.substr(2, eq - 2), value = s.substr(eq + 1);
                    if (values_.count(name))
                        r.values[name] = value;
                    else if (flags_.count(name))
                        throwfr("flag '%s' does not need a value", name.c_str());
                    else
                        throwfr("unknown value '%s'", name.c_str());
                } else {
                    std::string name = s.substr(2);
                    if (flags_.count(name))
                        r.flags.insert(name);
                    else if (values_.count(name))
                        throwfr("missing value for parameter '%s'", name.c_str());
                    else
                        throwfr("unknown flag '%s'", name.c_str());
                }
            } else {
                for (size_t k = 1; k < s.size(); ++k) {
                    auto it = short_.find(s[k]);
                    if (it == short_.end()) throwfr("unknown flag '%c'", s[k]);
                    r.flags.insert(it->second);
                }
            }
        } else {
            r.args.push_back(s);
        }
    }
    return r;
}

// ---------------------------------------------------------------------------------------
// Timer.cpp:11-77
// ---------------------------------------------------------------------------------------
static double now_s() {
    timeval tv;
    gettimeofday(&tv, nullptr);
    return tv.tv_sec + tv.tv_usec * 1e-6;
}

Timer::~Timer() { stop(); }

void Timer::stop() {
    if (open_) {
        std::fprintf(stderr, "(%.3f s)\n", now_s() - t0_);
        std::fflush(stderr);
        open_ = false;
    }
}

void Timer::start(const char* msg) {
    stop();
    std::fprintf(stderr, "%s... ", msg);
    std::fflush(stderr);
    open_ = true;
    t0_ = now_s();
}

// ---------------------------------------------------------------------------------------
// coulombo.cpp:213-262: one file per e/h class with values, rows in (ni, nj, nk, nl) order with
// the hole numbering reversed, "%2d %2d %2d %2d   %17.14f %17.14f\n".  The lines of a class are
// formatted in parallel chunks of (ni, nj) on the host threads and written in order; a class
// file is created only when it has a line, as the reference opens it at its first line.
// ---------------------------------------------------------------------------------------
void write_integrals(const std::string& out_prefix, const std::vector<int16_t>& specs, const double* values,
                     int n_holes, int n_electrons, int threads) {
    const size_t n_int = specs.size() / 4;
    const int n = n_holes + n_electrons;
    // spec -> integral index: a flat table while n^4 is small, else a hash map
    const unsigned long long n4 = (unsigned long long)n * n * n * n;
    const bool flat = n4 <= (1ull << 25);
    std::vector<int64_t> table(flat ? (size_t)n4 : 0, -1);
    std::unordered_map<unsigned long long, int64_t> hashed;
    const auto key_of = [n](int a, int b, int c, int d) {
        return (((unsigned long long)(a - 1) * n + (b - 1)) * n + (c - 1)) * n + (d - 1);
    };
    for (size_t i = 0; i < n_int; ++i) {
        const int16_t* sp = &specs[4 * i];
        for (int q = 0; q < 4; ++q)
            if (sp[q] < 1 || sp[q] > n) throwfr("integral index out of range");
        const unsigned long long k = key_of(sp[0], sp[1], sp[2], sp[3]);
        if (flat)
            table[k] = (int64_t)i;
        else
            hashed[k] = (int64_t)i;
    }
    const auto find = [&](unsigned long long k) -> int64_t {
        if (flat) return table[k];
        auto it = hashed.find(k);
        return it == hashed.end() ? -1 : it->second;
    };
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    char core[5];
    core[4] = 0;
    for (int ti = 0; ti < 2; ++ti)
        for (int tj = 0; tj < 2; ++tj)
            for (int tk = 0; tk < 2; ++tk)
                for (int tl = 0; tl < 2; ++tl) {
                    const int t[4] = {ti, tj, tk, tl};
                    int cnt[4];
                    for (int q = 0; q < 4; ++q) {
                        core[q] = t[q] ? 'e' : 'h';
                        cnt[q] = t[q] ? n_electrons : n_holes;
                    }
                    const long long units = (long long)cnt[0] * cnt[1];  // (ni, nj) pairs
                    if (units == 0 || cnt[2] == 0 || cnt[3] == 0) continue;
                    const int nt = (int)std::min<long long>(threads, units);
                    std::vector<std::string> bufs((size_t)nt);
                    const auto work = [&](int w) {
                        std::string& buf = bufs[(size_t)w];
                        char line[128];
                        for (long long u = units * w / nt; u < units * (w + 1) / nt; ++u) {
                            const int ni = (int)(u / cnt[1]) + 1, nj = (int)(u % cnt[1]) + 1;
                            for (int nk = 1; nk <= cnt[2]; ++nk)
                                for (int nl = 1; nl <= cnt[3]; ++nl) {
                                    const int idx[4] = {ni, nj, nk, nl};
                                    int sp[4];
                                    for (int q = 0; q < 4; ++q)
                                        sp[q] = t[q] ? n_holes + idx[q] : n_holes + 1 - idx[q];
                                    const int64_t i = find(key_of(sp[0], sp[1], sp[2], sp[3]));
                                    if (i < 0) continue;
                                    const int len = std::snprintf(line, sizeof line, "%2d %2d %2d %2d   %17.14f %17.14f\n",
                                                                  ni, nj, nk, nl, values[2 * i], values[2 * i + 1]);
                                    buf.append(line, (size_t)len);
                                }
                        }
                    };
                    if (nt == 1) {
                        work(0);
                    } else {
                        std::vector<std::thread> pool;
                        for (int w = 0; w < nt; ++w) pool.emplace_back(work, w);
                        for (auto& th : pool) th.join();
                    }
                    bool any = false;
                    for (const auto& b2 : bufs) any = any || !b2.empty();
                    if (!any) continue;
                    const std::string path = out_prefix + core + ".txt";
                    FILE* file = std::fopen(path.c_str(), "w");
                    if (!file) throwfr("cannot open file %s for writing", path.c_str());
                    for (const auto& b2 : bufs) std::fwrite(b2.data(), 1, b2.size(), file);
                    std::fclose(file);
                }
}

}  // namespace clio
