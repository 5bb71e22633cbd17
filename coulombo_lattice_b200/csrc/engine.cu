// Context, orchestration and the GPU half of the C ABI (include/coulombo_lattice.h).
#include <algorithm>
#include <array>
#include <memory>
#include <map>
#include <mutex>
#include <tuple>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include "coulombo_lattice.h"
#include "host/host_logic.hpp"
#include "host/status.hpp"
#include "kernels.cuh"
#include "passes.hpp"
#include "gram_dmma.cuh"
#include "gram_tc.cuh"
#include "sublattice.cuh"

using clk::cx;
using clk::FftPlan;

namespace {

// ---------------------------------------------------------------------------------------
// CUDA helpers
// ---------------------------------------------------------------------------------------
#define CL_CUDA(call)                                                                           \
    do {                                                                                        \
        cudaError_t err_ = (call);                                                              \
        if (err_ != cudaSuccess)                                                                \
            cl::fail(err_ == cudaErrorMemoryAllocation ? CL_ERR_MEMORY : CL_ERR_CUDA,           \
                     "CUDA error %s at %s:%d: %s", cudaGetErrorName(err_), __FILE__, __LINE__,  \
                     cudaGetErrorString(err_));                                                 \
    } while (0)

#define CL_LAUNCHED() CL_CUDA(cudaGetLastError())

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count) {
        if (count == n && p) return;
        release();
        if (count == 0) return;
        CL_CUDA(cudaMalloc(&p, count * sizeof(T)));
        n = count;
    }
    void upload(const T* host, size_t count, cudaStream_t s) {
        alloc(count);
        if (count) CL_CUDA(cudaMemcpyAsync(p, host, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
};

int device_count() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

void require_gpu() {
    if (device_count() == 0) cl::fail(CL_ERR_CUDA, "no CUDA device is available");
}

int grid_for(long long n, int threads = 256) {
    long long b = (n + threads - 1) / threads;
    return (int)std::max(1LL, std::min(b, 148LL * 32));
}

// ---------------------------------------------------------------------------------------
// FFT plans and host-built tables
// ---------------------------------------------------------------------------------------
bool smooth235(int n) {
    if (n < 1) return false;
    for (int p : {2, 3, 5})
        while (n % p == 0) n /= p;
    return n == 1;
}

FftPlan make_plan(int n) {
    FftPlan p{};
    p.n = n;
    int m = n;
    auto push = [&](int r) {
        if (p.nst >= 16) cl::fail(CL_ERR_UNSUPPORTED, "FFT length %d needs too many stages", n);
        p.radix[p.nst++] = r;
        m /= r;
    };
    // fewest shared-memory round trips: radix 16 first, then 8/4, a lone 2 joined with a
    // 3 (-> 6) or 5 (-> 10), a lone 4 with a 3 (-> 12), then 3s and 5s
    int twos = 0, threes = 0, fives = 0;
    for (; m % 2 == 0; m /= 2) ++twos;
    for (; m % 3 == 0; m /= 3) ++threes;
    for (; m % 5 == 0; m /= 5) ++fives;
    if (m != 1) cl::fail(CL_ERR_UNSUPPORTED, "FFT length %d is not a product of 2, 3 and 5", n);
    m = n;
    while (twos >= 4) { push(16); twos -= 4; }
    if (twos == 3) { push(8); twos = 0; }
    if (twos == 2) {
        if (threes > 0) { push(12); --threes; } else push(4);
        twos = 0;
    }
    if (twos == 1) {
        if (threes > 0) { push(6); --threes; }
        else if (fives > 0) { push(10); --fives; }
        else push(2);
        twos = 0;
    }
    while (threes-- > 0) push(3);
    while (fives-- > 0) push(5);
    int ns = 1;
    for (int s = 0; s < p.nst; ++s) {
        p.ns_magic[s] = clk::fdiv_magic(ns);
        ns *= p.radix[s];
    }
    return p;
}

// tw[t] = exp(-2 pi i t / n), built in extended precision and rounded once.
std::vector<cx<double>> twiddles64(int n) {
    std::vector<cx<double>> t(n);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int i = 0; i < n; ++i) {
        long double ang = -2.0L * pi * (long double)i / (long double)n;
        t[i].re = (double)std::cos(ang);
        t[i].im = (double)std::sin(ang);
    }
    return t;
}

// phase(i) = exp(i pi i / n) (CoulombCalculator.cpp:45-54).
std::vector<cx<double>> phases64(int n) {
    std::vector<cx<double>> t(n);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int i = 0; i < n; ++i) {
        long double ang = pi * (long double)i / (long double)n;
        t[i].re = (double)std::cos(ang);
        t[i].im = (double)std::sin(ang);
    }
    return t;
}

// Thomas-Fermi-Resta radius (Interaction.cpp:18-32, same Newton iteration and stop rule).
void thomas_fermi(double dielectric, double lattice, double* r_tf, double* q_tf) {
    const double eps = 1.0e-12;
    const double q = 2.0 / std::sqrt(M_PI) * std::cbrt(96.0 * M_PI * M_PI) / lattice;
    double x = std::sqrt(6.0 * (dielectric - 1.0)), dx;
    int guard = 0;
    do {
        double F = std::sinh(x) - dielectric * x;
        double dF = std::cosh(x) - dielectric;
        dx = (std::fabs(F) < eps) ? 0 : F / dF;
        x -= dx;
        if (++guard > 10000) cl::fail(CL_ERR_ARGUMENT, "Thomas-Fermi radius did not converge");
    } while (dx / q > eps);
    *q_tf = q;
    *r_tf = x / q;
}

struct Axis {
    FftPlan plan;
    DevBuf<cx<double>> tw64;
    DevBuf<cx<float>> tw32;
    DevBuf<cx<double>> phase;
};

// Per-launch geometry of the x passes and the y/z passes.
struct XTile {
    int rows, ld;
    size_t smem;
};
struct LTile {
    int W;
    size_t smem;
};

template <typename T>
XTile x_tile(int nx, int nrows) {
    const int elems = sizeof(T) == 4 ? 4096 : 2048;
    int rows = std::max(1, std::min(elems / std::max(nx, 1), 64));
    rows = std::min(rows, nrows);
    int ld = (rows % 2 == 0) ? rows + 1 : rows;
    XTile t{rows, ld, sizeof(cx<T>) * ((size_t)nx + 2ull * nx * ld)};
    return t;
}

template <typename T>
LTile l_tile(int n, bool with_khat) {
    int W = sizeof(T) == 4 ? 16 : 8;
    auto bytes = [&](int w) {
        return sizeof(cx<T>) * ((size_t)n + 2ull * n * w) + (with_khat ? sizeof(T) * (size_t)n * w : 0);
    };
    while (W > 1 && bytes(W) > 200 * 1024) W /= 2;
    return LTile{W, bytes(W)};
}

unsigned zgroups(long long zblocks, int cnt) { return clp::density_groups(zblocks, cnt); }

// Bytes of grids a chunk may hold so that consecutive passes meet in L2 (CL_L2_CHUNK_MB;
// off by default: measured on B200 it gave no gain at 96^3 over whole-request chunks).
size_t l2_chunk_bytes() {
    const char* e = std::getenv("CL_L2_CHUNK_MB");
    double mb = e ? std::atof(e) : 0.0;
    return (size_t)(std::max(0.0, mb) * 1024 * 1024);
}

template <typename K>
void ensure_smem(K kernel, size_t bytes) {
    if (bytes > 227 * 1024) cl::fail(CL_ERR_UNSUPPORTED, "tile needs %zu bytes of shared memory", bytes);
    CL_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

}  // namespace

// ---------------------------------------------------------------------------------------
// The context
// ---------------------------------------------------------------------------------------
// State of the sub-lattice decomposition (sublattice.cuh) for the loaded structure.
struct Sublattice {
    bool active = false;  // the request paths use the decomposition (a sub-lattice mode whose structure qualifies)
    bool zb = false;      // the classes are the zinc-blende set: compiled mixing table, canonical class order
    int m = 0, S = 0;
    int off[clk::kSlMaxClasses][3] = {};  // offset (x, y, z) of each class, in the order used on the GPU
    int sub[3] = {0, 0, 0};               // sub-grid points per axis, n/m
    int pad[3] = {0, 0, 0};               // transform length per axis, 2n/m
    int vn[3] = {0, 0, 0};                // virtual grid of the x and y passes: (pad x, pad y, S * sub z)
    long long vM = 0;
    clk::SlTable table;
    Axis ax[3];                           // plans and twiddles of the transform lengths
    DevBuf<cx<double>> H64, phxy64, phz64;
    DevBuf<cx<float>> H32, phxy32, phz32;
    long long tables_version = -1;        // kernel version the tables were built from
};

struct cl_ctx {
    int device = 0;
    int mode = CL_MODE_FP64_PLAIN;
    Sublattice sl;
    long long kernel_version = 0;  // bumped at every kernel build
    // grid the register passes run on (the real grid, or the sub-lattice virtual grid), the key
    // of the autotuner's choices
    int tune_dims[3] = {0, 0, 0};
    int tune_form = 0;  // 2 on the virtual grid
    int n[3] = {0, 0, 0};
    long long M = 0;
    double step[3] = {1, 1, 1};
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[5] = {};
    Axis ax[3];

    bool kernel_ready = false;
    DevBuf<double> ghat;
    DevBuf<double> khat64[8];
    DevBuf<float> khat32[8];

    // grid API ("every cell is an atom")
    DevBuf<int> grid_cell, grid_row_ptr;
    DevBuf<cx<double>> grid_rho, grid_V, grid_rho2;
    DevBuf<cx<float>> grid_rho32;  // the grid density in the FP32 form
    bool grid_prepared = false;

    // states
    int n_states = 0, n_holes = 0, n_orb = 0;
    long long n_atoms = 0, n_sorted = 0;
    DevBuf<cx<double>> coeff;
    DevBuf<int> cell_sorted, orig_sorted, row_ptr;
    DevBuf<cx<double>> coeff_stage;  // two states of caller coefficients, input atom order
    long long live_rows = 0;           // rows (y, z) holding at least one atom
    std::vector<long long> atom_slot;  // input atom -> sorted (deduplicated) slot
    std::vector<int64_t> cells_seen;   // the cells of the last load (an identical list skips the sort)
    cudaStream_t copy_stream = nullptr;  // coefficient uploads of cl_compute_states
    std::vector<cudaEvent_t> state_ev;   // one per state: its coefficients are on the device

    // work buffers, kept across requests (grown on demand)
    DevBuf<unsigned char> work;
    DevBuf<unsigned char> rounds;  // per-round values at the atoms of a chunk of densities
    DevBuf<cx<double>> req_rho, req_V;
    DevBuf<double> req_o4;
    DevBuf<int> req_ridx;
    DevBuf<float> tc_buf;  // TF32 hi/lo operands of the tensor-core Gram
    double timings[4] = {0, 0, 0, 0};

    // per-kernel profiling (events recorded around launches on `stream`)
    struct ProfEntry {
        int cls;
        cudaEvent_t a, b;
        double bytes;
    };
    bool profiling = false;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    std::vector<ProfEntry> prof_pending;
    // while a batch captures this context with profiling on: event pairs go to the batch
    std::vector<ProfEntry>* prof_sink = nullptr;
    std::vector<cudaEvent_t>* prof_owned = nullptr;
    double prof_ms[CL_NUM_KCLASS] = {};
    double prof_bytes[CL_NUM_KCLASS] = {};
    int64_t prof_launches[CL_NUM_KCLASS] = {};

    ~cl_ctx() {
        if (copy_stream) {
            cudaStreamSynchronize(copy_stream);
            for (auto& e : state_ev) cudaEventDestroy(e);
            cudaStreamDestroy(copy_stream);
        }
        if (stream) {
            cudaStreamSynchronize(stream);
            for (auto& e : ev)
                if (e) cudaEventDestroy(e);
            for (auto& e : ev_pool) cudaEventDestroy(e);
            cudaStreamDestroy(stream);
        }
    }
};

namespace {

// Precision of a form: the all-FP64 forms against the FP32-transform forms.
bool fp64_form(const cl_ctx* c) { return c->mode == CL_MODE_FP64_PLAIN || c->mode == CL_MODE_FP64_SUBLATTICE; }
bool sublattice_mode(const cl_ctx* c) {
    return c->mode == CL_MODE_FP64_SUBLATTICE || c->mode == CL_MODE_FP32_SUBLATTICE;
}

size_t free_device_bytes() {
    size_t fr = 0, tot = 0;
    CL_CUDA(cudaMemGetInfo(&fr, &tot));
    return fr;
}

cudaEvent_t prof_event(cl_ctx* c) {
    if (c->prof_owned) {  // captured into a graph: the event lives as long as the graph
        cudaEvent_t e;
        CL_CUDA(cudaEventCreate(&e));
        c->prof_owned->push_back(e);
        return e;
    }
    if (c->ev_used == c->ev_pool.size()) {
        cudaEvent_t e;
        CL_CUDA(cudaEventCreate(&e));
        c->ev_pool.push_back(e);
    }
    return c->ev_pool[c->ev_used++];
}

// Marks the start of a launch of class `cls`; returns the start event (or nullptr).
// Inside a capture an event must be recorded as an external event-record node, so that
// every replay of the graph records it.
void prof_record(cl_ctx* c, cudaEvent_t e) {
    if (c->prof_owned)
        CL_CUDA(cudaEventRecordWithFlags(e, c->stream, cudaEventRecordExternal));
    else
        CL_CUDA(cudaEventRecord(e, c->stream));
}

cudaEvent_t prof_begin(cl_ctx* c) {
    if (!c->profiling) return nullptr;
    cudaEvent_t a = prof_event(c);
    prof_record(c, a);
    return a;
}

void prof_end(cl_ctx* c, cudaEvent_t a, int cls, double bytes) {
    if (!a) return;
    cudaEvent_t b = prof_event(c);
    prof_record(c, b);
    (c->prof_sink ? *c->prof_sink : c->prof_pending).push_back({cls, a, b, bytes});
}

// After the stream has been synchronised: fold the pending pairs into the totals.
void prof_collect(cl_ctx* c) {
    for (const auto& e : c->prof_pending) {
        float ms = 0;
        CL_CUDA(cudaEventElapsedTime(&ms, e.a, e.b));
        c->prof_ms[e.cls] += ms;
        c->prof_bytes[e.cls] += e.bytes;
        c->prof_launches[e.cls] += 1;
    }
    c->prof_pending.clear();
    c->ev_used = 0;
}

void build_khat(cl_ctx* c) {
    const int nx = c->n[0], ny = c->n[1], nz = c->n[2];
    const double denom = (double)((unsigned long long)c->M * 8ull);
    for (int r = 0; r < 8; ++r) {
        const int kx = r & 1, ky = (r >> 1) & 1, kz = (r >> 2) & 1;
        if (fp64_form(c)) {
            c->khat64[r].alloc(c->M);
            clk::k_khat<double><<<grid_for(c->M), 256, 0, c->stream>>>(c->ghat.p, nx, ny, nz, kx, ky, kz, denom,
                                                                       c->khat64[r].p);
        } else {
            c->khat32[r].alloc(c->M);
            clk::k_khat<float><<<grid_for(c->M), 256, 0, c->stream>>>(c->ghat.p, nx, ny, nz, kx, ky, kz, denom,
                                                                      c->khat32[r].p);
        }
        CL_LAUNCHED();
    }
}

// 3D DCT-I of the octant held in c->ghat (three separable passes), then Khat per round.
void transform_kernel(cl_ctx* c) {
    const int n1[3] = {c->n[0] + 1, c->n[1] + 1, c->n[2] + 1};
    const long long total = (long long)n1[0] * n1[1] * n1[2];
    DevBuf<double> tmp;
    tmp.alloc(total);
    double* src = c->ghat.p;
    double* dst = tmp.p;
    long long inner = 1;
    for (int d = 0; d < 3; ++d) {
        const int L = n1[d];
        const int np = L - 1;
        std::vector<double> ct(2 * (size_t)np);
        const long double pi = 3.141592653589793238462643383279502884L;
        for (int t = 0; t < 2 * np; ++t) ct[t] = (double)std::cos(pi * (long double)t / (long double)np);
        DevBuf<double> dct;
        dct.upload(ct.data(), ct.size(), c->stream);
        const long long nlines = total / L;
        int nl = 16;
        while (nl > 1 && (size_t)(L * nl + 2 * np) * sizeof(double) > 160 * 1024) nl /= 2;
        const size_t smem = (size_t)(L * nl + 2 * np) * sizeof(double);
        ensure_smem(clk::k_dct1, smem);
        const long long blocks = (nlines + nl - 1) / nl;
        clk::k_dct1<<<(unsigned)blocks, 256, smem, c->stream>>>(src, dst, L, inner, nlines, nl, dct.p);
        CL_LAUNCHED();
        CL_CUDA(cudaStreamSynchronize(c->stream));  // dct table lifetime
        std::swap(src, dst);
        inner *= L;
    }
    if (src != c->ghat.p)
        CL_CUDA(cudaMemcpyAsync(c->ghat.p, src, total * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    build_khat(c);
    CL_CUDA(cudaStreamSynchronize(c->stream));
    c->kernel_ready = true;
    ++c->kernel_version;
}

// ---------------------------------------------------------------------------------------
// Autotuner of the register passes (passes.hpp).  For each pass of a grid shape and
// precision, every compiled variant (radix split of the line length x lines per block) is
// timed with CUDA events on the request's own buffers, and the fastest is kept for the rest of
// the process.  Tuning runs at the first eager request of a shape (never inside a graph
// capture); CL_AUTOTUNE=0 keeps the default variants.
// ---------------------------------------------------------------------------------------
struct TuneKey {
    int pass, fp32, nx, ny, nz;
    bool operator<(const TuneKey& o) const {
        return std::tie(pass, fp32, nx, ny, nz) < std::tie(o.pass, o.fp32, o.nx, o.ny, o.nz);
    }
};
struct TuneEntry {
    clp::Variant v;
    int candidates = 0;
    double ms = 0, ms_default = 0;  // per launch of the tuning sample
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneEntry> g_tune;

// Key of a pass on the grid the context's passes currently run on; fp32 carries the form: bit 0
// FP32 transforms, bit 1 the sub-lattice virtual grid.
TuneKey tune_key(const cl_ctx* c, int pass, bool fp32) {
    return TuneKey{pass, (fp32 ? 1 : 0) | c->tune_form, c->tune_dims[0], c->tune_dims[1], c->tune_dims[2]};
}
bool g_tune_loaded = false;

// CL_TUNE_FILE: choices persist across processes.  Lines "pass fp32 nx ny nz split half pad";
// the file is read once (before the first lookup) and every new choice is appended.
const char* tune_file() {
    const char* f = std::getenv("CL_TUNE_FILE");
    return (f && *f) ? f : nullptr;
}

void tune_load_locked() {  // g_tune_mu held
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char* path = tune_file();
    if (!path) return;
    FILE* fh = std::fopen(path, "r");
    if (!fh) return;
    TuneKey k{};
    TuneEntry e;
    while (std::fscanf(fh, "%d %d %d %d %d %d %d %d", &k.pass, &k.fp32, &k.nx, &k.ny, &k.nz, &e.v.split, &e.v.half,
                       &e.v.pad) == 8) {
        if (k.pass < 0 || k.pass >= clp::kNumPasses) continue;
        e.candidates = 0;  // loaded, not timed in this process
        g_tune[k] = e;
    }
    std::fclose(fh);
}

void tune_save(const TuneKey& k, const TuneEntry& e) {
    const char* path = tune_file();
    if (!path) return;
    if (FILE* fh = std::fopen(path, "a")) {
        std::fprintf(fh, "%d %d %d %d %d %d %d %d\n", k.pass, k.fp32, k.nx, k.ny, k.nz, e.v.split, e.v.half,
                     e.v.pad);
        std::fclose(fh);
    }
}

bool autotune_enabled() {
    const char* e = std::getenv("CL_AUTOTUNE");
    return !(e && e[0] == '0');
}

bool register_passes_enabled() { return !std::getenv("CL_NO_REGISTER_FFT"); }

clp::Variant tuned_variant(const cl_ctx* c, int pass, bool fp32) {
    if (const char* f = std::getenv("CL_TUNE_FORCE")) {  // "split,half[,pad]": one variant for every pass
        clp::Variant v;
        if (std::sscanf(f, "%d,%d,%d", &v.split, &v.half, &v.pad) >= 2) return v;
    }
    std::lock_guard<std::mutex> g(g_tune_mu);
    tune_load_locked();
    auto it = g_tune.find(tune_key(c, pass, fp32));
    return it == g_tune.end() ? clp::Variant{} : it->second.v;
}

bool stream_capturing(cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    CL_CUDA(cudaStreamIsCapturing(s, &st));
    return st != cudaStreamCaptureStatusNone;
}

// Times launch(variant) -- one warm-up and three timed launches per candidate -- and records
// the fastest variant of the pass.  Candidates: the split variants of the line length `len`,
// each with the default and (FP32) the half lines per block; the default is tried first.
template <typename F>
void tune_pass(cl_ctx* c, int pass, bool fp32, int len, F&& launch) {
    const TuneKey key = tune_key(c, pass, fp32);
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        tune_load_locked();
        if (g_tune.count(key)) return;
    }
    std::vector<clp::Variant> cands;
    const int pads = (fp32 && pass == clp::kXFwd) ? 2 : 1;
    for (int sv = 0; sv < clp::split_variants(len); ++sv)
        for (int h = 0; h < (fp32 ? 2 : 1); ++h)
            for (int pd = 0; pd < pads; ++pd) cands.push_back(clp::Variant{sv, h, pd});
    TuneEntry best;
    best.candidates = (int)cands.size();
    if (cands.size() >= 2) {
        cudaEvent_t a, b;
        CL_CUDA(cudaEventCreate(&a));
        CL_CUDA(cudaEventCreate(&b));
        double best_ms = 1e30;
        for (size_t i = 0; i < cands.size(); ++i) {
            launch(cands[i]);
            CL_LAUNCHED();
            CL_CUDA(cudaEventRecord(a, c->stream));
            for (int k = 0; k < 3; ++k) launch(cands[i]);
            CL_LAUNCHED();
            CL_CUDA(cudaEventRecord(b, c->stream));
            CL_CUDA(cudaEventSynchronize(b));
            float ms = 0;
            CL_CUDA(cudaEventElapsedTime(&ms, a, b));
            const double per = ms / 3.0;
            if (i == 0) best.ms_default = per;
            if (per < best_ms) {
                best_ms = per;
                best.v = cands[i];
            }
        }
        best.ms = best_ms;
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_tune[key] = best;
    tune_save(key, best);
}

// Fused plane passes against the separate passes they replace: times launch() like
// tune_pass and records split = 1 (use the fused kernel) when it beats sep_ms, the sum of the
// tuned separate passes' times on the same sample.
template <typename F>
void tune_plane(cl_ctx* c, int pass, bool fp32, double sep_ms, F&& launch) {
    const TuneKey key = tune_key(c, pass, fp32);
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        tune_load_locked();
        if (g_tune.count(key)) return;
    }
    cudaEvent_t a, b;
    CL_CUDA(cudaEventCreate(&a));
    CL_CUDA(cudaEventCreate(&b));
    launch();
    CL_LAUNCHED();
    CL_CUDA(cudaEventRecord(a, c->stream));
    for (int k = 0; k < 3; ++k) launch();
    CL_LAUNCHED();
    CL_CUDA(cudaEventRecord(b, c->stream));
    CL_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    CL_CUDA(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    TuneEntry e;
    e.candidates = 2;
    e.ms = ms / 3.0;
    e.ms_default = sep_ms;
    e.v.split = (sep_ms <= 0 || e.ms < sep_ms) ? 1 : 0;  // ms: the fused pass; ms_default: separate
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_tune[key] = e;
    tune_save(key, e);
}

double tuned_ms(const cl_ctx* c, int pass, bool fp32) {
    std::lock_guard<std::mutex> g(g_tune_mu);
    auto it = g_tune.find(tune_key(c, pass, fp32));
    return it == g_tune.end() ? 0.0 : it->second.ms;
}

// Whether the fused plane pass replaces the separate ones: CL_XY_PLANE=0/1 decides outright;
// with forced variants (CL_TUNE_FORCE) the separate passes run; otherwise the tuned choice,
// and the fused pass when nothing was tuned.
bool use_plane(const cl_ctx* c, int pass, bool fp32, bool supported) {
    if (!supported) return false;
    if (const char* e = std::getenv("CL_XY_PLANE")) return e[0] != '0';
    if (std::getenv("CL_TUNE_FORCE")) return false;
    std::lock_guard<std::mutex> g(g_tune_mu);
    tune_load_locked();
    auto it = g_tune.find(tune_key(c, pass, fp32));
    return it == g_tune.end() ? true : it->second.v.split != 0;
}

// Number of atoms listed by a row CSR (host-side copy kept with the CSR).
long long row_ptr_count(cl_ctx* c, const int* row_ptr) {
    return row_ptr == c->row_ptr.p ? c->n_sorted : c->M;
}

// One request's transforms: for every density p in [0, np) (rho rows), V[p] = the 8-round
// convolution (the rounds of round_mask) at the atoms of the row CSR.  For a chunk of densities,
// each round's inverse x pass writes its values at the atoms (type T) to a slot of the rounds
// buffer; k_round_sum then forms V in FP64.  buf holds `chunk` grids of type T.
template <typename T>
void run_rounds(cl_ctx* c, const cx<T>* rho, long long rho_stride, int np, const int* row_ptr,
                const int* cell, cx<double>* V, long long v_stride, int round_mask) {
    const int nx = c->n[0], ny = c->n[1], nz = c->n[2];
    const int nrows = ny * nz;
    const long long nxy = (long long)nx * ny;
    const size_t grid_bytes = sizeof(cx<T>) * (size_t)c->M;
    for (int d = 0; d < 3; ++d) c->tune_dims[d] = c->n[d];
    c->tune_form = 0;
    // Densities per chunk.  When a few grids fit in L2, chunks are sized so that the passes of
    // one round hand their output to the next pass through L2; otherwise chunks are as large
    // as 60% of the free memory allows (fewer, larger launches and Khat reuse in the z pass).
    const long long n_at = row_ptr_count(c, row_ptr);
    const int n_rounds = __builtin_popcount(round_mask & 0xFF);
    if (n_rounds == 0) {  // no round of this share (a split over more ranks than rounds)
        CL_CUDA(cudaMemset2DAsync(V, sizeof(cx<double>) * v_stride, 0, sizeof(cx<double>) * n_at, np, c->stream));
        return;
    }
    const size_t round_bytes = sizeof(cx<T>) * (size_t)n_at * n_rounds;  // per density
    const size_t l2_budget = l2_chunk_bytes();
    size_t budget = (size_t)(0.6 * (double)(free_device_bytes() + c->work.n + c->rounds.n));
    size_t by_mem = std::max<size_t>(1, budget / (grid_bytes + round_bytes));
    size_t by_l2 = l2_budget / grid_bytes;
    int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)np, by_l2 >= 2 ? by_l2 : by_mem));
    c->work.alloc(std::max(c->work.n, (size_t)chunk * grid_bytes));
    c->rounds.alloc(std::max(c->rounds.n, (size_t)chunk * round_bytes));
    cx<T>* buf = reinterpret_cast<cx<T>*>(c->work.p);
    cx<T>* tr = reinterpret_cast<cx<T>*>(c->rounds.p);
    const long long tr_slot = (long long)chunk * n_at;  // elements per round slot

    const Axis& X = c->ax[0];
    const Axis& Y = c->ax[1];
    const Axis& Z = c->ax[2];
    const cx<T>* twx = sizeof(T) == 4 ? (const cx<T>*)X.tw32.p : (const cx<T>*)X.tw64.p;
    const cx<T>* twy = sizeof(T) == 4 ? (const cx<T>*)Y.tw32.p : (const cx<T>*)Y.tw64.p;
    const cx<T>* twz = sizeof(T) == 4 ? (const cx<T>*)Z.tw32.p : (const cx<T>*)Z.tw64.p;

    const XTile xt = x_tile<T>(nx, nrows);
    const LTile yt = l_tile<T>(ny, false);
    const LTile zt = l_tile<T>(nz, true);
    ensure_smem(clk::k_xfwd<T>, xt.smem);
    ensure_smem(clk::k_xinv<T>, xt.smem);
    ensure_smem(clk::k_ypass<-1, T>, yt.smem);
    ensure_smem(clk::k_ypass<+1, T>, yt.smem);
    ensure_smem(clk::k_zpass<T>, zt.smem);
    const int xblocks = (nrows + xt.rows - 1) / xt.rows;
    const int ychunks = (nx + yt.W - 1) / yt.W;
    const long long zblocks = (nxy + zt.W - 1) / zt.W;
    // Rows without atoms are skipped (not stored / not loaded) when the x and y passes are both
    // the register ones, which agree on it; CL_NO_ROW_SKIP turns it off.
    const bool reg_x = register_passes_enabled() && clp::split_variants(nx) > 0;
    const bool reg_y = register_passes_enabled() && clp::split_variants(ny) > 0;
    const bool reg_z = register_passes_enabled() && clp::split_variants(nz) > 0;
    const int skip_empty = (reg_x && reg_y && !std::getenv("CL_NO_ROW_SKIP")) ? 1 : 0;
    const bool fp32 = sizeof(T) == 4;
    const bool plane_ok = reg_x && reg_y && clp::plane_supported(fp32, nx, ny);

    // Autotuning at the first eager request of this shape: the variants run on the first
    // densities of the request (about 512 MB of grids) in the work and rounds buffers, which
    // the request's own passes overwrite afterwards.
    if (autotune_enabled() && !std::getenv("CL_TUNE_FORCE") && np > 0 && !stream_capturing(c->stream)) {
        const int cnt_t = (int)std::max<size_t>(1, std::min<size_t>((size_t)chunk, (512ull << 20) / grid_bytes));
        const clk::RoundPhase rp0{c->ax[0].phase.p, c->ax[1].phase.p, c->ax[2].phase.p, 0, 0, 0};
        const T* kh0 = sizeof(T) == 4 ? (const T*)c->khat32[0].p : (const T*)c->khat64[0].p;
        const int* rp_skip = skip_empty ? row_ptr : nullptr;
        if (reg_x)
            tune_pass(c, clp::kXFwd, fp32, nx, [&](clp::Variant v) {
                clp::xfwd<T>(c->stream, v, rho, rho_stride, row_ptr, cell, buf, c->M, twx, rp0, nx, ny, nrows, cnt_t,
                             skip_empty);
            });
        if (reg_y) {
            tune_pass(c, clp::kYFwd, fp32, ny, [&](clp::Variant v) {
                clp::ycol<-1, T>(c->stream, v, buf, c->M, twy, nx, ny, nz, cnt_t, rp_skip);
            });
            tune_pass(c, clp::kYInv, fp32, ny, [&](clp::Variant v) {
                clp::ycol<+1, T>(c->stream, v, buf, c->M, twy, nx, ny, nz, cnt_t, rp_skip);
            });
        }
        if (reg_z)
            tune_pass(c, clp::kZConv, fp32, nz, [&](clp::Variant v) {
                clp::zconv<T>(c->stream, v, buf, c->M, twz, kh0, nxy, nz, cnt_t);
            });
        if (reg_x)
            tune_pass(c, clp::kXInv, fp32, nx, [&](clp::Variant v) {
                clp::xinv<T>(c->stream, v, buf, c->M, twx, row_ptr, cell, tr, n_at, nx, nrows, cnt_t);
            });
        if (plane_ok && !std::getenv("CL_XY_PLANE")) {
            tune_plane(c, clp::kXYFwd, fp32, tuned_ms(c, clp::kXFwd, fp32) + tuned_ms(c, clp::kYFwd, fp32), [&] {
                clp::xyfwd<T>(c->stream, rho, rho_stride, row_ptr, cell, buf, c->M, twx, rp0, nx, ny, nz, cnt_t);
            });
            tune_plane(c, clp::kXYInv, fp32, tuned_ms(c, clp::kYInv, fp32) + tuned_ms(c, clp::kXInv, fp32), [&] {
                clp::xyinv<T>(c->stream, buf, c->M, twx, row_ptr, cell, tr, n_at, nx, ny, nz, cnt_t);
            });
        }
    }
    const bool xy_fwd = use_plane(c, clp::kXYFwd, fp32, plane_ok);
    const bool xy_inv = use_plane(c, clp::kXYInv, fp32, plane_ok);
    const clp::Variant v_xf = tuned_variant(c, clp::kXFwd, fp32), v_yf = tuned_variant(c, clp::kYFwd, fp32),
                       v_z = tuned_variant(c, clp::kZConv, fp32), v_yi = tuned_variant(c, clp::kYInv, fp32),
                       v_xi = tuned_variant(c, clp::kXInv, fp32);

    // algorithmic bytes per density of each pass (minimum HBM traffic of its work); with
    // skipped rows only the live fraction of a row-side sweep counts
    const double gbytes = (double)grid_bytes;
    const double atoms = (double)(row_ptr_count(c, row_ptr));
    const double live = (skip_empty && row_ptr == c->row_ptr.p) ? (double)c->live_rows / nrows : 1.0;
    const double row_side = (row_ptr == c->row_ptr.p) ? (double)c->live_rows / nrows : 1.0;
    for (int p0 = 0; p0 < np; p0 += chunk) {
        const int cnt = std::min(chunk, np - p0);
        const cx<T>* rho_c = rho + (long long)p0 * rho_stride;
        cx<double>* V_c = V + (long long)p0 * v_stride;
        int slot = 0;
        for (int r = 0; r < 8; ++r) {
            if (!((round_mask >> r) & 1)) continue;
            cx<T>* tr_r = tr + slot++ * tr_slot;
            clk::RoundPhase rp{c->ax[0].phase.p, c->ax[1].phase.p, c->ax[2].phase.p, r & 1, (r >> 1) & 1,
                               (r >> 2) & 1};
            const T* kh = sizeof(T) == 4 ? (const T*)c->khat32[r].p : (const T*)c->khat64[r].p;
            cudaEvent_t e = prof_begin(c);
            if (xy_fwd) {
                clp::xyfwd<T>(c->stream, rho_c, rho_stride, row_ptr, cell, buf, c->M, twx, rp, nx, ny, nz, cnt);
            } else if (!(reg_x && clp::xfwd<T>(c->stream, v_xf, rho_c, rho_stride, row_ptr, cell, buf, c->M, twx,
                                                rp, nx, ny, nrows, cnt, skip_empty))) {
                clk::k_xfwd<T><<<xblocks, 256, xt.smem, c->stream>>>(rho_c, rho_stride, row_ptr, cell, buf, c->M,
                                                                     X.plan, twx, rp, nx, ny, nrows, xt.rows, xt.ld,
                                                                     cnt);
            }
            CL_LAUNCHED();
            prof_end(c, e, CL_KCLASS_XFWD,
                     cnt * (atoms * (double)sizeof(cx<T>) + (xy_fwd ? 1.0 : live) * gbytes) + atoms * 4.0);
            if (!xy_fwd) {
                e = prof_begin(c);
                if (!(reg_y &&
                      clp::ycol<-1, T>(c->stream, v_yf, buf, c->M, twy, nx, ny, nz, cnt, skip_empty ? row_ptr : nullptr)))
                    clk::k_ypass<-1, T><<<dim3(ychunks * nz, cnt), 256, yt.smem, c->stream>>>(buf, c->M, Y.plan, twy,
                                                                                              nx, ny, yt.W, ychunks);
                CL_LAUNCHED();
                prof_end(c, e, CL_KCLASS_YPASS, cnt * (1.0 + live) * gbytes);
            }
            e = prof_begin(c);
            if (!(reg_z && clp::zconv<T>(c->stream, v_z, buf, c->M, twz, kh, nxy, nz, cnt)))
                clk::k_zpass<T><<<dim3((unsigned)zblocks, zgroups(zblocks, cnt)), 256, zt.smem, c->stream>>>(
                    buf, c->M, Z.plan, twz, kh, nxy, nz, zt.W, cnt, 0);
            CL_LAUNCHED();
            prof_end(c, e, CL_KCLASS_ZPASS, cnt * 2.0 * gbytes + (double)c->M * sizeof(T));
            if (!xy_inv) {
                e = prof_begin(c);
                if (!(reg_y &&
                      clp::ycol<+1, T>(c->stream, v_yi, buf, c->M, twy, nx, ny, nz, cnt, skip_empty ? row_ptr : nullptr)))
                    clk::k_ypass<+1, T><<<dim3(ychunks * nz, cnt), 256, yt.smem, c->stream>>>(buf, c->M, Y.plan, twy,
                                                                                              nx, ny, yt.W, ychunks);
                CL_LAUNCHED();
                prof_end(c, e, CL_KCLASS_YPASS, cnt * (1.0 + live) * gbytes);
            }
            e = prof_begin(c);
            if (xy_inv) {
                clp::xyinv<T>(c->stream, buf, c->M, twx, row_ptr, cell, tr_r, n_at, nx, ny, nz, cnt);
            } else if (!(reg_x && clp::xinv<T>(c->stream, v_xi, buf, c->M, twx, row_ptr, cell, tr_r, n_at, nx, nrows,
                                                cnt))) {
                clk::k_xinv<T><<<xblocks, 256, xt.smem, c->stream>>>(buf, c->M, X.plan, twx, row_ptr, cell, tr_r,
                                                                     n_at, nx, nrows, xt.rows, xt.ld, cnt);
            }
            CL_LAUNCHED();
            prof_end(c, e, CL_KCLASS_XINV,
                     cnt * ((xy_inv ? 1.0 : row_side) * gbytes + atoms * (double)sizeof(cx<T>)) + atoms * 4.0);
        }
        if (n_rounds > 0) {
            const clk::RoundPhase base{c->ax[0].phase.p, c->ax[1].phase.p, c->ax[2].phase.p, 0, 0, 0};
            const long long blocks = std::min<long long>((n_at + 255) / 256, 148LL * 16);
            cudaEvent_t e = prof_begin(c);
            clk::k_round_sum<T><<<dim3((unsigned)blocks, zgroups(blocks, cnt)), 256, 0, c->stream>>>(
                tr, tr_slot, n_at, round_mask & 0xFF, base, cell, nx, ny, n_at, V_c, v_stride, cnt);
            CL_LAUNCHED();
            prof_end(c, e, CL_KCLASS_ROUND_SUM,
                     cnt * atoms * (n_rounds * (double)sizeof(cx<T>) + 16.0) + atoms * 4.0);
        }
    }
}

// Pair densities are complex128 in the plain form and complex64 in the FP32 form (rounded
// once from their FP64 sums); buffers are addressed in elements of the form's type.
size_t rho_bytes(const cl_ctx* c) { return fp64_form(c) ? sizeof(cx<double>) : sizeof(cx<float>); }
void* rho_at(const cl_ctx* c, void* base, long long elems) {
    return static_cast<unsigned char*>(base) + elems * (long long)rho_bytes(c);
}

void run_rounds_mode(cl_ctx* c, const void* rho, long long rho_stride, int np, const int* row_ptr, const int* cell,
                     cx<double>* V, long long v_stride, int round_mask = 0xFF) {
    if (fp64_form(c))
        run_rounds<double>(c, static_cast<const cx<double>*>(rho), rho_stride, np, row_ptr, cell, V, v_stride,
                           round_mask);
    else
        run_rounds<float>(c, static_cast<const cx<float>*>(rho), rho_stride, np, row_ptr, cell, V, v_stride,
                          round_mask);
}


// ---------------------------------------------------------------------------------------
// Sub-lattice decomposition (sublattice.cuh)
// ---------------------------------------------------------------------------------------

// Plans and twiddles of the transform lengths, the class kernels H (from the kernel spectrum in
// c->ghat) and the class phases, built once per kernel and class set.  Not during a capture.
void ensure_sl_tables(cl_ctx* c) {
    Sublattice& sl = c->sl;
    if (sl.tables_version == c->kernel_version) return;
    if (stream_capturing(c->stream))
        cl::fail(CL_ERR_STATE, "the sub-lattice tables must be built by an eager call before a capture");
    const bool fp32 = !fp64_form(c);
    for (int d = 0; d < 3; ++d) {
        Axis& A = sl.ax[d];
        A.plan = make_plan(sl.pad[d]);
        auto t64 = twiddles64(sl.pad[d]);
        std::vector<cx<float>> t32(t64.size());
        for (size_t i = 0; i < t64.size(); ++i) t32[i] = cx<float>{(float)t64[i].re, (float)t64[i].im};
        A.tw64.upload(t64.data(), t64.size(), c->stream);
        A.tw32.upload(t32.data(), t32.size(), c->stream);
    }
    const int px = sl.pad[0], py = sl.pad[1], pz = sl.pad[2];
    const long long nxy = (long long)px * py, nq = nxy * pz;
    // class kernels H_r(q): the residue representatives and the m-th roots of unity
    clk::SlRes res{};
    res.nh = sl.table.nh;
    res.m = sl.m;
    for (int h = 0; h < res.nh; ++h)
        for (int d = 0; d < 3; ++d) res.rep[h][d] = sl.table.rep[h][d];
    for (int e = 0; e < 4; ++e) {  // exact: m is 2 or 4
        const int q = (sl.m == 4) ? e : 2 * e;  // quarter turns
        static const double cq[4] = {1.0, 0.0, -1.0, 0.0}, sq[4] = {0.0, 1.0, 0.0, -1.0};
        res.wc[e] = cq[q & 3];
        res.ws[e] = sq[q & 3];
    }
    const double denom = (double)((unsigned long long)c->M * 8ull);
    const int blocks = grid_for(nq);
    if (sl.zb) {
        // raw class kernels in FP64, then their Walsh-Hadamard form (sublattice.cuh) rounded once
        DevBuf<cx<double>> raw;
        raw.alloc((size_t)res.nh * nq);
        clk::k_sl_build_h<double><<<blocks, 256, 0, c->stream>>>(c->ghat.p, c->n[0], c->n[1], c->n[2], px, py, pz,
                                                                 res, denom, raw.p);
        CL_LAUNCHED();
        clk::SlWht w{};
        for (int k = 0; k < 8; ++k) {
            w.src[k] = sl.table.h[k * clk::kSlMaxClasses];  // (class k, class 0): alpha_k, then beta_k
            w.cj[k] = sl.table.cj[k * clk::kSlMaxClasses];
        }
        if (fp32) {
            sl.H32.alloc((size_t)8 * nq);
            clk::k_sl_zb_wht<float><<<blocks, 256, 0, c->stream>>>(raw.p, nq, w, sl.H32.p);
        } else {
            sl.H64.alloc((size_t)8 * nq);
            clk::k_sl_zb_wht<double><<<blocks, 256, 0, c->stream>>>(raw.p, nq, w, sl.H64.p);
        }
        CL_LAUNCHED();
        CL_CUDA(cudaStreamSynchronize(c->stream));  // raw goes out of scope
    } else if (fp32) {
        sl.H32.alloc((size_t)res.nh * nq);
        clk::k_sl_build_h<float><<<blocks, 256, 0, c->stream>>>(c->ghat.p, c->n[0], c->n[1], c->n[2], px, py, pz, res,
                                                                denom, sl.H32.p);
    } else {
        sl.H64.alloc((size_t)res.nh * nq);
        clk::k_sl_build_h<double><<<blocks, 256, 0, c->stream>>>(c->ghat.p, c->n[0], c->n[1], c->n[2], px, py, pz,
                                                                 res, denom, sl.H64.p);
    }
    CL_LAUNCHED();
    // phases: phxy[s][ky][kx] = exp(-i pi (kx bx/nx + ky by/ny)), phz[b][kz] = exp(-i pi kz b/nz) (b < m;
    // rows up to 4), in extended precision and rounded once
    const long double pi = 3.141592653589793238462643383279502884L;
    std::vector<cx<double>> phxy((size_t)sl.S * nxy), phz((size_t)4 * pz, cx<double>{0.0, 0.0});
    for (int s2 = 0; s2 < sl.S; ++s2)
        for (int ky = 0; ky < py; ++ky)
            for (int kx = 0; kx < px; ++kx) {
                const long double a = -pi * ((long double)kx * sl.off[s2][0] / c->n[0] +
                                             (long double)ky * sl.off[s2][1] / c->n[1]);
                phxy[(size_t)s2 * nxy + (size_t)ky * px + kx] = cx<double>{(double)std::cos(a), (double)std::sin(a)};
            }
    for (int b = 0; b < sl.m; ++b)
        for (int kz = 0; kz < pz; ++kz) {
            const long double a = -pi * (long double)kz * b / c->n[2];
            phz[(size_t)b * pz + kz] = cx<double>{(double)std::cos(a), (double)std::sin(a)};
        }
    if (fp32) {
        std::vector<cx<float>> f1(phxy.size()), f2(phz.size());
        for (size_t i = 0; i < phxy.size(); ++i) f1[i] = cx<float>{(float)phxy[i].re, (float)phxy[i].im};
        for (size_t i = 0; i < phz.size(); ++i) f2[i] = cx<float>{(float)phz[i].re, (float)phz[i].im};
        sl.phxy32.upload(f1.data(), f1.size(), c->stream);
        sl.phz32.upload(f2.data(), f2.size(), c->stream);
        CL_CUDA(cudaStreamSynchronize(c->stream));
    } else {
        sl.phxy64.upload(phxy.data(), phxy.size(), c->stream);
        sl.phz64.upload(phz.data(), phz.size(), c->stream);
        CL_CUDA(cudaStreamSynchronize(c->stream));
    }
    sl.tables_version = c->kernel_version;
}

// One request's transforms in the sub-lattice form: for every density p in [0, np), V[p] at the
// atoms (virtual-grid order).  Per chunk of densities: x and y forward passes on the virtual
// grid (fused plane pass where compiled and faster), the z pass with class mixing, the y and x
// inverse passes writing the values at the atoms; in the FP32 form they are widened to V.
template <typename T>
void run_sublattice(cl_ctx* c, const cx<T>* rho, long long rho_stride, int np, void* V_any, long long v_stride,
                    bool v32) {
    cx<double>* V = static_cast<cx<double>*>(V_any);
    ensure_sl_tables(c);
    const Sublattice& sl = c->sl;
    const int nx = sl.vn[0], ny = sl.vn[1], nz = sl.vn[2];
    const int nrows = ny * nz;
    const long long nxy = (long long)nx * ny;
    const long long vM = sl.vM;
    const size_t grid_bytes = sizeof(cx<T>) * (size_t)vM;
    const bool fp32 = sizeof(T) == 4;
    for (int d = 0; d < 3; ++d) c->tune_dims[d] = sl.vn[d];
    c->tune_form = 2;
    const int* row_ptr = c->row_ptr.p;
    const int* cell = c->cell_sorted.p;
    const long long n_at = c->n_sorted;
    // values at the atoms: straight into V in FP64, and in FP32 when the reductions read FP32
    // potentials (v32); otherwise through the rounds buffer, widened to V
    const bool via_tr = fp32 && !v32;
    const size_t at_bytes = via_tr ? sizeof(cx<T>) * (size_t)n_at : 0;
    size_t budget = (size_t)(0.6 * (double)(free_device_bytes() + c->work.n + c->rounds.n));
    int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)std::max(np, 1), budget / (grid_bytes + at_bytes)));
    c->work.alloc(std::max(c->work.n, (size_t)chunk * grid_bytes));
    if (via_tr) c->rounds.alloc(std::max(c->rounds.n, (size_t)chunk * at_bytes));
    cx<T>* buf = reinterpret_cast<cx<T>*>(c->work.p);
    cx<T>* tr = reinterpret_cast<cx<T>*>(c->rounds.p);
    const cx<T>* twx = fp32 ? (const cx<T>*)sl.ax[0].tw32.p : (const cx<T>*)sl.ax[0].tw64.p;
    const cx<T>* twy = fp32 ? (const cx<T>*)sl.ax[1].tw32.p : (const cx<T>*)sl.ax[1].tw64.p;
    const cx<T>* twz = fp32 ? (const cx<T>*)sl.ax[2].tw32.p : (const cx<T>*)sl.ax[2].tw64.p;
    const cx<T>* H = fp32 ? (const cx<T>*)sl.H32.p : (const cx<T>*)sl.H64.p;
    const cx<T>* phxy = fp32 ? (const cx<T>*)sl.phxy32.p : (const cx<T>*)sl.phxy64.p;
    const cx<T>* phz = fp32 ? (const cx<T>*)sl.phz32.p : (const cx<T>*)sl.phz64.p;
    clk::SlMix mix{};
    mix.S = sl.S;
    for (int s2 = 0; s2 < clk::kSlMaxClasses; ++s2) mix.offz[s2] = s2 < sl.S ? sl.off[s2][2] : 0;
    for (int i = 0; i < clk::kSlMaxClasses * clk::kSlMaxClasses; ++i) {
        mix.h[i] = sl.table.h[i];
        mix.cj[i] = sl.table.cj[i];
    }
    const XTile xt = x_tile<T>(nx, nrows);
    const LTile yt = l_tile<T>(ny, false);
    ensure_smem(clk::k_xfwd<T>, xt.smem);
    ensure_smem(clk::k_xinv<T>, xt.smem);
    ensure_smem(clk::k_ypass<-1, T>, yt.smem);
    ensure_smem(clk::k_ypass<+1, T>, yt.smem);
    const int xblocks = (nrows + xt.rows - 1) / xt.rows;
    const int ychunks = (nx + yt.W - 1) / yt.W;
    const bool reg_x = register_passes_enabled() && clp::split_variants(nx) > 0;
    const bool reg_y = register_passes_enabled() && clp::split_variants(ny) > 0;
    const int skip_empty = (reg_x && reg_y && !std::getenv("CL_NO_ROW_SKIP")) ? 1 : 0;
    const bool plane_ok = reg_x && reg_y && clp::plane_supported(fp32, nx, ny);
    // 128 x 128 FP32 class planes: the quadrant forward plane pass (two blocks an SM);
    // CL_NO_QPLANE=1 keeps the general one
    const bool qplane = clp::quadrant_supported(fp32, nx, ny) && !std::getenv("CL_NO_QPLANE");
    // no phase in any pass: the rounds' phase tables are never read with kappa = 0
    const clk::RoundPhase rp0{c->ax[0].phase.p, c->ax[1].phase.p, c->ax[2].phase.p, 0, 0, 0};
    cx<T>* out0 = via_tr ? tr : static_cast<cx<T>*>(V_any);
    const long long out_stride = via_tr ? n_at : v_stride;
    if (autotune_enabled() && !std::getenv("CL_TUNE_FORCE") && np > 0 && !stream_capturing(c->stream)) {
        const int cnt_t = (int)std::max<size_t>(1, std::min<size_t>((size_t)chunk, (512ull << 20) / grid_bytes));
        const int* rp_skip = skip_empty ? row_ptr : nullptr;
        if (reg_x)
            tune_pass(c, clp::kXFwd, fp32, nx, [&](clp::Variant v) {
                clp::xfwd<T>(c->stream, v, rho, rho_stride, row_ptr, cell, buf, vM, twx, rp0, nx, ny, nrows, cnt_t,
                             skip_empty);
            });
        if (reg_y) {
            tune_pass(c, clp::kYFwd, fp32, ny, [&](clp::Variant v) {
                clp::ycol<-1, T>(c->stream, v, buf, vM, twy, nx, ny, nz, cnt_t, rp_skip);
            });
            tune_pass(c, clp::kYInv, fp32, ny, [&](clp::Variant v) {
                clp::ycol<+1, T>(c->stream, v, buf, vM, twy, nx, ny, nz, cnt_t, rp_skip);
            });
        }
        if (reg_x)
            tune_pass(c, clp::kXInv, fp32, nx, [&](clp::Variant v) {
                clp::xinv<T>(c->stream, v, buf, vM, twx, row_ptr, cell, out0, out_stride, nx, nrows, cnt_t);
            });
        if (plane_ok && !std::getenv("CL_XY_PLANE")) {
            tune_plane(c, clp::kXYFwd, fp32, tuned_ms(c, clp::kXFwd, fp32) + tuned_ms(c, clp::kYFwd, fp32), [&] {
                clp::xyfwd<T>(c->stream, rho, rho_stride, row_ptr, cell, buf, vM, twx, rp0, nx, ny, nz, cnt_t);
            });
            tune_plane(c, clp::kXYInv, fp32, tuned_ms(c, clp::kYInv, fp32) + tuned_ms(c, clp::kXInv, fp32), [&] {
                clp::xyinv<T>(c->stream, buf, vM, twx, row_ptr, cell, out0, out_stride, nx, ny, nz, cnt_t);
            });
        }
    }
    const bool xy_fwd = use_plane(c, clp::kXYFwd, fp32, plane_ok);
    const bool xy_inv = use_plane(c, clp::kXYInv, fp32, plane_ok);
    const clp::Variant v_xf = tuned_variant(c, clp::kXFwd, fp32), v_yf = tuned_variant(c, clp::kYFwd, fp32),
                       v_yi = tuned_variant(c, clp::kYInv, fp32), v_xi = tuned_variant(c, clp::kXInv, fp32);
    const double gbytes = (double)grid_bytes;
    const double atoms = (double)n_at;
    const double live = skip_empty ? (double)c->live_rows / nrows : 1.0;
    const double row_side = (double)c->live_rows / nrows;
    const double h_bytes = (double)sl.table.nh * sl.pad[2] * nxy * sizeof(cx<T>);
    for (int p0 = 0; p0 < np; p0 += chunk) {
        const int cnt = std::min(chunk, np - p0);
        const cx<T>* rho_c = rho + (long long)p0 * rho_stride;
        cx<T>* out_c = via_tr ? tr : static_cast<cx<T>*>(V_any) + (long long)p0 * v_stride;
        cudaEvent_t e = prof_begin(c);
        if (qplane) {
            clp::qfwd(c->stream, reinterpret_cast<const cx<float>*>(rho_c), rho_stride, row_ptr, cell,
                      reinterpret_cast<cx<float>*>(buf), vM, reinterpret_cast<const cx<float>*>(twx), nz, cnt);
        } else if (xy_fwd) {
            clp::xyfwd<T>(c->stream, rho_c, rho_stride, row_ptr, cell, buf, vM, twx, rp0, nx, ny, nz, cnt);
        } else if (!(reg_x && clp::xfwd<T>(c->stream, v_xf, rho_c, rho_stride, row_ptr, cell, buf, vM, twx, rp0, nx,
                                            ny, nrows, cnt, skip_empty))) {
            clk::k_xfwd<T><<<xblocks, 256, xt.smem, c->stream>>>(rho_c, rho_stride, row_ptr, cell, buf, vM,
                                                                 sl.ax[0].plan, twx, rp0, nx, ny, nrows, xt.rows,
                                                                 xt.ld, cnt);
        }
        CL_LAUNCHED();
        prof_end(c, e, CL_KCLASS_XFWD,
                 cnt * (atoms * (double)sizeof(cx<T>) + (xy_fwd || qplane ? 1.0 : live) * gbytes) + atoms * 4.0);
        if (!xy_fwd && !qplane) {
            e = prof_begin(c);
            if (!(reg_y && clp::ycol<-1, T>(c->stream, v_yf, buf, vM, twy, nx, ny, nz, cnt,
                                             skip_empty ? row_ptr : nullptr)))
                clk::k_ypass<-1, T><<<dim3(ychunks * nz, cnt), 256, yt.smem, c->stream>>>(buf, vM, sl.ax[1].plan, twy,
                                                                                          nx, ny, yt.W, ychunks);
            CL_LAUNCHED();
            prof_end(c, e, CL_KCLASS_YPASS, cnt * (1.0 + live) * gbytes);
        }
        e = prof_begin(c);
        if (!clp::zmix<T>(c->stream, buf, vM, twz, H, phxy, phz, mix, sl.zb, nxy, sl.pad[2], cnt))
            cl::fail(CL_ERR_UNSUPPORTED, "no sub-lattice z pass for %d points", sl.pad[2]);
        CL_LAUNCHED();
        prof_end(c, e, CL_KCLASS_ZPASS, cnt * 2.0 * gbytes + h_bytes);
        if (!xy_inv) {
            e = prof_begin(c);
            if (!(reg_y && clp::ycol<+1, T>(c->stream, v_yi, buf, vM, twy, nx, ny, nz, cnt,
                                             skip_empty ? row_ptr : nullptr)))
                clk::k_ypass<+1, T><<<dim3(ychunks * nz, cnt), 256, yt.smem, c->stream>>>(buf, vM, sl.ax[1].plan, twy,
                                                                                          nx, ny, yt.W, ychunks);
            CL_LAUNCHED();
            prof_end(c, e, CL_KCLASS_YPASS, cnt * (1.0 + live) * gbytes);
        }
        e = prof_begin(c);
        if (xy_inv) {
            clp::xyinv<T>(c->stream, buf, vM, twx, row_ptr, cell, out_c, out_stride, nx, ny, nz, cnt);
        } else if (!(reg_x && clp::xinv<T>(c->stream, v_xi, buf, vM, twx, row_ptr, cell, out_c, out_stride, nx, nrows,
                                            cnt))) {
            clk::k_xinv<T><<<xblocks, 256, xt.smem, c->stream>>>(buf, vM, sl.ax[0].plan, twx, row_ptr, cell, out_c,
                                                                 out_stride, nx, nrows, xt.rows, xt.ld, cnt);
        }
        CL_LAUNCHED();
        prof_end(c, e, CL_KCLASS_XINV,
                 cnt * ((xy_inv ? 1.0 : row_side) * gbytes + atoms * (double)sizeof(cx<T>)) + atoms * 4.0);
        if (via_tr) {
            e = prof_begin(c);
            clk::k_sl_widen<T><<<dim3((unsigned)std::min<long long>((n_at + 255) / 256, 148LL * 8), cnt), 256, 0,
                                 c->stream>>>(tr, n_at, V + (long long)p0 * v_stride, v_stride, n_at);
            CL_LAUNCHED();
            prof_end(c, e, CL_KCLASS_ROUND_SUM, cnt * atoms * ((double)sizeof(cx<T>) + 16.0));
        }
    }
}

// The transforms of a request on the context's loaded atoms: the sub-lattice decomposition when
// it is in use, else the 8 rounds (of the rounds in round_mask).
// V is complex128 [np][v_stride], or complex64 when v32 (the FP32 sub-lattice form whose
// reductions read FP32 potentials, see v_fp32).
void run_transforms(cl_ctx* c, const void* rho, long long rho_stride, int np, void* V, long long v_stride, bool v32,
                    int round_mask = 0xFF) {
    if (c->sl.active) {
        if ((round_mask & 0xFF) != 0xFF)
            cl::fail(CL_ERR_UNSUPPORTED, "the sub-lattice form has no rounds to split (use an 8-round form)");
        if (fp64_form(c))
            run_sublattice<double>(c, static_cast<const cx<double>*>(rho), rho_stride, np, V, v_stride, false);
        else
            run_sublattice<float>(c, static_cast<const cx<float>*>(rho), rho_stride, np, V, v_stride, v32);
        return;
    }
    if (v32) cl::fail(CL_ERR_STATE, "the 8-round forms write FP64 potentials");
    run_rounds_mode(c, rho, rho_stride, np, c->row_ptr.p, c->cell_sorted.p, static_cast<cx<double>*>(V), v_stride,
                    round_mask);
}

// ---------------------------------------------------------------------------------------
// Tensor-core Gram (FP32 form): TF32 split pass + tcgen05 GEMM, see gram_tc.cuh.
// ---------------------------------------------------------------------------------------
bool use_tc_gram(const cl_ctx* c) { return !fp64_form(c) && !std::getenv("CL_NO_TC_GRAM"); }

// The FP32 sub-lattice form keeps the potentials at the atoms in FP32 (as the inverse passes
// produce them) when the tensor-core Gram reads them: its split rounds them to TF32 parts
// directly, with no FP64 copy in between.
bool v_fp32(const cl_ctx* c) { return c->sl.active && !fp64_form(c) && use_tc_gram(c); }
void* v_at(void* base, long long elems, bool v32) {
    return static_cast<unsigned char*>(base) + elems * (long long)(v32 ? sizeof(cx<float>) : sizeof(cx<double>));
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    if (!fn) cl::fail(CL_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    return fn;
}

// 3D FP32 tensor [2 parts][rows][k_pad] viewed in boxes of 32 atoms x box_rows rows x 1 part,
// 128-byte swizzle; rows of a box beyond `rows` are zero-filled by the copy (not read).
CUtensorMap tc_tensor_map(float* base, long long k_pad, long long rows, int box_rows) {
    CUtensorMap m;
    const cuuint64_t dims[3] = {(cuuint64_t)k_pad, (cuuint64_t)rows, 2};
    const cuuint64_t strides[2] = {(cuuint64_t)k_pad * sizeof(float), (cuuint64_t)(rows * k_pad) * sizeof(float)};
    const cuuint32_t box[3] = {(cuuint32_t)clk::tc::BK, (cuuint32_t)box_rows, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = tensor_map_encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, estr,
                                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) cl::fail(CL_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return m;
}

struct TcShape {
    int rowsA = 0, rowsB = 0;        // real operand rows: re and im of each density
    long long chunk = 0, k_pad = 0;  // atoms per operand chunk, chunk rounded up to a k-tile
};

long long tc_bytes_per_atom(int rowsA, int rowsB) { return 2LL * (rowsA + rowsB) * (long long)sizeof(float); }

TcShape tc_shape(const cl_ctx* c, int nl, int nr, long long n_atoms) {
    TcShape s;
    s.rowsA = 2 * nl;
    s.rowsB = 2 * nr;
    const long long per_atom = tc_bytes_per_atom(s.rowsA, s.rowsB);
    const long long fit = (long long)(c->tc_buf.n * sizeof(float)) / per_atom / clk::tc::BK * clk::tc::BK;
    const long long full = (n_atoms + clk::tc::BK - 1) / clk::tc::BK * clk::tc::BK;
    s.k_pad = std::min(full, fit);
    s.chunk = std::min(n_atoms, s.k_pad);
    return s;
}

// FP32 potentials and FP32 densities in one tile of each operand (at most 64 left and 64 right
// densities): the Gram splits its operands itself (k_gram_tc_fused) and needs no operand
// buffer.  With more tiles a block would convert its operands once per tile of the other
// side, and the split pass + k_gram_tc is used.  CL_TC_SPLIT=1 keeps the split pass
// everywhere; CL_TC_FUSED=1 takes the fused Gram at any tile count.
bool fused_gram(bool v_f32, bool rho_f32, int nl, int nr) {
    if (!v_f32 || !rho_f32 || std::getenv("CL_TC_SPLIT")) return false;
    if (std::getenv("CL_TC_FUSED")) return true;
    return 2 * nl <= clk::tc::BM && 2 * nr <= clk::tc::BN;
}

// Reductions of the FP32 forms over fewer than 65,536 atoms (CL_TC_MIN_ATOMS) are summed in
// FP64: the FP64 tensor-core Gram (k_gram_dmma) on FP32 potentials and densities, k_gram on FP64
// potentials.  The TF32x3 Gram's error is ~2^-23 of each product, random in sign, so relative to
// the sum of the terms' magnitudes it falls as 1/sqrt(atoms): at 2M atoms it is far below the
// FP32 gate even where the terms cancel 1000:1, while on a box of a hundred atoms it can reach
// the 1e-9 eV floor on integrals that small.  Below the threshold the FP64 Gram costs little.
long long tc_min_atoms() {
    const char* e = std::getenv("CL_TC_MIN_ATOMS");
    return e ? std::atoll(e) : 65536LL;
}
bool small_gram(const cl_ctx* c, long long n_atoms) {
    return !fp64_form(c) && n_atoms < tc_min_atoms() && !std::getenv("CL_TC_FUSED") && !std::getenv("CL_TC_SPLIT");
}

// Operand buffer for (nl, nr, n_atoms): whole atom range when it fits in a quarter of the free
// device memory (at most 8 GiB), else chunks of the atom range.  Called outside any capture.
void tc_reserve(cl_ctx* c, int nl, int nr, long long n_atoms, bool v_f32, bool rho_f32) {
    if (!use_tc_gram(c) || nl <= 0 || nr <= 0 || n_atoms <= 0 || fused_gram(v_f32, rho_f32, nl, nr) ||
        small_gram(c, n_atoms))
        return;
    const int rowsA = 2 * nl, rowsB = 2 * nr;
    const long long per_atom = tc_bytes_per_atom(rowsA, rowsB);
    const long long full = (n_atoms + clk::tc::BK - 1) / clk::tc::BK * clk::tc::BK;
    const long long have = (long long)(c->tc_buf.n * sizeof(float)) / per_atom;
    if (have >= full) return;
    const long long budget = std::min<long long>(8LL << 30, (long long)(free_device_bytes() / 4));
    long long atoms = std::min(full, std::max<long long>(budget / per_atom, 64LL * clk::tc::BK));
    if (const char* e = std::getenv("CL_TC_MAX_ATOMS"))  // cap per chunk (exercises the chunked path)
        atoms = std::min(atoms, std::max<long long>(clk::tc::BK, std::atoll(e)));
    atoms = atoms / clk::tc::BK * clk::tc::BK;
    if (atoms <= have) return;
    c->tc_buf.alloc((size_t)(atoms * per_atom / (long long)sizeof(float)));
}

// Atom splits of a Gram launch: whole waves of 148 blocks, each split at least 16 k-tiles long.
int gram_splits(int tiles, int kt_total) {
    int best_s = 1;
    double best = -1e30;
    const int s_max = std::max(1, std::min(256, kt_total / 16));
    for (int s = 1; s <= s_max; ++s) {
        const int per = (kt_total + s - 1) / s;
        const int used = (kt_total + per - 1) / per;
        const long long items = (long long)tiles * used;
        const long long waves = (items + 147) / 148;
        const double score = (double)items / (double)(waves * 148) - 0.01 * (double)waves;
        if (score > best) {
            best = score;
            best_s = used;
        }
    }
    return best_s;
}

// The FP64 tensor-core Gram on FP32 operands over the whole atom range (see k_gram_dmma).
void gram_dmma(cl_ctx* c, const cx<float>* V, long long v_stride, int nl, const cx<float>* rho, long long r_stride,
               const int* ridx_dev, int nr, long long n_atoms, double* out4_dev) {
    using namespace clk::dm;
    static std::once_flag once;
    std::call_once(once, [] {
        CL_CUDA(cudaFuncSetAttribute(k_gram_dmma, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    });
    const int tilesA = (2 * nl + TILE - 1) / TILE, tilesB = (2 * nr + TILE - 1) / TILE;
    const int nA4 = (std::min(TILE / 2, nl) + 3) & ~3, nB4 = (std::min(TILE / 2, nr) + 3) & ~3;
    GramArgs g{};
    g.V = reinterpret_cast<const float2*>(V);
    g.v_stride = v_stride;
    g.rho = reinterpret_cast<const float2*>(rho);
    g.r_stride = r_stride;
    g.ridx = ridx_dev;
    g.nl = nl;
    g.nr = nr;
    g.na = n_atoms;
    g.nd_max = nA4 + nB4;
    g.out4 = out4_dev;
    const int chunks = (int)std::min<long long>((n_atoms + KC - 1) / KC, 1LL << 30);
    // small boxes: enough atom splits to occupy every SM (at least 2 chunks a block)
    const int splits0 = std::max(gram_splits(tilesA * tilesB, chunks),
                                 std::min(chunks / 2, (148 + tilesA * tilesB - 1) / (tilesA * tilesB)));
    const long long per_chunks = (chunks + splits0 - 1) / splits0;
    g.atoms_per_split = per_chunks * KC;
    const int splits = (int)((n_atoms + g.atoms_per_split - 1) / g.atoms_per_split);
    const size_t smem = smem_bytes(g.nd_max);
    if (smem > 227 * 1024) cl::fail(CL_ERR_UNSUPPORTED, "FP64 Gram needs %zu bytes of shared memory", smem);
    cudaEvent_t e = prof_begin(c);
    k_gram_dmma<<<dim3(tilesA, tilesB, splits), THREADS, smem, c->stream>>>(g);
    CL_LAUNCHED();
    prof_end(c, e, CL_KCLASS_GRAM, (double)n_atoms * (nl + nr) * (double)sizeof(cx<float>));
}

// The fused Gram on FP32 operands over the whole atom range (see k_gram_tc_fused).
void gram_tc_fused(cl_ctx* c, const cx<float>* V, long long v_stride, int nl, const cx<float>* rho,
                   long long r_stride, const int* ridx_dev, int nr, long long n_atoms, double* out4_dev) {
    using namespace clk::tc;
    static std::once_flag once;
    std::call_once(once, [] {
        CL_CUDA(cudaFuncSetAttribute(k_gram_tc_fused<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
        CL_CUDA(cudaFuncSetAttribute(k_gram_tc_fused<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
        CL_CUDA(cudaFuncSetAttribute(k_gram_tc_fused<5>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
        CL_CUDA(cudaFuncSetAttribute(k_gram_tc_ws<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
        CL_CUDA(cudaFuncSetAttribute(k_gram_tc_ws<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
        CL_CUDA(cudaFuncSetAttribute(k_gram_tc_ws<5>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    });
    const int tilesA = (2 * nl + BM - 1) / BM, tilesB = (2 * nr + BN - 1) / BN;
    const int nA = std::min(BM / 2, nl), nB = std::min(BN / 2, nr);
    const int nb = std::max(16, (2 * nB + 15) / 16 * 16);
    FusedGram g{};
    g.V = reinterpret_cast<const float2*>(V);
    g.v_stride = v_stride;
    g.rho = reinterpret_cast<const float2*>(rho);
    g.r_stride = r_stride;
    g.ridx = ridx_dev;
    g.nl = nl;
    g.nr = nr;
    g.na = n_atoms;
    g.out4 = out4_dev;
    g.kt_total = (int)((n_atoms + BK - 1) / BK);
    g.stage_bytes = (uint32_t)(2 * BM * 128 + 2 * nb * 128);
    g.raw_slot_bytes = (uint32_t)((nA + nB) * BK * 8);
    // CL_TC_COPY8=1: 8-byte copies even where the rows allow 16 (zinc-blende boxes always do)
    g.aligned16 = (reinterpret_cast<uintptr_t>(V) % 16 == 0 && reinterpret_cast<uintptr_t>(rho) % 16 == 0 &&
                   v_stride % 2 == 0 && r_stride % 2 == 0 && !std::getenv("CL_TC_COPY8"))
                      ? 1
                      : 0;
    const int splits0 = gram_splits(tilesA * tilesB, g.kt_total);
    g.kt_per = (g.kt_total + splits0 - 1) / splits0;
    const int splits = (g.kt_total + g.kt_per - 1) / g.kt_per;
    // the deepest copy ring that fits: 5 k-tiles ahead (6 slots) at the 2.1M-atom box's 72 densities
    const size_t smem5 = fused_smem_bytes(g.stage_bytes, g.raw_slot_bytes, 5);
    const size_t smem3 = fused_smem_bytes(g.stage_bytes, g.raw_slot_bytes, 3);
    const size_t smem2 = fused_smem_bytes(g.stage_bytes, g.raw_slot_bytes, 2);
    if (smem2 > 227 * 1024) cl::fail(CL_ERR_UNSUPPORTED, "fused Gram needs %zu bytes of shared memory", smem2);
    cudaEvent_t e = prof_begin(c);
    const dim3 grid(tilesA, tilesB, splits);
    // up to 40 right densities a block (N <= 80): the warp-specialised kernel; CL_TC_NO_WS=1
    // keeps the kernel whose warps take every role in turn
    const bool ws = nb <= WS_MAX_NB && !std::getenv("CL_TC_NO_WS");
    const size_t ws5 = ws_smem_bytes(g.stage_bytes, g.raw_slot_bytes, 5);
    const size_t ws3 = ws_smem_bytes(g.stage_bytes, g.raw_slot_bytes, 3);
    const size_t ws2 = ws_smem_bytes(g.stage_bytes, g.raw_slot_bytes, 2);
    if (ws && ws2 > 227 * 1024) cl::fail(CL_ERR_UNSUPPORTED, "fused Gram needs %zu bytes of shared memory", ws2);
    if (ws && ws5 <= 227 * 1024)
        k_gram_tc_ws<5><<<grid, WS_THREADS, ws5, c->stream>>>(g);
    else if (ws && ws3 <= 227 * 1024)
        k_gram_tc_ws<3><<<grid, WS_THREADS, ws3, c->stream>>>(g);
    else if (ws)
        k_gram_tc_ws<2><<<grid, WS_THREADS, ws2, c->stream>>>(g);
    else if (smem5 <= 227 * 1024)
        k_gram_tc_fused<5><<<grid, FUSED_THREADS, smem5, c->stream>>>(g);
    else if (smem3 <= 227 * 1024)
        k_gram_tc_fused<3><<<grid, FUSED_THREADS, smem3, c->stream>>>(g);
    else
        k_gram_tc_fused<2><<<grid, FUSED_THREADS, smem2, c->stream>>>(g);
    CL_LAUNCHED();
    prof_end(c, e, CL_KCLASS_GRAM, (double)n_atoms * (nl + nr) * (double)sizeof(cx<float>));
}

// out4[l][r] += {sum ac, bd, ad, bc} (out4 zeroed by the caller, error slot included).
void gram_tc(cl_ctx* c, const void* V, bool v_f32, long long v_stride, int nl, const void* rho, bool rho_f32,
             long long r_stride, const int* ridx_dev, int nr, long long n_atoms, double* out4_dev) {
    using namespace clk::tc;
    if (fused_gram(v_f32, rho_f32, nl, nr)) {
        gram_tc_fused(c, static_cast<const cx<float>*>(V), v_stride, nl, static_cast<const cx<float>*>(rho), r_stride,
                      ridx_dev, nr, n_atoms, out4_dev);
        return;
    }
    const TcShape sh = tc_shape(c, nl, nr, n_atoms);
    if (sh.k_pad < BK) cl::fail(CL_ERR_STATE, "tensor-core Gram operands not reserved");
    static bool smem_set = false;
    if (!smem_set) {
        ensure_smem(clk::tc::k_gram_tc, SMEM_BYTES);
        smem_set = true;
    }
    float* A = c->tc_buf.p;
    float* B = A + 2LL * sh.rowsA * sh.k_pad;
    const CUtensorMap mapA = tc_tensor_map(A, sh.k_pad, sh.rowsA, BM);
    const CUtensorMap mapB = tc_tensor_map(B, sh.k_pad, sh.rowsB, BN);
    const int tilesA = (sh.rowsA + BM - 1) / BM, tilesB = (sh.rowsB + BN - 1) / BN;
    const int tiles = tilesA * tilesB;
    for (long long a0 = 0; a0 < n_atoms; a0 += sh.chunk) {
        const long long na = std::min(sh.chunk, n_atoms - a0);
        const long long kp = (na + BK - 1) / BK * BK;  // k-tiles that hold atoms of this chunk
        const int kt_total = (int)(kp / BK);
        cudaEvent_t e0 = prof_begin(c);
        const int xblocks = (int)std::min<long long>((kp + 255) / 256, 64);
        if (v_f32)
            clk::tc::k_tf32_split<float><<<dim3(xblocks, nl), 256, 0, c->stream>>>(
                static_cast<const cx<float>*>(V), v_stride, nullptr, nl, a0, na, sh.k_pad, A);
        else
            clk::tc::k_tf32_split<double><<<dim3(xblocks, nl), 256, 0, c->stream>>>(
                static_cast<const cx<double>*>(V), v_stride, nullptr, nl, a0, na, sh.k_pad, A);
        CL_LAUNCHED();
        if (rho_f32)
            clk::tc::k_tf32_split<float><<<dim3(xblocks, nr), 256, 0, c->stream>>>(
                static_cast<const cx<float>*>(rho), r_stride, ridx_dev, nr, a0, na, sh.k_pad, B);
        else
            clk::tc::k_tf32_split<double><<<dim3(xblocks, nr), 256, 0, c->stream>>>(
                static_cast<const cx<double>*>(rho), r_stride, ridx_dev, nr, a0, na, sh.k_pad, B);
        CL_LAUNCHED();
        prof_end(c, e0, CL_KCLASS_GRAM_SPLIT,
                 (double)na * (nl * (v_f32 ? 8.0 : 16.0) + nr * (rho_f32 ? 8.0 : 16.0)) +
                     (double)tc_bytes_per_atom(sh.rowsA, sh.rowsB) * kp);
        const int best_s = gram_splits(tiles, kt_total);
        const int kt_per = (kt_total + best_s - 1) / best_s;
        const int splits = (kt_total + kt_per - 1) / kt_per;
        cudaEvent_t e1 = prof_begin(c);
        clk::tc::k_gram_tc<<<dim3(tilesA, tilesB, splits), THREADS, SMEM_BYTES, c->stream>>>(
            mapA, mapB, kt_total, kt_per, nl, nr, out4_dev);
        CL_LAUNCHED();
        prof_end(c, e1, CL_KCLASS_GRAM, (double)tc_bytes_per_atom(sh.rowsA, sh.rowsB) * kp);
    }
}

// Error slot after the 4 * nl * nr results: non-zero when a device-side wait gave up.
void check_gram_slot(double slot) {
    if (slot != 0.0) cl::fail(CL_ERR_TIMEOUT, "tensor-core Gram: a device-side wait timed out");
}

// out4[l][r] = {sum ac, bd, ad, bc} over atoms (see k_gram); out4 holds 4 * nl * nr + 1
// doubles, the last one an error slot.  The FP32 form runs the tensor-core Gram; the plain
// form runs k_gram in FP64, whose register block IB (tile 16*IB) is the one that pads
// max(nl, nr) least, preferring larger blocks.
// rho: the right densities, complex64 when rho_f32 (the FP32 form's pair densities), else
// complex128 (the plain form's, and the grid API's caller-given density).
void gram(cl_ctx* c, const void* V_any, bool v_f32, long long v_stride, int nl, const void* rho_any, bool rho_f32,
          long long r_stride, const int* ridx_dev, int nr, long long n_atoms, double* out4_dev) {
    CL_CUDA(cudaMemsetAsync(out4_dev, 0, sizeof(double) * (4 * (size_t)nl * nr + 1), c->stream));
    const bool small = small_gram(c, n_atoms);
    if (small && v_f32 && rho_f32) {
        gram_dmma(c, static_cast<const cx<float>*>(V_any), v_stride, nl, static_cast<const cx<float>*>(rho_any),
                  r_stride, ridx_dev, nr, n_atoms, out4_dev);
        return;
    }
    if (use_tc_gram(c) && !small) {
        gram_tc(c, V_any, v_f32, v_stride, nl, rho_any, rho_f32, r_stride, ridx_dev, nr, n_atoms, out4_dev);
        return;
    }
    if (v_f32) cl::fail(CL_ERR_STATE, "the FP64 Gram needs FP64 potentials");
    const cx<double>* V = static_cast<const cx<double>*>(V_any);
    const int pmax = std::max(nl, nr);
    int ib = 4;
    long long best = -1;
    for (int cand = 4; cand >= 1; --cand) {
        const long long ts = 16 * cand, padded = (pmax + ts - 1) / ts * ts;
        if (best < 0 || padded < best) { best = padded; ib = cand; }
    }
    const int ts = 16 * ib;
    const int tl = (nl + ts - 1) / ts, tr = (nr + ts - 1) / ts;
    long long want = std::max(1LL, (148LL * 4) / std::max(1, tl * tr));
    long long per = std::max(256LL, (n_atoms + want - 1) / want);
    per = (per + 15) / 16 * 16;
    long long splits = std::max(1LL, (n_atoms + per - 1) / per);
    if (splits > 65535) {
        splits = 65535;
        per = ((n_atoms + splits - 1) / splits + 15) / 16 * 16;
    }
    cudaEvent_t e = prof_begin(c);
    const dim3 grid(tl, tr, (unsigned)splits);
    // FP32 densities (the FP32 form with CL_NO_TC_GRAM) are widened as they are loaded
    const auto launch = [&](auto tag) {
        using RT = decltype(tag);
        const cx<RT>* rho = static_cast<const cx<RT>*>(rho_any);
        switch (ib) {
            case 1: clk::k_gram<1, RT><<<grid, 256, 0, c->stream>>>(V, v_stride, nl, rho, r_stride, ridx_dev, nr, n_atoms, per, out4_dev); break;
            case 2: clk::k_gram<2, RT><<<grid, 256, 0, c->stream>>>(V, v_stride, nl, rho, r_stride, ridx_dev, nr, n_atoms, per, out4_dev); break;
            case 3: clk::k_gram<3, RT><<<grid, 256, 0, c->stream>>>(V, v_stride, nl, rho, r_stride, ridx_dev, nr, n_atoms, per, out4_dev); break;
            default: clk::k_gram<4, RT><<<grid, 256, 0, c->stream>>>(V, v_stride, nl, rho, r_stride, ridx_dev, nr, n_atoms, per, out4_dev); break;
        }
    };
    if (rho_f32)
        launch(float{});
    else
        launch(double{});
    CL_LAUNCHED();
    prof_end(c, e, CL_KCLASS_GRAM, (double)n_atoms * (nl * 16.0 + nr * (rho_f32 ? 8.0 : 16.0)));
}

// Pair densities rho[p][atom] for products (fl[p], fr[p]) (0-based state indices): the
// device lists and launch shape are set up once (setup synchronises), the launch itself only
// enqueues (it can be captured in a CUDA graph).
struct PairSetup {
    DevBuf<clk::PairSeg> segs;  // products grouped by left state, indices into `states` (FP64 kernel)
    clk::PairTri tri{};  // products over at most 12 states (register kernel)
    bool reg_ok = false;
    int grid_reg = 1;
    // tiles of 4 x 4 states (more than 8 used states, see k_pair_density_tile)
    bool tile_ok = false;
    DevBuf<int> tile_states, tiles, tile_prod;
    int ns_pad = 0, n_tiles = 0, tile_atoms = 0, tile_threads = 0, tile_blocks = 0;
    size_t tile_smem = 0;
    DevBuf<int> states;
    int np = 0, n_segs = 0, n_used = 0, chunk = 1, blocks = 1;
    size_t smem = 0;
};

// Tables of the 4 x 4-state tile kernel: used states ascending, padded to a multiple of 4
// (-1: zero rows); the requested tiles (bi | bj << 16, bi >= bj); and per ordered state pair
// (i >= j) the density row 2p (rho_p = conj(c_i) c_j) or 2p + 1 (rho_p = conj(c_j) c_i).  The
// atoms a block stages (A) are the most, of 64, 32, 16, 8, whose coefficients fit 110 KB (two
// blocks an SM), else 8 atoms in up to 227 KB; beyond that, or when two products name the same
// pair of states both ways, the segment kernel runs instead (as it does with CL_NO_PAIR_TILE=1).
void pair_tile_setup(cl_ctx* c, const std::vector<int2>& fl, const std::vector<int>& used,
                     const std::vector<int>& where, PairSetup& ps) {
    const int n = (int)used.size();
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int a, int b) { return used[a] < used[b]; });
    std::vector<int> pos(n);
    const int ns_pad = (n + clk::kPairTile - 1) / clk::kPairTile * clk::kPairTile;
    std::vector<int> st(ns_pad, -1);
    for (int k = 0; k < n; ++k) {
        pos[order[k]] = k;
        st[k] = used[order[k]];
    }
    std::vector<int> prod((size_t)ns_pad * ns_pad, -1);
    const int nblk = ns_pad / clk::kPairTile;
    std::vector<char> want((size_t)nblk * nblk, 0);
    for (int p = 0; p < ps.np; ++p) {
        int i = pos[where[fl[p].x]], j = pos[where[fl[p].y]];
        int code = 2 * p;
        if (i < j) {
            std::swap(i, j);
            code += 1;
        }
        int& slot = prod[(size_t)i * ns_pad + j];
        if (slot >= 0) return;  // the same pair both ways: the segment kernel
        slot = code;
        want[(size_t)(i / clk::kPairTile) * nblk + j / clk::kPairTile] = 1;
    }
    std::vector<int> tiles;
    for (int bi = 0; bi < nblk; ++bi)
        for (int bj = 0; bj <= bi; ++bj)
            if (want[(size_t)bi * nblk + bj]) tiles.push_back(bi | (bj << 16));
    const size_t per_atom = sizeof(cx<double>) * (size_t)ns_pad * (size_t)(c->n_orb | 1);
    int A = 0;
    for (int cand : {64, 32, 16, 8})
        if (per_atom * cand <= 110 * 1024) {
            A = cand;
            break;
        }
    if (A == 0 && per_atom * 8 <= 227 * 1024) A = 8;
    if (A == 0) return;
    ps.tile_ok = true;
    ps.ns_pad = ns_pad;
    ps.n_tiles = (int)tiles.size();
    ps.tile_atoms = A;
    ps.tile_smem = per_atom * A;
    ps.tile_threads = (int)std::min<long long>(256, ((long long)ps.n_tiles * A + 31) / 32 * 32);
    ps.tile_blocks = (int)std::max<long long>(1, std::min<long long>((c->n_sorted + A - 1) / A, 148LL * 8));
    ps.tile_states.upload(st.data(), st.size(), c->stream);
    ps.tiles.upload(tiles.data(), tiles.size(), c->stream);
    ps.tile_prod.upload(prod.data(), prod.size(), c->stream);
}

void pair_setup(cl_ctx* c, const std::vector<int2>& fl, PairSetup& ps) {
    ps.np = (int)fl.size();
    std::vector<int> used;
    std::vector<int> where(c->n_states, -1);
    for (const auto& f : fl)
        for (int s : {f.x, f.y})
            if (where[s] < 0) { where[s] = (int)used.size(); used.push_back(s); }
    // segments: the products of each left state, kPairSeg at a time (product order kept)
    std::vector<std::vector<int>> by_left(used.size());
    for (int p = 0; p < ps.np; ++p) by_left[where[fl[p].x]].push_back(p);
    std::vector<clk::PairSeg> segs;
    for (int u = 0; u < (int)used.size(); ++u)
        for (size_t k0 = 0; k0 < by_left[u].size(); k0 += clk::kPairSeg) {
            clk::PairSeg sg{};
            sg.left = u;
            sg.cnt = (int)std::min<size_t>(clk::kPairSeg, by_left[u].size() - k0);
            for (int j = 0; j < sg.cnt; ++j) {
                const int p = by_left[u][k0 + j];
                sg.right[j] = where[fl[p].y];
                sg.prod[j] = p;
            }
            segs.push_back(sg);
        }
    ps.n_segs = (int)segs.size();
    ps.segs.upload(segs.data(), segs.size(), c->stream);
    // register kernel (at most 12 used states): the used states in ascending order, and the
    // density row of each product (i, j), i >= j in that order (rows are conj(c_x) c_y, x >= y)
    // (CL_NO_PAIR_REG12=1: at most 8, the 4 x 4-state tile kernel above that)
    const size_t reg_max = std::getenv("CL_NO_PAIR_REG12") ? 8 : (size_t)clk::kPairRegStates;
    ps.reg_ok = !used.empty() && used.size() <= reg_max;
    if (ps.reg_ok) {
        std::vector<int> order(used.size());
        std::iota(order.begin(), order.end(), 0);
        std::sort(order.begin(), order.end(), [&](int a, int b) { return used[a] < used[b]; });
        std::vector<int> pos(used.size());
        for (size_t k = 0; k < order.size(); ++k) {
            pos[order[k]] = (int)k;
            ps.tri.states[k] = used[order[k]];
        }
        for (size_t k = order.size(); k < (size_t)clk::kPairRegStates; ++k) ps.tri.states[k] = used[order[0]];
        for (int& v : ps.tri.prod) v = -1;
        for (int p = 0; p < ps.np; ++p) {
            const int i = pos[where[fl[p].x]], j = pos[where[fl[p].y]];
            if (i < j) cl::fail(CL_ERR_STATE, "pair density with its lower state first");
            ps.tri.prod[i * (i + 1) / 2 + j] = p;
        }
        ps.grid_reg = (int)std::max<long long>(
            1, std::min<long long>((c->n_sorted + clk::kPairAtoms - 1) / clk::kPairAtoms, 148LL * 2 * 4));
    }
    if (!ps.reg_ok && !used.empty() && !std::getenv("CL_NO_PAIR_TILE")) pair_tile_setup(c, fl, used, where, ps);
    ps.states.upload(used.data(), used.size(), c->stream);
    ps.n_used = (int)used.size();
    // two stages of `chunk` atoms, each up to 48 KB (about two blocks per SM)
    const int os = c->n_orb | 1;
    const size_t per_atom = sizeof(cx<double>) * (size_t)used.size() * os;
    // the chunk (at most the 48 KB stage) whose item rounds -- segments x atoms over the 256
    // threads of a block -- cost least per atom
    const int max_chunk = (int)std::max<size_t>(1, std::min<size_t>(64, (48 * 1024) / per_atom));
    ps.chunk = max_chunk;
    double best = 1e300;
    for (int ch = max_chunk; ch >= std::max(1, max_chunk / 2); --ch) {
        const double rounds = (double)(((long long)ps.n_segs * ch + 255) / 256);
        if (rounds / ch < best - 1e-12) {
            best = rounds / ch;
            ps.chunk = ch;
        }
    }
    ps.smem = 2 * per_atom * ps.chunk;
    ensure_smem(clk::k_pair_density<double>, ps.smem);
    ensure_smem(clk::k_pair_density<float>, ps.smem);
    const long long chunks = (c->n_sorted + ps.chunk - 1) / ps.chunk;
    ps.blocks = (int)std::min<long long>(chunks, 148LL * 8);
    CL_CUDA(cudaStreamSynchronize(c->stream));
}

// f(std::integral_constant<int, n>) for 1 <= n <= 12 used states
template <typename F>
void with_states(int n, F&& f) {
    switch (n) {
        case 1: f(std::integral_constant<int, 1>{}); break;
        case 2: f(std::integral_constant<int, 2>{}); break;
        case 3: f(std::integral_constant<int, 3>{}); break;
        case 4: f(std::integral_constant<int, 4>{}); break;
        case 5: f(std::integral_constant<int, 5>{}); break;
        case 6: f(std::integral_constant<int, 6>{}); break;
        case 7: f(std::integral_constant<int, 7>{}); break;
        case 8: f(std::integral_constant<int, 8>{}); break;
        case 9: f(std::integral_constant<int, 9>{}); break;
        case 10: f(std::integral_constant<int, 10>{}); break;
        case 11: f(std::integral_constant<int, 11>{}); break;
        default: f(std::integral_constant<int, 12>{}); break;
    }
}

void pair_launch(cl_ctx* c, const PairSetup& ps, void* rho) {
    // the shared-memory attribute is per kernel, so another setup (of another group or
    // request) may have lowered it since this one was prepared
    cudaEvent_t e = prof_begin(c);
    if (fp64_form(c) && ps.reg_ok) {
        cx<double>* out = static_cast<cx<double>*>(rho);
        const auto go = [&](auto ns) {
            constexpr int NS = decltype(ns)::value;
            const size_t smem = 2 * sizeof(cx<double>) * clk::pair_stage_elems(NS);
            ensure_smem(clk::k_pair_density_reg<NS, double>, smem);
            clk::k_pair_density_reg<NS, double><<<ps.grid_reg, clk::kPairAtoms * clk::pair_parts(NS), smem, c->stream>>>(
                c->coeff.p, c->n_sorted, c->n_orb, nullptr, c->n_sorted, ps.tri, out);
        };
        with_states(ps.n_used, go);
    } else if (fp64_form(c) && !ps.tile_ok) {
        ensure_smem(clk::k_pair_density<double>, ps.smem);
        clk::k_pair_density<double><<<ps.blocks, 256, ps.smem, c->stream>>>(
            c->coeff.p, c->n_sorted, c->n_orb, nullptr, c->n_sorted, ps.segs.p, ps.n_segs, ps.states.p,
            ps.n_used, ps.chunk, static_cast<cx<double>*>(rho));
    } else if (ps.reg_ok) {
        cx<float>* out = static_cast<cx<float>*>(rho);
        const auto go = [&](auto ns) {
            constexpr int NS = decltype(ns)::value;
            const size_t smem = 2 * sizeof(cx<double>) * clk::pair_stage_elems(NS);
            ensure_smem(clk::k_pair_density_reg<NS, float>, smem);
            clk::k_pair_density_reg<NS, float><<<ps.grid_reg, clk::kPairAtoms * clk::pair_parts(NS), smem, c->stream>>>(
                c->coeff.p, c->n_sorted, c->n_orb, nullptr, c->n_sorted, ps.tri, out);
        };
        with_states(ps.n_used, go);
    } else if (ps.tile_ok) {  // more than 12 states: 4 x 4-state tiles (FP64 sums, rounded once)
        const auto go = [&](auto tag) {
            using RT = decltype(tag);
            ensure_smem(clk::k_pair_density_tile<RT>, ps.tile_smem);
            clk::k_pair_density_tile<RT><<<ps.tile_blocks, ps.tile_threads, ps.tile_smem, c->stream>>>(
                c->coeff.p, c->n_sorted, c->n_orb, nullptr, c->n_sorted, ps.tile_states.p, ps.ns_pad,
                ps.tiles.p, ps.n_tiles, ps.tile_prod.p, ps.tile_atoms, static_cast<cx<RT>*>(rho));
        };
        if (fp64_form(c))
            go(double{});
        else
            go(float{});
    } else {  // the segment kernel (FP64 sums, rounded once)
        ensure_smem(clk::k_pair_density<float>, ps.smem);
        clk::k_pair_density<float><<<ps.blocks, 256, ps.smem, c->stream>>>(
            c->coeff.p, c->n_sorted, c->n_orb, nullptr, c->n_sorted, ps.segs.p, ps.n_segs, ps.states.p,
            ps.n_used, ps.chunk, static_cast<cx<float>*>(rho));
    }
    CL_LAUNCHED();
    prof_end(c, e, CL_KCLASS_DENSITY,
             (double)ps.n_used * c->n_sorted * c->n_orb * 16.0 + (double)ps.np * c->n_sorted * rho_bytes(c));
}

void pair_densities(cl_ctx* c, const std::vector<int2>& fl, void* rho) {
    PairSetup ps;
    pair_setup(c, fl, ps);
    pair_launch(c, ps, rho);
    CL_CUDA(cudaStreamSynchronize(c->stream));  // device lists go out of scope
}

// Device buffer of at least `count` elements, reallocated only when it must grow.
template <typename T>
void grow(DevBuf<T>& b, size_t count) {
    if (b.n >= count && b.p) return;
    b.alloc(count);
}

void check_ctx(cl_ctx* c) {
    if (!c) cl::fail(CL_ERR_ARGUMENT, "null context");
    CL_CUDA(cudaSetDevice(c->device));
}

void check_kernel(cl_ctx* c) {
    if (!c->kernel_ready) cl::fail(CL_ERR_STATE, "the Coulomb kernel is not initialised (call cl_set_kernel_*)");
}

void identity_atoms(cl_ctx* c) {
    if (c->grid_cell.p) return;
    const int nrows = c->n[1] * c->n[2];
    std::vector<int> cell((size_t)c->M), rp((size_t)nrows + 1);
    std::iota(cell.begin(), cell.end(), 0);
    for (int r = 0; r <= nrows; ++r) rp[r] = r * c->n[0];
    c->grid_cell.upload(cell.data(), cell.size(), c->stream);
    c->grid_row_ptr.upload(rp.data(), rp.size(), c->stream);
    CL_CUDA(cudaStreamSynchronize(c->stream));
}

}  // namespace

// =======================================================================================
// C ABI
// =======================================================================================
extern "C" {

int cl_create(cl_ctx** out, int nx, int ny, int nz, double sx, double sy, double sz, int mode) {
    if (out) *out = nullptr;
    cl_ctx* c = nullptr;
    int st = cl::guarded([&] {
        if (!out) cl::fail(CL_ERR_ARGUMENT, "null output pointer");
        if (nx <= 0 || ny <= 0 || nz <= 0) cl::fail(CL_ERR_ARGUMENT, "dimensions must be positive");
        if (mode < CL_MODE_FP64_PLAIN || mode > CL_MODE_FP32_SUBLATTICE) cl::fail(CL_ERR_ARGUMENT, "unknown mode %d", mode);
        const int dims[3] = {nx, ny, nz};
        for (int d = 0; d < 3; ++d) {
            if (!smooth235(dims[d]))
                cl::fail(CL_ERR_UNSUPPORTED, "grid size %d is not a product of 2, 3 and 5", dims[d]);
            if (dims[d] > 4096) cl::fail(CL_ERR_UNSUPPORTED, "grid size %d exceeds 4096", dims[d]);
        }
        const long long M = (long long)nx * ny * nz;
        if (M >= (1LL << 31)) cl::fail(CL_ERR_UNSUPPORTED, "grid of %lld cells exceeds 2^31", M);
        if (!(sx > 0 && sy > 0 && sz > 0)) cl::fail(CL_ERR_ARGUMENT, "step lengths must be positive");
        require_gpu();
        c = new cl_ctx();
        CL_CUDA(cudaGetDevice(&c->device));
        c->mode = mode;
        c->n[0] = nx;
        c->n[1] = ny;
        c->n[2] = nz;
        c->M = M;
        c->step[0] = sx;
        c->step[1] = sy;
        c->step[2] = sz;
        CL_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        for (auto& e : c->ev) CL_CUDA(cudaEventCreate(&e));
        for (int d = 0; d < 3; ++d) {
            Axis& A = c->ax[d];
            A.plan = make_plan(dims[d]);
            auto t64 = twiddles64(dims[d]);
            std::vector<cx<float>> t32(t64.size());
            for (size_t i = 0; i < t64.size(); ++i) {
                t32[i].re = (float)t64[i].re;
                t32[i].im = (float)t64[i].im;
            }
            A.tw64.upload(t64.data(), t64.size(), c->stream);
            A.tw32.upload(t32.data(), t32.size(), c->stream);
            auto ph = phases64(dims[d]);
            A.phase.upload(ph.data(), ph.size(), c->stream);
        }
        CL_CUDA(cudaStreamSynchronize(c->stream));
        *out = c;
    });
    if (st != CL_OK) delete c;
    return st;
}

void cl_destroy(cl_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    delete ctx;
}

int cl_set_kernel_coulomb(cl_ctx* c, double dielectric, double onsite, double tf_lattice) {
    return cl::guarded([&] {
        check_ctx(c);
        clk::KernelModel km{dielectric, onsite, 0, 0.0, 0.0};
        if (tf_lattice > 0) {
            if (!(dielectric > 1.0)) cl::fail(CL_ERR_ARGUMENT, "dielectric constant must be >1 to use Thomas-Fermi model");
            km.thomas_fermi = 1;
            thomas_fermi(dielectric, tf_lattice, &km.r_tf, &km.q_tf);
        }
        const int n1x = c->n[0] + 1, n1y = c->n[1] + 1, n1z = c->n[2] + 1;
        const long long total = (long long)n1x * n1y * n1z;
        c->kernel_ready = false;
        c->ghat.alloc(total);
        cudaEvent_t pe = prof_begin(c);
        clk::k_kernel_octant<<<grid_for(total), 256, 0, c->stream>>>(c->ghat.p, n1x, n1y, n1z, c->step[0], c->step[1],
                                                                     c->step[2], km);
        CL_LAUNCHED();
        transform_kernel(c);
        prof_end(c, pe, CL_KCLASS_KERNEL, (double)total * 8.0 * 7.0 + (double)c->M * 8.0 * (fp64_form(c) ? 8.0 : 4.0));
        CL_CUDA(cudaStreamSynchronize(c->stream));
        prof_collect(c);
    });
}

int cl_set_kernel_grid(cl_ctx* c, const double* G) {
    return cl::guarded([&] {
        check_ctx(c);
        if (!G) cl::fail(CL_ERR_ARGUMENT, "null kernel grid");
        const long long total = (long long)(c->n[0] + 1) * (c->n[1] + 1) * (c->n[2] + 1);
        c->kernel_ready = false;
        c->ghat.upload(G, total, c->stream);
        transform_kernel(c);
    });
}

int cl_prepare_grid(cl_ctx* c, const double* rho) {
    return cl::guarded([&] {
        check_ctx(c);
        check_kernel(c);
        if (!rho) cl::fail(CL_ERR_ARGUMENT, "null density");
        identity_atoms(c);
        c->grid_rho.upload(reinterpret_cast<const cx<double>*>(rho), c->M, c->stream);
        c->grid_V.alloc(c->M);
        const void* rho_in = c->grid_rho.p;
        if (!fp64_form(c)) {  // the FP32 forms' densities are complex64
            c->grid_rho32.alloc(c->M);
            clk::k_narrow<float><<<grid_for(c->M), 256, 0, c->stream>>>(c->grid_rho.p, c->grid_rho32.p, c->M);
            CL_LAUNCHED();
            rho_in = c->grid_rho32.p;
        }
        run_rounds_mode(c, rho_in, c->M, 1, c->grid_row_ptr.p, c->grid_cell.p, c->grid_V.p, c->M);
        CL_CUDA(cudaStreamSynchronize(c->stream));
        c->grid_prepared = true;
    });
}

int cl_calculate_grid(cl_ctx* c, const double* rho2, double out[2]) {
    return cl::guarded([&] {
        check_ctx(c);
        if (!c->grid_prepared) cl::fail(CL_ERR_STATE, "calculate() called before prepare()");
        if (!rho2 || !out) cl::fail(CL_ERR_ARGUMENT, "null argument");
        c->grid_rho2.upload(reinterpret_cast<const cx<double>*>(rho2), c->M, c->stream);
        DevBuf<double> o4;
        o4.alloc(5);
        DevBuf<int> ridx;
        int zero = 0;
        ridx.upload(&zero, 1, c->stream);
        tc_reserve(c, 1, 1, c->M, false, false);
        gram(c, c->grid_V.p, false, c->M, 1, c->grid_rho2.p, false, c->M, ridx.p, 1, c->M, o4.p);
        double h[5];
        CL_CUDA(cudaMemcpyAsync(h, o4.p, sizeof h, cudaMemcpyDeviceToHost, c->stream));
        CL_CUDA(cudaStreamSynchronize(c->stream));
        check_gram_slot(h[4]);
        out[0] = h[0] - h[1];
        out[1] = h[2] + h[3];
    });
}

int cl_potential_grid(cl_ctx* c, double* V) {
    return cl::guarded([&] {
        check_ctx(c);
        if (!c->grid_prepared) cl::fail(CL_ERR_STATE, "potential() called before prepare()");
        if (!V) cl::fail(CL_ERR_ARGUMENT, "null argument");
        CL_CUDA(cudaMemcpyAsync(V, c->grid_V.p, sizeof(cx<double>) * c->M, cudaMemcpyDeviceToHost, c->stream));
        CL_CUDA(cudaStreamSynchronize(c->stream));
    });
}

}  // extern "C"

namespace {

void check_states_args(int n_states, int n_holes, int64_t n_atoms, int n_orb, const double* coeff,
                       const int64_t* cells) {
    if (n_states <= 0 || n_holes < 0 || n_holes > n_states || n_atoms <= 0 || n_orb <= 0 || !coeff || !cells)
        cl::fail(CL_ERR_ARGUMENT, "invalid states description");
    if (n_atoms >= (1LL << 31)) cl::fail(CL_ERR_UNSUPPORTED, "too many atoms");
}

// Sub-lattice decomposition for the (deduplicated) atom cells, in the sub-lattice modes: the
// modulus m in {4, 2} dividing every grid size whose classes need the least transform work,
// S / m^3 of the 8 rounds' (S occupied classes, each transformed at (2n/m)^3 points), kept when
// at most half of it, with at most 8 classes and a compiled z-mix length.  Classes go in
// class-id order, or in the canonical zinc-blende order when they are that set (shifted).
// CL_NO_SUBLATTICE=1 keeps the 8 rounds.
void plan_sublattice(cl_ctx* c, const std::vector<int>& cell_s) {
    Sublattice& sl = c->sl;
    const int old_m = sl.m, old_S = sl.S;
    int old_off[clk::kSlMaxClasses][3];
    std::memcpy(old_off, sl.off, sizeof old_off);
    sl.active = false;
    sl.zb = false;
    if (!sublattice_mode(c) || std::getenv("CL_NO_SUBLATTICE")) return;
    const int nx = c->n[0], ny = c->n[1], nz = c->n[2];
    double best = 0.5;
    int best_m = 0;
    std::vector<int> best_ids;
    for (int m : {4, 2}) {
        if (nx % m || ny % m || nz % m) continue;
        if (!clp::zmix_supported(2 * nz / m)) continue;
        std::vector<char> seen((size_t)m * m * m, 0);
        for (int cs : cell_s) {
            const int x = cs % nx, y = (cs / nx) % ny, z = cs / (nx * ny);
            seen[((z % m) * m + y % m) * m + x % m] = 1;
        }
        std::vector<int> ids;
        for (int id = 0; id < m * m * m; ++id)
            if (seen[id]) ids.push_back(id);
        if (ids.empty() || (int)ids.size() > clk::kSlMaxClasses) continue;
        const double cost = (double)ids.size() / (double)(m * m * m);
        if (cost <= best) {
            best = cost;
            best_m = m;
            best_ids = ids;
        }
    }
    if (!best_m) return;
    const int m = best_m, S = (int)best_ids.size();
    sl.m = m;
    sl.S = S;
    for (int s = 0; s < S; ++s) {
        sl.off[s][0] = best_ids[s] % m;
        sl.off[s][1] = (best_ids[s] / m) % m;
        sl.off[s][2] = best_ids[s] / (m * m);
    }
    if (m == 4 && S == 8) {  // the zinc-blende set, shifted by t?
        for (int t = 0; t < 64 && !sl.zb; ++t) {
            const int tx = t % 4, ty = (t / 4) % 4, tz = t / 16;
            int cand[8][3];
            bool all = true;
            for (int s = 0; s < 8 && all; ++s) {
                cand[s][0] = (clk::ZincBlende::off[s][0] + tx) % 4;
                cand[s][1] = (clk::ZincBlende::off[s][1] + ty) % 4;
                cand[s][2] = (clk::ZincBlende::off[s][2] + tz) % 4;
                all = std::binary_search(best_ids.begin(), best_ids.end(),
                                         (cand[s][2] * 4 + cand[s][1]) * 4 + cand[s][0]);
            }
            if (all) {
                sl.zb = true;
                std::memcpy(sl.off, cand, sizeof cand);
            }
        }
    }
    for (int d = 0; d < 3; ++d) {
        sl.sub[d] = c->n[d] / m;
        sl.pad[d] = 2 * c->n[d] / m;
    }
    sl.vn[0] = sl.pad[0];
    sl.vn[1] = sl.pad[1];
    sl.vn[2] = S * sl.sub[2];
    sl.vM = (long long)sl.vn[0] * sl.vn[1] * sl.vn[2];
    sl.table = clk::sl_table(sl.off, S, m);
    if (m != old_m || S != old_S || std::memcmp(old_off, sl.off, sizeof old_off) != 0) sl.tables_version = -1;
    sl.active = true;
}

// Atoms sorted by cell; where several atoms share a cell the one listed last wins, as with
// F[cell] = value in atom order (Product.cpp:16-30).  Builds the sorted cell list, the input
// atom of each slot, the row CSR and the live-row count, and uploads them (synchronously).  With
// the sub-lattice decomposition the atoms are then ordered by their cell of the virtual grid
// (class-stacked sub-grids), which is the order every later pass and reduction uses.  A list
// identical to the previous load's is not processed again.
void load_cells(cl_ctx* c, int64_t n_atoms, const int64_t* cells) {
    if ((int64_t)c->cells_seen.size() == n_atoms && c->n_sorted > 0 &&
        std::memcmp(c->cells_seen.data(), cells, sizeof(int64_t) * (size_t)n_atoms) == 0)
        return;
    c->cells_seen.clear();
    std::vector<int> order((size_t)n_atoms);
    std::iota(order.begin(), order.end(), 0);
    for (int64_t a = 0; a < n_atoms; ++a)
        if (cells[a] < 0 || cells[a] >= c->M) cl::fail(CL_ERR_ARGUMENT, "atom %lld lies outside the grid", (long long)a);
    bool sorted = true;
    for (int64_t a = 1; a < n_atoms && sorted; ++a) sorted = cells[a - 1] < cells[a];
    if (!sorted) std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cells[x] < cells[y]; });
    std::vector<int> cell_s, orig_s;
    cell_s.reserve((size_t)n_atoms);
    orig_s.reserve((size_t)n_atoms);
    c->atom_slot.assign((size_t)n_atoms, 0);
    for (size_t i = 0; i < order.size(); ++i) {
        const int a = order[i];
        if (!cell_s.empty() && cell_s.back() == (int)cells[a]) {
            orig_s.back() = a;  // later atom of the same cell replaces the earlier one
        } else {
            cell_s.push_back((int)cells[a]);
            orig_s.push_back(a);
        }
        c->atom_slot[a] = (long long)cell_s.size() - 1;
    }
    plan_sublattice(c, cell_s);
    int nx = c->n[0];
    int nrows = c->n[1] * c->n[2];
    if (c->sl.active) {
        const Sublattice& sl = c->sl;
        const int m = sl.m, gx = c->n[0], gy = c->n[1];
        int cls_of[64];
        for (int s = 0; s < sl.S; ++s) cls_of[(sl.off[s][2] * m + sl.off[s][1]) * m + sl.off[s][0]] = s;
        std::vector<int> vcell(cell_s.size()), perm(cell_s.size());
        for (size_t i = 0; i < cell_s.size(); ++i) {
            const int cs = cell_s[i];
            const int x = cs % gx, y = (cs / gx) % gy, z = cs / (gx * gy);
            const int s = cls_of[((z % m) * m + y % m) * m + x % m];
            vcell[i] = ((s * sl.sub[2] + z / m) * sl.pad[1] + y / m) * sl.pad[0] + x / m;
        }
        std::iota(perm.begin(), perm.end(), 0);
        std::sort(perm.begin(), perm.end(), [&](int a, int b) { return vcell[a] < vcell[b]; });
        std::vector<int> new_pos(cell_s.size());
        std::vector<int> vc(cell_s.size()), vo(cell_s.size());
        for (size_t k = 0; k < perm.size(); ++k) {
            new_pos[perm[k]] = (int)k;
            vc[k] = vcell[perm[k]];
            vo[k] = orig_s[perm[k]];
        }
        for (auto& slot : c->atom_slot) slot = new_pos[slot];
        cell_s.swap(vc);
        orig_s.swap(vo);
        nx = sl.vn[0];
        nrows = sl.vn[1] * sl.vn[2];
    }
    std::vector<int> rp((size_t)nrows + 1, 0);
    for (int cs : cell_s) rp[cs / nx + 1]++;
    for (int r = 0; r < nrows; ++r) rp[r + 1] += rp[r];
    long long live = 0;
    for (int r = 0; r < nrows; ++r) live += rp[r + 1] > rp[r];
    c->live_rows = live;
    c->n_sorted = (long long)cell_s.size();
    c->cell_sorted.upload(cell_s.data(), cell_s.size(), c->stream);
    c->orig_sorted.upload(orig_s.data(), orig_s.size(), c->stream);
    c->row_ptr.upload(rp.data(), rp.size(), c->stream);
    CL_CUDA(cudaStreamSynchronize(c->stream));
    c->cells_seen.assign(cells, cells + n_atoms);
}

// Uploads state s of the caller's coefficients ([state][atom][orb], input atom order) through
// a staging slot and stores it in the cell-sorted atom order the pair-density kernels read
// (k_gather_atoms): consecutive slots of a block are then contiguous rows in HBM.  Both on
// `stream`, so slot s & 1 is free again once the gather of state s - 2 has run.
void upload_state_sorted(cl_ctx* c, int s, const double* coeff, cudaStream_t stream) {
    const size_t per_in = (size_t)c->n_atoms * c->n_orb, per_s = (size_t)c->n_sorted * c->n_orb;
    cx<double>* slot = c->coeff_stage.p + (size_t)(s & 1) * per_in;
    CL_CUDA(cudaMemcpyAsync(slot, coeff + 2 * (size_t)s * per_in, sizeof(cx<double>) * per_in, cudaMemcpyHostToDevice,
                            stream));
    const int blocks = (int)std::max<long long>(1, std::min<long long>(((long long)per_s + 255) / 256, 148LL * 16));
    clk::k_gather_atoms<<<blocks, 256, 0, stream>>>(slot, c->orig_sorted.p, c->n_sorted, c->n_orb,
                                                    c->coeff.p + (size_t)s * per_s);
    CL_LAUNCHED();
}
void reserve_coeff(cl_ctx* c, int n_states) {
    grow(c->coeff, (size_t)n_states * c->n_sorted * c->n_orb);
    grow(c->coeff_stage, 2 * (size_t)c->n_atoms * c->n_orb);
}

}  // namespace

extern "C" {

int cl_set_states(cl_ctx* c, int n_states, int n_holes, int64_t n_atoms, int n_orb, const double* coeff,
                  const int64_t* cells) {
    return cl::guarded([&] {
        check_ctx(c);
        check_states_args(n_states, n_holes, n_atoms, n_orb, coeff, cells);
        load_cells(c, n_atoms, cells);
        c->n_states = n_states;
        c->n_holes = n_holes;
        c->n_orb = n_orb;
        c->n_atoms = n_atoms;
        reserve_coeff(c, n_states);
        for (int s = 0; s < n_states; ++s) upload_state_sorted(c, s, coeff, c->stream);
        CL_CUDA(cudaStreamSynchronize(c->stream));
    });
}

}  // extern "C"

namespace {

// Step values (coulombo.cpp:199-207): step s takes the Gram entry of its (left, right) pair,
// combined for the pair's conjugation flags and conjugated when the left product is.  Long
// integral lists are mapped on several host threads.
void map_step_values(const std::vector<cl::PlanStep>& plan, const std::vector<int>& slot,
                     const std::vector<int>& rcol, int nr, const double* h, double* out) {
    const auto work = [&](size_t i0, size_t i1) {
        for (size_t i = i0; i < i1; ++i) {
            const auto& st = plan[i];
            const int l = slot[st.left.product], r = rcol[st.right.product];
            const double* q = &h[((size_t)l * nr + r) * 4];
            const bool rconj = st.left.conjugate != st.right.conjugate;
            const double re = rconj ? q[0] + q[1] : q[0] - q[1];
            double im = rconj ? q[3] - q[2] : q[2] + q[3];
            if (st.left.conjugate) im = -im;
            out[2 * st.id] = re;
            out[2 * st.id + 1] = im;
        }
    };
    const size_t n = plan.size();
    const size_t hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t nt = std::min<size_t>(std::min<size_t>(hw, 32), n / 65536 + 1);
    if (nt <= 1) {
        work(0, n);
        return;
    }
    std::vector<std::thread> pool;
    for (size_t t = 0; t < nt; ++t) pool.emplace_back([&, t] { work(n * t / nt, n * (t + 1) / nt); });
    for (auto& th : pool) th.join();
}

// The steps of shard `shard` of `n_shards`: the plan's prepared (left) densities, in ascending
// product order, are dealt round-robin, and a step belongs to the shard of its left density.
// Every step is in exactly one shard, so the shards' integrals add up to the whole request's.
std::vector<cl::PlanStep> shard_steps(std::vector<cl::PlanStep> plan, int n_states, int shard, int n_shards) {
    if (n_shards < 1 || shard < 0 || shard >= n_shards) cl::fail(CL_ERR_ARGUMENT, "invalid shard %d of %d", shard, n_shards);
    if (n_shards == 1) return plan;
    const int P = n_states * (n_states + 1) / 2;
    std::vector<int> owner(P, -1);
    for (const auto& st : plan) owner[st.left.product] = 0;
    int k = 0;
    for (int p = 0; p < P; ++p)
        if (owner[p] == 0) owner[p] = k++ % n_shards;
        else owner[p] = -1;
    std::vector<cl::PlanStep> mine;
    for (const auto& st : plan)
        if (owner[st.left.product] == shard) mine.push_back(st);
    return mine;
}

void compute_impl(cl_ctx* c, int64_t n_int, const int16_t* spec, double* out, int round_mask, int shard = 0,
                  int n_shards = 1) {
    {
        check_ctx(c);
        check_kernel(c);
        if (c->n_states == 0) cl::fail(CL_ERR_STATE, "no states loaded (call cl_set_states)");
        if (n_int < 0 || (n_int && (!spec || !out))) cl::fail(CL_ERR_ARGUMENT, "invalid integral list");
        std::memset(c->timings, 0, sizeof c->timings);
        if (n_int == 0) return;
        std::vector<std::array<int16_t, 4>> specs((size_t)n_int);
        for (int64_t i = 0; i < n_int; ++i)
            for (int k = 0; k < 4; ++k) specs[i][k] = spec[4 * i + k];
        const auto plan = shard_steps(cl::orient_steps(c->n_states, specs), c->n_states, shard, n_shards);
        if (n_shards > 1) std::memset(out, 0, sizeof(double) * 2 * (size_t)n_int);
        if (plan.empty()) return;
        // densities: prepared (left) products first, then right-only products
        const int P = c->n_states * (c->n_states + 1) / 2;
        std::vector<int> slot(P, -1), is_left(P, 0), is_right(P, 0);
        for (const auto& s : plan) {
            is_left[s.left.product] = 1;
            is_right[s.right.product] = 1;
        }
        std::vector<int> prods;
        for (int p = 0; p < P; ++p)
            if (is_left[p]) { slot[p] = (int)prods.size(); prods.push_back(p); }
        const int nl = (int)prods.size();
        for (int p = 0; p < P; ++p)
            if (is_right[p] && slot[p] < 0) { slot[p] = (int)prods.size(); prods.push_back(p); }
        std::vector<int> rights, rcol(P, -1);
        for (int p = 0; p < P; ++p)
            if (is_right[p]) { rcol[p] = (int)rights.size(); rights.push_back(slot[p]); }
        const int nu = (int)prods.size(), nr = (int)rights.size();
        std::vector<int2> fl(nu);
        for (int i = 0; i < nu; ++i) {
            int a, b;
            cl::product_states(prods[i], &a, &b);
            fl[i] = make_int2(a - 1, b - 1);
        }
        const long long As = c->n_sorted;
        DevBuf<int>& dr = c->req_ridx;
        grow(dr, rights.size());
        CL_CUDA(cudaMemcpyAsync(dr.p, rights.data(), rights.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
        DevBuf<cx<double>>& rho = c->req_rho;
        DevBuf<cx<double>>& V = c->req_V;
        grow(rho, (size_t)nu * As);
        grow(V, (size_t)nl * As);
        DevBuf<double>& o4 = c->req_o4;
        grow(o4, (size_t)4 * nl * nr + 1);
        tc_reserve(c, nl, nr, As, v_fp32(c), rho_bytes(c) == sizeof(cx<float>));
        CL_CUDA(cudaEventRecord(c->ev[0], c->stream));
        pair_densities(c, fl, rho.p);
        CL_CUDA(cudaEventRecord(c->ev[1], c->stream));
        const bool v32 = v_fp32(c);
        run_transforms(c, rho.p, As, nl, V.p, As, v32, round_mask);
        CL_CUDA(cudaEventRecord(c->ev[2], c->stream));
        gram(c, V.p, v32, As, nl, rho.p, rho_bytes(c) == sizeof(cx<float>), As, dr.p, nr, As, o4.p);
        CL_CUDA(cudaEventRecord(c->ev[3], c->stream));
        std::vector<double> h((size_t)4 * nl * nr + 1);
        CL_CUDA(cudaMemcpyAsync(h.data(), o4.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CL_CUDA(cudaStreamSynchronize(c->stream));
        check_gram_slot(h.back());
        float t01, t12, t23, t03;
        CL_CUDA(cudaEventElapsedTime(&t01, c->ev[0], c->ev[1]));
        CL_CUDA(cudaEventElapsedTime(&t12, c->ev[1], c->ev[2]));
        CL_CUDA(cudaEventElapsedTime(&t23, c->ev[2], c->ev[3]));
        CL_CUDA(cudaEventElapsedTime(&t03, c->ev[0], c->ev[3]));
        c->timings[0] = t01;
        c->timings[1] = t12;
        c->timings[2] = t23;
        c->timings[3] = t03;
        prof_collect(c);
        map_step_values(plan, slot, rcol, nr, h.data(), out);
    }
}

// cl_compute_states: the states' coefficients are uploaded one state at a time on a copy stream
// while the densities whose states have arrived are transformed.  Left densities are grouped by
// their higher state index; a group's pair densities and rounds wait only for its last state.
void compute_states_impl(cl_ctx* c, int n_states, int n_holes, int64_t n_atoms, int n_orb, const double* coeff,
                         const int64_t* cells, int64_t n_int, const int16_t* spec, double* out) {
    check_ctx(c);
    check_kernel(c);
    check_states_args(n_states, n_holes, n_atoms, n_orb, coeff, cells);
    if (n_int < 0 || (n_int && (!spec || !out))) cl::fail(CL_ERR_ARGUMENT, "invalid integral list");
    load_cells(c, n_atoms, cells);
    c->n_states = n_states;
    c->n_holes = n_holes;
    c->n_orb = n_orb;
    c->n_atoms = n_atoms;
    reserve_coeff(c, n_states);
    std::memset(c->timings, 0, sizeof c->timings);
    if (!c->copy_stream) CL_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    while ((int)c->state_ev.size() < n_states) {
        cudaEvent_t e;
        CL_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        c->state_ev.push_back(e);
    }
    if (n_int == 0) {
        for (int s = 0; s < n_states; ++s) upload_state_sorted(c, s, coeff, c->stream);
        CL_CUDA(cudaStreamSynchronize(c->stream));
        return;
    }
    // The integral list is checked (and planned) before any copy reads the caller's buffer.
    std::vector<std::array<int16_t, 4>> specs((size_t)n_int);
    for (int64_t i = 0; i < n_int; ++i)
        for (int k = 0; k < 4; ++k) specs[i][k] = spec[4 * i + k];
    const auto plan = cl::orient_steps(n_states, specs);
    // On every error path below, the copies already queued from the caller's buffer (and the
    // work waiting on them) finish before the call returns, so the buffer is free for reuse
    // once the call has returned, whatever its status.
    struct DrainOnError {
        cudaStream_t a, b;
        bool armed = true;
        ~DrainOnError() {
            if (!armed) return;
            cudaStreamSynchronize(a);
            cudaStreamSynchronize(b);
            cudaGetLastError();
        }
    } drain{c->copy_stream, c->stream};
    // Uploads, one state at a time on the copy stream.  From pinned memory they are all enqueued
    // now and overlap the planning below; from pageable memory a copy returns only once staged,
    // so they are interleaved with the groups that need them (the groups already enqueued run
    // meanwhile).
    CL_CUDA(cudaEventRecord(c->ev[0], c->stream));
    CL_CUDA(cudaStreamWaitEvent(c->copy_stream, c->ev[0], 0));
    int uploaded = 0;
    const auto upload_through = [&](int last) {
        for (; uploaded <= last && uploaded < n_states; ++uploaded) {
            upload_state_sorted(c, uploaded, coeff, c->copy_stream);
            CL_CUDA(cudaEventRecord(c->state_ev[uploaded], c->copy_stream));
        }
    };
    {
        cudaPointerAttributes attr{};
        if (cudaPointerGetAttributes(&attr, coeff) == cudaSuccess && attr.type == cudaMemoryTypeHost)
            upload_through(n_states - 1);
        cudaGetLastError();  // pageable memory is not an error
    }
    const int P = n_states * (n_states + 1) / 2;
    std::vector<int> is_left(P, 0), is_right(P, 0);
    for (const auto& st : plan) {
        is_left[st.left.product] = 1;
        is_right[st.right.product] = 1;
    }
    // product -> (higher, lower) 0-based state
    auto states_of = [](int p) {
        int a, b;
        cl::product_states(p, &a, &b);
        return std::make_pair(a - 1, b - 1);
    };
    // left densities ordered by their higher state (stable), then right-only densities
    std::vector<int> lefts, prods, slot(P, -1);
    for (int p = 0; p < P; ++p)
        if (is_left[p]) lefts.push_back(p);
    std::stable_sort(lefts.begin(), lefts.end(),
                     [&](int x, int y) { return states_of(x).first < states_of(y).first; });
    for (int p : lefts) { slot[p] = (int)prods.size(); prods.push_back(p); }
    const int nl = (int)lefts.size();
    for (int p = 0; p < P; ++p)
        if (is_right[p] && slot[p] < 0) { slot[p] = (int)prods.size(); prods.push_back(p); }
    std::vector<int> rights, rcol(P, -1);
    for (int p = 0; p < P; ++p)
        if (is_right[p]) { rcol[p] = (int)rights.size(); rights.push_back(slot[p]); }
    const int nu = (int)prods.size(), nr = (int)rights.size();
    // groups of left densities: cut at a state boundary once a group holds nl/6 densities
    struct Group {
        int begin, end, last_state;
        PairSetup ps;
    };
    std::vector<std::unique_ptr<Group>> groups;
    const int min_group = std::max(1, nl / 6);
    for (int i = 0; i < nl;) {
        int j = i;
        int hi = states_of(prods[i]).first;
        while (j < nl && (j - i < min_group || states_of(prods[j]).first == hi)) {
            hi = std::max(hi, states_of(prods[j]).first);
            ++j;
        }
        auto g = std::make_unique<Group>();
        g->begin = i;
        g->end = j;
        g->last_state = hi;
        groups.push_back(std::move(g));
        i = j;
    }
    auto pairs_of = [&](int b, int e) {
        std::vector<int2> fl;
        for (int i = b; i < e; ++i) {
            const auto st = states_of(prods[i]);
            fl.push_back(make_int2(st.first, st.second));
        }
        return fl;
    };
    for (auto& g : groups) pair_setup(c, pairs_of(g->begin, g->end), g->ps);
    PairSetup ps_right;
    if (nu > nl) pair_setup(c, pairs_of(nl, nu), ps_right);
    const long long As = c->n_sorted;
    const bool v32 = v_fp32(c);
    DevBuf<int>& dr = c->req_ridx;
    grow(dr, rights.size());
    CL_CUDA(cudaMemcpyAsync(dr.p, rights.data(), rights.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    DevBuf<cx<double>>& rho = c->req_rho;
    DevBuf<cx<double>>& V = c->req_V;
    grow(rho, (size_t)nu * As);
    grow(V, (size_t)nl * As);
    DevBuf<double>& o4 = c->req_o4;
    grow(o4, (size_t)4 * nl * nr + 1);
    tc_reserve(c, nl, nr, As, v_fp32(c), rho_bytes(c) == sizeof(cx<float>));
    CL_CUDA(cudaStreamSynchronize(c->stream));
    for (auto& g : groups) {
        upload_through(g->last_state);
        CL_CUDA(cudaStreamWaitEvent(c->stream, c->state_ev[g->last_state], 0));
        pair_launch(c, g->ps, rho_at(c, rho.p, (long long)g->begin * As));
        run_transforms(c, rho_at(c, rho.p, (long long)g->begin * As), As, g->end - g->begin,
                       v_at(V.p, (long long)g->begin * As, v32), As, v32);
    }
    upload_through(n_states - 1);
    CL_CUDA(cudaStreamWaitEvent(c->stream, c->state_ev[n_states - 1], 0));
    if (nu > nl) pair_launch(c, ps_right, rho_at(c, rho.p, (long long)nl * As));
    CL_CUDA(cudaEventRecord(c->ev[2], c->stream));
    gram(c, V.p, v32, As, nl, rho.p, rho_bytes(c) == sizeof(cx<float>), As, dr.p, nr, As, o4.p);
    CL_CUDA(cudaEventRecord(c->ev[3], c->stream));
    std::vector<double> h((size_t)4 * nl * nr + 1);
    CL_CUDA(cudaMemcpyAsync(h.data(), o4.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CL_CUDA(cudaStreamSynchronize(c->stream));  // after the wait on the last upload: all copies done
    drain.armed = false;
    check_gram_slot(h.back());
    float t02, t23, t03;
    CL_CUDA(cudaEventElapsedTime(&t02, c->ev[0], c->ev[2]));
    CL_CUDA(cudaEventElapsedTime(&t23, c->ev[2], c->ev[3]));
    CL_CUDA(cudaEventElapsedTime(&t03, c->ev[0], c->ev[3]));
    c->timings[0] = 0;  // pair densities are interleaved with the uploads and the rounds
    c->timings[1] = t02;
    c->timings[2] = t23;
    c->timings[3] = t03;
    prof_collect(c);
    map_step_values(plan, slot, rcol, nr, h.data(), out);
}
}  // namespace

extern "C" {

int cl_compute_states(cl_ctx* c, int n_states, int n_holes, int64_t n_atoms, int n_orb, const double* coeff,
                      const int64_t* cells, int64_t n_int, const int16_t* spec, double* out) {
    return cl::guarded(
        [&] { compute_states_impl(c, n_states, n_holes, n_atoms, n_orb, coeff, cells, n_int, spec, out); });
}

int cl_compute(cl_ctx* c, int64_t n_int, const int16_t* spec, double* out) {
    return cl::guarded([&] { compute_impl(c, n_int, spec, out, 0xFF); });
}

int cl_compute_rounds(cl_ctx* c, int64_t n_int, const int16_t* spec, int round_mask, double* out) {
    return cl::guarded([&] {
        if (round_mask < 0 || round_mask > 0xFF) cl::fail(CL_ERR_ARGUMENT, "round mask must be within 0..255");
        compute_impl(c, n_int, spec, out, round_mask);
    });
}

int cl_compute_shard(cl_ctx* c, int64_t n_int, const int16_t* spec, int shard, int n_shards, double* out) {
    return cl::guarded([&] { compute_impl(c, n_int, spec, out, 0xFF, shard, n_shards); });
}

int cl_set_profiling(cl_ctx* c, int enable) {
    return cl::guarded([&] {
        check_ctx(c);
        CL_CUDA(cudaStreamSynchronize(c->stream));
        prof_collect(c);
        c->profiling = enable != 0;
        if (c->profiling) {
            std::fill(std::begin(c->prof_ms), std::end(c->prof_ms), 0.0);
            std::fill(std::begin(c->prof_bytes), std::end(c->prof_bytes), 0.0);
            std::fill(std::begin(c->prof_launches), std::end(c->prof_launches), (int64_t)0);
        }
    });
}

int cl_kernel_profile(cl_ctx* c, double ms[CL_NUM_KCLASS], int64_t launches[CL_NUM_KCLASS],
                      double bytes[CL_NUM_KCLASS]) {
    return cl::guarded([&] {
        check_ctx(c);
        CL_CUDA(cudaStreamSynchronize(c->stream));
        prof_collect(c);
        for (int k = 0; k < CL_NUM_KCLASS; ++k) {
            if (ms) ms[k] = c->prof_ms[k];
            if (launches) launches[k] = c->prof_launches[k];
            if (bytes) bytes[k] = c->prof_bytes[k];
        }
    });
}

int cl_potentials(cl_ctx* c, double* out) {
    return cl::guarded([&] {
        check_ctx(c);
        check_kernel(c);
        if (c->n_states == 0) cl::fail(CL_ERR_STATE, "no states loaded (call cl_set_states)");
        if (!out) cl::fail(CL_ERR_ARGUMENT, "null output");
        const int n = c->n_states;
        const long long As = c->n_sorted;
        std::vector<int2> fl(n);
        for (int s = 0; s < n; ++s) fl[s] = make_int2(s, s);
        DevBuf<cx<double>> rho, V;
        rho.alloc((size_t)n * As);
        V.alloc((size_t)n * As);
        CL_CUDA(cudaEventRecord(c->ev[0], c->stream));
        pair_densities(c, fl, rho.p);
        CL_CUDA(cudaEventRecord(c->ev[1], c->stream));
        run_transforms(c, rho.p, As, n, V.p, As, false);
        CL_CUDA(cudaEventRecord(c->ev[2], c->stream));
        std::vector<cx<double>> h((size_t)n * As);
        CL_CUDA(cudaMemcpyAsync(h.data(), V.p, h.size() * sizeof(cx<double>), cudaMemcpyDeviceToHost, c->stream));
        CL_CUDA(cudaStreamSynchronize(c->stream));
        for (int s = 0; s < n; ++s)
            for (long long a = 0; a < c->n_atoms; ++a) out[(size_t)s * c->n_atoms + a] = h[(size_t)s * As + c->atom_slot[a]].re;
        float t01, t12;
        CL_CUDA(cudaEventElapsedTime(&t01, c->ev[0], c->ev[1]));
        CL_CUDA(cudaEventElapsedTime(&t12, c->ev[1], c->ev[2]));
        prof_collect(c);
        c->timings[0] = t01;
        c->timings[1] = t12;
        c->timings[2] = 0;
        c->timings[3] = t01 + t12;
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// Prepared requests and graph-captured batches
// ---------------------------------------------------------------------------------------
struct cl_request {
    cl_ctx* ctx = nullptr;
    int64_t n_int = 0;
    std::vector<cl::PlanStep> plan;
    std::vector<int> slot, rcol;
    int nl = 0, nr = 0;
    PairSetup ps;
    DevBuf<int> ridx;
    DevBuf<cx<double>> rho, V;
    DevBuf<double> o4;
    double* o4_host = nullptr;  // pinned
    bool warm = false;
    int n_shards = 1;  // out entries of other shards' steps are zero
    ~cl_request() {
        if (o4_host) cudaFreeHost(o4_host);
    }
};

struct cl_batch {
    std::vector<cl_request*> reqs;
    cudaStream_t master = nullptr;
    cudaEvent_t fork = nullptr, t0 = nullptr, t1 = nullptr;
    std::vector<cudaEvent_t> joins;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    double last_ms = 0;
    // per-launch event pairs captured into the graph for requests whose context profiles
    std::vector<std::vector<cl_ctx::ProfEntry>> prof;
    std::vector<cudaEvent_t> prof_events;
    ~cl_batch() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (auto e : prof_events) cudaEventDestroy(e);
        for (auto e : joins) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        if (t0) cudaEventDestroy(t0);
        if (t1) cudaEventDestroy(t1);
        if (master) cudaStreamDestroy(master);
    }
};

namespace {

// Stream-ordered work of a prepared request: no allocation, no host synchronisation, no
// pageable copies -- it can be captured.
void request_enqueue(cl_request* r) {
    cl_ctx* c = r->ctx;
    if (r->nl == 0) return;  // a shard without densities
    const long long As = c->n_sorted;
    pair_launch(c, r->ps, r->rho.p);
    const bool v32 = v_fp32(c);
    run_transforms(c, r->rho.p, As, r->nl, r->V.p, As, v32);
    gram(c, r->V.p, v32, As, r->nl, r->rho.p, rho_bytes(c) == sizeof(cx<float>), As, r->ridx.p, r->nr, As, r->o4.p);
    CL_CUDA(cudaMemcpyAsync(r->o4_host, r->o4.p, sizeof(double) * (4 * (size_t)r->nl * r->nr + 1),
                            cudaMemcpyDeviceToHost, c->stream));
}

void request_finish(cl_request* r, double* out) {
    if (r->n_shards > 1) std::memset(out, 0, sizeof(double) * 2 * (size_t)r->n_int);
    if (r->nl == 0) return;
    check_gram_slot(r->o4_host[4 * (size_t)r->nl * r->nr]);
    map_step_values(r->plan, r->slot, r->rcol, r->nr, r->o4_host, out);
}

}  // namespace

extern "C" {

int cl_request_create(cl_ctx* c, int64_t n_int, const int16_t* spec, cl_request** out) {
    return cl_request_create_shard(c, n_int, spec, 0, 1, out);
}

int cl_request_create_shard(cl_ctx* c, int64_t n_int, const int16_t* spec, int shard, int n_shards,
                            cl_request** out) {
    if (out) *out = nullptr;
    cl_request* r = nullptr;
    int st = cl::guarded([&] {
        check_ctx(c);
        check_kernel(c);
        if (!out) cl::fail(CL_ERR_ARGUMENT, "null output pointer");
        if (c->n_states == 0) cl::fail(CL_ERR_STATE, "no states loaded (call cl_set_states)");
        if (n_int <= 0 || !spec) cl::fail(CL_ERR_ARGUMENT, "invalid integral list");
        r = new cl_request();
        r->ctx = c;
        r->n_int = n_int;
        std::vector<std::array<int16_t, 4>> specs((size_t)n_int);
        for (int64_t i = 0; i < n_int; ++i)
            for (int k = 0; k < 4; ++k) specs[i][k] = spec[4 * i + k];
        r->plan = shard_steps(cl::orient_steps(c->n_states, specs), c->n_states, shard, n_shards);
        r->n_shards = n_shards;
        if (r->plan.empty()) {  // a shard without densities: runs produce zeros
            *out = r;
            return;
        }
        const int P = c->n_states * (c->n_states + 1) / 2;
        std::vector<int> is_left(P, 0), is_right(P, 0);
        r->slot.assign(P, -1);
        r->rcol.assign(P, -1);
        for (const auto& s : r->plan) {
            is_left[s.left.product] = 1;
            is_right[s.right.product] = 1;
        }
        std::vector<int> prods, rights;
        for (int p = 0; p < P; ++p)
            if (is_left[p]) { r->slot[p] = (int)prods.size(); prods.push_back(p); }
        r->nl = (int)prods.size();
        for (int p = 0; p < P; ++p)
            if (is_right[p] && r->slot[p] < 0) { r->slot[p] = (int)prods.size(); prods.push_back(p); }
        for (int p = 0; p < P; ++p)
            if (is_right[p]) { r->rcol[p] = (int)rights.size(); rights.push_back(r->slot[p]); }
        r->nr = (int)rights.size();
        std::vector<int2> fl(prods.size());
        for (size_t i = 0; i < prods.size(); ++i) {
            int a, b;
            cl::product_states(prods[i], &a, &b);
            fl[i] = make_int2(a - 1, b - 1);
        }
        const long long As = c->n_sorted;
        pair_setup(c, fl, r->ps);
        r->ridx.upload(rights.data(), rights.size(), c->stream);
        r->rho.alloc((size_t)prods.size() * As);
        r->V.alloc((size_t)r->nl * As);
        r->o4.alloc((size_t)4 * r->nl * r->nr + 1);
        CL_CUDA(cudaMallocHost(&r->o4_host, sizeof(double) * (4 * (size_t)r->nl * r->nr + 1)));
        tc_reserve(c, r->nl, r->nr, As, v_fp32(c), rho_bytes(c) == sizeof(cx<float>));
        CL_CUDA(cudaStreamSynchronize(c->stream));
        *out = r;
    });
    if (st != CL_OK) delete r;
    return st;
}

void cl_request_destroy(cl_request* r) {
    if (!r) return;
    cudaSetDevice(r->ctx->device);
    delete r;
}

int cl_request_run(cl_request* r, double* out) {
    return cl::guarded([&] {
        if (!r || !out) cl::fail(CL_ERR_ARGUMENT, "null argument");
        check_ctx(r->ctx);
        request_enqueue(r);
        CL_CUDA(cudaStreamSynchronize(r->ctx->stream));
        prof_collect(r->ctx);
        r->warm = true;
        request_finish(r, out);
    });
}

int cl_batch_create(cl_request** reqs, int n, cl_batch** out) {
    if (out) *out = nullptr;
    cl_batch* b = nullptr;
    int st = cl::guarded([&] {
        if (!reqs || n <= 0 || !out) cl::fail(CL_ERR_ARGUMENT, "invalid batch");
        const int dev = reqs[0]->ctx->device;
        for (int i = 0; i < n; ++i) {
            if (!reqs[i]) cl::fail(CL_ERR_ARGUMENT, "null request");
            if (reqs[i]->ctx->device != dev) cl::fail(CL_ERR_ARGUMENT, "all requests of a batch must share one device");
            for (int j = 0; j < i; ++j)
                if (reqs[j]->ctx == reqs[i]->ctx)
                    cl::fail(CL_ERR_ARGUMENT, "requests of one batch need distinct contexts (one stream each)");
        }
        CL_CUDA(cudaSetDevice(dev));
        b = new cl_batch();
        b->reqs.assign(reqs, reqs + n);
        CL_CUDA(cudaStreamCreateWithFlags(&b->master, cudaStreamNonBlocking));
        CL_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
        CL_CUDA(cudaEventCreate(&b->t0));
        CL_CUDA(cudaEventCreate(&b->t1));
        b->joins.resize(n);
        for (auto& e : b->joins) CL_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        *out = b;
    });
    if (st != CL_OK) delete b;
    return st;
}

void cl_batch_destroy(cl_batch* b) {
    if (!b) return;
    if (!b->reqs.empty()) cudaSetDevice(b->reqs[0]->ctx->device);
    delete b;
}

int cl_batch_run(cl_batch* b, double** outs) {
    return cl::guarded([&] {
        if (!b || !outs) cl::fail(CL_ERR_ARGUMENT, "null argument");
        CL_CUDA(cudaSetDevice(b->reqs[0]->ctx->device));
        if (!b->exec) {
            // one eager run of every request sizes every buffer and sets every kernel
            // attribute; then the whole batch is captured once as parallel branches
            for (cl_request* r : b->reqs)
                if (!r->warm) {
                    request_enqueue(r);
                    CL_CUDA(cudaStreamSynchronize(r->ctx->stream));
                    prof_collect(r->ctx);
                    r->warm = true;
                }
            // contexts that profile record their launch events inside the graph
            b->prof.assign(b->reqs.size(), {});
            for (size_t i = 0; i < b->reqs.size(); ++i) {
                cl_ctx* c = b->reqs[i]->ctx;
                if (c->profiling) {
                    c->prof_sink = &b->prof[i];
                    c->prof_owned = &b->prof_events;
                }
            }
            CL_CUDA(cudaStreamBeginCapture(b->master, cudaStreamCaptureModeRelaxed));
            CL_CUDA(cudaEventRecord(b->fork, b->master));
            for (size_t i = 0; i < b->reqs.size(); ++i) {
                cl_request* r = b->reqs[i];
                CL_CUDA(cudaStreamWaitEvent(r->ctx->stream, b->fork, 0));
                request_enqueue(r);
                CL_CUDA(cudaEventRecord(b->joins[i], r->ctx->stream));
                CL_CUDA(cudaStreamWaitEvent(b->master, b->joins[i], 0));
            }
            CL_CUDA(cudaStreamEndCapture(b->master, &b->graph));
            for (cl_request* r : b->reqs) {
                r->ctx->prof_sink = nullptr;
                r->ctx->prof_owned = nullptr;
            }
            CL_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
        }
        CL_CUDA(cudaEventRecord(b->t0, b->master));
        CL_CUDA(cudaGraphLaunch(b->exec, b->master));
        CL_CUDA(cudaEventRecord(b->t1, b->master));
        CL_CUDA(cudaStreamSynchronize(b->master));
        float ms = 0;
        CL_CUDA(cudaEventElapsedTime(&ms, b->t0, b->t1));
        b->last_ms = ms;
        for (size_t i = 0; i < b->reqs.size(); ++i) {
            cl_ctx* c = b->reqs[i]->ctx;
            if (!c->profiling) continue;
            for (const auto& e : b->prof[i]) {
                float kms = 0;
                CL_CUDA(cudaEventElapsedTime(&kms, e.a, e.b));
                c->prof_ms[e.cls] += kms;
                c->prof_bytes[e.cls] += e.bytes;
                c->prof_launches[e.cls] += 1;
            }
        }
        for (size_t i = 0; i < b->reqs.size(); ++i) request_finish(b->reqs[i], outs[i]);
    });
}

int cl_batch_last_ms(cl_batch* b, double* ms) {
    return cl::guarded([&] {
        if (!b || !ms) cl::fail(CL_ERR_ARGUMENT, "null argument");
        *ms = b->last_ms;
    });
}

int cl_autotune_report(char* buf, int64_t len, int64_t* needed) {
    // precision and grid of a tuning key: "fp32" / "fp64" on the real grid, "fp32 sub-lattice" /
    // "fp64 sub-lattice" on the virtual grid of the sub-lattice forms
    const auto form_name = [](int f) {
        static const char* n[4] = {"fp64", "fp32", "fp64 sub-lattice", "fp32 sub-lattice"};
        return n[f & 3];
    };
    return cl::guarded([&] {
        static const char* names[clp::kNumPasses] = {"x_forward", "y_forward", "z_pass",   "y_inverse",
                                                     "x_inverse", "xy_forward", "xy_inverse"};
        std::string out;
        {
            std::lock_guard<std::mutex> g(g_tune_mu);
            for (const auto& kv : g_tune) {
                char line[256];
                const char* pn = names[kv.first.pass];
                if (kv.first.pass == clp::kXYFwd || kv.first.pass == clp::kXYInv) {
                    const char* ch = kv.second.v.split ? "fused plane pass" : "separate passes";
                    if (kv.second.candidates == 0)
                        std::snprintf(line, sizeof line, "%s %s %dx%dx%d: %s, from CL_TUNE_FILE\n", pn,
                                      form_name(kv.first.fp32), kv.first.nx, kv.first.ny, kv.first.nz, ch);
                    else
                        std::snprintf(line, sizeof line,
                                      "%s %s %dx%dx%d: %s, 2 candidates, fused %.4f ms, separate %.4f ms\n", pn,
                                      form_name(kv.first.fp32), kv.first.nx, kv.first.ny, kv.first.nz, ch,
                                      kv.second.ms, kv.second.ms_default);
                    out += line;
                    continue;
                }
                const char* pr = form_name(kv.first.fp32);
                const char* sp = kv.second.v.split ? "swapped" : "balanced";
                const char* ln = kv.second.v.half ? "half" : "default";
                const char* pd = kv.second.v.pad ? ", padded tile" : "";
                if (kv.second.candidates == 0)
                    std::snprintf(line, sizeof line, "%s %s %dx%dx%d: split %s, lines %s%s, from CL_TUNE_FILE\n", pn,
                                  pr, kv.first.nx, kv.first.ny, kv.first.nz, sp, ln, pd);
                else
                    std::snprintf(line, sizeof line,
                                  "%s %s %dx%dx%d: split %s, lines %s%s, %d candidates, %.4f ms (default %.4f ms)\n",
                                  pn, pr, kv.first.nx, kv.first.ny, kv.first.nz, sp, ln, pd, kv.second.candidates,
                                  kv.second.ms, kv.second.ms_default);
                out += line;
            }
        }
        if (needed) *needed = (int64_t)out.size() + 1;
        if (buf && len > 0) {
            const size_t n = std::min<size_t>(out.size(), (size_t)len - 1);
            std::memcpy(buf, out.data(), n);
            buf[n] = 0;
        }
    });
}

int cl_form_info(cl_ctx* c, int info[8]) {
    return cl::guarded([&] {
        check_ctx(c);
        if (!info) cl::fail(CL_ERR_ARGUMENT, "null output");
        const Sublattice& sl = c->sl;
        info[0] = sl.active ? 1 : 0;
        info[1] = sl.active ? sl.m : 0;
        info[2] = sl.active ? sl.S : 0;
        info[3] = sl.active && sl.zb ? 1 : 0;
        for (int d = 0; d < 3; ++d) info[4 + d] = sl.active ? sl.pad[d] : 0;
        info[7] = sl.active ? sl.table.nh : 0;
    });
}

int cl_last_timings(cl_ctx* c, double t[4]) {
    return cl::guarded([&] {
        if (!c || !t) cl::fail(CL_ERR_ARGUMENT, "null argument");
        for (int i = 0; i < 4; ++i) t[i] = c->timings[i];
    });
}

int cl_fft3d(int nx, int ny, int nz, int batch, int sign, int fp32, double* data) {
    return cl::guarded([&] {
        if (nx <= 0 || ny <= 0 || nz <= 0 || batch <= 0 || !data || (sign != -1 && sign != 1))
            cl::fail(CL_ERR_ARGUMENT, "invalid FFT arguments");
        cl_ctx* raw = nullptr;
        if (cl_create(&raw, nx, ny, nz, 1, 1, 1, fp32 ? CL_MODE_FP32_ROUNDS : CL_MODE_FP64_PLAIN) != CL_OK)
            cl::fail(CL_ERR_ARGUMENT, "%s", cl_last_error());
        std::unique_ptr<cl_ctx> c(raw);
        const long long M = c->M;
        const size_t n = (size_t)M * batch;
        DevBuf<cx<double>> d64;
        d64.upload(reinterpret_cast<const cx<double>*>(data), n, c->stream);
        auto run = [&](auto tag) {
            using T = decltype(tag);
            DevBuf<cx<T>> dT;
            cx<T>* buf;
            if constexpr (sizeof(T) == 4) {
                dT.alloc(n);
                clk::k_narrow<float><<<grid_for((long long)n), 256, 0, c->stream>>>(d64.p, dT.p, (long long)n);
                CL_LAUNCHED();
                buf = dT.p;
            } else {
                buf = d64.p;
            }
            const Axis& X = c->ax[0];
            const Axis& Y = c->ax[1];
            const Axis& Z = c->ax[2];
            const cx<T>* twx = sizeof(T) == 4 ? (const cx<T>*)X.tw32.p : (const cx<T>*)X.tw64.p;
            const cx<T>* twy = sizeof(T) == 4 ? (const cx<T>*)Y.tw32.p : (const cx<T>*)Y.tw64.p;
            const cx<T>* twz = sizeof(T) == 4 ? (const cx<T>*)Z.tw32.p : (const cx<T>*)Z.tw64.p;
            const int nrows = ny * nz;
            const XTile xt = x_tile<T>(nx, nrows);
            const LTile yt = l_tile<T>(ny, false);
            const LTile zt = l_tile<T>(nz, false);
            const int xblocks = (nrows + xt.rows - 1) / xt.rows;
            const int ychunks = (nx + yt.W - 1) / yt.W;
            const long long nxy = (long long)nx * ny;
            const long long zblocks = (nxy + zt.W - 1) / zt.W;
            // the x and y passes take the grid index from blockIdx.y (at most 65535): slices of grids
            for (int b0 = 0; b0 < batch; b0 += 65535) {
                const int nb = std::min(65535, batch - b0);
                cx<T>* slice = buf + (long long)b0 * M;
                if (sign < 0) {
                    ensure_smem(clk::k_xpass<-1, T>, xt.smem);
                    ensure_smem(clk::k_ypass<-1, T>, yt.smem);
                    clk::k_xpass<-1, T><<<dim3(xblocks, nb), 256, xt.smem, c->stream>>>(slice, M, X.plan, twx, nx,
                                                                                       nrows, xt.rows, xt.ld);
                    CL_LAUNCHED();
                    clk::k_ypass<-1, T><<<dim3(ychunks * nz, nb), 256, yt.smem, c->stream>>>(slice, M, Y.plan, twy,
                                                                                            nx, ny, yt.W, ychunks);
                    CL_LAUNCHED();
                } else {
                    ensure_smem(clk::k_xpass<+1, T>, xt.smem);
                    ensure_smem(clk::k_ypass<+1, T>, yt.smem);
                    clk::k_xpass<+1, T><<<dim3(xblocks, nb), 256, xt.smem, c->stream>>>(slice, M, X.plan, twx, nx,
                                                                                       nrows, xt.rows, xt.ld);
                    CL_LAUNCHED();
                    clk::k_ypass<+1, T><<<dim3(ychunks * nz, nb), 256, yt.smem, c->stream>>>(slice, M, Y.plan, twy,
                                                                                            nx, ny, yt.W, ychunks);
                    CL_LAUNCHED();
                }
            }
            ensure_smem(clk::k_zpass<T>, zt.smem);
            clk::k_zpass<T><<<(unsigned)zblocks, 256, zt.smem, c->stream>>>(buf, M, Z.plan, twz, nullptr, nxy, nz,
                                                                             zt.W, batch, sign);
            CL_LAUNCHED();
            if constexpr (sizeof(T) == 4) {
                clk::k_widen<float><<<grid_for((long long)n), 256, 0, c->stream>>>(dT.p, d64.p, (long long)n);
                CL_LAUNCHED();
            }
            CL_CUDA(cudaMemcpyAsync(data, d64.p, n * sizeof(cx<double>), cudaMemcpyDeviceToHost, c->stream));
            CL_CUDA(cudaStreamSynchronize(c->stream));
        };
        if (fp32)
            run(float{});
        else
            run(double{});
    });
}

}  // extern "C"
