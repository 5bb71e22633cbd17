// cl_fft3d_noalloc: the batched 3D FFT of cl_fft3d on a caller-owned device buffer, with no
// device allocation at all.
//
// Who needs it: callers that own every byte of device memory through their own pool or
// arena (a cudaMalloc behind their back bypasses their accounting and can fail against
// their memory cap), and callers on latency-critical paths, where cudaMalloc/cudaFree may
// synchronise the whole device.  They pass the data already on the GPU; the only other
// global memory the transform needs -- its twiddle tables -- lives in a fixed array inside
// this library.
//
// The scratch: g_fft_scratch below, three tables (x, y, z) of at most kMaxAxis complex
// doubles each, 192 KiB in total.  It is a file-scope __device__ array, so every GPU that
// loads the library holds it until the process exits.  In host code its name is only a
// host-side stand-in; every call looks the device address up with cudaGetSymbolAddress on the
// current device (no allocation, no stream work), so a device reset that reloads the module
// and moves the array leaves no stale address behind.  Every call rewrites all table
// entries it reads, so nothing has to start at zero; but all calls share the one array, so
// calls that overlap on the GPU (e.g. from threads using per-thread default streams) race on
// it.
#include <algorithm>
#include <cstdint>

#include <cuda_runtime.h>

#include "coulombo_lattice.h"
#include "host/status.hpp"
#include "kernels.cuh"

namespace {

constexpr int kMaxAxis = 4096;

__device__ __align__(256) clk::cx<double> g_fft_scratch[3 * kMaxAxis];


#define NA_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t err_ = (call);                                                             \
        if (err_ != cudaSuccess)                                                               \
            cl::fail(CL_ERR_CUDA, "CUDA error %s at %s:%d: %s", cudaGetErrorName(err_), __FILE__, \
                     __LINE__, cudaGetErrorString(err_));                                      \
    } while (0)

// Device address of the scratch array on the current device.
clk::cx<double>* scratch_on_current_device() {
    void* p = nullptr;
    NA_CUDA(cudaGetSymbolAddress(&p, g_fft_scratch));
    return static_cast<clk::cx<double>*>(p);
}

// tw[t] = exp(-2 pi i t / n)
__global__ void k_fill_twiddles(clk::cx<double>* __restrict__ tw, int n) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(-2.0 * (double)t / (double)n, &s, &c);
        tw[t] = clk::mk(c, s);
    }
}

bool smooth(int n) {
    for (int p : {2, 3, 5})
        while (n % p == 0) n /= p;
    return n == 1;
}

clk::FftPlan plan_for(int n) {
    clk::FftPlan p{};
    p.n = n;
    int m = n;
    for (int r : {8, 4, 2, 3, 5})
        while (m % r == 0 && p.nst < 16) {
            p.radix[p.nst++] = r;
            m /= r;
        }
    int ns = 1;
    for (int s = 0; s < p.nst; ++s) {
        p.ns_magic[s] = clk::fdiv_magic(ns);
        ns *= p.radix[s];
    }
    return p;
}

template <typename K>
void allow_smem(K kernel, size_t bytes) {
    if (bytes > 227 * 1024) cl::fail(CL_ERR_UNSUPPORTED, "tile needs %zu bytes of shared memory", bytes);
    NA_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

template <int S>
void run(int nx, int ny, int nz, int batch, clk::cx<double>* data, const clk::cx<double>* twx,
         const clk::cx<double>* twy, const clk::cx<double>* twz) {
    using C = clk::cx<double>;
    const long long M = (long long)nx * ny * nz;
    const int nrows = ny * nz;
    // x: rows of nx points, transposed into shared memory
    int rows = std::max(1, std::min(2048 / nx, 64));
    rows = std::min(rows, nrows);
    const int ld = (rows % 2 == 0) ? rows + 1 : rows;
    const size_t xs = sizeof(C) * ((size_t)nx + 2ull * nx * ld);
    // y and z: tiles of W adjacent lines
    auto tile = [](int n) {
        int W = 8;
        while (W > 1 && sizeof(C) * ((size_t)n + 2ull * n * W) > 200 * 1024) W /= 2;
        return W;
    };
    const int wy = tile(ny), wz = tile(nz);
    const size_t ys = sizeof(C) * ((size_t)ny + 2ull * ny * wy);
    const size_t zs = sizeof(C) * ((size_t)nz + 2ull * nz * wz);
    allow_smem(clk::k_xpass<S, double>, xs);
    allow_smem(clk::k_ypass<S, double>, ys);
    allow_smem(clk::k_zpass<double>, zs);
    const clk::FftPlan px = plan_for(nx), py = plan_for(ny), pz = plan_for(nz);
    const int ychunks = (nx + wy - 1) / wy;
    const long long nxy = (long long)nx * ny;
    // the x and y passes take the grid index from blockIdx.y (at most 65535): slices of grids
    for (int b0 = 0; b0 < batch; b0 += 65535) {
        const int nb = std::min(65535, batch - b0);
        C* slice = data + (long long)b0 * M;
        clk::k_xpass<S, double><<<dim3((nrows + rows - 1) / rows, nb), 256, xs>>>(slice, M, px, twx, nx, nrows, rows,
                                                                                  ld);
        NA_CUDA(cudaGetLastError());
        clk::k_ypass<S, double><<<dim3(ychunks * nz, nb), 256, ys>>>(slice, M, py, twy, nx, ny, wy, ychunks);
        NA_CUDA(cudaGetLastError());
    }
    clk::k_zpass<double><<<(unsigned)((nxy + wz - 1) / wz), 256, zs>>>(data, M, pz, twz, nullptr, nxy, nz, wz, batch, S);
    NA_CUDA(cudaGetLastError());
}

}  // namespace

extern "C" int cl_fft3d_noalloc(int nx, int ny, int nz, int batch, int sign, double* data) {
    return cl::guarded([&] {
        if (nx <= 0 || ny <= 0 || nz <= 0 || batch <= 0 || (sign != -1 && sign != 1))
            cl::fail(CL_ERR_ARGUMENT, "invalid FFT arguments");
        if (!data) cl::fail(CL_ERR_ARGUMENT, "null data pointer");
        if (reinterpret_cast<uintptr_t>(data) % 16 != 0) cl::fail(CL_ERR_ARGUMENT, "data must be 16-byte aligned");
        const int dims[3] = {nx, ny, nz};
        for (int d = 0; d < 3; ++d) {
            if (dims[d] > kMaxAxis)
                cl::fail(CL_ERR_UNSUPPORTED,
                         "axis length %d exceeds the %d-point twiddle scratch of the allocation-free FFT", dims[d],
                         kMaxAxis);
            if (!smooth(dims[d])) cl::fail(CL_ERR_UNSUPPORTED, "FFT length %d is not a product of 2, 3 and 5", dims[d]);
        }
        if ((long long)nx * ny * nz * batch >= (1LL << 31)) cl::fail(CL_ERR_UNSUPPORTED, "too many points");
        clk::cx<double>* scratch = scratch_on_current_device();
        clk::cx<double>* tw[3] = {scratch, scratch + kMaxAxis, scratch + 2 * kMaxAxis};
        for (int d = 0; d < 3; ++d) {
            k_fill_twiddles<<<(dims[d] + 255) / 256, 256>>>(tw[d], dims[d]);
            NA_CUDA(cudaGetLastError());
        }
        clk::cx<double>* c = reinterpret_cast<clk::cx<double>*>(data);
        if (sign < 0)
            run<-1>(nx, ny, nz, batch, c, tw[0], tw[1], tw[2]);
        else
            run<+1>(nx, ny, nz, batch, c, tw[0], tw[1], tw[2]);
        NA_CUDA(cudaStreamSynchronize(0));
    });
}
