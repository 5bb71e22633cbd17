// Register-resident two-factor line FFTs for the column passes (y and z).
//
// A line of N = R1*R2 points is transformed as two Stockham stages whose butterflies live in
// registers; the only shared-memory traffic is one exchange between the stages:
//   phase A  thread t < R2 of a line loads x[t + R2 j], j < R1, straight from HBM and does an
//            R1-point DFT; outputs go to shared memory at t*R1 + r;
//   phase B  thread j < R1 reads positions j + r*R1, r < R2, multiplies by W_N^(r j) and does
//            an R2-point DFT; its outputs are X[j + r*R1] in natural order.
// Tiles hold L adjacent columns (consecutive x, or consecutive xy positions for z), so every
// global access of a warp covers whole 128-byte lines.
//
// The z pass of a round fuses forward transform, x Khat_kappa and inverse transform: after
// phase B a thread holds X[j + r*R1], which is exactly the input of the first stage of an
// inverse transform planned as (R2, R1); the Khat values of those positions stay in
// registers for all densities of the block.  Each density costs one HBM read, one HBM write
// and two shared-memory exchanges.
#pragma once

#include "fft.cuh"

namespace clk {

template <int A, int B>
struct cmax {
    static constexpr int value = A > B ? A : B;
};

// ---------------------------------------------------------------------------------------
// z pass: forward FFT along z, x Khat, inverse FFT along z; block = L adjacent xy columns,
// densities [blockIdx.y * per, ...).
// ---------------------------------------------------------------------------------------
template <typename T, int R1, int R2, int L>
__global__ void __launch_bounds__(L * cmax<R1, R2>::value)
    k_zconv_rf(cx<T>* __restrict__ buf, long long stride, const cx<T>* __restrict__ tw_g,
               const T* __restrict__ khat, long long nxy, int np) {
    constexpr int N = R1 * R2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* tw = reinterpret_cast<cx<T>*>(smem_raw);
    cx<T>* s0 = tw + N;
    cx<T>* s1 = s0 + N * L;
    const int line = threadIdx.x % L;
    const int q = threadIdx.x / L;
    const long long c = (long long)blockIdx.x * L + line;
    const bool valid = c < nxy;
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = tw_g[i];
    T kv[R2];
#pragma unroll
    for (int r = 0; r < R2; ++r) kv[r] = (q < R1 && valid) ? khat[(long long)(q + r * R1) * nxy + c] : T(0);
    __syncthreads();
    const int per = (np + gridDim.y - 1) / gridDim.y;
    const int p_begin = blockIdx.y * per, p_end = min(np, p_begin + per);
    for (int p = p_begin; p < p_end; ++p) {
        cx<T>* base = buf + (long long)p * stride + c;
        if (q < R2) {
            cx<T> v[R1];
#pragma unroll
            for (int j = 0; j < R1; ++j) v[j] = valid ? base[(long long)(q + R2 * j) * nxy] : mk(T(0), T(0));
            dft<R1, -1>(v);
#pragma unroll
            for (int r = 0; r < R1; ++r) s0[(q * R1 + r) * L + line] = v[r];
        }
        __syncthreads();
        if (q < R1) {
            cx<T> u[R2];
#pragma unroll
            for (int r = 0; r < R2; ++r) u[r] = s0[(q + r * R1) * L + line];
#pragma unroll
            for (int r = 1; r < R2; ++r) u[r] = cmul(u[r], tw[r * q]);
            dft<R2, -1>(u);
#pragma unroll
            for (int r = 0; r < R2; ++r) u[r] = mk(u[r].re * kv[r], u[r].im * kv[r]);
            dft<R2, +1>(u);
#pragma unroll
            for (int r = 0; r < R2; ++r) s1[(q * R2 + r) * L + line] = u[r];
        }
        __syncthreads();
        if (q < R2) {
            cx<T> w[R1];
#pragma unroll
            for (int r = 0; r < R1; ++r) w[r] = s1[(q + r * R2) * L + line];
#pragma unroll
            for (int r = 1; r < R1; ++r) w[r] = cmulc(w[r], tw[r * q]);
            dft<R1, +1>(w);
            if (valid) {
#pragma unroll
                for (int r = 0; r < R1; ++r) base[(long long)(q + R2 * r) * nxy] = w[r];
            }
        }
    }
}

// ---------------------------------------------------------------------------------------
// y pass (one direction): block = L adjacent x of one z-plane, densities
// [blockIdx.y * per, ...).
// ---------------------------------------------------------------------------------------
template <int S, typename T, int R1, int R2, int L>
__global__ void __launch_bounds__(L * cmax<R1, R2>::value)
    k_ycol_rf(cx<T>* __restrict__ buf, long long stride, const cx<T>* __restrict__ tw_g, int nx, int ny,
              int xchunks, int np) {
    constexpr int N = R1 * R2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* tw = reinterpret_cast<cx<T>*>(smem_raw);
    cx<T>* s0 = tw + N;
    const int line = threadIdx.x % L;
    const int q = threadIdx.x / L;
    const int xc = blockIdx.x % xchunks, z = blockIdx.x / xchunks;
    const int x = xc * L + line;
    const bool valid = x < nx;
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = tw_g[i];
    __syncthreads();
    const int per = (np + gridDim.y - 1) / gridDim.y;
    const int p_begin = blockIdx.y * per, p_end = min(np, p_begin + per);
    for (int p = p_begin; p < p_end; ++p) {
        cx<T>* base = buf + (long long)p * stride + (long long)z * nx * ny + x;
        if (q < R2) {
            cx<T> v[R1];
#pragma unroll
            for (int j = 0; j < R1; ++j) v[j] = valid ? base[(long long)(q + R2 * j) * nx] : mk(T(0), T(0));
            dft<R1, S>(v);
#pragma unroll
            for (int r = 0; r < R1; ++r) s0[(q * R1 + r) * L + line] = v[r];
        }
        __syncthreads();
        if (q < R1) {
            cx<T> u[R2];
#pragma unroll
            for (int r = 0; r < R2; ++r) u[r] = s0[(q + r * R1) * L + line];
#pragma unroll
            for (int r = 1; r < R2; ++r) u[r] = S < 0 ? cmul(u[r], tw[r * q]) : cmulc(u[r], tw[r * q]);
            dft<R2, S>(u);
            if (valid) {
#pragma unroll
                for (int r = 0; r < R2; ++r) base[(long long)(q + r * R1) * nx] = u[r];
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------
// Host-side dispatch: calls f(SplitTag<R1, R2>{}) for a length with a compiled two-factor
// split (factors are register codelets 2..16, as balanced as possible); false otherwise.
// ---------------------------------------------------------------------------------------
template <int A, int B>
struct SplitTag {
    static constexpr int r1 = A, r2 = B;
};

template <typename F>
bool with_split2(int n, F&& f) {
    switch (n) {
#define CLK_SPLIT(N, A, B) \
    case N: f(SplitTag<A, B>{}); return true;
        CLK_SPLIT(16, 4, 4)
        CLK_SPLIT(20, 4, 5)
        CLK_SPLIT(24, 4, 6)
        CLK_SPLIT(25, 5, 5)
        CLK_SPLIT(27, 3, 9)
        CLK_SPLIT(30, 5, 6)
        CLK_SPLIT(32, 4, 8)
        CLK_SPLIT(36, 6, 6)
        CLK_SPLIT(40, 8, 5)
        CLK_SPLIT(45, 5, 9)
        CLK_SPLIT(48, 6, 8)
        CLK_SPLIT(50, 5, 10)
        CLK_SPLIT(54, 6, 9)
        CLK_SPLIT(60, 6, 10)
        CLK_SPLIT(64, 8, 8)
        CLK_SPLIT(72, 8, 9)
        CLK_SPLIT(75, 5, 15)
        CLK_SPLIT(80, 8, 10)
        CLK_SPLIT(81, 9, 9)
        CLK_SPLIT(90, 9, 10)
        CLK_SPLIT(96, 8, 12)
        CLK_SPLIT(100, 10, 10)
        CLK_SPLIT(108, 9, 12)
        CLK_SPLIT(120, 10, 12)
        CLK_SPLIT(128, 8, 16)
        CLK_SPLIT(135, 9, 15)
        CLK_SPLIT(144, 12, 12)
        CLK_SPLIT(150, 10, 15)
        CLK_SPLIT(160, 10, 16)
        CLK_SPLIT(180, 12, 15)
        CLK_SPLIT(192, 12, 16)
        CLK_SPLIT(225, 15, 15)
        CLK_SPLIT(240, 15, 16)
        CLK_SPLIT(256, 16, 16)
#undef CLK_SPLIT
        default: return false;
    }
}

}  // namespace clk
