// Quadrant forward plane pass of the sub-lattice forms for 128-point FP32 planes (the 2.1M-atom
// box).
//
// A class plane of the sub-lattice virtual grid holds atoms only in its [0, 64)^2 quadrant (a
// class line of n/m points zero-padded to P = 2n/m = 128).  So the forward pass transforms y
// first -- 64 columns, half-input 128-point FFTs -- into a 128 x 64 buffer, then x in batches of
// rows, straight to HBM.  The block needs 64 KB for that buffer and 35 KB of row scratch, so two
// blocks of 256 threads share an SM and one block's barriers overlap the other's stages (the
// general plane pass holds a whole 128 x 128 plane, one block an SM).  Measured on the 2.1M-atom
// box: 0.88 ms per request against 0.94 ms for the general pass.  The inverse kept the general
// pass: a quadrant inverse (x from HBM first, half-output, then y on 64 columns) measured
// 0.94 ms against 0.90 ms, and 1.01 ms with its rows staged through shared memory.
//
// 128-point FFTs in two stages, 128 = 8 x 16 (as in plane_rf.cuh): phase A, item t < 16 reads
// points t + 16 m, does an 8-point DFT and writes output j to point t + 16 j; phase B, item
// j < 8 reads points 16 j + t, multiplies by W^(t j), does a 16-point DFT and writes output s to
// point 16 j + s, which holds frequency j + 8 s.
//
// Buffers: I[128][64] (row = y or frequency, column = x < 64), the row scratch S[32][136]
// (point n of a row at n + n / 16: the 8 lanes of a phase-B item group on distinct banks), the
// twiddles W^(t j) at [t][j].
#pragma once

#include "fft.cuh"

namespace clk {
namespace qp {

constexpr int N = 128, Q = 64, R1 = 8, R2 = 16;
constexpr int THREADS = 256;
constexpr int RB = 32;    // rows of the x stage per batch
constexpr int SP = 136;   // scratch row pitch
__host__ __device__ constexpr int spos(int n) { return n + n / 16; }
constexpr size_t SMEM = sizeof(cx<float>) * ((size_t)N * Q + (size_t)RB * SP + N);

// Forward: atoms of plane z (virtual rows z*N .. z*N + N - 1) of each density -> the plane's
// 2D spectrum in out[p][z][ky][kx].
__global__ void __launch_bounds__(THREADS, 2)
    k_qfwd(const cx<float>* __restrict__ rho, long long rho_stride, const int* __restrict__ row_ptr,
           const int* __restrict__ cell, cx<float>* __restrict__ out, long long out_stride,
           const cx<float>* __restrict__ tw_g, int np) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<float>* I = reinterpret_cast<cx<float>*>(smem_raw);
    cx<float>* S = I + N * Q;
    cx<float>* tw = S + RB * SP;
    const int tid = threadIdx.x, z = blockIdx.x;
    for (int i = tid; i < N; i += THREADS) tw[i] = tw_g[(i / R1) * (i % R1)];
    const int a0 = row_ptr[z * N], a1 = row_ptr[z * N + N];
    const bool full = (a1 - a0) == Q * Q;  // every quadrant point an atom: no zeroing needed
    const int per = (np + gridDim.y - 1) / gridDim.y;
    const int p_begin = blockIdx.y * per, p_end = min(np, p_begin + per);
    __syncthreads();
    for (int p = p_begin; p < p_end; ++p) {
        if (!full) {
            float4* I4 = reinterpret_cast<float4*>(I);
            for (int e = tid; e < Q * Q / 2; e += THREADS) I4[e] = make_float4(0.f, 0.f, 0.f, 0.f);
            __syncthreads();
        }
        const cx<float>* src = rho + (long long)p * rho_stride;
        for (int i = a0 + tid; i < a1; i += THREADS) {
            const int c = cell[i];
            const int x = c % N, y = (c / N) % N;
            if (x < Q && y < Q) I[y * Q + x] = src[i];
        }
        __syncthreads();
        // y, phase A: columns x < 64, inputs y < 64 (m < 4)
        for (int e = tid; e < Q * R2; e += THREADS) {
            const int x = e % Q, t = e / Q;
            cx<float> v[R1];
#pragma unroll
            for (int m = 0; m < R1 / 2; ++m) v[m] = I[(t + R2 * m) * Q + x];
#pragma unroll
            for (int m = R1 / 2; m < R1; ++m) v[m] = mk(0.f, 0.f);
            dft8_half_in<-1>(v);
#pragma unroll
            for (int j = 0; j < R1; ++j) I[(t + R2 * j) * Q + x] = v[j];
        }
        __syncthreads();
        // y, phase B: row 16 j + s then holds frequency ky = j + 8 s
        for (int e = tid; e < Q * R1; e += THREADS) {
            const int x = e % Q, j = e / Q;
            cx<float> u[R2];
#pragma unroll
            for (int t = 0; t < R2; ++t) u[t] = I[(R2 * j + t) * Q + x];
#pragma unroll
            for (int t = 1; t < R2; ++t) u[t] = cmul(u[t], tw[t * R1 + j]);
            dft<R2, -1>(u);
#pragma unroll
            for (int s = 0; s < R2; ++s) I[(R2 * j + s) * Q + x] = u[s];
        }
        __syncthreads();
        // x, in batches of RB rows: phase A into the scratch, phase B to HBM
        cx<float>* o = out + (long long)p * out_stride + (long long)z * N * N;
        for (int r0 = 0; r0 < N; r0 += RB) {
            for (int e = tid; e < RB * R2; e += THREADS) {
                const int t = e % R2, rr = e / R2;
                const cx<float>* row = I + (r0 + rr) * Q;
                cx<float> v[R1];
#pragma unroll
                for (int m = 0; m < R1 / 2; ++m) v[m] = row[t + R2 * m];
#pragma unroll
                for (int m = R1 / 2; m < R1; ++m) v[m] = mk(0.f, 0.f);
                dft8_half_in<-1>(v);
#pragma unroll
                for (int j = 0; j < R1; ++j) S[rr * SP + spos(t + R2 * j)] = v[j];
            }
            __syncthreads();
            for (int e = tid; e < RB * R1; e += THREADS) {
                const int j = e % R1, rr = e / R1;
                const int r = r0 + rr;
                const int ky = r / R2 + R1 * (r % R2);
                cx<float> u[R2];
#pragma unroll
                for (int t = 0; t < R2; ++t) u[t] = S[rr * SP + spos(R2 * j + t)];
#pragma unroll
                for (int t = 1; t < R2; ++t) u[t] = cmul(u[t], tw[t * R1 + j]);
                dft<R2, -1>(u);
                cx<float>* orow = o + (long long)ky * N;
#pragma unroll
                for (int s = 0; s < R2; ++s) orow[j + R1 * s] = u[s];
            }
            __syncthreads();  // the scratch is refilled by the next batch; I by the next density
        }
    }
}

}  // namespace qp
}  // namespace clk
