// FP64 tensor-core Gram over atoms for FP32 operands (FP32 potentials and pair densities).
//
// The reductions of CoulombCalculator::calculate (CoulombCalculator.cpp:165-172) restricted to
// atom cells and batched over every (left, right) pair of a request, as in gram_tc.cuh:
//   C = A . B^T,  A rows = {Re V_l, Im V_l},  B rows = {Re rho_r, Im rho_r},  K = atoms,
// here with FP64 products and FP64 sums on the FP64 tensor cores (mma.sync m8n8k4 .f64): the
// FP32 operands are widened exactly, so the only rounding left is that of FP64 accumulation.
//
// A block takes up to 64 left and 64 right densities (a 128 x 128 tile of C) and an atom range,
// in chunks of 32 atoms:
//   copy     8-byte cp.async of the chunk's raw complex values into one of two raw slots, a
//            chunk ahead ([density][36] complex float; thread e takes element e + 256 j, atom
//            e % 32 of density e / 32: 256 contiguous bytes a warp);
//   widen    each thread widens the elements it copied itself into the FP64 stage of the next
//            chunk ([density][36] complex double; the pitch of 36 puts the 16 lanes of a
//            fragment load on distinct banks);
//   multiply 8 warps in a 2 x 4 grid over the C tiles of 8 x 8: warp (wr, wc) holds the tiles
//            (wr + 2a, wc + 4b); per k-step of 4 atoms it loads one A fragment per row tile and
//            one B fragment per column tile and issues one mma per tile.
// One barrier per chunk separates the widening of chunk c + 1 from the reads of chunk c - 1's
// stage.  Left densities are staged at [0, nA4), right ones at [nA4, nA4 + nB4), each count
// rounded up to 4 with zero rows, so every fragment of a partial 8-row tile reads staged zeros.
#pragma once

#include <cstdint>

#include "fft.cuh"

namespace clk {
namespace dm {

constexpr int TILE = 128;          // C rows (left re/im rows) and columns per block
constexpr int KC = 32;             // atoms per chunk
constexpr int PITCH = KC + 4;      // complex elements per staged density
constexpr int THREADS = 256;
constexpr int MAX_DENS = TILE;     // staged densities per block (64 left + 64 right, rounded)

struct GramArgs {
    const float2* V;      // left densities: V[l * v_stride + atom]
    long long v_stride;
    const float2* rho;    // right densities: rho[(ridx ? ridx[r] : r) * r_stride + atom]
    long long r_stride;
    const int* ridx;
    int nl, nr;
    long long na;               // atoms
    long long atoms_per_split;  // a multiple of KC
    int nd_max;                 // staged densities of the largest block (nA4 + nB4)
    double* out4;               // out4[l][r] += {ac, bd, ad, bc}
};

__host__ __device__ constexpr size_t smem_bytes(int nd_max) {
    return (size_t)nd_max * PITCH * (2 * 16 + 2 * 8) + sizeof(void*) * MAX_DENS;
}

__device__ __forceinline__ void mma_f64(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}
__device__ __forceinline__ void cp_async8_zfill(void* dst, const void* src, bool in) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(in ? 8u : 0u) : "memory");
}

__global__ void __launch_bounds__(THREADS, 1) k_gram_dmma(const GramArgs g) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* stage = reinterpret_cast<double2*>(smem_raw);                 // [2][nd_max][PITCH]
    float2* raw = reinterpret_cast<float2*>(stage + 2 * g.nd_max * PITCH);  // [2][nd_max][PITCH]
    const float2** src_tab = reinterpret_cast<const float2**>(raw + 2 * g.nd_max * PITCH);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * TILE, n0 = blockIdx.y * TILE;
    const int la0 = m0 / 2, rb0 = n0 / 2;
    const int nA = min(TILE / 2, g.nl - la0), nB = min(TILE / 2, g.nr - rb0);
    const int nA4 = (nA + 3) & ~3, nB4 = (nB + 3) & ~3;
    const int nd = nA4 + nB4;
    const int ta = (2 * nA + 7) / 8, tb = (2 * nB + 7) / 8;  // 8-row tiles of C
    const long long k_begin = (long long)blockIdx.z * g.atoms_per_split;
    const long long k_end = min(g.na, k_begin + g.atoms_per_split);
    const int nc = (int)((k_end - k_begin + KC - 1) / KC);

    for (int i = tid; i < nd; i += THREADS) {
        const float2* p = nullptr;
        if (i < nA) {
            p = g.V + (long long)(la0 + i) * g.v_stride;
        } else if (i >= nA4 && i < nA4 + nB) {
            const int r = rb0 + (i - nA4);
            p = g.rho + (long long)(g.ridx ? g.ridx[r] : r) * g.r_stride;
        }
        src_tab[i] = p;  // null: a zero row
    }
    __syncthreads();

    // this thread's elements of a chunk: e = tid + 256 j < nd * KC
    const auto issue = [&](int c) {
        float2* slot = raw + (c & 1) * g.nd_max * PITCH;
        const long long k0 = k_begin + (long long)c * KC;
        for (int e = tid; e < nd * KC; e += THREADS) {
            const int i = e / KC, k = e % KC;
            const float2* p = src_tab[i];
            const bool in = p != nullptr && k0 + k < k_end;
            cp_async8_zfill(slot + i * PITCH + k, in ? p + k0 + k : g.V, in);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    const auto widen_chunk = [&](int c) {
        const float2* slot = raw + (c & 1) * g.nd_max * PITCH;
        double2* st = stage + (c & 1) * g.nd_max * PITCH;
        for (int e = tid; e < nd * KC; e += THREADS) {
            const int i = e / KC, k = e % KC;
            const float2 v = slot[i * PITCH + k];
            st[i * PITCH + k] = make_double2((double)v.x, (double)v.y);
        }
    };

    // warp grid 2 x 4 over the C tiles
    const int wr = warp & 1, wc = warp >> 1;
    const int grp = lane >> 2, tig = lane & 3;
    double acc[8][4][2];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;

    if (nc > 0) {
        issue(0);
        if (nc > 1) issue(1);
        if (nc > 1)
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        else
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        widen_chunk(0);
    }
    __syncthreads();
#pragma unroll 1
    for (int c = 0; c < nc; ++c) {
        if (c + 1 < nc) {
            asm volatile("cp.async.wait_group 0;" ::: "memory");  // chunk c + 1 (this thread's copies)
            widen_chunk(c + 1);
            if (c + 2 < nc) issue(c + 2);  // into the raw slot of chunk c, widened last iteration
        }
        const double2* st = stage + (c & 1) * g.nd_max * PITCH;
#pragma unroll 2
        for (int ks = 0; ks < KC / 4; ++ks) {
            const int k = ks * 4 + tig;
            double af[8], bf[4];
#pragma unroll
            for (int a = 0; a < 8; ++a) {
                const int ti = wr + 2 * a;
                const int row = ti * 8 + grp;  // re/im row of left density row / 2 (< nA4)
                af[a] = 0.0;
                if (ti < ta) {
                    const double2 v = st[(row >> 1) * PITCH + k];
                    af[a] = (row & 1) ? v.y : v.x;
                }
            }
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int tj = wc + 4 * b;
                const int col = tj * 8 + grp;  // re/im row of right density col / 2 (< nB4)
                bf[b] = 0.0;
                if (tj < tb) {
                    const double2 v = st[(nA4 + (col >> 1)) * PITCH + k];
                    bf[b] = (col & 1) ? v.y : v.x;
                }
            }
#pragma unroll
            for (int a = 0; a < 8; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b)
                    if (wr + 2 * a < ta && wc + 4 * b < tb) mma_f64(acc[a][b], af[a], bf[b]);
        }
        __syncthreads();  // stage c & 1 is rewritten by the widening of chunk c + 2
    }

#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int ti = wr + 2 * a, tj = wc + 4 * b;
            if (ti >= ta || tj >= tb) continue;
            const int R = m0 + ti * 8 + grp;
            const int l = R >> 1, pa = R & 1;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int Cg = n0 + tj * 8 + 2 * tig + h;
                const int r = Cg >> 1, pc = Cg & 1;
                if (l < g.nl && r < g.nr) {
                    const int qi = (pa == pc) ? pa : 2 + pa;  // ac, bd, ad, bc
                    atomicAdd(g.out4 + ((long long)l * g.nr + r) * 4 + qi, acc[a][b][h]);
                }
            }
        }
}

}  // namespace dm
}  // namespace clk
