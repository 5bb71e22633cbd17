// Device kernels of the Coulomb-integral path (sm_100a).
//
// Data layout in HBM
//   grid buffers   [density][z][y][x]   cx<T>, x fastest (T = double for the plain form,
//                                        float for the FP32 form)
//   pair densities [density][atom]      cx<double>, atoms sorted by grid cell
//   potentials     [density][atom]      cx<double>, accumulated over the 8 rounds
//   Ghat           [(nz+1)][(ny+1)][(nx+1)] double (DCT-I of the kernel octant)
//   Khat_kappa     [z][y][x] T           Ghat folded for round kappa, divided by 8M
//
// One round kappa of the convolution for every density is five passes:
//   k_xfwd   scatter atoms -> rows, x conj(phase_kappa), FFT along x     (reads atoms only)
//   k_ypass  FFT along y
//   k_zpass  FFT along z, x Khat_kappa, inverse FFT along z             (Khat tile reused
//                                                                        for all densities)
//   k_ypass  inverse FFT along y
//   k_xinv   inverse FFT along x, x phase_kappa, accumulate V at atoms  (writes atoms only)
#pragma once

#include "fft.cuh"

namespace clk {

constexpr double kE2_4PE0 = 14.39963737103201;  // e^2/(4 pi eps0) in eV*A (src/base.hpp:28)

struct RoundPhase {
    const cx<double>* px;  // exp(i pi x / nx)
    const cx<double>* py;
    const cx<double>* pz;
    int kx, ky, kz;
};

__device__ __forceinline__ cx<double> round_phase(const RoundPhase& rp, int x, int y, int z) {
    cx<double> p = mk(1.0, 0.0);
    if (rp.kz) p = rp.pz[z];
    if (rp.ky) p = cmul(rp.py[y], p);
    if (rp.kx) p = cmul(rp.px[x], p);
    return p;
}

template <typename T>
__device__ __forceinline__ cx<T> narrow(cx<double> v) {
    return mk(static_cast<T>(v.re), static_cast<T>(v.im));
}
template <typename T>
__device__ __forceinline__ cx<double> widen(cx<T> v) {
    return mk(static_cast<double>(v.re), static_cast<double>(v.im));
}
template <typename T>
__device__ __forceinline__ cx<T> czero() {
    return mk(T(0), T(0));
}

// ---------------------------------------------------------------------------------------
// Coulomb kernel on the octant: Interaction.hpp:32-51 with Interaction.cpp:8-39.
// ---------------------------------------------------------------------------------------
struct KernelModel {
    double dielectric;
    double onsite;
    int thomas_fermi;
    double r_tf, q_tf;
};

static __global__ void k_kernel_octant(double* __restrict__ G, int n1x, int n1y, int n1z, double sx, double sy,
                                double sz, KernelModel km) {
    const long long total = (long long)n1x * n1y * n1z;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(idx % n1x);
        const int iy = (int)((idx / n1x) % n1y);
        const int iz = (int)(idx / ((long long)n1x * n1y));
        // same association as the reference, with no contraction into FMA
        const double z = __dmul_rn((double)iz, sz), z2 = __dmul_rn(z, z);
        const double y = __dmul_rn((double)iy, sy), y2z2 = __dadd_rn(z2, __dmul_rn(y, y));
        const double x = __dmul_rn((double)ix, sx);
        const double r = sqrt(__dadd_rn(y2z2, __dmul_rn(x, x)));
        double eps = km.dielectric;
        if (km.thomas_fermi && r < km.r_tf)
            eps = km.dielectric * (km.q_tf * km.r_tf / (sinh(km.q_tf * (km.r_tf - r)) + km.q_tf * r));
        G[idx] = idx == 0 ? km.onsite : kE2_4PE0 / (eps * r);
    }
}

// ---------------------------------------------------------------------------------------
// REDFT00 along one axis (FFTW's DCT-I definition):
//   Y_k = X_0 + (-1)^k X_{L-1} + 2 sum_{j=1}^{L-2} X_j cos(pi j k / (L-1)),  L = points.
// Line l = (o, i) has element j at (o*L + j)*inner + i.  A block handles `nl` consecutive
// lines staged in shared memory; ctab[t] = cos(pi t / (L-1)), t < 2(L-1).
// ---------------------------------------------------------------------------------------
static __global__ void k_dct1(const double* __restrict__ in, double* __restrict__ out, int L, long long inner,
                       long long nlines, int nl, const double* __restrict__ ctab) {
    extern __shared__ double dsm[];
    const int np = L - 1;  // N'
    double* ct = dsm;       // 2*np
    double* s = dsm + 2 * np;  // [L][nl]
    for (int t = threadIdx.x; t < 2 * np; t += blockDim.x) ct[t] = ctab[t];
    const long long l0 = (long long)blockIdx.x * nl;
    const int cnt = (int)min((long long)nl, nlines - l0);
    const bool rows = (inner == 1);
    for (int e = threadIdx.x; e < L * nl; e += blockDim.x) {
        int j, l;
        if (rows) { l = e / L; j = e - l * L; } else { j = e / nl; l = e - j * nl; }
        double v = 0.0;
        if (l < cnt) {
            const long long line = l0 + l;
            const long long o = line / inner, i = line - o * inner;
            v = in[(o * L + j) * inner + i];
        }
        s[j * nl + l] = v;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < L * nl; e += blockDim.x) {
        int k, l;
        if (rows) { l = e / L; k = e - l * L; } else { k = e / nl; l = e - k * nl; }
        if (l >= cnt) continue;
        double acc = 0.0;
        int t = k % (2 * np);
        int idx = t;
        for (int j = 1; j < np; ++j) {
            acc += s[j * nl + l] * ct[idx];
            idx += t;
            if (idx >= 2 * np) idx -= 2 * np;
        }
        double y = s[l] + ((k & 1) ? -s[np * nl + l] : s[np * nl + l]) + 2.0 * acc;
        const long long line = l0 + l;
        const long long o = line / inner, i = line - o * inner;
        out[(o * L + k) * inner + i] = y;
    }
}

// Khat_kappa(x,y,z) = Ghat(f(2x+kx), f(2y+ky), f(2z+kz)) / (8M), f(q) = min(q, 2n-q)
// (CoulombCalculator.cpp:130-144 and :102).
template <typename T>
__global__ void k_khat(const double* __restrict__ ghat, int nx, int ny, int nz, int kx, int ky, int kz,
                       double denom, T* __restrict__ out) {
    const long long M = (long long)nx * ny * nz;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < M;
         idx += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(idx % nx);
        const int y = (int)((idx / nx) % ny);
        const int z = (int)(idx / ((long long)nx * ny));
        const int qx = 2 * x + kx, qy = 2 * y + ky, qz = 2 * z + kz;
        const int fx = min(qx, 2 * nx - qx), fy = min(qy, 2 * ny - qy), fz = min(qz, 2 * nz - qz);
        out[idx] = static_cast<T>(ghat[((long long)fz * (ny + 1) + fy) * (nx + 1) + fx] / denom);
    }
}

// ---------------------------------------------------------------------------------------
// Pair densities at atoms: rho_p(a) = sum_o conj(c_fl[a][o]) c_fr[a][o]  (Product.cpp:16-30).
// coeff is [state][atom][orb] with n_atoms atoms a state; the atom of sorted slot i is
// orig[i], or i itself when orig is null (coefficients already in sorted order: the library
// stores them so, see k_gather_atoms).
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ long long atom_of(const int* __restrict__ orig, long long i) {
    return orig ? (long long)orig[i] : i;
}

// dst[i][o] = src[orig[i]][o] for the n_sorted slots and n_orb orbitals of one state: the
// coefficients of a state in the cell-sorted order of the atoms (consecutive threads on
// consecutive orbitals: whole 16-byte values, rows of n_orb contiguous on both sides).
static __global__ void __launch_bounds__(256) k_gather_atoms(const cx<double>* __restrict__ src,
                                                     const int* __restrict__ orig, long long n_sorted, int n_orb,
                                                     cx<double>* __restrict__ dst) {
    const long long n = n_sorted * n_orb;
    for (long long e = blockIdx.x * 256LL + threadIdx.x; e < n; e += (long long)gridDim.x * 256) {
        const long long i = e / n_orb;
        const int o = (int)(e - i * n_orb);
        dst[e] = src[(long long)orig[i] * n_orb + o];
    }
}
__device__ __forceinline__ void pd_cp_async16(void* smem_dst, const void* gmem_src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(
                     static_cast<unsigned>(__cvta_generic_to_shared(smem_dst))),
                 "l"(gmem_src));
}

// Products of one left state, up to kPairSeg of them: rho_prod[k] = conj(c_left) c_right[k].
constexpr int kPairSeg = 4;
struct PairSeg {
    int left, cnt;              // indices into the used-state list; products in this segment
    int right[kPairSeg];        // right state of each product (used-state index)
    int prod[kPairSeg];         // product index (row of rho)
};

// rho is written in the working precision RT of the form (rounded once from the FP64 sum).
template <typename RT>
__global__ void __launch_bounds__(256) k_pair_density(const cx<double>* __restrict__ coeff, long long n_atoms,
                                                    int n_orb, const int* __restrict__ orig, long long n_sorted,
                                                    const PairSeg* __restrict__ segs, int n_segs,
                                                    const int* __restrict__ states, int n_used, int chunk,
                                                    cx<RT>* __restrict__ rho) {
    // A block stages the coefficients of `chunk` consecutive (cell-sorted) atoms for every used
    // state in shared memory -- each coefficient is read from HBM once, a warp copying one
    // (state, atom) row of orbitals with 16-byte cp.async -- and forms every product of the
    // chunk while the next chunk is being copied (two stages).  A thread takes one segment
    // (a left state and up to kPairSeg right states) at one atom, so each orbital of the left
    // state is read from shared memory once for all the segment's products.  Atom pitch `os`
    // is odd (in 16-byte units), so threads on consecutive atoms hit distinct banks.
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int os = n_orb | 1;
    const int stage = n_used * chunk * os;
    cx<double>* sc0 = reinterpret_cast<cx<double>*>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    const long long n_chunks = (n_sorted + chunk - 1) / chunk;
    const auto load = [&](long long ci, cx<double>* sc) {
        const long long i0 = ci * chunk;
        const int ca = (int)min((long long)chunk, n_sorted - i0);
        for (int row = warp; row < n_used * ca; row += nwarps) {
            const int su = row / ca, a = row - su * ca;
            const cx<double>* src = coeff + ((long long)states[su] * n_atoms + atom_of(orig, i0 + a)) * n_orb;
            cx<double>* dst = sc + (su * chunk + a) * os;
            for (int k = lane; k < n_orb; k += 32) pd_cp_async16(dst + k, src + k);
        }
        asm volatile("cp.async.commit_group;\n" ::);
    };
    long long ci = blockIdx.x;
    int buf = 0;
    if (ci < n_chunks) load(ci, sc0);
    for (; ci < n_chunks; ci += gridDim.x) {
        cx<double>* sc = sc0 + buf * stage;
        const long long next = ci + gridDim.x;
        if (next < n_chunks) {
            load(next, sc0 + (buf ^ 1) * stage);
            asm volatile("cp.async.wait_group 1;\n" ::);
        } else {
            asm volatile("cp.async.wait_group 0;\n" ::);
        }
        __syncthreads();
        const long long i0 = ci * chunk;
        const int ca = (int)min((long long)chunk, n_sorted - i0);
        for (int e = threadIdx.x; e < n_segs * ca; e += blockDim.x) {
            const int q = e / ca, a = e - q * ca;
            const PairSeg& sg = segs[q];
            const cx<double>* L = sc + (sg.left * chunk + a) * os;
            const cx<double>* R[kPairSeg];
#pragma unroll
            for (int j = 0; j < kPairSeg; ++j) R[j] = sc + ((j < sg.cnt ? sg.right[j] : sg.left) * chunk + a) * os;
            cx<double> acc[kPairSeg];
#pragma unroll
            for (int j = 0; j < kPairSeg; ++j) acc[j] = mk(0.0, 0.0);
            // four orbitals in flight: the chain of shared-memory loads, not their bandwidth,
            // bounds this loop at the occupancy the staged chunks allow
#pragma unroll 4
            for (int k = 0; k < n_orb; ++k) {
                const cx<double> l = L[k];
#pragma unroll
                for (int j = 0; j < kPairSeg; ++j)
                    if (j < sg.cnt) {
                        const cx<double> r = R[j][k];
                        acc[j] = acc[j] + mk(l.re * r.re + l.im * r.im, l.re * r.im - l.im * r.re);
                    }
            }
#pragma unroll
            for (int j = 0; j < kPairSeg; ++j)
                if (j < sg.cnt) rho[(long long)sg.prod[j] * n_sorted + i0 + a] = narrow<RT>(acc[j]);
        }
        __syncthreads();  // the stage is refilled by the load issued next iteration
        buf ^= 1;
    }
}

// ---------------------------------------------------------------------------------------
// Pair densities for requests over at most 12 states, summed in FP64 and rounded once to the
// form's precision RT; products t = i (i + 1) / 2 + j of states i >= j (ascending order) go to
// rows prod[t] of rho.
// ---------------------------------------------------------------------------------------
constexpr int kPairRegStates = 12;
struct PairTri {
    int states[kPairRegStates];                             // used states, ascending (coefficient rows)
    int prod[kPairRegStates * (kPairRegStates + 1) / 2];    // row of product (i, j), i >= j; -1: not requested
};

// Block = 64 atoms x PARTS warp pairs: the products are split into PARTS parts (t mod PARTS),
// each taken by the two warps of one part (the part is uniform over a warp: no predicated work;
// at most 10 FP64 sums per thread: 4 parts up to 8 states, 8 parts up to 12).  The coefficients
// are staged through shared memory four orbitals at a time: per (state, atom) the 64 contiguous
// bytes of those orbitals are copied with 16-byte cp.async (coalesced; the next slice is in
// flight while this one is used), at an 80-byte pitch per atom so that threads on consecutive
// atoms read distinct banks.  Every coefficient leaves HBM once and each part reads the slice
// from shared memory.  The barriers are in the kernel body, reached by every thread; only the
// arithmetic is specialised per part.
constexpr int kPairAtoms = 64;      // atoms per block and step
constexpr int kPairOrbSlice = 4;    // orbitals per stage
__host__ __device__ constexpr int pair_stage_elems(int ns) { return ns * kPairAtoms * (kPairOrbSlice + 1); }
__host__ __device__ constexpr int pair_parts(int ns) { return ns <= 8 ? 4 : 8; }
__host__ __device__ constexpr int pair_min_blocks(int ns) { return ns <= 8 ? 2 : 1; }  // <= 128 registers

template <int NS, int PARTS, int H>
__device__ __forceinline__ void pair_accumulate(const cx<double>* __restrict__ st, int a, double* ar, double* ai) {
    constexpr int NT = NS * (NS + 1) / 2;
#pragma unroll
    for (int o = 0; o < kPairOrbSlice; ++o) {
        cx<double> c[NS];
#pragma unroll
        for (int i = 0; i < NS; ++i) c[i] = st[(i * kPairAtoms + a) * (kPairOrbSlice + 1) + o];
#pragma unroll
        for (int i = 0; i < NS; ++i)
#pragma unroll
            for (int j = 0; j <= i; ++j) {
                const int t = i * (i + 1) / 2 + j;
                if (t % PARTS == H && t < NT) {  // compile-time after unrolling
                    ar[t / PARTS] += c[i].re * c[j].re + c[i].im * c[j].im;  // conj(c_i) c_j
                    ai[t / PARTS] += c[i].re * c[j].im - c[i].im * c[j].re;
                }
            }
    }
}

template <int NS, int PARTS, int H, typename RT>
__device__ __forceinline__ void pair_store(const PairTri& tri, const double* ar, const double* ai, long long slot,
                                           long long n_sorted, cx<RT>* __restrict__ rho) {
    constexpr int NT = NS * (NS + 1) / 2, NH = (NT - H + PARTS - 1) / PARTS;
#pragma unroll
    for (int k = 0; k < NH; ++k) {
        const int p = tri.prod[PARTS * k + H];
        if (p >= 0) rho[(long long)p * n_sorted + slot] = narrow<RT>(mk(ar[k], ai[k]));
    }
}

// The part `part` of the thread, dispatched to the compile-time part H.
template <int NS, int PARTS, int H = 0>
__device__ __forceinline__ void pair_accumulate_part(int part, const cx<double>* __restrict__ st, int a, double* ar,
                                                     double* ai) {
    if constexpr (H < PARTS) {
        if (part == H)
            pair_accumulate<NS, PARTS, H>(st, a, ar, ai);
        else
            pair_accumulate_part<NS, PARTS, H + 1>(part, st, a, ar, ai);
    }
}
template <int NS, int PARTS, typename RT, int H = 0>
__device__ __forceinline__ void pair_store_part(int part, const PairTri& tri, const double* ar, const double* ai,
                                                long long slot, long long n_sorted, cx<RT>* __restrict__ rho) {
    if constexpr (H < PARTS) {
        if (part == H)
            pair_store<NS, PARTS, H, RT>(tri, ar, ai, slot, n_sorted, rho);
        else
            pair_store_part<NS, PARTS, RT, H + 1>(part, tri, ar, ai, slot, n_sorted, rho);
    }
}

template <int NS, typename RT>
__global__ void __launch_bounds__(kPairAtoms * pair_parts(NS), pair_min_blocks(NS))
    k_pair_density_reg(const cx<double>* __restrict__ coeff, long long n_atoms, int n_orb,
                       const int* __restrict__ orig, long long n_sorted, const PairTri tri,
                       cx<RT>* __restrict__ rho) {
    constexpr int PARTS = pair_parts(NS), THREADS = kPairAtoms * PARTS;
    constexpr int NT = NS * (NS + 1) / 2, NHM = (NT + PARTS - 1) / PARTS;
    constexpr int SE = pair_stage_elems(NS);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<double>* sm = reinterpret_cast<cx<double>*>(smem_raw);
    const int part = threadIdx.x / kPairAtoms;
    const int a = threadIdx.x % kPairAtoms;
    const int n_slices = (n_orb + kPairOrbSlice - 1) / kPairOrbSlice;
    // the copies of one stage: NS states x 64 atoms x 4 orbitals, 16 bytes each
    const auto issue = [&](long long a0, int slice, cx<double>* st) {
        const int na = (int)min((long long)kPairAtoms, n_sorted - a0);
        for (int e = threadIdx.x; e < NS * kPairAtoms * kPairOrbSlice; e += THREADS) {
            const int o = e % kPairOrbSlice, r = e / kPairOrbSlice;
            const int at = r % kPairAtoms, i = r / kPairAtoms;
            const int orb = slice * kPairOrbSlice + o;
            cx<double>* dst = st + (i * kPairAtoms + at) * (kPairOrbSlice + 1) + o;
            if (at < na && orb < n_orb)
                pd_cp_async16(dst, coeff + ((long long)tri.states[i] * n_atoms + atom_of(orig, a0 + at)) * n_orb + orb);
            else
                *dst = mk(0.0, 0.0);
        }
        asm volatile("cp.async.commit_group;\n" ::);
    };
    const long long gstep = (long long)gridDim.x * kPairAtoms;
    long long a0 = (long long)blockIdx.x * kPairAtoms;
    int stage = 0;
    if (a0 < n_sorted) issue(a0, 0, sm);
    for (; a0 < n_sorted; a0 += gstep) {
        double ar[NHM], ai[NHM];
#pragma unroll
        for (int k = 0; k < NHM; ++k) ar[k] = ai[k] = 0.0;
        for (int sl = 0; sl < n_slices; ++sl) {
            // next stage: this group's next slice, or the next group's first one
            const long long na0 = sl + 1 < n_slices ? a0 : a0 + gstep;
            if (na0 < n_sorted) {
                issue(na0, sl + 1 < n_slices ? sl + 1 : 0, sm + (stage ^ 1) * SE);
                asm volatile("cp.async.wait_group 1;\n" ::);
            } else {
                asm volatile("cp.async.wait_group 0;\n" ::);
            }
            __syncthreads();
            pair_accumulate_part<NS, PARTS>(part, sm + stage * SE, a, ar, ai);
            __syncthreads();  // the stage is refilled two slices on
            stage ^= 1;
        }
        const long long slot = a0 + a;
        if (slot < n_sorted) pair_store_part<NS, PARTS, RT>(part, tri, ar, ai, slot, n_sorted, rho);
    }
}

// ---------------------------------------------------------------------------------------
// Pair densities for requests over more than 8 states, in tiles of 4 x 4 states.  The used
// states, ascending and padded to a multiple of 4 (padding rows are zero), form blocks of 4;
// tile (bi, bj), bi >= bj, holds the products conj(c_i) c_j, i = 4 bi + u, j = 4 bj + v, of
// which prod[i * ns_pad + j] names the density row (2 p, or 2 p + 1 where the row is the
// conjugate, conj(c_j) c_i; -1: not requested).  Only tiles with a requested product are
// listed.  A block stages every orbital of its A atoms for every used state in shared memory
// ([state][atom][orbital], odd atom pitch: consecutive atoms on distinct banks; each
// coefficient leaves HBM once), then each thread takes (tile, atom) work items: per orbital
// 8 coefficient loads feed 16 complex FP64 products (the FP64 pipe, not shared memory, bounds
// it), and the sums are rounded once to RT on the store.
// ---------------------------------------------------------------------------------------
constexpr int kPairTile = 4;

template <typename RT>
__global__ void __launch_bounds__(256, 2) k_pair_density_tile(const cx<double>* __restrict__ coeff,
                                                             long long n_atoms, int n_orb,
                                                             const int* __restrict__ orig, long long n_sorted,
                                                             const int* __restrict__ states, int ns_pad,
                                                             const int* __restrict__ tiles, int n_tiles,
                                                             const int* __restrict__ prod, int A,
                                                             cx<RT>* __restrict__ rho) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<double>* sm = reinterpret_cast<cx<double>*>(smem_raw);
    const int P = n_orb | 1;
    const int items = n_tiles * A;
    const long long AP = (long long)A * P;
    for (long long a0 = (long long)blockIdx.x * A; a0 < n_sorted; a0 += (long long)gridDim.x * A) {
        const int na = (int)min((long long)A, n_sorted - a0);
        for (int e = threadIdx.x; e < ns_pad * A * n_orb; e += blockDim.x) {
            const int o = e % n_orb, r = e / n_orb;
            const int at = r % A, i = r / A;
            cx<double>* dst = sm + (i * A + at) * P + o;
            const int st = states[i];
            if (st >= 0 && at < na)
                pd_cp_async16(dst, coeff + ((long long)st * n_atoms + atom_of(orig, a0 + at)) * n_orb + o);
            else
                *dst = mk(0.0, 0.0);
        }
        asm volatile("cp.async.commit_group;\n" ::);
        asm volatile("cp.async.wait_group 0;\n" ::);
        __syncthreads();
        for (int w = threadIdx.x; w < items; w += blockDim.x) {
            const int t = w / A, a = w - t * A;
            const int code = tiles[t];
            const int bi = code & 0xffff, bj = code >> 16;
            const cx<double>* L = sm + (long long)(kPairTile * bi) * AP + (long long)a * P;
            const cx<double>* R = sm + (long long)(kPairTile * bj) * AP + (long long)a * P;
            double ar[kPairTile * kPairTile], ai[kPairTile * kPairTile];
#pragma unroll
            for (int k = 0; k < kPairTile * kPairTile; ++k) ar[k] = ai[k] = 0.0;
#pragma unroll 1
            for (int o = 0; o < n_orb; ++o) {
                cx<double> l[kPairTile], r[kPairTile];
#pragma unroll
                for (int u = 0; u < kPairTile; ++u) {
                    l[u] = L[u * AP + o];
                    r[u] = R[u * AP + o];
                }
#pragma unroll
                for (int u = 0; u < kPairTile; ++u)
#pragma unroll
                    for (int v = 0; v < kPairTile; ++v) {
                        ar[u * kPairTile + v] += l[u].re * r[v].re + l[u].im * r[v].im;  // conj(c_i) c_j
                        ai[u * kPairTile + v] += l[u].re * r[v].im - l[u].im * r[v].re;
                    }
            }
            if (a < na) {
                const long long slot = a0 + a;
#pragma unroll
                for (int u = 0; u < kPairTile; ++u)
#pragma unroll
                    for (int v = 0; v < kPairTile; ++v) {
                        const int pc = prod[(kPairTile * bi + u) * ns_pad + kPairTile * bj + v];
                        if (pc >= 0) {
                            const double im = (pc & 1) ? -ai[u * kPairTile + v] : ai[u * kPairTile + v];
                            rho[(long long)(pc >> 1) * n_sorted + slot] = narrow<RT>(mk(ar[u * kPairTile + v], im));
                        }
                    }
            }
        }
        __syncthreads();  // the stage is refilled for the next atoms
    }
}

// ---------------------------------------------------------------------------------------
// Pass 1: scatter + conj(phase) + forward FFT along x.  A block owns `rows` consecutive
// rows (row = z*ny + y); atoms of those rows are [row_ptr[r0], row_ptr[r0+rows]) in the
// cell-sorted atom list.  Densities are processed one after another by the same block.
// ---------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_xfwd(const cx<T>* __restrict__ rho, long long rho_stride,
                                             const int* __restrict__ row_ptr, const int* __restrict__ cell,
                                             cx<T>* __restrict__ out, long long out_stride, FftPlan plan,
                                             const cx<T>* __restrict__ tw_g, RoundPhase rp, int nx, int ny,
                                             int nrows, int rows, int ld, int np) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* tw = reinterpret_cast<cx<T>*>(smem_raw);
    cx<T>* a = tw + nx;
    cx<T>* b = a + (size_t)nx * ld;
    const int r0 = blockIdx.x * rows;
    const int nr = min(rows, nrows - r0);
    for (int i = threadIdx.x; i < nx; i += blockDim.x) tw[i] = tw_g[i];
    const int a0 = row_ptr[r0], a1 = row_ptr[r0 + nr];
    for (int p = 0; p < np; ++p) {
        for (int e = threadIdx.x; e < nx * ld; e += blockDim.x) a[e] = czero<T>();
        __syncthreads();
        const cx<T>* rp_ = rho + (long long)p * rho_stride;
        for (int i = a0 + threadIdx.x; i < a1; i += blockDim.x) {
            const int c = cell[i];
            const int row = c / nx, x = c - row * nx;
            const int y = row % ny, z = row / ny;
            a[x * ld + (row - r0)] = narrow<T>(cmulc(widen(rp_[i]), round_phase(rp, x, y, z)));
        }
        __syncthreads();
        const cx<T>* res = fft_lines<-1>(a, b, tw, plan, rows, ld);
        cx<T>* o = out + (long long)p * out_stride + (long long)r0 * nx;
        for (int e = threadIdx.x; e < nr * nx; e += blockDim.x) {
            const int lr = e / nx, x = e - lr * nx;
            o[e] = res[x * ld + lr];
        }
        __syncthreads();
    }
}

// Dense in-place FFT along x of whole rows (the standalone FFT entry point).
template <int S, typename T>
__global__ void __launch_bounds__(256) k_xpass(cx<T>* __restrict__ buf, long long stride, FftPlan plan,
                                              const cx<T>* __restrict__ tw_g, int nx, int nrows, int rows,
                                              int ld) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* tw = reinterpret_cast<cx<T>*>(smem_raw);
    cx<T>* a = tw + nx;
    cx<T>* b = a + (size_t)nx * ld;
    const int r0 = blockIdx.x * rows;
    const int nr = min(rows, nrows - r0);
    cx<T>* base = buf + (long long)blockIdx.y * stride + (long long)r0 * nx;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) tw[i] = tw_g[i];
    for (int e = threadIdx.x; e < rows * nx; e += blockDim.x) {
        const int lr = e / nx, x = e - lr * nx;
        a[x * ld + lr] = lr < nr ? base[e] : czero<T>();
    }
    __syncthreads();
    const cx<T>* res = fft_lines<S>(a, b, tw, plan, rows, ld);
    for (int e = threadIdx.x; e < nr * nx; e += blockDim.x) {
        const int lr = e / nx, x = e - lr * nx;
        base[e] = res[x * ld + lr];
    }
}

// ---------------------------------------------------------------------------------------
// Pass along y (or any axis with stride `step` between points and W adjacent lines):
// block = (tile of W consecutive x, one z, one density).
// ---------------------------------------------------------------------------------------
template <int S, typename T>
__global__ void __launch_bounds__(256) k_ypass(cx<T>* __restrict__ buf, long long stride, FftPlan plan,
                                              const cx<T>* __restrict__ tw_g, int nx, int ny, int W,
                                              int xchunks) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* tw = reinterpret_cast<cx<T>*>(smem_raw);
    cx<T>* a = tw + ny;
    cx<T>* b = a + (size_t)ny * W;
    const int xc = blockIdx.x % xchunks, z = blockIdx.x / xchunks;
    const int x0 = xc * W, w = min(W, nx - x0);
    cx<T>* base = buf + (long long)blockIdx.y * stride + (long long)z * nx * ny + x0;
    for (int i = threadIdx.x; i < ny; i += blockDim.x) tw[i] = tw_g[i];
    for (int e = threadIdx.x; e < ny * W; e += blockDim.x) {
        const int y = e / W, l = e - y * W;
        a[e] = l < w ? base[(long long)y * nx + l] : czero<T>();
    }
    __syncthreads();
    const cx<T>* res = fft_lines<S>(a, b, tw, plan, W, W);
    for (int e = threadIdx.x; e < ny * W; e += blockDim.x) {
        const int y = e / W, l = e - y * W;
        if (l < w) base[(long long)y * nx + l] = res[e];
    }
}

// ---------------------------------------------------------------------------------------
// Pass along z: forward FFT, x Khat_kappa (tile loaded once per block and reused for all
// densities), inverse FFT.  With khat == nullptr only the forward (S<0) or backward
// transform is done (standalone FFT).  Block = W consecutive xy positions, all z.
// ---------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_zpass(cx<T>* __restrict__ buf, long long stride, FftPlan plan,
                                              const cx<T>* __restrict__ tw_g, const T* __restrict__ khat,
                                              long long nxy, int nz, int W, int np, int sign) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* tw = reinterpret_cast<cx<T>*>(smem_raw);
    cx<T>* a = tw + nz;
    cx<T>* b = a + (size_t)nz * W;
    T* kt = reinterpret_cast<T*>(b + (size_t)nz * W);
    const long long c0 = (long long)blockIdx.x * W;
    const int w = (int)min((long long)W, nxy - c0);
    for (int i = threadIdx.x; i < nz; i += blockDim.x) tw[i] = tw_g[i];
    if (khat) {
        for (int e = threadIdx.x; e < nz * W; e += blockDim.x) {
            const int z = e / W, l = e - z * W;
            kt[e] = l < w ? khat[(long long)z * nxy + c0 + l] : T(0);
        }
    }
    // densities of this block: gridDim.y groups share the np densities
    const int per = (np + gridDim.y - 1) / gridDim.y;
    const int p_begin = blockIdx.y * per, p_end = min(np, p_begin + per);
    for (int p = p_begin; p < p_end; ++p) {
        cx<T>* base = buf + (long long)p * stride + c0;
        for (int e = threadIdx.x; e < nz * W; e += blockDim.x) {
            const int z = e / W, l = e - z * W;
            a[e] = l < w ? base[(long long)z * nxy + l] : czero<T>();
        }
        __syncthreads();
        cx<T>* res;
        if (khat) {
            res = fft_lines<-1>(a, b, tw, plan, W, W);
            for (int e = threadIdx.x; e < nz * W; e += blockDim.x) {
                const T k = kt[e];
                res[e] = mk(res[e].re * k, res[e].im * k);
            }
            __syncthreads();
            res = fft_lines<+1>(res, res == a ? b : a, tw, plan, W, W);
        } else if (sign < 0) {
            res = fft_lines<-1>(a, b, tw, plan, W, W);
        } else {
            res = fft_lines<+1>(a, b, tw, plan, W, W);
        }
        for (int e = threadIdx.x; e < nz * W; e += blockDim.x) {
            const int z = e / W, l = e - z * W;
            if (l < w) base[(long long)z * nxy + l] = res[e];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------
// Last pass: inverse FFT along x; the round's value at every atom of the rows is written to
// out[p][atom] (write-only, the pass's working precision).  k_round_sum multiplies by
// phase_kappa and adds the rounds in FP64.
// ---------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_xinv(const cx<T>* __restrict__ buf, long long stride, FftPlan plan,
                                             const cx<T>* __restrict__ tw_g, const int* __restrict__ row_ptr,
                                             const int* __restrict__ cell, cx<T>* __restrict__ out,
                                             long long o_stride, int nx, int nrows, int rows, int ld, int np) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* tw = reinterpret_cast<cx<T>*>(smem_raw);
    cx<T>* a = tw + nx;
    cx<T>* b = a + (size_t)nx * ld;
    const int r0 = blockIdx.x * rows;
    const int nr = min(rows, nrows - r0);
    for (int i = threadIdx.x; i < nx; i += blockDim.x) tw[i] = tw_g[i];
    const int a0 = row_ptr[r0], a1 = row_ptr[r0 + nr];
    for (int p = 0; p < np; ++p) {
        const cx<T>* base = buf + (long long)p * stride + (long long)r0 * nx;
        for (int e = threadIdx.x; e < rows * nx; e += blockDim.x) {
            const int lr = e / nx, x = e - lr * nx;
            a[x * ld + lr] = lr < nr ? base[e] : czero<T>();
        }
        __syncthreads();
        const cx<T>* res = fft_lines<+1>(a, b, tw, plan, rows, ld);
        cx<T>* op = out + (long long)p * o_stride;
        for (int i = a0 + threadIdx.x; i < a1; i += blockDim.x) {
            const int c = cell[i];
            const int row = c / nx, x = c - row * nx;
            op[i] = res[x * ld + (row - r0)];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------
// Round sum (CoulombCalculator.cpp:155-160, V += T . phi over the rounds): for every atom i
// and density p, V[p][i] = sum over the rounds present, in ascending kappa, of
// widen(t_kappa[p][i]) x phase_kappa(cell i), in FP64.  The rounds' values t_kappa come from the
// inverse x pass (slot s = kappa's rank among the present rounds; slot stride r_stride).  A
// thread owns one atom: its (at most 8) phases are formed once and reused for the densities
// [blockIdx.y * per, ...) of its block.
// ---------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256, 8) k_round_sum(const cx<T>* __restrict__ t, long long r_stride,
                                                  long long p_stride, int round_mask, RoundPhase base,
                                                  const int* __restrict__ cell, int nx, int ny, long long n_atoms,
                                                  cx<double>* __restrict__ V, long long v_stride, int np) {
    const int per = (np + gridDim.y - 1) / gridDim.y;
    const int p_begin = blockIdx.y * per, p_end = min(np, p_begin + per);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_atoms;
         i += (long long)gridDim.x * blockDim.x) {
        const int c = cell[i];
        const int row = c / nx, x = c - row * nx;
        const int y = row % ny, z = row / ny;
        // Only the three axis phases are kept; round r's phase is formed from them in
        // round_phase's order when it is used.  The kernel is bound by load latency, so it is
        // launched for full occupancy (32 registers a thread, eight blocks an SM): what does
        // not fit is reloaded from L1 each density, and the warps' loads in flight double
        // (measured at 128^3: 5.46 -> 4.10 ms a request; 96^3: 0.226 -> 0.203 ms).
        const cx<double> qx = base.px[x], qy = base.py[y], qz = base.pz[z];
        const auto phase = [&](int r) {
            cx<double> ph = mk(1.0, 0.0);
            if ((r >> 2) & 1) ph = qz;
            if ((r >> 1) & 1) ph = cmul(qy, ph);
            if (r & 1) ph = cmul(qx, ph);
            return ph;
        };
        for (int p = p_begin; p < p_end; ++p) {
            const cx<T>* tp = t + (long long)p * p_stride + i;
            cx<double> acc = mk(0.0, 0.0);
            long long s = 0;
#pragma unroll
            for (int r = 0; r < 8; ++r)
                if ((round_mask >> r) & 1) {
                    acc = acc + cmul(widen(tp[s]), phase(r));
                    s += r_stride;
                }
            V[(long long)p * v_stride + i] = acc;
        }
    }
}

// ---------------------------------------------------------------------------------------
// Real-space reductions in FP64 (CoulombCalculator.cpp:165-172 restricted to the atom
// cells, where the right density is non-zero): for left l and right r with V = a+ib and
// rho = c+id, out[l][r] += {sum ac, sum bd, sum ad, sum bc}; then
//   sum V rho       = (ac - bd) + i (ad + bc)
//   sum V conj(rho) = (ac + bd) + i (bc - ad).
// 64x64 (l, r) tiles, 4x4 per thread, atoms staged 16 at a time; split over atoms with one
// FP64 atomicAdd per result per block.
// ---------------------------------------------------------------------------------------
template <int IB, typename RT>
__global__ void __launch_bounds__(256) k_gram(const cx<double>* __restrict__ V, long long v_stride, int nl,
                                             const cx<RT>* __restrict__ rho, long long r_stride,
                                             const int* __restrict__ ridx, int nr, long long n_atoms,
                                             long long atoms_per_split, double* __restrict__ out) {
    // (16*IB) x (16*IB) tile of (left, right) pairs, IB x IB per thread; IB is chosen on the host
    // so the tiles waste little of a small density count.
    constexpr int TS = 16 * IB;
    __shared__ cx<double> vs[16][TS];
    __shared__ cx<double> rs[16][TS];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int l0 = blockIdx.x * TS, r0 = blockIdx.y * TS;
    const long long k_begin = (long long)blockIdx.z * atoms_per_split;
    const long long k_end = min(n_atoms, k_begin + atoms_per_split);
    double acc[IB][IB][4];
#pragma unroll
    for (int i = 0; i < IB; ++i)
#pragma unroll
        for (int j = 0; j < IB; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.0;
    for (long long k0 = k_begin; k0 < k_end; k0 += 16) {
        for (int e = threadIdx.x; e < 16 * TS; e += 256) {
            const int row = e >> 4, k = e & 15;
            const long long atom = k0 + k;
            const bool ok = atom < k_end;
            const int l = l0 + row, r = r0 + row;
            vs[k][row] = (ok && l < nl) ? V[(long long)l * v_stride + atom] : mk(0.0, 0.0);
            rs[k][row] = (ok && r < nr) ? widen(rho[(long long)ridx[r] * r_stride + atom]) : mk(0.0, 0.0);
        }
        __syncthreads();
#pragma unroll 4
        for (int k = 0; k < 16; ++k) {
            cx<double> v[IB], r[IB];
#pragma unroll
            for (int i = 0; i < IB; ++i) v[i] = vs[k][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < IB; ++j) r[j] = rs[k][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < IB; ++i)
#pragma unroll
                for (int j = 0; j < IB; ++j) {
                    acc[i][j][0] += v[i].re * r[j].re;
                    acc[i][j][1] += v[i].im * r[j].im;
                    acc[i][j][2] += v[i].re * r[j].im;
                    acc[i][j][3] += v[i].im * r[j].re;
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < IB; ++i)
#pragma unroll
        for (int j = 0; j < IB; ++j) {
            const int l = l0 + ty + 16 * i, r = r0 + tx + 16 * j;
            if (l < nl && r < nr) {
                double* o = out + ((long long)l * nr + r) * 4;
#pragma unroll
                for (int q = 0; q < 4; ++q) atomicAdd(o + q, acc[i][j][q]);
            }
        }
}

// Grid-API scatter of a dense density into the "every cell is an atom" list is the identity;
// its dot product reuses k_gram with nl = nr = 1.

// Widening / narrowing copies for the standalone FFT entry point.
template <typename T>
__global__ void k_narrow(const cx<double>* __restrict__ in, cx<T>* __restrict__ out, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = narrow<T>(in[i]);
}
template <typename T>
__global__ void k_widen(const cx<T>* __restrict__ in, cx<double>* __restrict__ out, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = widen(in[i]);
}

}  // namespace clk
