// Sub-lattice decomposition of the aperiodic convolution (the CL_MODE_*_SUBLATTICE forms).
//
// The atoms of a crystal occupy few residue classes of the grid modulo m per axis: zinc-blende
// and diamond on the a/4 grid fill 8 of the 64 classes modulo 4.  Class b (offset b in [0, m)^3)
// holds the dense sub-grid of points b + m c, c < s = n/m per axis.  The aperiodic convolution
// that the reference computes with 8 rounds of N-point FFTs (CoulombCalculator.cpp:105-163),
//     V(r) = sum_r' G(|r - r'|) rho(r'),
// restricted to atom points, is exactly
//     V_a(c') = sum_b sum_c G(b_a - b_b + m (c' - c)) rho_b(c),
// one aperiodic convolution per class pair on the sub-grids.  With zero padding to P = 2s = 2n/m
// points per axis it becomes, with unnormalised transforms,
//     A_b(q) = FFT_P(rho_b)(q)
//     u_a(q) = e^{+i pi q.b_a/n} sum_b H_{(b_a - b_b) mod m}(q) e^{-i pi q.b_b/n} A_b(q)
//     V_a(c') = IFFT_P(u_a)(c'),  c' < s,
// where H_r(q) = sum_{j in [0,m)^3} Khat(q + P j) w^{j.r}, w = e^{2 pi i/m}, and Khat(k) =
// Ghat(f(kx), f(ky), f(kz)) / (8M), f(k) = min(k, 2n - k): the kernel spectrum of the 8-round
// method (REDFT00 of the octant, CoulombCalculator.cpp:57-103, folded as at :130-144) sampled at
// all 2n frequencies per axis.  (The sub-grid kernel G(delta + m d) is the inverse 2n-point DFT
// of Khat sampled on the sub-lattice; its P-point DFT aliases the m^3 frequencies q + P j.)
//
// Work per density: S classes x P^3 points each way, against 8 rounds x n^3 -- for zinc-blende
// (S = 8, m = 4) one eighth -- and the padded halves of each axis are neither loaded nor stored.
//
// On the GPU the classes are stacked along z into a virtual grid (P, P, S*s): class b's plane cz
// is virtual plane b*s + cz, and its atoms sit at x, y < s.  The forward and inverse x and y
// passes of the 8-round forms run unchanged on that grid (rows without atoms are neither stored
// nor read); k_zmix_rf below does the z transforms and the class mixing in one pass.
#pragma once

#include "fft.cuh"
#include "kernels.cuh"
#include "rfft.cuh"

namespace clk {

constexpr int kSlMaxClasses = 8;
constexpr int kSlMaxResidues = 64;

// Residue kernels of a class set: rep[h] are the representatives (x, y, z) of the class
// differences (b_a - b_b) mod m up to sign; entry (a, b) uses H_{h(a,b)}, conjugated when the
// difference is the negative of its representative (H_{-r} = conj(H_r): Khat is real).
struct SlTable {
    int S = 0, m = 0, nh = 0;
    int rep[kSlMaxResidues][3] = {};
    int h[kSlMaxClasses * kSlMaxClasses] = {};
    int cj[kSlMaxClasses * kSlMaxClasses] = {};
};

// Builds the table for S classes with offsets off[s] (the same rule on host and device, so the
// compiled zinc-blende table below and the host's H layout agree): representatives in order of
// first appearance over (a, b) row-major, each the lexicographically smaller of r and -r.
__host__ __device__ constexpr int sl_res_id(int x, int y, int z, int m) { return (z * m + y) * m + x; }

__host__ __device__ constexpr SlTable sl_table(const int (*off)[3], int S, int m) {
    SlTable t{};
    t.S = S;
    t.m = m;
    for (int a = 0; a < S; ++a)
        for (int b = 0; b < S; ++b) {
            int r[3] = {0, 0, 0}, nr[3] = {0, 0, 0};
            for (int d = 0; d < 3; ++d) {
                r[d] = ((off[a][d] - off[b][d]) % m + m) % m;
                nr[d] = (m - r[d]) % m;
            }
            const int id = sl_res_id(r[0], r[1], r[2], m), nid = sl_res_id(nr[0], nr[1], nr[2], m);
            const int rid = id < nid ? id : nid;
            int found = -1;
            for (int h = 0; h < t.nh; ++h)
                if (sl_res_id(t.rep[h][0], t.rep[h][1], t.rep[h][2], m) == rid) found = h;
            if (found < 0) {
                found = t.nh++;
                for (int d = 0; d < 3; ++d) t.rep[found][d] = (id <= nid) ? r[d] : nr[d];
            }
            t.h[a * kSlMaxClasses + b] = found;
            t.cj[a * kSlMaxClasses + b] = (id != rid) ? 1 : 0;
        }
    return t;
}

// The zinc-blende / diamond classes on the a/4 grid in canonical order: the fcc sites, then the
// fcc sites + (1,1,1).  A structure whose classes are this set shifted by t (mod 4) -- every
// zinc-blende or diamond box, whatever the grid origin -- uses the compiled table (differences
// do not depend on t); the shift only enters the phases, through the actual offsets.
struct ZincBlende {
    static constexpr int off[8][3] = {{0, 0, 0}, {0, 2, 2}, {2, 0, 2}, {2, 2, 0},
                                      {1, 1, 1}, {1, 3, 3}, {3, 1, 3}, {3, 3, 1}};
};
__host__ __device__ constexpr SlTable zb_table() { return sl_table(ZincBlende::off, 8, 4); }

// Mixing description passed to the kernel (uniform over threads).
struct SlMix {
    int S;                                   // occupied classes (<= 8)
    int offz[kSlMaxClasses];                 // z offset of each class (z phases)
    int h[kSlMaxClasses * kSlMaxClasses];    // residue kernel of (a, b)   (generic table only)
    int cj[kSlMaxClasses * kSlMaxClasses];   // 1: conjugated              (generic table only)
};

// H_r(q) for every representative r of `t`, q over the padded grid (px, py, pz), from the raw
// REDFT00 octant ghat[(nz+1)][(ny+1)][(nx+1)] (CoulombCalculator.cpp:57-103) divided by 8M.
// Layout H[h][qz][qy][qx].  Summed in FP64 in a fixed order; rounded once to T.
struct SlRes {
    int nh, m;
    int rep[kSlMaxResidues][3];
    double wc[4], ws[4];  // w^e = cos + i sin of 2 pi e / m, e < m (m <= 4)
};

template <typename T>
__global__ void k_sl_build_h(const double* __restrict__ ghat, int nx, int ny, int nz, int px, int py, int pz,
                             SlRes res, double denom, cx<T>* __restrict__ H) {
    const long long nq = (long long)px * py * pz;
    const int m = res.m;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
         q += (long long)gridDim.x * blockDim.x) {
        const int qx = (int)(q % px);
        const long long t = q / px;
        const int qy = (int)(t % py);
        const int qz = (int)(t / py);
        for (int h = 0; h < res.nh; ++h) {
            double re = 0.0, im = 0.0;
            for (int jz = 0; jz < m; ++jz) {
                const int kz = qz + pz * jz;
                const int fz = min(kz, 2 * nz - kz);
                for (int jy = 0; jy < m; ++jy) {
                    const int ky = qy + py * jy;
                    const int fy = min(ky, 2 * ny - ky);
                    for (int jx = 0; jx < m; ++jx) {
                        const int kx = qx + px * jx;
                        const int fx = min(kx, 2 * nx - kx);
                        const double K = ghat[((long long)fz * (ny + 1) + fy) * (nx + 1) + fx] / denom;
                        const int e = (jx * res.rep[h][0] + jy * res.rep[h][1] + jz * res.rep[h][2]) % m;
                        re += K * res.wc[e];
                        im += K * res.ws[e];
                    }
                }
            }
            H[h * nq + q] = mk(T(re), T(im));
        }
    }
}

// 4-point Walsh-Hadamard transform y[c] = sum_a (-1)^popcount(c & a) x[a].
template <typename T>
__device__ __forceinline__ void wht4(const cx<T>* x, cx<T>* y) {
    const cx<T> s01 = x[0] + x[1], d01 = x[0] - x[1], s23 = x[2] + x[3], d23 = x[2] - x[3];
    y[0] = s01 + s23;
    y[1] = d01 + d23;
    y[2] = s01 - s23;
    y[3] = d01 - d23;
}

// The zinc-blende mixing in Walsh-Hadamard form.  In the canonical class order the fcc offsets
// f_0..f_3 form a group under addition mod 4 (f_a + f_b = f_{a xor b}, -f = f), so the 8 x 8
// mixing matrix is [[A, C], [B, A]] with A_ab = alpha_{a^b}, B_ab = beta_{a^b}, C_ab =
// conj(beta_{a^b}), alpha_k = H_{f_k} (real), beta_k = H_{f_k + (1,1,1)}.  The 4-point
// Walsh-Hadamard transform W (W W = 4) diagonalises such matrices: with x^ = W x per half,
//     u^_fcc = alpha^ x^_fcc + conj(beta^) x^_other,   u^_other = beta^ x^_fcc + alpha^ x^_other,
// u = W u^ / 4, alpha^ = W alpha, beta^ = W beta.  This kernel turns the raw FP64 class kernels
// (entries h of the table, e.g. alpha_k = Hraw[src[k]] conjugated if cj[k]) into
// H[c] = alpha^_c / 4 and H[4 + c] = beta^_c / 4, rounded once to T.
struct SlWht {
    int src[8], cj[8];  // raw table entry (and conjugation) of alpha_0..3, beta_0..3
};
template <typename T>
__global__ void k_sl_zb_wht(const cx<double>* __restrict__ Hraw, long long nq, SlWht w, cx<T>* __restrict__ H) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
         q += (long long)gridDim.x * blockDim.x) {
        cx<double> v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            v[k] = Hraw[w.src[k] * nq + q];
            if (w.cj[k]) v[k].im = -v[k].im;
        }
        cx<double> a[4], b[4];
        wht4(v, a);
        wht4(v + 4, b);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            H[c * nq + q] = mk(T(0.25 * a[c].re), T(0));  // alpha is real (self-conjugate residues)
            H[(4 + c) * nq + q] = mk(T(0.25 * b[c].re), T(0.25 * b[c].im));
        }
    }
}

// V[p][i] = widen(src[p][i]) for the densities p = blockIdx.y (FP32 forms: the values at the
// atoms from the inverse passes, into the FP64 potentials the reductions read).
template <typename T>
__global__ void k_sl_widen(const cx<T>* __restrict__ src, long long s_stride, cx<double>* __restrict__ dst,
                           long long d_stride, long long n) {
    const cx<T>* s = src + blockIdx.y * s_stride;
    cx<double>* d = dst + blockIdx.y * d_stride;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        d[i] = widen(s[i]);
}

// Shared-memory layout of k_zmix_rf: twiddles, z phases, xy phases of the block's columns, the
// stage exchange and the spectra being mixed.  LL = 8 L lines (class-major, column-minor);
// LPM pads the spectra so the mixing step's reads (L columns x 32/L frequencies a warp) hit
// distinct banks.
template <typename T, int R1, int R2, int L>
struct ZmixLayout {
    static constexpr int N = R1 * R2;
    static constexpr int LL = kSlMaxClasses * L;
    static constexpr int LP0 = LL;
    static constexpr int LPM = LL + L;
    static constexpr size_t off_phz = N;
    static constexpr size_t off_phxy = off_phz + 4 * (size_t)N;
    static constexpr size_t off_s0 = off_phxy + (size_t)LL;
    static constexpr size_t off_sm = off_s0 + (size_t)N * LP0;
    static constexpr size_t elems = off_sm + (size_t)N * LPM;
    static constexpr size_t smem = sizeof(cx<T>) * elems;
};

// ---------------------------------------------------------------------------------------
// z pass of the sub-lattice forms: block = L adjacent (kx, ky) columns x 8 classes x P threads
// a line; densities [blockIdx.y * per, ...).  Per density:
//   phase A   loads each class line's s = N/2 stored planes (the rest is zero padding) and does
//             the R1-point DFTs of the first stage;
//   phase B   twiddles and R2-point DFTs: line spectra in natural order, to shared memory;
//   mix       per (column, kz): the classes' spectra times their pre-phases, mixed with the
//             residue kernels H, times the post-phases (u_a above);
//   phase B'  first stage of the inverse transform (R2-point inverse DFTs);
//   phase A'  twiddles and R1-point inverse DFTs; only the outputs z < N/2 are stored.
// ZB: the compiled zinc-blende table, whose eight H values per point stay in registers for all
// densities; otherwise the table of `mix` with H read through L1 per density.
// Requires R1 even (the stored half of a line is then j < R1/2 in every phase-A item).
// ---------------------------------------------------------------------------------------
template <typename T, int R1, int R2, int L, bool ZB>
__global__ void __launch_bounds__(kSlMaxClasses * L * ColShape<R1, R2>::P, 1)
    k_zmix_rf(cx<T>* __restrict__ buf, long long stride, const cx<T>* __restrict__ tw_g,
              const cx<T>* __restrict__ H, const cx<T>* __restrict__ phxy_g, const cx<T>* __restrict__ phz_g,
              const SlMix mix, long long nxy, int np) {
    static_assert(R1 % 2 == 0, "the stored half of a line must be whole R1/2 runs");
    using Sh = ColShape<R1, R2>;
    using Lay = ZmixLayout<T, R1, R2, L>;
    constexpr int N = R1 * R2, P = Sh::P, IA = Sh::IA, IB = Sh::IB, LL = Lay::LL, LP0 = Lay::LP0,
                  LPM = Lay::LPM, HALF = R1 / 2;
    constexpr int NT = LL * P;
    constexpr int NPT = (L * N + NT - 1) / NT;  // mixing points per thread
    constexpr int sz = N / 2;                    // stored planes per class
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* base_s = reinterpret_cast<cx<T>*>(smem_raw);
    cx<T>* tw = base_s;
    cx<T>* phz = base_s + Lay::off_phz;
    cx<T>* phxy = base_s + Lay::off_phxy;
    cx<T>* s0 = base_s + Lay::off_s0;
    cx<T>* sm = base_s + Lay::off_sm;
    const int S = ZB ? kSlMaxClasses : mix.S;
    const int line = threadIdx.x % LL;
    const int qt = threadIdx.x / LL;
    const int cls = line / L, col = line % L;
    const long long c = (long long)blockIdx.x * L + col;
    const bool valid = c < nxy && cls < S;
    const long long h_stride = (long long)N * nxy;

    for (int i = threadIdx.x; i < N; i += NT) tw[i] = tw_g[i];
    for (int i = threadIdx.x; i < 4 * N; i += NT) phz[i] = phz_g[i];
    for (int i = threadIdx.x; i < LL; i += NT) {
        const int s = i / L;
        const long long cc = (long long)blockIdx.x * L + (i % L);
        phxy[i] = (s < S && cc < nxy) ? phxy_g[(long long)s * nxy + cc] : mk(T(0), T(0));
    }
    // the residue kernels of this thread's mixing points, for every density (zinc-blende)
    constexpr int NHR = ZB ? 8 : 1;
    cx<T> hv[NPT][NHR];
#pragma unroll
    for (int j = 0; j < NPT; ++j) {
        const int i = threadIdx.x + j * NT;
        const long long cc = (long long)blockIdx.x * L + (i % L);
        const int k = i / L;
#pragma unroll
        for (int h = 0; h < NHR; ++h)
            hv[j][h] = (ZB && i < L * N && cc < nxy) ? H[h * h_stride + (long long)k * nxy + cc] : mk(T(0), T(0));
    }
    __syncthreads();

    const int per = (np + gridDim.y - 1) / gridDim.y;
    const int p_begin = blockIdx.y * per, p_end = min(np, p_begin + per);
    // a class line's stored planes z < N/2 are cls*sz + z of the virtual grid
    const auto load = [&](int p, cx<T>(&v)[IA][HALF]) {
        const cx<T>* src = buf + (long long)p * stride + (long long)cls * sz * nxy + c;
#pragma unroll
        for (int a = 0; a < IA; ++a) {
            const int q = qt + a * P;
#pragma unroll
            for (int j = 0; j < HALF; ++j)
                v[a][j] = (valid && q < R2) ? src[(long long)(q + R2 * j) * nxy] : mk(T(0), T(0));
        }
    };
    cx<T> v[IA][HALF], vn[IA][HALF];
    if (p_begin < p_end) load(p_begin, v);
    for (int p = p_begin; p < p_end; ++p) {
        cx<T>* dst = buf + (long long)p * stride + (long long)cls * sz * nxy + c;
        if (p + 1 < p_end) load(p + 1, vn);
        // phase A: R1-point DFTs, upper half of the inputs zero
#pragma unroll
        for (int a = 0; a < IA; ++a) {
            const int q = qt + a * P;
            if (q < R2) {
                cx<T> w[R1];
#pragma unroll
                for (int j = 0; j < R1; ++j) w[j] = j < HALF ? v[a][j] : mk(T(0), T(0));
                if constexpr (R1 == 8)
                    dft8_half_in<-1>(w);
                else
                    dft<R1, -1>(w);
#pragma unroll
                for (int r = 0; r < R1; ++r) s0[(q * R1 + r) * LP0 + line] = w[r];
            }
        }
        __syncthreads();
        // phase B: spectra in natural order to sm
#pragma unroll
        for (int b = 0; b < IB; ++b) {
            const int q = qt + b * P;
            if (q < R1) {
                cx<T> u[R2];
#pragma unroll
                for (int r = 0; r < R2; ++r) u[r] = s0[(q + r * R1) * LP0 + line];
#pragma unroll
                for (int r = 1; r < R2; ++r) u[r] = cmul(u[r], tw[r * q]);
                dft<R2, -1>(u);
#pragma unroll
                for (int r = 0; r < R2; ++r) sm[(q + r * R1) * LPM + line] = u[r];
            }
        }
        __syncthreads();
        // mixing: per (column, kz) point
#pragma unroll
        for (int j = 0; j < NPT; ++j) {
            const int i = threadIdx.x + j * NT;
            const int l = i % L, k = i / L;
            const long long cc = (long long)blockIdx.x * L + l;
            if (i < L * N && cc < nxy) {
                cx<T> xt[kSlMaxClasses], tb[kSlMaxClasses];
#pragma unroll
                for (int b = 0; b < kSlMaxClasses; ++b) {
                    if (b < S) {
                        tb[b] = cmul(phxy[b * L + l], phz[mix.offz[b] * N + k]);
                        xt[b] = cmul(sm[k * LPM + b * L + l], tb[b]);
                    } else {
                        tb[b] = mk(T(0), T(0));
                        xt[b] = mk(T(0), T(0));
                    }
                }
                if constexpr (ZB) {
                    // Walsh-Hadamard form (see k_sl_build_h): fcc classes 0-3, fcc + (1,1,1) 4-7;
                    // hv = alpha^/4 (real, 0-3) and beta^/4 (4-7) per character
                    cx<T> xf[4], xa[4];
                    wht4(xt, xf);
                    wht4(xt + 4, xa);
                    cx<T> uf[4], ua[4];
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        const T al = hv[j][c].re;
                        const cx<T> be = hv[j][4 + c];
                        uf[c] = mk(al * xf[c].re + be.re * xa[c].re + be.im * xa[c].im,
                                   al * xf[c].im + be.re * xa[c].im - be.im * xa[c].re);  // + conj(be) xa
                        ua[c] = mk(al * xa[c].re + be.re * xf[c].re - be.im * xf[c].im,
                                   al * xa[c].im + be.re * xf[c].im + be.im * xf[c].re);  // + be xf
                    }
                    cx<T> u8[8];
                    wht4(uf, u8);
                    wht4(ua, u8 + 4);
#pragma unroll
                    for (int a = 0; a < kSlMaxClasses; ++a) sm[k * LPM + a * L + l] = cmulc(u8[a], tb[a]);
                } else {
#pragma unroll
                    for (int a = 0; a < kSlMaxClasses; ++a) {
                        if (a >= S) continue;
                        cx<T> u = mk(T(0), T(0));
#pragma unroll
                        for (int b = 0; b < kSlMaxClasses; ++b) {
                            if (b >= S) continue;
                            cx<T> g = H[mix.h[a * kSlMaxClasses + b] * h_stride + (long long)k * nxy + cc];
                            if (mix.cj[a * kSlMaxClasses + b]) g.im = -g.im;
                            u.re += g.re * xt[b].re - g.im * xt[b].im;
                            u.im += g.re * xt[b].im + g.im * xt[b].re;
                        }
                        sm[k * LPM + a * L + l] = cmulc(u, tb[a]);
                    }
                }
            }
        }
        __syncthreads();
        // phase B': first stage of the inverse transform
#pragma unroll
        for (int b = 0; b < IB; ++b) {
            const int q = qt + b * P;
            if (q < R1) {
                cx<T> u[R2];
#pragma unroll
                for (int r = 0; r < R2; ++r) u[r] = sm[(q + r * R1) * LPM + line];
                dft<R2, +1>(u);
#pragma unroll
                for (int r = 0; r < R2; ++r) s0[(q * R2 + r) * LP0 + line] = u[r];
            }
        }
        __syncthreads();
        // phase A': twiddles, R1-point inverse DFTs, outputs z = q + R2 r < N/2 stored
#pragma unroll
        for (int a = 0; a < IA; ++a) {
            const int q = qt + a * P;
            if (q < R2) {
                cx<T> w[R1];
#pragma unroll
                for (int r = 0; r < R1; ++r) w[r] = s0[(q + r * R2) * LP0 + line];
#pragma unroll
                for (int r = 1; r < R1; ++r) w[r] = cmulc(w[r], tw[r * q]);
                if constexpr (R1 == 8)
                    dft8_half_out<+1>(w);  // outputs r < 4 only
                else
                    dft<R1, +1>(w);
                if (valid) {
#pragma unroll
                    for (int r = 0; r < HALF; ++r) dst[(long long)(q + R2 * r) * nxy] = w[r];
                }
            }
        }
        __syncthreads();  // s0 is rewritten by the next density's phase A
#pragma unroll
        for (int a = 0; a < IA; ++a)
#pragma unroll
            for (int j = 0; j < HALF; ++j) v[a][j] = vn[a][j];
    }
}

// The z-mix kernel's radix split of an even line length N = R1 * R2 with R1 even; f is called
// with SplitTag<R1, R2>.  Returns false when N has no compiled split.
template <typename F>
bool with_zmix_split(int n, F&& f) {
    switch (n) {
#define CLK_ZSPLIT(N, A, B)  \
    case N:                  \
        f(SplitTag<A, B>{}); \
        return true;
        CLK_ZSPLIT(2, 2, 1)
        CLK_ZSPLIT(4, 2, 2)
        CLK_ZSPLIT(6, 2, 3)
        CLK_ZSPLIT(8, 4, 2)
        CLK_ZSPLIT(10, 2, 5)
        CLK_ZSPLIT(12, 4, 3)
        CLK_ZSPLIT(16, 4, 4)
        CLK_ZSPLIT(18, 6, 3)
        CLK_ZSPLIT(20, 4, 5)
        CLK_ZSPLIT(24, 4, 6)
        CLK_ZSPLIT(30, 6, 5)
        CLK_ZSPLIT(32, 4, 8)
        CLK_ZSPLIT(36, 6, 6)
        CLK_ZSPLIT(40, 8, 5)
        CLK_ZSPLIT(48, 6, 8)
        CLK_ZSPLIT(50, 10, 5)
        CLK_ZSPLIT(54, 6, 9)
        CLK_ZSPLIT(60, 6, 10)
        CLK_ZSPLIT(64, 8, 8)
        CLK_ZSPLIT(72, 8, 9)
        CLK_ZSPLIT(80, 8, 10)
        CLK_ZSPLIT(90, 10, 9)
        CLK_ZSPLIT(96, 8, 12)
        CLK_ZSPLIT(100, 10, 10)
        CLK_ZSPLIT(108, 12, 9)
        CLK_ZSPLIT(120, 10, 12)
        CLK_ZSPLIT(128, 8, 16)
        CLK_ZSPLIT(144, 12, 12)
        CLK_ZSPLIT(150, 10, 15)
        CLK_ZSPLIT(160, 10, 16)
        CLK_ZSPLIT(180, 12, 15)
        CLK_ZSPLIT(192, 12, 16)
        CLK_ZSPLIT(240, 16, 15)
        CLK_ZSPLIT(256, 16, 16)
#undef CLK_ZSPLIT
        default: return false;
    }
}

}  // namespace clk
