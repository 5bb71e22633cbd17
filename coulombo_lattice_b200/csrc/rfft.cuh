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
#include "kernels.cuh"

namespace clk {

template <int A, int B>
struct cmax {
    static constexpr int value = A > B ? A : B;
};

// Minimum resident blocks asked of the compiler: with a radix-16 factor two (<= 128 registers
// for 256 threads; left alone those passes grow past it, one block per SM); otherwise none
// (0: the compiler's own choice, measured lower than with any explicit minimum).
template <int A, int B, int THREADS>
struct col_min_blocks {
    static constexpr int value = (A >= 16 || B >= 16) ? 2 : 0;
};

// ---------------------------------------------------------------------------------------
// Thread layout of the column passes.  A line of N = R1*R2 points has R2 phase-A items
// (R1-point DFTs) and R1 phase-B items (R2-point DFTs).  When one factor divides the other,
// P = the smaller factor threads serve a line and each takes IA = R2/P phase-A items and
// IB = R1/P phase-B items, so no thread idles at the barriers between the phases; otherwise
// P = the larger factor and the threads beyond a phase's item count sit that phase out.
// ---------------------------------------------------------------------------------------
template <int R1, int R2>
struct ColShape {
    static constexpr int lo = R1 < R2 ? R1 : R2;
    static constexpr int hi = R1 < R2 ? R2 : R1;
    static constexpr int P = (hi % lo == 0) ? lo : hi;
    static constexpr int IA = (R2 + P - 1) / P;
    static constexpr int IB = (R1 + P - 1) / P;
};

// Minimum resident blocks of the column passes when a factor is a radix-16 codelet: about 512
// threads per SM in FP32 (<= 128 registers a thread) and 256 in FP64 (<= 256, room for the
// 16-point butterflies and the prefetched column without spilling); otherwise the compiler's
// choice.
template <typename T, int R1, int R2, int THREADS>
struct colp_min_blocks {
    static constexpr int per_sm = sizeof(T) == 4 ? 512 : 256;
    static constexpr int value = (R1 >= 16 || R2 >= 16) ? (per_sm / THREADS > 0 ? per_sm / THREADS : 1) : 0;
};

// Point pitch LP of an exchange buffer [pos][line] (address pos*LP + line), written at
// pos = q*RW + r by items q < QW and read at pos = q + r*RW by items q < QR: the pitch in
// [L, L + W) with the fewest bank conflicts over the thread groups served by one
// shared-memory wavefront (W = 128 B / element; the r terms shift every thread alike).
template <int L, int P, int RW, int QW, int QR, int ES>
struct ColPitch {
    static constexpr int W = 128 / ES;
    static constexpr int degree(int lp, int write) {
        int worst = 0;
        for (int g0 = 0; g0 < L * P; g0 += W) {
            int count[32] = {};
            for (int tid = g0; tid < g0 + W && tid < L * P; ++tid) {
                const int line = tid % L, q = tid / L;
                if (q >= (write ? QW : QR)) continue;
                const int pos = write ? q * RW : q;
                const int slot = (pos * lp + line) % W;
                if (++count[slot] > worst) worst = count[slot];
            }
        }
        return worst;
    }
    static constexpr int pick() {
        int best = L, bd = 1 << 30;
        for (int lp = L; lp < L + W; ++lp) {
            const int d = degree(lp, 1) > degree(lp, 0) ? degree(lp, 1) : degree(lp, 0);
            if (d < bd) {
                bd = d;
                best = lp;
            }
        }
        return best;
    }
    static constexpr int LP = pick();
};

template <typename T, int R1, int R2, int L>
struct ZconvLayout {
    using S = ColShape<R1, R2>;
    static constexpr int LP0 = ColPitch<L, S::P, R1, R2, R1, sizeof(cx<T>)>::LP;  // phase A -> B
    static constexpr int LP1 = ColPitch<L, S::P, R2, R1, R2, sizeof(cx<T>)>::LP;  // phase B -> C
    static constexpr size_t smem = sizeof(cx<T>) * ((size_t)R1 * R2 * (1 + LP0 + LP1));
};

template <typename T, int R1, int R2, int L>
struct YcolLayout {
    using S = ColShape<R1, R2>;
    static constexpr int LP0 = ColPitch<L, S::P, R1, R2, R1, sizeof(cx<T>)>::LP;
    static constexpr size_t smem = sizeof(cx<T>) * ((size_t)R1 * R2 * (1 + LP0));
};

// ---------------------------------------------------------------------------------------
// z pass: forward FFT along z, x Khat, inverse FFT along z; block = L adjacent xy columns
// x P threads, densities [blockIdx.y * per, ...).
// ---------------------------------------------------------------------------------------
template <typename T, int R1, int R2, int L>
__global__ void __launch_bounds__(L * ColShape<R1, R2>::P, colp_min_blocks<T, R1, R2, L * ColShape<R1, R2>::P>::value)
    k_zconv_rf(cx<T>* __restrict__ buf, long long stride, const cx<T>* __restrict__ tw_g,
               const T* __restrict__ khat, long long nxy, int np) {
    using S = ColShape<R1, R2>;
    using Lay = ZconvLayout<T, R1, R2, L>;
    constexpr int N = R1 * R2, P = S::P, IA = S::IA, IB = S::IB, LP0 = Lay::LP0, LP1 = Lay::LP1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* tw = reinterpret_cast<cx<T>*>(smem_raw);
    cx<T>* s0 = tw + N;
    cx<T>* s1 = s0 + N * LP0;
    const int line = threadIdx.x % L;
    const int qt = threadIdx.x / L;
    const long long c = (long long)blockIdx.x * L + line;
    const bool valid = c < nxy;
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = tw_g[i];
    // Khat of the positions q + r*R1 that phase-B item q holds, for all densities
    T kv[IB][R2];
#pragma unroll
    for (int b = 0; b < IB; ++b) {
        const int q = qt + b * P;
#pragma unroll
        for (int r = 0; r < R2; ++r) kv[b][r] = (q < R1 && valid) ? khat[(long long)(q + r * R1) * nxy + c] : T(0);
    }
    __syncthreads();
    const int per = (np + gridDim.y - 1) / gridDim.y;
    const int p_begin = blockIdx.y * per, p_end = min(np, p_begin + per);
    // the next density's column is loaded into registers while the current one is transformed
    const auto load = [&](int p, cx<T>(&v)[IA][R1]) {
        const cx<T>* src = buf + (long long)p * stride + c;
#pragma unroll
        for (int a = 0; a < IA; ++a) {
            const int q = qt + a * P;
#pragma unroll
            for (int j = 0; j < R1; ++j)
                v[a][j] = (valid && q < R2) ? src[(long long)(q + R2 * j) * nxy] : mk(T(0), T(0));
        }
    };
    cx<T> v[IA][R1], vn[IA][R1];
    if (p_begin < p_end) load(p_begin, v);
    for (int p = p_begin; p < p_end; ++p) {
        cx<T>* base = buf + (long long)p * stride + c;
        if (p + 1 < p_end) load(p + 1, vn);
#pragma unroll
        for (int a = 0; a < IA; ++a) {
            const int q = qt + a * P;
            if (q < R2) {
                dft<R1, -1>(v[a]);
#pragma unroll
                for (int r = 0; r < R1; ++r) s0[(q * R1 + r) * LP0 + line] = v[a][r];
            }
        }
        __syncthreads();
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
                for (int r = 0; r < R2; ++r) u[r] = mk(u[r].re * kv[b][r], u[r].im * kv[b][r]);
                dft<R2, +1>(u);
#pragma unroll
                for (int r = 0; r < R2; ++r) s1[(q * R2 + r) * LP1 + line] = u[r];
            }
        }
        __syncthreads();
#pragma unroll
        for (int a = 0; a < IA; ++a) {
            const int q = qt + a * P;
            if (q < R2) {
                cx<T> w[R1];
#pragma unroll
                for (int r = 0; r < R1; ++r) w[r] = s1[(q + r * R2) * LP1 + line];
#pragma unroll
                for (int r = 1; r < R1; ++r) w[r] = cmulc(w[r], tw[r * q]);
                dft<R1, +1>(w);
                if (valid) {
#pragma unroll
                    for (int r = 0; r < R1; ++r) base[(long long)(q + R2 * r) * nxy] = w[r];
                }
            }
        }
#pragma unroll
        for (int a = 0; a < IA; ++a)
#pragma unroll
            for (int j = 0; j < R1; ++j) v[a][j] = vn[a][j];
    }
}

// ---------------------------------------------------------------------------------------
// y pass (one direction): block = L adjacent x of one z-plane x P threads, densities
// [blockIdx.y * per, ...).
// ---------------------------------------------------------------------------------------
template <int S, typename T, int R1, int R2, int L>
__global__ void __launch_bounds__(L * ColShape<R1, R2>::P, colp_min_blocks<T, R1, R2, L * ColShape<R1, R2>::P>::value)
    k_ycol_rf(cx<T>* __restrict__ buf, long long stride, const cx<T>* __restrict__ tw_g, int nx, int ny,
              int xchunks, int np, const int* __restrict__ row_ptr) {
    using Sh = ColShape<R1, R2>;
    constexpr int N = R1 * R2, P = Sh::P, IA = Sh::IA, IB = Sh::IB;
    constexpr int LP0 = YcolLayout<T, R1, R2, L>::LP0;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* tw = reinterpret_cast<cx<T>*>(smem_raw);
    cx<T>* s0 = tw + N;
    const int line = threadIdx.x % L;
    const int qt = threadIdx.x / L;
    const int xc = blockIdx.x % xchunks, z = blockIdx.x / xchunks;
    const int x = xc * L + line;
    const bool valid = x < nx;
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = tw_g[i];
    // Rows (y, z) without atoms: after the forward x pass they are zero and were not stored;
    // after the inverse y pass nothing reads them.  row_ptr == nullptr: every row is live.
    unsigned live_in[IA], live_out[IB];
#pragma unroll
    for (int a = 0; a < IA; ++a) {
        const int q = qt + a * P;
        live_in[a] = 0;
        if (q < R2) {
#pragma unroll
            for (int j = 0; j < R1; ++j) {
                const int r = z * ny + q + R2 * j;
                if (!row_ptr || row_ptr[r + 1] > row_ptr[r]) live_in[a] |= 1u << j;
            }
        }
    }
#pragma unroll
    for (int b = 0; b < IB; ++b) {
        const int q = qt + b * P;
        live_out[b] = 0;
        if (q < R1) {
#pragma unroll
            for (int j = 0; j < R2; ++j) {
                const int r = z * ny + q + j * R1;
                if (!row_ptr || row_ptr[r + 1] > row_ptr[r]) live_out[b] |= 1u << j;
            }
        }
    }
    __syncthreads();
    const int per = (np + gridDim.y - 1) / gridDim.y;
    const int p_begin = blockIdx.y * per, p_end = min(np, p_begin + per);
    // the next density's column is loaded into registers while the current one is transformed
    const auto load = [&](int p, cx<T>(&v)[IA][R1]) {
        const cx<T>* src = buf + (long long)p * stride + (long long)z * nx * ny + x;
#pragma unroll
        for (int a = 0; a < IA; ++a) {
            const int q = qt + a * P;
#pragma unroll
            for (int j = 0; j < R1; ++j) {
                const bool ld = valid && q < R2 && (S > 0 || ((live_in[a] >> j) & 1u));
                v[a][j] = ld ? src[(long long)(q + R2 * j) * nx] : mk(T(0), T(0));
            }
        }
    };
    cx<T> v[IA][R1], vn[IA][R1];
    if (p_begin < p_end) load(p_begin, v);
    for (int p = p_begin; p < p_end; ++p) {
        cx<T>* base = buf + (long long)p * stride + (long long)z * nx * ny + x;
        if (p + 1 < p_end) load(p + 1, vn);
#pragma unroll
        for (int a = 0; a < IA; ++a) {
            const int q = qt + a * P;
            if (q < R2) {
                dft<R1, S>(v[a]);
#pragma unroll
                for (int r = 0; r < R1; ++r) s0[(q * R1 + r) * LP0 + line] = v[a][r];
            }
        }
        __syncthreads();
#pragma unroll
        for (int b = 0; b < IB; ++b) {
            const int q = qt + b * P;
            if (q < R1) {
                cx<T> u[R2];
#pragma unroll
                for (int r = 0; r < R2; ++r) u[r] = s0[(q + r * R1) * LP0 + line];
#pragma unroll
                for (int r = 1; r < R2; ++r) u[r] = S < 0 ? cmul(u[r], tw[r * q]) : cmulc(u[r], tw[r * q]);
                dft<R2, S>(u);
                if (valid) {
#pragma unroll
                    for (int r = 0; r < R2; ++r)
                        if (S < 0 || ((live_out[b] >> r) & 1u)) base[(long long)(q + r * R1) * nx] = u[r];
                }
            }
        }
        __syncthreads();
#pragma unroll
        for (int a = 0; a < IA; ++a)
#pragma unroll
            for (int j = 0; j < R1; ++j) v[a][j] = vn[a][j];
    }
}


// ---------------------------------------------------------------------------------------
// Row passes (x) with the same two-factor register FFT.  A block owns LR consecutive rows
// (row = z*ny + y) held transposed in shared memory, T[x*(LR+1) + row]: phase A maps
// consecutive threads to consecutive rows and phase B to consecutive x, both free of bank
// conflicts thanks to the odd row pitch.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem_dst, const void* gmem_src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(smem_u32(smem_dst)), "l"(gmem_src), "n"(BYTES));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Forward: scatter the rows' atoms x conj(phase_kappa), FFT along x, store whole rows.
// The transposed tile holds point x of a row at pos(x)*(LR+1) + row.  With PAD there is one
// spare point every 4 points, so that atoms 4 points apart along a row (zinc-blende) scatter
// to distinct banks; dense rows then see 2-way conflicts instead, and the tile grows by a
// quarter, so the autotuner decides per shape.
template <int N, bool PAD>
struct XfwdTile {
    __host__ __device__ static constexpr int pos(int x) { return PAD ? x + x / 4 : x; }
    static constexpr int points = pos(N - 1) + 1;
};

// Pitches of the forward row pass, chosen at compile time by simulating the bank mapping
// (W-element slots, one wavefront per group of W lanes; cost = the wavefronts of all of a
// block's accesses):
//   tile     T[pos(x)*TP + row]: phase A reads (lanes: LR rows fastest, then t) and the atom
//            scatter (consecutive lanes on atoms 1, 2 or 4 points apart along a row);
//   exchange item t's output r at t*EP + r*XP + row: phase A writes it (lanes as above),
//            phase B reads position j + r*R1, i.e. item r's output j (lanes: j fastest, then
//            rows).  The item pitch EP is separate from R1*XP so that items t do not all start
//            on the same bank.
template <int R1, int R2, int LR, bool PAD, int ES>
struct XfwdPitch {
    static constexpr int N = R1 * R2;
    static constexpr int Q = R1 > R2 ? R1 : R2;
    static constexpr int TH = LR * Q;
    static constexpr int W = 128 / ES;
    using Tile = XfwdTile<N, PAD>;
    template <typename F>
    static constexpr int groups(F addr) {  // sum over W-lane groups of the worst slot count
        int total = 0;
        for (int g0 = 0; g0 < TH; g0 += W) {
            int cnt[32] = {};
            int worst = 0;
            for (int tid = g0; tid < g0 + W && tid < TH; ++tid) {
                const int a = addr(tid);
                if (a < 0) continue;
                const int sl = a % W;
                if (++cnt[sl] > worst) worst = cnt[sl];
            }
            total += worst;
        }
        return total;
    }
    static constexpr int tile_cost(int tp) {
        int c = 0;
        for (int j = 0; j < R1; ++j)
            c += groups([&](int tid) {
                const int lr = tid % LR, t = tid / LR;
                return t < R2 ? Tile::pos(t + R2 * j) * tp + lr : -1;
            });
        for (int s = 1; s <= 4; s *= 2)  // scatter of atoms s points apart, one row
            c += groups([&](int tid) { return tid * s < N ? Tile::pos(tid * s) * tp : -1; });
        return c;
    }
    static constexpr int ex_cost(int xp, int ep) {
        const int w = groups([&](int tid) {
            const int lr = tid % LR, t = tid / LR;
            return t < R2 ? t * ep + lr : -1;
        });
        const int r = groups([&](int tid) {
            const int j = tid % R1, lr = tid / R1;
            return lr < LR ? j * xp + lr : -1;
        });
        return R1 * w + R2 * r;
    }
    static constexpr int pick_tp() {
        int best = LR, bc = 1 << 30;
        for (int tp = LR; tp < LR + W; ++tp) {
            const int c = tile_cost(tp);
            if (c < bc) {
                bc = c;
                best = tp;
            }
        }
        return best;
    }
    static constexpr int pick_ex(int which) {  // 0: XP, 1: EP
        int bx = LR, be = R1 * LR, bc = 1 << 30;
        for (int xp = LR; xp < LR + W; ++xp)
            for (int ep = R1 * xp; ep < R1 * xp + W; ++ep) {
                const int c = ex_cost(xp, ep);
                if (c < bc) {
                    bc = c;
                    bx = xp;
                    be = ep;
                }
            }
        return which ? be : bx;
    }
    static constexpr int TP = pick_tp();
    static constexpr int XP = pick_ex(0);
    static constexpr int EP = pick_ex(1);
    static constexpr size_t elems = (size_t)N + (size_t)Tile::points * TP + (size_t)R2 * EP;
};

template <typename T, int R1, int R2, int LR, bool PAD>
__global__ void __launch_bounds__(LR * cmax<R1, R2>::value, col_min_blocks<R1, R2, LR * cmax<R1, R2>::value>::value)
    k_xfwd_rf(const cx<T>* __restrict__ rho, long long rho_stride, const int* __restrict__ row_ptr,
              const int* __restrict__ cell, cx<T>* __restrict__ out, long long out_stride,
              const cx<T>* __restrict__ tw_g, RoundPhase rp, int ny, int nrows, int np, int skip_empty) {
    constexpr int N = R1 * R2;
    using Pitch = XfwdPitch<R1, R2, LR, PAD, sizeof(cx<T>)>;
    constexpr int TP = Pitch::TP, XP = Pitch::XP, EP = Pitch::EP;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using Tile = XfwdTile<N, PAD>;
    cx<T>* tw = reinterpret_cast<cx<T>*>(smem_raw);
    cx<T>* tile = tw + N;
    cx<T>* ex = tile + Tile::points * TP;
    const int r0 = blockIdx.x * LR;
    const int nr = min(LR, nrows - r0);
    // twiddles laid out [r][j] = W_N^(r j), so that phase B's lanes on consecutive j read
    // consecutive words
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = tw_g[(i / R1) * (i % R1)];
    const int a0 = row_ptr[r0], a1 = row_ptr[r0 + nr];
    const int per = (np + gridDim.y - 1) / gridDim.y;
    const int p_begin = blockIdx.y * per, p_end = min(np, p_begin + per);
    // a row without atoms transforms to zero; with skip_empty the consumer (the forward y
    // pass) reads zero for it instead of loading it, so it is not stored
    bool store_row;
    {
        const int lr = threadIdx.x / R1;
        store_row = lr < nr && (!skip_empty || row_ptr[r0 + lr + 1] > row_ptr[r0 + lr]);
    }
    // the block's atoms (at most KA per thread): shared-memory slot and phase, computed once
    // for all densities
    constexpr int KA = 4;
    const bool pre = (a1 - a0) <= KA * (int)blockDim.x;
    int slot[KA];
    cx<double> ph[KA];
    if (pre) {
#pragma unroll
        for (int k = 0; k < KA; ++k) {
            const int i = a0 + threadIdx.x + k * blockDim.x;
            slot[k] = -1;
            if (i < a1) {
                const int c = cell[i];
                const int row = c / N, x = c - row * N;
                slot[k] = Tile::pos(x) * TP + (row - r0);
                ph[k] = round_phase(rp, x, row % ny, row / ny);
            }
        }
    }
    // cells without an atom stay zero for every density: the tile is cleared once
    for (int e = threadIdx.x; e < Tile::points * TP; e += blockDim.x) tile[e] = mk(T(0), T(0));
    __syncthreads();
    // the next density's atom values are loaded into registers while the current one is
    // transformed
    cx<T> rv[KA], rn[KA];
    const auto load = [&](int p, cx<T>(&v)[KA]) {
        const cx<T>* src = rho + (long long)p * rho_stride + a0 + threadIdx.x;
#pragma unroll
        for (int k = 0; k < KA; ++k) v[k] = slot[k] >= 0 ? src[k * blockDim.x] : mk(T(0), T(0));
    };
    if (pre && p_begin < p_end) load(p_begin, rv);
    for (int p = p_begin; p < p_end; ++p) {
        const cx<T>* rp_ = rho + (long long)p * rho_stride;
        if (pre) {
            if (p + 1 < p_end) load(p + 1, rn);
#pragma unroll
            for (int k = 0; k < KA; ++k)
                if (slot[k] >= 0) tile[slot[k]] = narrow<T>(cmulc(widen(rv[k]), ph[k]));
        } else {
            for (int i = a0 + threadIdx.x; i < a1; i += blockDim.x) {
                const int c = cell[i];
                const int row = c / N, x = c - row * N;
                const int y = row % ny, z = row / ny;
                tile[Tile::pos(x) * TP + (row - r0)] = narrow<T>(cmulc(widen(rp_[i]), round_phase(rp, x, y, z)));
            }
        }
        __syncthreads();
        {
            const int lr = threadIdx.x % LR, t = threadIdx.x / LR;
            if (t < R2) {
                cx<T> v[R1];
#pragma unroll
                for (int j = 0; j < R1; ++j) v[j] = tile[Tile::pos(t + R2 * j) * TP + lr];
                dft<R1, -1>(v);
#pragma unroll
                for (int r = 0; r < R1; ++r) ex[t * EP + r * XP + lr] = v[r];
            }
        }
        __syncthreads();
        {
            const int j = threadIdx.x % R1, lr = threadIdx.x / R1;
            if (store_row) {
                cx<T> u[R2];
#pragma unroll
                for (int r = 0; r < R2; ++r) u[r] = ex[r * EP + j * XP + lr];
#pragma unroll
                for (int r = 1; r < R2; ++r) u[r] = cmul(u[r], tw[r * R1 + j]);
                dft<R2, -1>(u);
                cx<T>* o = out + (long long)p * out_stride + (long long)(r0 + lr) * N + j;
#pragma unroll
                for (int r = 0; r < R2; ++r) o[r * R1] = u[r];
            }
        }
        if (pre) {
#pragma unroll
            for (int k = 0; k < KA; ++k) rv[k] = rn[k];
        }
    }
}

// Row pitches of the inverse row pass, chosen at compile time: every pad in [0, W) is tried
// and the one whose worst shared-memory bank conflict (over the thread groups served by one
// wavefront, W = 128 B / element) is lowest is kept -- for the exchange (phase A writes
// la*PP + ta*(R1+1) + r, phase B reads lb*PP + jb + r*(R1+1)) and for the natural-order rows
// (phase B writes point x = jb + r*R1 at lb*NP + pos(x)).
template <int R1, int R2, int LR, int ES>
struct XinvPitch {
    static constexpr int N = R1 * R2;
    static constexpr int Q = R1 > R2 ? R1 : R2;
    static constexpr int T = LR * Q;
    static constexpr int W = 128 / ES;
    // Row position of point x: one pad slot after every W points, so that gathers of atoms
    // spaced 1, 2 or 4 points apart along a row hit distinct banks.
    __host__ __device__ static constexpr int pos(int x) { return x + x / W; }
    // worst number of distinct elements per bank slot over the wavefront groups;
    // which: 0 phase-A exchange write, 1 phase-B exchange read, 2 phase-B row write
    static constexpr int degree(int pitch, int which) {
        int worst = 0;
        for (int r = 0; r < (which == 2 ? R2 : 1); ++r) {
            for (int g0 = 0; g0 < T; g0 += W) {
                int count[32] = {};
                for (int tid = g0; tid < g0 + W && tid < T; ++tid) {
                    int e = -1;
                    if (which == 0) {
                        const int ta = tid % R2, la = tid / R2;
                        if (la < LR) e = la * pitch + ta * (R1 + 1);
                    } else if (which == 1) {
                        const int jb = tid % R1, lb = tid / R1;
                        if (lb < LR) e = lb * pitch + jb;  // the r terms shift every thread alike
                    } else {
                        const int jb = tid % R1, lb = tid / R1;
                        if (lb < LR) e = lb * pitch + pos(jb + r * R1);
                    }
                    if (e >= 0) {
                        const int slot = e % W;
                        if (++count[slot] > worst) worst = count[slot];
                    }
                }
            }
        }
        return worst;
    }
    static constexpr int ex_pitch() {
        int best = N + R2, bd = 1 << 30;
        for (int pad = 0; pad < W; ++pad) {
            const int pp = N + R2 + pad;
            const int d = degree(pp, 0) > degree(pp, 1) ? degree(pp, 0) : degree(pp, 1);
            if (d < bd) {
                bd = d;
                best = pp;
            }
        }
        return best;
    }
    static constexpr int row_pitch() {
        const int base = pos(N - 1) + 1;
        int best = base, bd = 1 << 30;
        for (int pad = 0; pad < W; ++pad) {
            const int d = degree(base + pad, 2);
            if (d < bd) {
                bd = d;
                best = base + pad;
            }
        }
        return best;
    }
    static constexpr int PP = ex_pitch();
    static constexpr int NP = row_pitch();
};

// Inverse: phase A loads a row's points straight from HBM into registers (thread t of a row
// reads x = t + R2*j, so a warp covers whole row segments), the next density's points being
// loaded while the current one is transformed; rows without atoms are not loaded.  The
// exchange between the stages uses a padded layout (one pad per R1 points, conflict-free in
// both directions); phase B writes the rows in natural order to shared memory, from which the
// round's values at the rows' atoms are gathered to out[p][atom] with consecutive threads on
// consecutive atoms (write-only; the phase and the round sum are applied in FP64 by
// k_round_sum).
template <typename T, int R1, int R2, int LR>
__global__ void __launch_bounds__(LR * cmax<R1, R2>::value, col_min_blocks<R1, R2, LR * cmax<R1, R2>::value>::value)
    k_xinv_rf(const cx<T>* __restrict__ buf, long long stride, const cx<T>* __restrict__ tw_g,
              const int* __restrict__ row_ptr, const int* __restrict__ cell, cx<T>* __restrict__ out,
              long long o_stride, int nrows, int np) {
    constexpr int N = R1 * R2;
    // exchange row: position x' at x' + x' / R1 (one pad per R1 points), rows PP apart
    using Pitch = XinvPitch<R1, R2, LR, sizeof(cx<T>)>;
    constexpr int PP = Pitch::PP;
    constexpr int NP = Pitch::NP;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* tw = reinterpret_cast<cx<T>*>(smem_raw);
    cx<T>* ex = tw + N;          // [LR][PP]
    cx<T>* rows = ex + LR * PP;  // [LR][NP], natural order
    const int r0 = blockIdx.x * LR;
    const int nr = min(LR, nrows - r0);
    // twiddles laid out [r][j] = W_N^(r j), so that phase B's lanes on consecutive j read
    // consecutive words
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = tw_g[(i / R1) * (i % R1)];
    const int a0 = row_ptr[r0], a1 = row_ptr[r0 + nr];
    const int per = (np + gridDim.y - 1) / gridDim.y;
    const int p_begin = blockIdx.y * per, p_end = min(np, p_begin + per);
    // phase A: thread (ta, la) transforms row la from points ta + R2*j
    const int ta = threadIdx.x % R2, la = threadIdx.x / R2;
    const bool load_row = la < nr && row_ptr[r0 + la + 1] > row_ptr[r0 + la];
    // phase B: thread (jb, lb) holds points jb + r*R1 of row lb
    const int jb = threadIdx.x % R1, lb = threadIdx.x / R1;
    const auto load = [&](int p, cx<T>(&v)[R1]) {
        const cx<T>* src = buf + (long long)p * stride + (long long)(r0 + la) * N + ta;
#pragma unroll
        for (int j = 0; j < R1; ++j) v[j] = load_row ? src[R2 * j] : mk(T(0), T(0));
    };
    cx<T> v[R1], vn[R1];
    if (la < LR && p_begin < p_end) load(p_begin, v);
    __syncthreads();
    for (int p = p_begin; p < p_end; ++p) {
        if (la < LR) {
            if (p + 1 < p_end) load(p + 1, vn);
            dft<R1, +1>(v);
#pragma unroll
            for (int r = 0; r < R1; ++r) ex[la * PP + ta * (R1 + 1) + r] = v[r];
        }
        __syncthreads();
        if (lb < LR) {
            cx<T> u[R2];
#pragma unroll
            for (int r = 0; r < R2; ++r) u[r] = ex[lb * PP + jb + r * (R1 + 1)];
#pragma unroll
            for (int r = 1; r < R2; ++r) u[r] = cmulc(u[r], tw[r * R1 + jb]);
            dft<R2, +1>(u);
#pragma unroll
            for (int r = 0; r < R2; ++r) rows[lb * NP + Pitch::pos(jb + r * R1)] = u[r];
        }
        __syncthreads();
        cx<T>* op = out + (long long)p * o_stride;
        for (int i = a0 + threadIdx.x; i < a1; i += blockDim.x) {
            const int c = cell[i];
            const int row = c / N, x = c - row * N;
            op[i] = rows[(row - r0) * NP + Pitch::pos(x)];
        }
#pragma unroll
        for (int j = 0; j < R1; ++j) v[j] = vn[j];
    }
}

// ---------------------------------------------------------------------------------------
// Host-side dispatch: calls f(SplitTag<R1, R2>{}) for a length with a compiled two-factor
// split (factors are register codelets 2..16, as balanced as possible, or swapped); false
// otherwise.
// ---------------------------------------------------------------------------------------
template <int A, int B>
struct SplitTag {
    static constexpr int r1 = A, r2 = B;
};

// variant 1 calls f with the two factors swapped (the same split when they are equal).
template <typename F>
bool with_split2(int n, F&& f, int variant = 0) {
    switch (n) {
#define CLK_SPLIT(N, A, B)                  \
    case N:                                 \
        if (variant != 0 && (A) != (B))     \
            f(SplitTag<B, A>{});            \
        else                                \
            f(SplitTag<A, B>{});            \
        return true;
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
