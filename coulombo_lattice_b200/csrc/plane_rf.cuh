// Fused x+y passes on whole xy-planes held in shared memory, with the register two-factor
// line FFTs of rfft.cuh.
//
// A block owns one z-plane (N x N points, N = R1*R2) and a run of densities.  Every stage of
// both line transforms runs in place in the plane buffer:
//   phase A  item t < R2 of a line reads points t + R2*m (m < R1), does an R1-point DFT and
//            writes output j back to point t + R2*j;
//   phase B  item j < R1 reads points R2*j + t (t < R2), multiplies by W_N^(t j), does an
//            R2-point DFT and writes output s back to point R2*j + s, which then holds
//            frequency j + R1*s ("digit order", dig(k) below).
// Each thread rewrites only the points it read, so a stage needs one barrier, before the
// next stage reads.  The inverse stages run the same patterns in the opposite order
// (B, then A), which takes a line from digit order back to natural order.
//
// Forward (per density): scatter the plane's atoms x conj(phase_kappa) into the zeroed plane,
// x transform of the rows with atoms only (natural order in, digit order out), y transform of
// every column (natural order in), and the phase-B outputs go straight to HBM in natural order
// (consecutive threads on consecutive x); the points a thread read in the last stage are
// zeroed as it goes, so the plane is clear for the next density.  One HBM write per point.
// Inverse: the y transform loads its columns straight from HBM (natural order in, digit-order
// rows out; only rows with atoms are kept), the x transform of those rows (digit order in,
// natural order out), and the round's values at the plane's atoms are gathered to
// out[p][atom] with consecutive threads on consecutive atoms.  One HBM read per point.
//
// Shared-memory layout: point n of a row at pos(n) = n + P*(n / R2) (P pad elements after
// every R2 points), physical row pr at pr*LDP + cls(pr)*D with cls(pr) = (pr >> 1) & 1.  The
// x-stage phase A serves 16 lanes per row and phase B 8 lanes per row, two rows of distinct
// classes in one 16-lane group (the pair list of plane_rows); with P and D below, the row
// accesses of both phases and the column accesses of the y stage (lanes on consecutive
// frequencies kx, points pos(dig(kx))) are free of bank conflicts -- checked at compile time
// by PlaneLayout::kConflictFree.
#pragma once

#include <type_traits>

#include "rfft.cuh"

namespace clk {

template <typename T, int R1, int R2>
struct PlaneLayout {
    static constexpr int N = R1 * R2;
    static constexpr int W = 128 / (int)sizeof(cx<T>);  // elements served by one wavefront
    static constexpr int P = sizeof(T) == 4 ? 2 : 1;
    static constexpr int D = sizeof(T) == 4 ? 1 : 0;
    __host__ __device__ static constexpr int pos(int n) { return n + P * (n / R2); }
    __host__ __device__ static constexpr int dig(int k) { return R2 * (k % R1) + k / R1; }
    __host__ __device__ static constexpr int cls(int pr) { return (pr >> 1) & 1; }
    // row pitch a multiple of W, so that a row's slot offset is cls(pr) * D whatever pr
    static constexpr int LDP = (pos(N - 1) + 1 + D + W - 1) / W * W;
    __host__ __device__ static constexpr int rowbase(int pr) { return pr * LDP + cls(pr) * D; }
    // With R2 a multiple of 4 (or no class shift), rows r + R2*k share the class of r, so the
    // rows a y-stage item touches are one base plus compile-time multiples of R2*LDP:
    // rowbase(r + R2*k) = rowbase(r) + k*RSTEP.
    static_assert(R2 % 4 == 0 || D == 0, "rows R2 apart must share their class");
    static constexpr int RSTEP = R2 * LDP;

    // Bank model: a wavefront serves W consecutive lanes; the degree is the largest number of
    // lanes of one group that hit the same W-element slot.
    static constexpr int deg_a() {  // x phase A: lanes t of one row, points t + R2*m
        int worst = 0;
        for (int m = 0; m < R1; ++m)
            for (int g0 = 0; g0 < 16; g0 += W) {
                int cnt[16] = {};
                for (int l = g0; l < g0 + W; ++l)
                    if (l < R2) {
                        const int s = pos(l + R2 * m) % W;
                        if (++cnt[s] > worst) worst = cnt[s];
                    }
            }
        return worst;
    }
    static constexpr int deg_b() {  // x phase B: 8 lanes j of a class-0 row, 8 of a class-1 row
        int worst = 0;
        for (int t = 0; t < R2; ++t)
            for (int g0 = 0; g0 < 16; g0 += W) {
                int cnt[16] = {};
                for (int l = g0; l < g0 + W; ++l) {
                    const int j = l & 7, off = (l >> 3) ? D : 0;
                    if (j >= R1) continue;
                    const int s = (off + pos(R2 * j + t)) % W;
                    if (++cnt[s] > worst) worst = cnt[s];
                }
            }
        return worst;
    }
    static constexpr int deg_c() {  // y stage: lanes on consecutive kx of one row
        int worst = 0;
        for (int g0 = 0; g0 < N; g0 += W) {
            int cnt[16] = {};
            for (int k = g0; k < g0 + W && k < N; ++k) {
                const int s = pos(dig(k)) % W;
                if (++cnt[s] > worst) worst = cnt[s];
            }
        }
        return worst;
    }
    static constexpr bool kConflictFree = deg_a() == 1 && deg_b() == 1 && deg_c() == 1;
};

// Shared memory of the plane kernels: the plane, the twiddles W_N^(t j) laid out [t][j], the atom phases (forward),
// the atom masks and the row and item tables; then (forward, one block an SM, where it holds
// more atoms than the register slots) the staging of a plane's atom values for the next
// density, KS of them, and their plane positions.
template <typename T, int R1, int R2, int THREADS, bool FWD, int MINB = 1>
struct PlaneSmem {
    using L = PlaneLayout<T, R1, R2>;
    static constexpr int KA = 4;                   // atoms a thread keeps (slots) across densities
    static constexpr int NI = L::N * R2;           // phase-A items of the x stage
    static constexpr int AW = (NI + 3) / 4;        // words of the byte masks amask
    static constexpr size_t elems = (size_t)L::N * L::LDP + L::N + (FWD ? (size_t)KA * THREADS : 0);
    static constexpr size_t shorts = 4 * (size_t)L::N + 2 + NI;  // prl, lst, tmask, items
    static constexpr size_t base_bytes = sizeof(cx<T>) * elems + 4 * (size_t)AW + 2 * shorts;
    static constexpr size_t stage_off = (base_bytes + 15) / 16 * 16;
    static constexpr long long ks_fit =
        (FWD && MINB == 1) ? ((227LL * 1024 - (long long)stage_off) / (long long)(sizeof(cx<T>) + 4)) / 256 * 256 : 0;
    static constexpr int KS = ks_fit > (long long)KA * THREADS ? (int)(ks_fit < 8192 ? ks_fit : 8192) : 0;
    static constexpr size_t bytes = KS ? stage_off + (size_t)KS * (sizeof(cx<T>) + 4) : base_bytes;
};

// Asynchronous copy of one complex value (8 or 16 bytes) from HBM to shared memory.
template <typename T>
__device__ __forceinline__ void cp_async_cx(cx<T>* dst, const cx<T>* src) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    if constexpr (sizeof(cx<T>) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
    else
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}

// Row tables of the block's plane (rp = the plane's slice of the row CSR): the physical rows
// (pr = y, or dig(y) for digit-order rows) of the rows with atoms, paired class 0 with class 1
// and flattened (prl[2q], prl[2q+1]; -1 where a pair has one row), and the live-row bit mask
// by natural y.  Returns the number of pairs.  Called by every thread of the block.
template <typename L>
__device__ int plane_rows(const int* __restrict__ rp, bool digit_rows, short* prl, short* lst, unsigned* live_mask,
                          int* cnt_sh) {
    constexpr int N = L::N;
    constexpr int NW = (N + 31) / 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    bool live = false;
    int pr = 0, g = 0;
    if (tid < N) {
        live = rp[tid + 1] > rp[tid];
        pr = digit_rows ? L::dig(tid) : tid;
        g = L::cls(pr);
    }
    unsigned b0 = 0, b1 = 0;
    if (warp < NW) {
        b0 = __ballot_sync(0xffffffffu, live && g == 0);
        b1 = __ballot_sync(0xffffffffu, live && g == 1);
        if (lane == 0) {
            cnt_sh[warp] = __popc(b0);
            cnt_sh[NW + warp] = __popc(b1);
            live_mask[warp] = b0 | b1;
        }
    }
    __syncthreads();
    if (tid < N && live) {
        int before = __popc((g ? b1 : b0) & ((1u << lane) - 1u));
        for (int w = 0; w < warp; ++w) before += cnt_sh[g * NW + w];
        lst[g * N + before] = (short)pr;
    }
    int n0 = 0, n1 = 0;
    for (int w = 0; w < NW; ++w) {
        n0 += cnt_sh[w];
        n1 += cnt_sh[NW + w];
    }
    __syncthreads();
    const int mn = min(n0, n1), nbig = max(n0, n1), big = n0 > n1 ? 0 : 1;
    const int npairs = mn + (nbig - mn + 1) / 2;
    for (int q = tid; q < npairs; q += blockDim.x) {
        short a, b;
        if (q < mn) {
            a = lst[q];
            b = lst[N + q];
        } else {  // rows left over in the longer class, paired among themselves
            const int u = mn + 2 * (q - mn);
            a = lst[big * N + u];
            b = (u + 1 < nbig) ? lst[big * N + u + 1] : (short)-1;
        }
        prl[2 * q] = a;
        prl[2 * q + 1] = b;
    }
    __syncthreads();
    return npairs;
}

// Atom tables of the block's plane (atoms a0..a1 of the sorted cell list, rows r0..r0+N):
// amask byte y*R2 + t has bit m set when an atom sits at x = t + R2*m of row y; tmask[y] has
// bit t set when that byte is nonzero; items[] lists y*16 + t for the nonzero bytes in
// row-major order.  Returns the item count.  Called by every thread of the block.
template <typename L, int R2, int THREADS>
__device__ int plane_items(const int* __restrict__ cell, int a0, int a1, int r0, unsigned* amask_w,
                           unsigned short* tmask, short* items, int* scan_sh) {
    constexpr int N = L::N, NI = N * R2, AW = (NI + 3) / 4, K = (NI + THREADS - 1) / THREADS;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int w = tid; w < AW; w += THREADS) amask_w[w] = 0u;
    __syncthreads();
    for (int i = a0 + tid; i < a1; i += THREADS) {
        const int c = cell[i];
        const int row = c / N, x = c - row * N, y = row - r0;
        const int e = y * R2 + x % R2;
        atomicOr(&amask_w[e >> 2], (1u << (x / R2)) << (8 * (e & 3)));
    }
    __syncthreads();
    const unsigned char* am = reinterpret_cast<const unsigned char*>(amask_w);
    for (int y = tid; y < N; y += THREADS) {
        unsigned tm = 0;
        for (int t = 0; t < R2; ++t)
            if (am[y * R2 + t]) tm |= 1u << t;
        tmask[y] = (unsigned short)tm;
    }
    // compaction: thread tid owns candidates [tid*K, tid*K + K); exclusive scan of the counts
    int cnt = 0;
    for (int k = 0; k < K; ++k) {
        const int e = tid * K + k;
        if (e < NI && am[e]) ++cnt;
    }
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) scan_sh[warp] = incl;
    __syncthreads();
    int before = 0, total = 0;
    for (int w = 0; w < THREADS / 32; ++w) {
        const int v = scan_sh[w];
        if (w < warp) before += v;
        total += v;
    }
    int o = before + incl - cnt;
    for (int k = 0; k < K; ++k) {
        const int e = tid * K + k;
        if (e < NI && am[e]) items[o++] = (short)((e / R2) * 16 + e % R2);
    }
    __syncthreads();
    return total;
}

// Bit y of the block's live-row mask, held in registers (planes of up to 128 rows).
__device__ __forceinline__ unsigned live_bit(const unsigned (&lw)[4], int y) {
    const unsigned w = y < 64 ? (y < 32 ? lw[0] : lw[1]) : (y < 96 ? lw[2] : lw[3]);
    return (w >> (y & 31)) & 1u;
}

// Carves the plane kernels' shared memory.
template <typename T, int R1, int R2, int THREADS, bool FWD>
struct PlaneTables {
    using Sm = PlaneSmem<T, R1, R2, THREADS, FWD>;
    static constexpr int N = Sm::L::N;
    cx<T>* plane;
    cx<T>* tw;
    cx<T>* phs;
    unsigned* amask_w;
    short* prl;
    short* lst;
    unsigned short* tmask;
    short* items;
    __device__ explicit PlaneTables(unsigned char* raw) {
        plane = reinterpret_cast<cx<T>*>(raw);
        tw = plane + N * Sm::L::LDP;
        phs = tw + N;
        amask_w = reinterpret_cast<unsigned*>(phs + (FWD ? Sm::KA * THREADS : 0));
        prl = reinterpret_cast<short*>(amask_w + Sm::AW);
        lst = prl + N + 2;
        tmask = reinterpret_cast<unsigned short*>(lst + 2 * N);
        items = reinterpret_cast<short*>(tmask + N);
    }
};

template <typename T, int R1, int R2, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB)
    k_xyfwd_plane(const cx<T>* __restrict__ rho, long long rho_stride, const int* __restrict__ row_ptr,
                  const int* __restrict__ cell, cx<T>* __restrict__ out, long long out_stride,
                  const cx<T>* __restrict__ tw_g, RoundPhase rp, int np) {
    using L = PlaneLayout<T, R1, R2>;
    using Sm = PlaneSmem<T, R1, R2, THREADS, true, MINB>;
    static_assert(R1 <= 8 && R2 <= 16 && L::N <= 128, "plane stages serve 16 lanes a row (phase A) and 8 (phase B)");
    static_assert(L::kConflictFree, "plane layout has bank conflicts");
    constexpr int N = L::N, KA = Sm::KA, NW = (N + 31) / 32, KS = Sm::KS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const PlaneTables<T, R1, R2, THREADS, true> tb(smem_raw);
    cx<T>* const stg = reinterpret_cast<cx<T>*>(smem_raw + Sm::stage_off);  // KS atom values
    int* const slt = reinterpret_cast<int*>(stg + KS);                      // their plane positions
    cx<T>* const plane = tb.plane;
    const cx<T>* const tw = tb.tw;
    __shared__ unsigned live_mask[4];
    __shared__ int cnt_sh[2 * NW];
    __shared__ int scan_sh[THREADS / 32];
    const int tid = threadIdx.x, z = blockIdx.x, r0 = z * N;
    // twiddles laid out [t][j] = W_N^(t j): the x stage's phase-B lanes on consecutive j read
    // consecutive words (the y stage's lanes share j: one broadcast)
    for (int i = tid; i < N; i += THREADS) tb.tw[i] = tw_g[(i / R1) * (i % R1)];
    if (tid < 4) live_mask[tid] = 0u;
    __syncthreads();
    const int npairs = plane_rows<L>(row_ptr + r0, false, tb.prl, tb.lst, live_mask, cnt_sh);
    const int a0 = row_ptr[r0], a1 = row_ptr[r0 + N];
    const int n_items = plane_items<L, R2, THREADS>(cell, a0, a1, r0, tb.amask_w, tb.tmask, tb.items, scan_sh);
    const unsigned char* am = reinterpret_cast<const unsigned char*>(tb.amask_w);
    const unsigned lw[4] = {live_mask[0], live_mask[1], live_mask[2], live_mask[3]};
    const bool pre = (a1 - a0) <= KA * THREADS;
    int slot[KA];
#pragma unroll
    for (int k = 0; k < KA; ++k) {
        const int i = a0 + tid + k * THREADS;
        slot[k] = -1;
        if (pre && i < a1) {
            const int c = cell[i];
            const int row = c / N, x = c - row * N, y = row - r0;
            slot[k] = L::rowbase(y) + L::pos(x);
            tb.phs[k * THREADS + tid] = narrow<T>(round_phase(rp, x, y, z));
        }
    }
    // planes with more atoms than the register slots: the next density's atom values are copied
    // into shared memory (cp.async, each thread the atoms it scatters) while this one is
    // transformed
    const bool staged = KS > 0 && !pre && (a1 - a0) <= KS;
    const bool has_phase = (rp.kx | rp.ky | rp.kz) != 0;
    if (staged) {
        for (int i = tid; i < a1 - a0; i += THREADS) {
            const int c = cell[a0 + i];
            const int row = c / N, x = c - row * N, y = row - r0;
            slt[i] = L::rowbase(y) + L::pos(x);
        }
    }
    const auto stage_issue = [&](int p) {
        const cx<T>* src = rho + (long long)p * rho_stride + a0;
        for (int i = tid; i < a1 - a0; i += THREADS) cp_async_cx(stg + i, src + i);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    const int per = (np + gridDim.y - 1) / gridDim.y;
    const int p_begin = blockIdx.y * per, p_end = min(np, p_begin + per);
    cx<T> rv[KA], rn[KA];
    const auto load = [&](int p, cx<T>(&v)[KA]) {
        const cx<T>* src = rho + (long long)p * rho_stride + a0 + tid;
#pragma unroll
        for (int k = 0; k < KA; ++k) v[k] = slot[k] >= 0 ? src[k * THREADS] : mk(T(0), T(0));
    };
    if (pre && p_begin < p_end) load(p_begin, rv);
    if (staged && p_begin < p_end) stage_issue(p_begin);
    __syncthreads();
    // The plane is never cleared: every read below takes only points written for the current
    // density (atom points, masked by amask / tmask / the live rows) and zero for the rest.
    for (int p = p_begin; p < p_end; ++p) {
        if (pre) {
#pragma unroll
            for (int k = 0; k < KA; ++k)
                if (slot[k] >= 0) plane[slot[k]] = cmulc(rv[k], tb.phs[k * THREADS + tid]);
            if (p + 1 < p_end) load(p + 1, rn);
        } else if (staged) {
            asm volatile("cp.async.wait_all;\n" ::: "memory");  // this thread's copies of density p
            for (int i = tid; i < a1 - a0; i += THREADS) {
                cx<T> v = stg[i];
                if (has_phase) {
                    const int c = cell[a0 + i];
                    const int row = c / N, x = c - row * N, y = row - r0;
                    v = narrow<T>(cmulc(widen(v), round_phase(rp, x, y, z)));
                }
                plane[slt[i]] = v;
            }
        } else {
            const cx<T>* rp_ = rho + (long long)p * rho_stride;
            for (int i = a0 + tid; i < a1; i += THREADS) {
                const int c = cell[i];
                const int row = c / N, x = c - row * N, y = row - r0;
                plane[L::rowbase(y) + L::pos(x)] = narrow<T>(cmulc(widen(rp_[i]), round_phase(rp, x, y, z)));
            }
        }
        __syncthreads();
        if (staged && p + 1 < p_end) stage_issue(p + 1);  // every value of density p is scattered
        // x, phase A: the items (row, t) with atoms, their atom points only
        for (int i = tid; i < n_items; i += THREADS) {
            const int code = tb.items[i];
            const int y = code >> 4, t = code & 15;
            const unsigned mm = am[y * R2 + t];
            cx<T>* row = plane + L::rowbase(y);
            cx<T> v[R1];
#pragma unroll
            for (int m = 0; m < R1; ++m) v[m] = ((mm >> m) & 1u) ? row[L::pos(t + R2 * m)] : mk(T(0), T(0));
            dft<R1, -1>(v);
#pragma unroll
            for (int m = 0; m < R1; ++m) row[L::pos(t + R2 * m)] = v[m];
        }
        __syncthreads();
        // x, phase B: rows with atoms, 8 lanes a row, two rows a 16-lane group
        for (int i = tid; i < npairs * 16; i += THREADS) {
            const int j = i & 7, pr = tb.prl[i >> 3];
            if (pr >= 0 && j < R1) {
                const unsigned tm = tb.tmask[pr];
                cx<T>* row = plane + L::rowbase(pr);
                cx<T> u[R2];
#pragma unroll
                for (int t = 0; t < R2; ++t) u[t] = ((tm >> t) & 1u) ? row[L::pos(R2 * j + t)] : mk(T(0), T(0));
#pragma unroll
                for (int t = 1; t < R2; ++t) u[t] = cmul(u[t], tw[t * R1 + j]);
                dft<R2, -1>(u);
#pragma unroll
                for (int s = 0; s < R2; ++s) row[L::pos(R2 * j + s)] = u[s];
            }
        }
        __syncthreads();
        // y, phase A: every column, lanes on consecutive kx; rows without atoms read as zero.
        // Where the launch leaves a thread 128 registers or more (FP32), the loads of all of its
        // items are issued before the first transform; otherwise one item at a time (measured:
        // batching spills at 80 registers and is slower there).
        constexpr bool kBatch = sizeof(T) == 4 && 65536 / (THREADS * MINB) >= 128;
        if constexpr (kBatch) {
            constexpr int IA = (N * R2 + THREADS - 1) / THREADS;
            cx<T> v[IA][R1];
#pragma unroll
            for (int a = 0; a < IA; ++a) {
                const int i = tid + a * THREADS;
                const int kx = i % N, t = i / N;
                const cx<T>* col = plane + L::pos(L::dig(kx));
#pragma unroll
                for (int m = 0; m < R1; ++m)
                    v[a][m] = (i < N * R2 && live_bit(lw, t + R2 * m)) ? col[L::rowbase(t) + m * L::RSTEP]
                                                                       : mk(T(0), T(0));
            }
#pragma unroll
            for (int a = 0; a < IA; ++a) {
                const int i = tid + a * THREADS;
                if (i < N * R2) {
                    const int kx = i % N, t = i / N;
                    dft<R1, -1>(v[a]);
                    cx<T>* col = plane + L::pos(L::dig(kx));
#pragma unroll
                    for (int m = 0; m < R1; ++m) col[L::rowbase(t) + m * L::RSTEP] = v[a][m];
                }
            }
        } else {
#pragma unroll 1
            for (int i = tid; i < N * R2; i += THREADS) {
                const int kx = i % N, t = i / N;
                cx<T>* col = plane + L::pos(L::dig(kx));
                cx<T> v[R1];
#pragma unroll
                for (int m = 0; m < R1; ++m)
                    v[m] = live_bit(lw, t + R2 * m) ? col[L::rowbase(t) + m * L::RSTEP] : mk(T(0), T(0));
                dft<R1, -1>(v);
#pragma unroll
                for (int m = 0; m < R1; ++m) col[L::rowbase(t) + m * L::RSTEP] = v[m];
            }
        }
        __syncthreads();
        // y, phase B: outputs to HBM in natural order
        cx<T>* o = out + (long long)p * out_stride + (long long)z * N * N;
#pragma unroll 1
        for (int i = tid; i < N * R1; i += THREADS) {
            const int kx = i % N, j = i / N;
            cx<T>* col = plane + L::pos(L::dig(kx));
            cx<T> u[R2];
#pragma unroll
            for (int t = 0; t < R2; ++t) u[t] = col[j * L::RSTEP + L::rowbase(t)];
#pragma unroll
            for (int t = 1; t < R2; ++t) u[t] = cmul(u[t], tw[t * R1 + j]);
            dft<R2, -1>(u);
#pragma unroll
            for (int s = 0; s < R2; ++s) o[(long long)(j + R1 * s) * N + kx] = u[s];
        }
        __syncthreads();
        if (pre) {
#pragma unroll
            for (int k = 0; k < KA; ++k) rv[k] = rn[k];
        }
    }
}

template <typename T, int R1, int R2, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB)
    k_xyinv_plane(const cx<T>* __restrict__ buf, long long stride, const cx<T>* __restrict__ tw_g,
                  const int* __restrict__ row_ptr, const int* __restrict__ cell, cx<T>* __restrict__ out,
                  long long o_stride, int np) {
    using L = PlaneLayout<T, R1, R2>;
    using Sm = PlaneSmem<T, R1, R2, THREADS, false>;
    static_assert(R1 <= 8 && R2 <= 16 && L::N <= 128, "plane stages serve 16 lanes a row (phase A) and 8 (phase B)");
    static_assert(L::kConflictFree, "plane layout has bank conflicts");
    constexpr int N = L::N, KA = Sm::KA, NW = (N + 31) / 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const PlaneTables<T, R1, R2, THREADS, false> tb(smem_raw);
    cx<T>* const plane = tb.plane;
    const cx<T>* const tw = tb.tw;
    __shared__ unsigned live_mask[4];
    __shared__ int cnt_sh[2 * NW];
    __shared__ int scan_sh[THREADS / 32];
    const int tid = threadIdx.x, z = blockIdx.x, r0 = z * N;
    // twiddles laid out [t][j] = W_N^(t j): the x stage's phase-B lanes on consecutive j read
    // consecutive words (the y stage's lanes share j: one broadcast)
    for (int i = tid; i < N; i += THREADS) tb.tw[i] = tw_g[(i / R1) * (i % R1)];
    if (tid < 4) live_mask[tid] = 0u;
    __syncthreads();
    const int npairs = plane_rows<L>(row_ptr + r0, true, tb.prl, tb.lst, live_mask, cnt_sh);
    const int a0 = row_ptr[r0], a1 = row_ptr[r0 + N];
    const int n_items = plane_items<L, R2, THREADS>(cell, a0, a1, r0, tb.amask_w, tb.tmask, tb.items, scan_sh);
    const unsigned char* am = reinterpret_cast<const unsigned char*>(tb.amask_w);
    const unsigned lw[4] = {live_mask[0], live_mask[1], live_mask[2], live_mask[3]};
    const bool pre = (a1 - a0) <= KA * THREADS;
    int slot[KA];
#pragma unroll
    for (int k = 0; k < KA; ++k) {
        const int i = a0 + tid + k * THREADS;
        slot[k] = -1;
        if (pre && i < a1) {
            const int c = cell[i];
            const int row = c / N, x = c - row * N, y = row - r0;
            slot[k] = L::rowbase(L::dig(y)) + L::pos(x);
        }
    }
    const int per = (np + gridDim.y - 1) / gridDim.y;
    const int p_begin = blockIdx.y * per, p_end = min(np, p_begin + per);
    for (int p = p_begin; p < p_end; ++p) {
        const cx<T>* src = buf + (long long)p * stride + (long long)z * N * N;
        // y, phase A: columns loaded from HBM (lanes on consecutive kx), natural order in; the
        // loads of all of a thread's items are issued before the first transform
        constexpr int IA = (N * R2 + THREADS - 1) / THREADS;
        cx<T> v[IA][R1];
#pragma unroll
        for (int a = 0; a < IA; ++a) {
            const int i = tid + a * THREADS;
            const int kx = i % N, t = i / N;
#pragma unroll
            for (int m = 0; m < R1; ++m)
                v[a][m] = i < N * R2 ? src[(long long)(t + R2 * m) * N + kx] : mk(T(0), T(0));
        }
#pragma unroll
        for (int a = 0; a < IA; ++a) {
            const int i = tid + a * THREADS;
            if (i < N * R2) {
                const int kx = i % N, t = i / N;
                dft<R1, +1>(v[a]);
                cx<T>* col = plane + L::pos(L::dig(kx));
#pragma unroll
                for (int m = 0; m < R1; ++m) col[L::rowbase(t) + m * L::RSTEP] = v[a][m];
            }
        }
        __syncthreads();
        // y, phase B: digit-order rows out, kept only for the rows with atoms
#pragma unroll 1
        for (int i = tid; i < N * R1; i += THREADS) {
            const int kx = i % N, j = i / N;
            cx<T>* col = plane + L::pos(L::dig(kx));
            cx<T> u[R2];
#pragma unroll
            for (int t = 0; t < R2; ++t) u[t] = col[j * L::RSTEP + L::rowbase(t)];
#pragma unroll
            for (int t = 1; t < R2; ++t) u[t] = cmulc(u[t], tw[t * R1 + j]);
            dft<R2, +1>(u);
#pragma unroll
            for (int s = 0; s < R2; ++s)
                if (live_bit(lw, j + R1 * s)) col[j * L::RSTEP + L::rowbase(s)] = u[s];
        }
        __syncthreads();
        // x, phase B pattern first (digit order in); only the points of items with atoms kept
        for (int i = tid; i < npairs * 16; i += THREADS) {
            const int j = i & 7, pr = tb.prl[i >> 3];
            if (pr >= 0 && j < R1) {
                const unsigned tm = tb.tmask[(pr % R2) * R1 + pr / R2];  // natural row of pr = dig(y)
                cx<T>* row = plane + L::rowbase(pr);
                cx<T> u[R2];
#pragma unroll
                for (int s = 0; s < R2; ++s) u[s] = row[L::pos(R2 * j + s)];
                dft<R2, +1>(u);
#pragma unroll
                for (int t = 1; t < R2; ++t) u[t] = cmulc(u[t], tw[t * R1 + j]);
#pragma unroll
                for (int t = 0; t < R2; ++t)
                    if ((tm >> t) & 1u) row[L::pos(R2 * j + t)] = u[t];
            }
        }
        __syncthreads();
        // x, phase A pattern (natural order out): the items with atoms, their atom points only
        for (int i = tid; i < n_items; i += THREADS) {
            const int code = tb.items[i];
            const int y = code >> 4, t = code & 15;
            const unsigned mm = am[y * R2 + t];
            cx<T>* row = plane + L::rowbase(L::dig(y));
            cx<T> v[R1];
#pragma unroll
            for (int j = 0; j < R1; ++j) v[j] = row[L::pos(R2 * j + t)];
            dft<R1, +1>(v);
#pragma unroll
            for (int m = 0; m < R1; ++m)
                if ((mm >> m) & 1u) row[L::pos(t + R2 * m)] = v[m];
        }
        __syncthreads();
        cx<T>* op = out + (long long)p * o_stride;
        if (pre) {
#pragma unroll
            for (int k = 0; k < KA; ++k)
                if (slot[k] >= 0) op[a0 + tid + k * THREADS] = plane[slot[k]];
        } else {
            for (int i = a0 + tid; i < a1; i += THREADS) {
                const int c = cell[i];
                const int row = c / N, x = c - row * N, y = row - r0;
                op[i] = plane[L::rowbase(L::dig(y)) + L::pos(x)];
            }
        }
        __syncthreads();
    }
}

// Compiled plane shapes (square planes): N = R1*R2 with R1 <= 8, R2 <= 16; threads per block
// and resident blocks per SM chosen so that the plane (and, forward, the atom phases) fits:
// FP32 64^2 (52 KB forward, three blocks an SM), FP32 96^2 (101 KB, two blocks), FP32 128^2
// (168 KB), FP64 64^2 (91 KB, two blocks), FP64 96^2 (186 KB).
template <typename T, typename F>
bool with_plane(int nx, int ny, F&& f) {
    if (nx != ny) return false;
    if constexpr (sizeof(T) == 4) {
        switch (nx) {
            case 64: f(SplitTag<8, 8>{}, std::integral_constant<int, 256>{}, std::integral_constant<int, 3>{}); return true;
            case 96: f(SplitTag<8, 12>{}, std::integral_constant<int, 384>{}, std::integral_constant<int, 2>{}); return true;
            case 128: f(SplitTag<8, 16>{}, std::integral_constant<int, 512>{}, std::integral_constant<int, 1>{}); return true;
            default: return false;
        }
    } else {
        switch (nx) {
            case 64: f(SplitTag<8, 8>{}, std::integral_constant<int, 256>{}, std::integral_constant<int, 2>{}); return true;
            case 96: f(SplitTag<8, 12>{}, std::integral_constant<int, 384>{}, std::integral_constant<int, 1>{}); return true;
            default: return false;
        }
    }
}

}  // namespace clk
