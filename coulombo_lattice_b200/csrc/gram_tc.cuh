// Split-precision tensor-core Gram over atoms (FP32 form).
//
// The reductions of CoulombCalculator::calculate (CoulombCalculator.cpp:165-172), restricted
// to atom cells and batched over every (left, right) pair of a request, form the real Gram
//   C = A . B^T,  A rows = {Re V_l, Im V_l} (2 per left density),
//                 B rows = {Re rho_r, Im rho_r} (2 per right density),  K = atoms,
// whose 2x2 blocks are {sum ac, sum ad; sum bc, sum bd} for V = a+ib, rho = c+id.
//
// Each FP64 operand is split into two TF32 parts, x = hi + lo (both rounded to nearest), and
// C = A_hi.B_hi + (A_hi.B_lo + A_lo.B_hi) is accumulated by tcgen05 MMAs (kind::tf32, M=128,
// N=128, K=8) in FP32 in tensor memory.  The tensor cores' FP32 accumulation rounds toward
// zero, a bias that grows with every MMA added into a running sum.  So the main products go to
// an accumulator that is drained into FP64 registers after every k-tile of 32 atoms (4 MMAs,
// double-buffered in tensor memory), while the two correction products -- 2^-11 of the main
// ones and of random sign, the lo parts being round-to-nearest residuals -- accumulate in a
// third accumulator over the block's whole atom range and are drained once.  The drained
// partial sums are added across the atom range in FP64 and then across atom splits with FP64
// atomics.  The dropped lo.lo term and
// the rounding of the parts are ~2^-22 of each product.
//
// Operands are staged by TMA (no multicast) into 128-byte-swizzled shared-memory tiles: one
// warp issues the copies, one lane issues the MMAs, eight warps drain the accumulator.
// Every wait is bounded by a clock deadline; on expiry the block records an error in the
// slot after the results, waits (again bounded) for its own copies and MMAs, frees its
// tensor memory and returns.
#pragma once

#include <cuda.h>
#include <cstdint>

#include "fft.cuh"

namespace clk {
namespace tc {

constexpr int BM = 128;          // A rows per tile (64 left densities)
constexpr int BN = 128;          // B rows per tile (64 right densities)
constexpr int BK = 32;           // atoms per k-tile: 32 x 4 B = one 128-byte swizzle row
constexpr int STAGES = 3;        // shared-memory pipeline depth
constexpr int CH = 1;            // k-tiles per FP32 accumulation chunk (32 atoms)
constexpr int A_BYTES = BM * BK * 4;
constexpr int B_BYTES = BN * BK * 4;
constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;  // hi and lo of both operands
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
constexpr int EPI_WARPS = 8;
constexpr int THREADS = 32 * (2 + EPI_WARPS);
constexpr uint32_t TMEM_COLS = 4 * BN;  // main x double buffer, correction, unused; FP32
constexpr long long TIMEOUT_CYCLES = 1LL << 32;  // ~2 s at B200 clocks

static_assert(BN == 128 && BM == 128, "epilogue mapping assumes 128x128 tiles");

// Instruction descriptor, kind::tf32: D F32 (bits 4-5 = 1), A and B TF32 (bits 7-9, 10-12
// = 2), both K-major (bits 15, 16 = 0), N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t a, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t a) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint32_t a, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the phase of parity `parity` to complete.  Returns false when the deadline
// passes (and raises the block's abort flag) or when another role has already aborted.
__device__ __forceinline__ bool mbar_wait(uint32_t a, uint32_t parity, volatile int* abort_flag) {
    const long long t0 = clock64();
    while (!mbar_test(a, parity)) {
        if (*abort_flag) return false;
        if (clock64() - t0 > TIMEOUT_CYCLES) {
            *abort_flag = 1;
            return false;
        }
    }
    return true;
}
// Teardown wait that ignores the abort flag (still bounded).
__device__ __forceinline__ void mbar_drain(uint32_t a, uint32_t parity) {
    const long long t0 = clock64();
    while (!mbar_test(a, parity))
        if (clock64() - t0 > TIMEOUT_CYCLES) return;
}

// Tile (x = atom, y = row, z = part) of a [part][row][atom] operand; rows beyond the operand's
// real rows are filled with zeros by the copy itself (nothing is read for them).
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y, int z,
                                            uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(mbar)
        : "memory");
}

// Shared-memory matrix descriptor of a K-major tile with the 128-byte swizzle: start address
// >> 4, leading offset 1 (unused for swizzled K-major), stride 1024 B between 8-row groups,
// descriptor version 1 (bit 46), layout type 2 = SWIZZLE_128B (bits 61-63).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) |
           (2ull << 61);
}

__device__ __forceinline__ void mma_tf32(uint32_t d, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(IDESC), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive FP32 accumulator columns of this thread's lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float tf32_rn(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// ---------------------------------------------------------------------------------------
// Split pass: density d of `src` (row idx[d], or d; complex of S) over atoms [a0, a0 + na) ->
//   dst[part][2d + {0: re, 1: im}][k], part 0 = hi, 1 = lo, 2n rows a part; k >= na are zero.
// grid.y = n densities, grid.x strides over k.  (The Gram's tiles are 128 rows; its copies fill
// the rows beyond 2n with zeros, so no padding is stored.)
// ---------------------------------------------------------------------------------------
template <typename S>
__global__ void __launch_bounds__(256) k_tf32_split(const cx<S>* __restrict__ src, long long stride,
                                                    const int* __restrict__ idx, int n, long long a0,
                                                    long long na, long long k_pad, float* __restrict__ dst) {
    const int d = blockIdx.y;
    const long long plane = (long long)(2 * n) * k_pad;
    float* hre = dst + (long long)(2 * d) * k_pad;
    float* him = hre + k_pad;
    const cx<S>* s = src + (long long)(idx ? idx[d] : d) * stride + a0;
    for (long long k = blockIdx.x * 256LL + threadIdx.x; k < k_pad; k += (long long)gridDim.x * 256) {
        double re = 0.0, im = 0.0;
        if (k < na) {
            const cx<S> z = s[k];
            re = (double)z.re;
            im = (double)z.im;
        }
        const float hr = tf32_rn((float)re), hi_ = tf32_rn((float)im);
        hre[k] = hr;
        him[k] = hi_;
        hre[plane + k] = tf32_rn((float)(re - (double)hr));
        him[plane + k] = tf32_rn((float)(im - (double)hi_));
    }
}

// ---------------------------------------------------------------------------------------
// The Gram.  grid = (ceil(2 nl / BM), ceil(2 nr / BN), splits); block z covers k-tiles
// [z * kt_per, min(kt_total, (z + 1) * kt_per)), never empty.  out4[l][r] += {ac, bd, ad, bc};
// out4[4 * nl * nr] (as int) is set to 1 if any wait expired.
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(THREADS, 1)
    k_gram_tc(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, int kt_total,
              int kt_per, int nl, int nr, double* __restrict__ out4) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    unsigned char* gbase = smem_raw + (base - raw);
    uint64_t* bars = reinterpret_cast<uint64_t*>(gbase + STAGES * STAGE_BYTES);
    // bars: full[STAGES], empty[STAGES], acc_full[2], acc_empty[2], drain
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * STAGES + 5);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    const auto bar = [&](int i) { return smem_u32(bars + i); };
    const int FULL = 0, EMPTY = STAGES, ACCF = 2 * STAGES, ACCE = 2 * STAGES + 2, DRAIN = 2 * STAGES + 4;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    const int kt0 = blockIdx.z * kt_per;
    const int kt1 = min(kt_total, kt0 + kt_per);
    const int nchunks = (kt1 - kt0 + CH - 1) / CH;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(bar(FULL + s), 1);
            mbar_init(bar(EMPTY + s), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(bar(ACCF + b), 1);
            mbar_init(bar(ACCE + b), EPI_WARPS);  // one arrival a warp, after __syncwarp
        }
        mbar_init(bar(DRAIN), 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // ---- TMA producer ----
            int s = 0;
            uint32_t ph = 0;
            int issued = 0;
            for (int kt = kt0; kt < kt1; ++kt) {
                if (!mbar_wait(bar(EMPTY + s), ph ^ 1u, abort_flag)) break;
                const uint32_t st = base + (uint32_t)(s * STAGE_BYTES);
                mbar_expect_tx(bar(FULL + s), STAGE_BYTES);
                const int x = kt * BK;
                tma_load_3d(st, &mapA, x, m0, 0, bar(FULL + s));
                tma_load_3d(st + A_BYTES, &mapA, x, m0, 1, bar(FULL + s));
                tma_load_3d(st + 2 * A_BYTES, &mapB, x, n0, 0, bar(FULL + s));
                tma_load_3d(st + 2 * A_BYTES + B_BYTES, &mapB, x, n0, 1, bar(FULL + s));
                ++issued;
                if (++s == STAGES) {
                    s = 0;
                    ph ^= 1u;
                }
            }
            if (*abort_flag) {
                // let the last (up to STAGES) copies land before the block's memory goes away
                for (int i = 1; i <= min(issued, STAGES); ++i) {
                    const int n = issued - i;
                    mbar_drain(bar(FULL + n % STAGES), (uint32_t)((n / STAGES) & 1));
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---- MMA issuer ----
            int s = 0;
            uint32_t ph = 0;
            int kt = kt0;
            bool issued_any = false;
            for (int ch = 0; ch < nchunks; ++ch) {
                const int b = ch & 1;
                if (!mbar_wait(bar(ACCE + b), (uint32_t)(((ch >> 1) & 1) ^ 1), abort_flag)) break;
                fence_after();
                const uint32_t dm = tmem + (uint32_t)(b * BN);  // main products of this chunk
                const uint32_t dc = tmem + (uint32_t)(2 * BN);  // correction products, whole range
                const int kend = min(kt1, kt + CH);
                bool ok = true;
                uint32_t acc = 0;
                for (; kt < kend; ++kt) {
                    if (!mbar_wait(bar(FULL + s), ph, abort_flag)) {
                        ok = false;
                        break;
                    }
                    fence_after();
                    const uint32_t st = base + (uint32_t)(s * STAGE_BYTES);
#pragma unroll
                    for (int kk = 0; kk < BK / 8; ++kk) {
                        const uint64_t ahi = sw128_desc(st + kk * 32);
                        const uint64_t alo = sw128_desc(st + A_BYTES + kk * 32);
                        const uint64_t bhi = sw128_desc(st + 2 * A_BYTES + kk * 32);
                        const uint64_t blo = sw128_desc(st + 2 * A_BYTES + B_BYTES + kk * 32);
                        mma_tf32(dm, ahi, bhi, acc);
                        mma_tf32(dc, alo, bhi, (ch > 0 || acc) ? 1u : 0u);
                        mma_tf32(dc, ahi, blo, 1u);
                        acc = 1u;
                    }
                    issued_any = true;
                    mma_commit(bar(EMPTY + s));  // the stage is free once these MMAs finish
                    if (++s == STAGES) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
                if (!ok) break;
                mma_commit(bar(ACCF + b));  // chunk complete in accumulator b
            }
            if (*abort_flag && issued_any) {
                mma_commit(bar(DRAIN));
                mbar_drain(bar(DRAIN), 0);
            }
        }
    } else {
        // ---- epilogue: FP32 accumulator -> FP64 registers ----
        const int q = warp & 3;             // tensor-memory lane quarter this warp may read
        const int h = (warp - 2) >> 2;      // column half
        double acc[64];
#pragma unroll
        for (int i = 0; i < 64; ++i) acc[i] = 0.0;
        bool ok = true;
        for (int ch = 0; ch < nchunks; ++ch) {
            const int b = ch & 1;
            bool got = mbar_wait(bar(ACCF + b), (uint32_t)((ch >> 1) & 1), abort_flag);
            got = __all_sync(0xffffffffu, got);
            if (!got) {
                ok = false;
                break;
            }
            fence_after();
            const uint32_t ta = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(b * BN + h * 64);
            float v[32];
            tmem_ld32(ta, v);
#pragma unroll
            for (int i = 0; i < 32; ++i) acc[i] += (double)v[i];
            tmem_ld32(ta + 32, v);
#pragma unroll
            for (int i = 0; i < 32; ++i) acc[32 + i] += (double)v[i];
            fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(bar(ACCE + b));
        }
        if (ok) {
            // the correction accumulator is complete with the last chunk's commit
            fence_after();
            const uint32_t tc_ = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(2 * BN + h * 64);
            float v[32];
            tmem_ld32(tc_, v);
#pragma unroll
            for (int i = 0; i < 32; ++i) acc[i] += (double)v[i];
            tmem_ld32(tc_ + 32, v);
#pragma unroll
            for (int i = 0; i < 32; ++i) acc[32 + i] += (double)v[i];
        }
        if (ok) {
            const int R = m0 + 32 * q + lane;
            const int l = R >> 1, pa = R & 1;
            if (l < nl) {
#pragma unroll
                for (int j = 0; j < 64; ++j) {
                    const int Cg = n0 + h * 64 + j;
                    const int r = Cg >> 1, pc = Cg & 1;
                    if (r < nr) {
                        const int qi = (pa == pc) ? pa : 2 + pa;  // ac, bd, ad, bc
                        atomicAdd(out4 + ((long long)l * nr + r) * 4 + qi, acc[j]);
                    }
                }
            }
        }
    }

    fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && *abort_flag)
        *reinterpret_cast<volatile int*>(out4 + (long long)4 * nl * nr) = 1;
    if (warp == 1) {
        __syncwarp();
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// ---------------------------------------------------------------------------------------
// Fused Gram for FP32 operands (the FP32 sub-lattice form: FP32 potentials and pair densities).
// The split happens inside the kernel, so neither the hi/lo operands nor any padding reach HBM.
// Sixteen warps, each with three jobs per k-tile of 32 atoms:
//   copy    8-byte cp.async of the raw complex values of its densities into a ring of AHEAD+1
//           raw slots, AHEAD tiles ahead: a lane takes 4 consecutive atoms of one density, 8
//           lanes a density, a warp 4 densities (4w + 64j + lane/8: left densities of the
//           block's A tile, then right densities of its B tile); a density's 256-byte raw row
//           holds each lane's first two atoms in its first half and the other two in its second;
//   convert round the lane's 4 values to TF32 hi and lo parts and store them with four 16-byte
//           stores (re hi, im hi, re lo, im lo) into the MMA stage in the 128-byte-swizzled
//           K-major layout the descriptors expect -- row r, atoms 4c..4c+3 at (r/8)*1024 +
//           (r%8)*128 + ((c ^ (r%8))*16): 8 lanes fill one row without bank conflicts -- fence
//           the stores to the async proxy and arrive on the stage's full barrier (then thread 0
//           issues the tile's MMAs as in k_gram_tc, with N = the block's right rows rounded up
//           to 16);
//   drain   the previous k-tile's main products, tensor memory -> FP64 registers: lane quarter
//           w % 4, accumulator columns 32 (w / 4) .. + 31.
// Rows beyond the real ones are zeroed once at the start and never written again.  Each thread
// reads back only the raw values it copied itself, so its own cp.async group wait is the only
// ordering the raw ring needs.
// ---------------------------------------------------------------------------------------
struct FusedGram {
    const float2* V;      // left densities: V[l * v_stride + atom]
    long long v_stride;
    const float2* rho;    // right densities: rho[(ridx ? ridx[r] : r) * r_stride + atom]
    long long r_stride;
    const int* ridx;
    int nl, nr;
    long long na;         // atoms
    int kt_total, kt_per;
    uint32_t stage_bytes;     // 2 * BM * 128 + 2 * nb_max * 128
    uint32_t raw_slot_bytes;  // (left + right densities of a block, at most) * 32 * 8
    double* out4;
    int aligned16;            // every density row starts on a 16-byte boundary (16-byte copies)
};

constexpr int FUSED_WARPS = 16;
constexpr int FUSED_THREADS = 32 * FUSED_WARPS;
constexpr int FUSED_MMA_STAGES = 2;
constexpr int FUSED_MAX_DENS = BM / 2 + BN / 2;  // densities a block converts per k-tile

__host__ __device__ constexpr uint32_t fused_idesc(int nb) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(nb >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}
// Bytes of dynamic shared memory: alignment slack, the MMA stages, the raw ring, the source
// table and the barriers.
__host__ __device__ constexpr size_t fused_smem_bytes(uint32_t stage_bytes, uint32_t raw_slot_bytes, int ahead) {
    return 1024 + (size_t)FUSED_MMA_STAGES * stage_bytes + (size_t)(ahead + 1) * raw_slot_bytes +
           sizeof(void*) * FUSED_MAX_DENS + 256;
}

// Byte offset of the 16-byte chunk c (atoms 4c..4c+3) of row r in a 128-byte-swizzled tile.
__device__ __forceinline__ uint32_t sw128_chunk(int row, int c) {
    return (uint32_t)((row >> 3) * 1024 + (row & 7) * 128 + ((c ^ (row & 7)) << 4));
}
__device__ __forceinline__ void mma_tf32_n(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
// 16 bytes, of which the first src_bytes (0, 8 or 16) are read and the rest zero-filled.
__device__ __forceinline__ void cp_async16z(uint32_t dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// grid = (ceil(2 nl / BM), ceil(2 nr / BN), splits); block z covers k-tiles
// [z * kt_per, min(kt_total, (z + 1) * kt_per)), never empty.  out4 as for k_gram_tc.
template <int AHEAD>
__global__ void __launch_bounds__(FUSED_THREADS, 1) k_gram_tc_fused(const FusedGram g) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    unsigned char* gbase = smem_raw + (base - raw);
    const uint32_t ring_off = FUSED_MMA_STAGES * g.stage_bytes;
    const float2** src_tab = reinterpret_cast<const float2**>(gbase + ring_off + (AHEAD + 1) * g.raw_slot_bytes);
    uint64_t* bars = reinterpret_cast<uint64_t*>(src_tab + FUSED_MAX_DENS);
    // bars: full[2], empty[2], acc_full[2], acc_empty[2], drain
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 9);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    const auto bar = [&](int i) { return smem_u32(bars + i); };
    constexpr int FULL = 0, EMPTY = 2, ACCF = 4, ACCE = 6, DRAIN = 8;
    constexpr uint32_t A_PART = BM * 128;  // bytes of one TF32 part of the A tile
    const uint32_t b_part = (g.stage_bytes - 2u * A_PART) / 2u;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    const int la0 = m0 / 2, rb0 = n0 / 2;
    const int nA = min(BM / 2, g.nl - la0), nB = min(BN / 2, g.nr - rb0);
    const int nd = nA + nB;
    const int nb = max(16, (2 * nB + 15) / 16 * 16);  // MMA N: the block's right rows, rounded up
    const uint32_t idesc = fused_idesc(nb);
    const int kt0 = blockIdx.z * g.kt_per;
    const int nt = min(g.kt_total, kt0 + g.kt_per) - kt0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < FUSED_MMA_STAGES; ++s) {
            mbar_init(bar(FULL + s), FUSED_WARPS);  // one arrival a warp, after __syncwarp
            mbar_init(bar(EMPTY + s), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(bar(ACCF + b), 1);
            mbar_init(bar(ACCE + b), FUSED_WARPS);
        }
        mbar_init(bar(DRAIN), 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    for (int i = threadIdx.x; i < nd; i += FUSED_THREADS) {
        if (i < nA) {
            src_tab[i] = g.V + (long long)(la0 + i) * g.v_stride;
        } else {
            const int r = rb0 + (i - nA);
            src_tab[i] = g.rho + (long long)(g.ridx ? g.ridx[r] : r) * g.r_stride;
        }
    }
    // zero both MMA stages once: rows beyond the real ones are never written again
    for (uint32_t o = threadIdx.x * 16u; o < ring_off; o += FUSED_THREADS * 16u)
        *reinterpret_cast<uint4*>(gbase + o) = make_uint4(0u, 0u, 0u, 0u);
    fence_proxy_async();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;

    const int dsub = lane >> 3;       // density of the warp's four this lane converts
    const int quad = lane & 7;        // atoms 4 quad .. 4 quad + 3 of the k-tile
    const int q = warp & 3;           // tensor-memory lane quarter this warp may read
    const int c0 = (warp >> 2) * 32;  // first accumulator column this warp drains
    bool issued_any = false;          // thread 0: MMAs issued
    // thread 0: the MMAs of k-tile t, once its stage is full and its accumulator drained
    const auto mma_tile = [&](int t) -> bool {
        const int s = t & 1, b = t & 1;
        const uint32_t ph = (uint32_t)((t >> 1) & 1);
        if (!mbar_wait(bar(ACCE + b), ph ^ 1u, abort_flag)) return false;
        if (!mbar_wait(bar(FULL + s), ph, abort_flag)) return false;
        fence_after();
        const uint32_t st = base + (uint32_t)s * g.stage_bytes;
        const uint32_t dm = tmem + (uint32_t)(b * BN);  // main products of this k-tile
        const uint32_t dc = tmem + (uint32_t)(2 * BN);  // correction products, whole range
#pragma unroll
        for (int kk = 0; kk < BK / 8; ++kk) {
            const uint64_t ahi = sw128_desc(st + kk * 32);
            const uint64_t alo = sw128_desc(st + A_PART + kk * 32);
            const uint64_t bhi = sw128_desc(st + 2 * A_PART + kk * 32);
            const uint64_t blo = sw128_desc(st + 2 * A_PART + b_part + kk * 32);
            mma_tf32_n(dm, ahi, bhi, idesc, kk > 0 ? 1u : 0u);
            mma_tf32_n(dc, alo, bhi, idesc, (t > 0 || kk > 0) ? 1u : 0u);
            mma_tf32_n(dc, ahi, blo, idesc, 1u);
        }
        issued_any = true;
        mma_commit(bar(EMPTY + s));  // the stage is free once these MMAs finish
        mma_commit(bar(ACCF + b));   // k-tile complete in accumulator b
        return true;
    };
    double acc[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) acc[i] = 0.0;
    const auto issue = [&](int t) {
        const long long at0 = (long long)(kt0 + t) * BK + 4 * quad;
        // raw density row (256 B): atoms 4q, 4q+1 at 16 q, atoms 4q+2, 4q+3 at 128 + 16 q, so that
        // the 8 lanes of a density read two contiguous 128-byte halves
        const uint32_t slot = base + ring_off + (uint32_t)(t % (AHEAD + 1)) * g.raw_slot_bytes + (uint32_t)quad * 16u;
        for (int i = 4 * warp + dsub; i < nd; i += 4 * FUSED_WARPS) {
            const float2* src = src_tab[i];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const bool in = at0 + e < g.na;
                cp_async8(slot + (uint32_t)i * 256u + 128u * (e >> 1) + 8u * (e & 1), src + (in ? at0 + e : 0LL),
                          in ? 8u : 0u);
            }
        }
    };
    // adds accumulator columns col + c0 .. + 31 of this warp's lanes to acc (after waiting for
    // the MMAs that complete the barrier `mbar`, phase `ph`)
    const auto drain = [&](uint32_t mbar, uint32_t ph, uint32_t col) -> bool {
        bool got = mbar_wait(mbar, ph, abort_flag);
        got = __all_sync(0xffffffffu, got);
        if (!got) return false;
        fence_after();
        if (c0 < nb) {
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + col + (uint32_t)c0, v);
#pragma unroll
            for (int i = 0; i < 32; ++i) acc[i] += (double)v[i];
        }
        fence_before();
        return true;
    };
#pragma unroll 1
    for (int t = 0; t < AHEAD; ++t) {
        if (t < nt) issue(t);
        cp_async_commit();
    }
    bool ok = true;
#pragma unroll 1
    for (int t = 0; t < nt; ++t) {
        if (t + AHEAD < nt) issue(t + AHEAD);
        cp_async_commit();
        cp_async_wait<AHEAD>();  // this thread's copies of k-tile t have landed
        const int s = t & 1;
        bool got = mbar_wait(bar(EMPTY + s), (uint32_t)(((t >> 1) & 1) ^ 1), abort_flag);
        if (!__all_sync(0xffffffffu, got)) {
            ok = false;
            break;
        }
        unsigned char* stg = gbase + (size_t)s * g.stage_bytes;
        const unsigned char* rs = gbase + ring_off + (size_t)(t % (AHEAD + 1)) * g.raw_slot_bytes + quad * 16;
        for (int i = 4 * warp + dsub; i < nd; i += 4 * FUSED_WARPS) {
            const float4 z0 = *reinterpret_cast<const float4*>(rs + i * 256);       // atoms 0, 1
            const float4 z1 = *reinterpret_cast<const float4*>(rs + i * 256 + 128);  // atoms 2, 3
            const float re[4] = {z0.x, z0.z, z1.x, z1.z}, im[4] = {z0.y, z0.w, z1.y, z1.w};
            float rh[4], ih[4], rl[4], il[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                rh[e] = tf32_rn(re[e]);
                ih[e] = tf32_rn(im[e]);
                rl[e] = tf32_rn(re[e] - rh[e]);
                il[e] = tf32_rn(im[e] - ih[e]);
            }
            const bool left = i < nA;
            unsigned char* hi_p = left ? stg : stg + 2 * A_PART;
            unsigned char* lo_p = hi_p + (left ? A_PART : b_part);
            const int row = 2 * (left ? i : i - nA);
            const uint32_t o0 = sw128_chunk(row, quad), o1 = sw128_chunk(row + 1, quad);
            *reinterpret_cast<float4*>(hi_p + o0) = make_float4(rh[0], rh[1], rh[2], rh[3]);
            *reinterpret_cast<float4*>(hi_p + o1) = make_float4(ih[0], ih[1], ih[2], ih[3]);
            *reinterpret_cast<float4*>(lo_p + o0) = make_float4(rl[0], rl[1], rl[2], rl[3]);
            *reinterpret_cast<float4*>(lo_p + o1) = make_float4(il[0], il[1], il[2], il[3]);
        }
        fence_proxy_async();  // the stores, seen by the tensor cores' async proxy
        __syncwarp();
        if (lane == 0) mbar_arrive(bar(FULL + s));
        if (warp == 0) {
            bool go = true;
            if (lane == 0) go = mma_tile(t);
            if (!__shfl_sync(0xffffffffu, go ? 1 : 0, 0)) {
                ok = false;
                break;
            }
        }
        if (t > 0) {
            const int tp = t - 1;
            if (!drain(bar(ACCF + (tp & 1)), (uint32_t)((tp >> 1) & 1), (uint32_t)((tp & 1) * BN))) {
                ok = false;
                break;
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(bar(ACCE + (tp & 1)));
        }
    }
    if (ok) {
        const int tp = nt - 1;
        ok = drain(bar(ACCF + (tp & 1)), (uint32_t)((tp >> 1) & 1), (uint32_t)((tp & 1) * BN));
        // the correction accumulator is complete with the last k-tile's commit
        if (ok) ok = drain(bar(ACCF + (tp & 1)), (uint32_t)((tp >> 1) & 1), (uint32_t)(2 * BN));
    }
    cp_async_wait_all();
    if (threadIdx.x == 0 && *abort_flag && issued_any) {
        mma_commit(bar(DRAIN));
        mbar_drain(bar(DRAIN), 0);
    }
    if (ok) {
        const int R = m0 + 32 * q + lane;
        const int l = R >> 1, pa = R & 1;
        if (l < g.nl) {
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                const int Cg = n0 + c0 + j;
                const int r = Cg >> 1, pc = Cg & 1;
                if (r < g.nr) {
                    const int qi = (pa == pc) ? pa : 2 + pa;  // ac, bd, ad, bc
                    atomicAdd(g.out4 + ((long long)l * g.nr + r) * 4 + qi, acc[j]);
                }
            }
        }
    }

    fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && *abort_flag)
        *reinterpret_cast<volatile int*>(g.out4 + (long long)4 * g.nl * g.nr) = 1;
    if (warp == 0) {
        __syncwarp();
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// ---------------------------------------------------------------------------------------
// The fused Gram with its roles in separate warps (at most 40 right densities a block: N <= 80),
// so that the conversion of k-tile t + 1, the MMAs of k-tile t and the drain of k-tile t - 1
// run at the same time instead of one after another in every warp:
//   warps 0-6    copy their items' raw values AHEAD k-tiles ahead with cp.async (16 bytes on
//                rows that start on a 16-byte boundary, else 8; each thread reads back only its
//                own copies) and convert them: item (density i, atoms 4q .. 4q + 3) -> TF32 hi
//                and lo of re and im, four 16-byte stores into the 128-byte-swizzled K-major
//                stage; then one arrival a warp on the stage's full barrier;
//   warp 7       lane 0 issues the tile's 12 MMAs once the stage is full and its accumulator
//                buffer drained (three main buffers in tensor memory, the correction in a
//                fourth), and commits them to the stage's empty and the buffer's full barrier;
//   warps 8-15   drain: warp w reads lane quarter w % 4, columns [h DC, h DC + DC) for h =
//                (w - 8) / 4, DC = N / 2, two k-tiles at a time: the two FP32 values of a
//                column summed once (round to nearest, unbiased, at most 2^-24 of the pair
//                against the TF32 parts' 2^-22 of each product) and added to FP64 registers;
//                the correction accumulator once after the last k-tile.
// TF32 rounding to nearest (ties away from zero, as cvt.rna.tf32.f32 for finite values) is done
// on the integer pipe: add half the weight of the 13 dropped mantissa bits, clear them.
// ---------------------------------------------------------------------------------------
constexpr int WS_CONV_WARPS = 7;
constexpr int WS_MMA_WARP = 7;
constexpr int WS_DRAIN_WARP0 = 8;
constexpr int WS_DRAIN_WARPS = 8;
constexpr int WS_THREADS = 32 * (WS_DRAIN_WARP0 + WS_DRAIN_WARPS);
constexpr int WS_NACC = 3;         // main accumulator buffers (128 columns apart)
constexpr int WS_STAGES = 2;       // MMA operand stages in shared memory
constexpr int WS_MAX_NB = 80;      // MMA N: at most 40 right densities
constexpr int WS_MAX_DC = WS_MAX_NB / 2;
// items of 4 atoms a converter thread takes: 64 left + 40 right densities, 8 items each
constexpr int WS_ITEMS = ((BM / 2 + WS_MAX_NB / 2) * (BK / 4) + 32 * WS_CONV_WARPS - 1) / (32 * WS_CONV_WARPS);

__host__ __device__ constexpr size_t ws_smem_bytes(uint32_t stage_bytes, uint32_t raw_slot_bytes, int ahead) {
    return 1024 + (size_t)WS_STAGES * stage_bytes + (size_t)(ahead + 1) * raw_slot_bytes +
           sizeof(void*) * FUSED_MAX_DENS + 256;
}

__device__ __forceinline__ uint32_t tf32_rna_bits(uint32_t b) { return (b + 0x1000u) & 0xFFFFE000u; }

// 8 consecutive FP32 accumulator columns of this thread's lane.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr)
                 : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// Issues the load of 8 consecutive FP32 accumulator columns of this thread's lane (no wait).
__device__ __forceinline__ void tmem_ld8_issue(uint32_t taddr, uint32_t* r) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr)
                 : "memory");
}
// Waits for this thread's tensor-memory loads; the 16 destination registers pass through the
// wait, so that no use of them is scheduled before it.
__device__ __forceinline__ void tmem_wait_ld16(uint32_t* r) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])
                 :
                 : "memory");
}

template <int AHEAD>
__global__ void __launch_bounds__(WS_THREADS, 1) k_gram_tc_ws(const FusedGram g) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    unsigned char* gbase = smem_raw + (base - raw);
    const uint32_t ring_off = WS_STAGES * g.stage_bytes;
    const float2** src_tab = reinterpret_cast<const float2**>(gbase + ring_off + (AHEAD + 1) * g.raw_slot_bytes);
    uint64_t* bars = reinterpret_cast<uint64_t*>(src_tab + FUSED_MAX_DENS);
    // bars: full[WS_STAGES], empty[WS_STAGES], acc_full[WS_NACC], acc_empty[WS_NACC], drain
    constexpr int FULL = 0, EMPTY = WS_STAGES, ACCF = 2 * WS_STAGES, ACCE = ACCF + WS_NACC, DRAIN = ACCE + WS_NACC;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + DRAIN + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    const auto bar = [&](int i) { return smem_u32(bars + i); };
    constexpr uint32_t A_PART = BM * 128;
    const uint32_t b_part = (g.stage_bytes - 2u * A_PART) / 2u;
    constexpr int CONV_THREADS = 32 * WS_CONV_WARPS;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    const int la0 = m0 / 2, rb0 = n0 / 2;
    const int nA = min(BM / 2, g.nl - la0), nB = min(BN / 2, g.nr - rb0);
    const int nd = nA + nB;
    const int nb = max(16, (2 * nB + 15) / 16 * 16);
    const uint32_t idesc = fused_idesc(nb);
    const int kt0 = blockIdx.z * g.kt_per;
    const int nt = min(g.kt_total, kt0 + g.kt_per) - kt0;

    if (threadIdx.x == 0) {
        // one arrival a warp (after __syncwarp): full by the converter warps, drained by the
        // drain warps
        for (int s = 0; s < WS_STAGES; ++s) {
            mbar_init(bar(FULL + s), WS_CONV_WARPS);
            mbar_init(bar(EMPTY + s), 1);
        }
        for (int b = 0; b < WS_NACC; ++b) {
            mbar_init(bar(ACCF + b), 1);
            mbar_init(bar(ACCE + b), WS_DRAIN_WARPS);
        }
        mbar_init(bar(DRAIN), 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    for (int i = threadIdx.x; i < nd; i += WS_THREADS) {
        if (i < nA) {
            src_tab[i] = g.V + (long long)(la0 + i) * g.v_stride;
        } else {
            const int r = rb0 + (i - nA);
            src_tab[i] = g.rho + (long long)(g.ridx ? g.ridx[r] : r) * g.r_stride;
        }
    }
    // zero both MMA stages once: rows beyond the real ones are never written again
    for (uint32_t o = threadIdx.x * 16u; o < ring_off; o += WS_THREADS * 16u)
        *reinterpret_cast<uint4*>(gbase + o) = make_uint4(0u, 0u, 0u, 0u);
    fence_proxy_async();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;
    bool ok = true;

    if (warp < WS_CONV_WARPS) {
        // ---- converters: item it = (density it / 8, atoms 4 (it % 8) .. + 3); the raw slot holds
        // atoms 4q, 4q + 1 of item it at 16 it and atoms 4q + 2, 4q + 3 at half + 16 it, so that
        // consecutive threads copy and read contiguous 16-byte pieces.  A thread's items, their
        // sources and their places in the stage are the same for every k-tile.
        const int items = nd * (BK / 4);
        const uint32_t half = (uint32_t)items * 16u;
        const float2* isrc[WS_ITEMS];
        uint32_t ihi[WS_ITEMS][2], ilo[WS_ITEMS][2];
#pragma unroll
        for (int k = 0; k < WS_ITEMS; ++k) {
            const int it = threadIdx.x + k * CONV_THREADS;
            const int i = min(it, items - 1) >> 3, qd = it & 7;
            const bool left = i < nA;
            const int row = 2 * (left ? i : i - nA);
            const uint32_t hi0 = left ? 0u : 2u * A_PART, lo0 = hi0 + (left ? A_PART : b_part);
            isrc[k] = src_tab[i] + 4 * qd;
            ihi[k][0] = hi0 + sw128_chunk(row, qd);
            ihi[k][1] = hi0 + sw128_chunk(row + 1, qd);
            ilo[k][0] = lo0 + sw128_chunk(row, qd);
            ilo[k][1] = lo0 + sw128_chunk(row + 1, qd);
        }
        const auto issue = [&](int t) {
            const long long at0 = (long long)(kt0 + t) * BK;
            const uint32_t slot = base + ring_off + (uint32_t)(t % (AHEAD + 1)) * g.raw_slot_bytes;
#pragma unroll
            for (int k = 0; k < WS_ITEMS; ++k) {
                const int it = threadIdx.x + k * CONV_THREADS;
                if (it < items) {
                    const long long a = at0 + 4 * (it & 7);  // first atom of the item
                    const uint32_t d0 = slot + (uint32_t)it * 16u;
                    if (g.aligned16) {
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const long long left_atoms = g.na - (a + 2 * h);
                            const uint32_t nbytes = left_atoms >= 2 ? 16u : (left_atoms == 1 ? 8u : 0u);
                            cp_async16z(d0 + h * half, isrc[k] + (nbytes ? at0 + 2 * h : -4LL * (it & 7)), nbytes);
                        }
                    } else {
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const bool in = a + e < g.na;
                            cp_async8(d0 + (e >> 1) * half + 8u * (e & 1), isrc[k] + (in ? at0 + e : -4LL * (it & 7)),
                                      in ? 8u : 0u);
                        }
                    }
                }
            }
        };
#pragma unroll 1
        for (int t = 0; t < AHEAD; ++t) {
            if (t < nt) issue(t);
            cp_async_commit();
        }
#pragma unroll 1
        for (int t = 0; t < nt; ++t) {
            if (t + AHEAD < nt) issue(t + AHEAD);
            cp_async_commit();
            cp_async_wait<AHEAD>();  // this thread's copies of k-tile t have landed
            const int s = t % WS_STAGES;
            const bool got = mbar_wait(bar(EMPTY + s), (uint32_t)(((t / WS_STAGES) & 1) ^ 1), abort_flag);
            if (!__all_sync(0xffffffffu, got)) {
                ok = false;
                break;
            }
            unsigned char* stg = gbase + (size_t)s * g.stage_bytes;
            const unsigned char* rs = gbase + ring_off + (size_t)(t % (AHEAD + 1)) * g.raw_slot_bytes;
#pragma unroll
            for (int k = 0; k < WS_ITEMS; ++k) {
                const int it = threadIdx.x + k * CONV_THREADS;
                if (it < items) {
                    const uint4 z0 = *reinterpret_cast<const uint4*>(rs + it * 16);         // re0 im0 re1 im1
                    const uint4 z1 = *reinterpret_cast<const uint4*>(rs + half + it * 16);  // re2 im2 re3 im3
                    const uint32_t re[4] = {z0.x, z0.z, z1.x, z1.z}, im[4] = {z0.y, z0.w, z1.y, z1.w};
                    uint32_t rh[4], ih[4], rl[4], il[4];
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        rh[e] = tf32_rna_bits(re[e]);
                        ih[e] = tf32_rna_bits(im[e]);
                        rl[e] = tf32_rna_bits(__float_as_uint(__uint_as_float(re[e]) - __uint_as_float(rh[e])));
                        il[e] = tf32_rna_bits(__float_as_uint(__uint_as_float(im[e]) - __uint_as_float(ih[e])));
                    }
                    *reinterpret_cast<uint4*>(stg + ihi[k][0]) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
                    *reinterpret_cast<uint4*>(stg + ihi[k][1]) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
                    *reinterpret_cast<uint4*>(stg + ilo[k][0]) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
                    *reinterpret_cast<uint4*>(stg + ilo[k][1]) = make_uint4(il[0], il[1], il[2], il[3]);
                }
            }
            fence_proxy_async();  // the stores, seen by the tensor cores' async proxy
            __syncwarp();
            if (lane == 0) mbar_arrive(bar(FULL + s));
        }
        cp_async_wait_all();
    } else if (warp == WS_MMA_WARP) {
        // ---- MMA issuer
        bool issued_any = false;
        if (lane == 0) {
#pragma unroll 1
            for (int t = 0; t < nt; ++t) {
                const int s = t % WS_STAGES, b = t % WS_NACC;
                if (!mbar_wait(bar(ACCE + b), (uint32_t)(((t / WS_NACC) & 1) ^ 1), abort_flag)) {
                    ok = false;
                    break;
                }
                if (!mbar_wait(bar(FULL + s), (uint32_t)((t / WS_STAGES) & 1), abort_flag)) {
                    ok = false;
                    break;
                }
                fence_after();
                const uint32_t st = base + (uint32_t)s * g.stage_bytes;
                const uint32_t dm = tmem + (uint32_t)(b * BN);
                const uint32_t dc = tmem + (uint32_t)(WS_NACC * BN);
#pragma unroll
                for (int kk = 0; kk < BK / 8; ++kk) {
                    const uint64_t ahi = sw128_desc(st + kk * 32);
                    const uint64_t alo = sw128_desc(st + A_PART + kk * 32);
                    const uint64_t bhi = sw128_desc(st + 2 * A_PART + kk * 32);
                    const uint64_t blo = sw128_desc(st + 2 * A_PART + b_part + kk * 32);
                    mma_tf32_n(dm, ahi, bhi, idesc, kk > 0 ? 1u : 0u);
                    mma_tf32_n(dc, alo, bhi, idesc, (t > 0 || kk > 0) ? 1u : 0u);
                    mma_tf32_n(dc, ahi, blo, idesc, 1u);
                }
                issued_any = true;
                mma_commit(bar(EMPTY + s));
                mma_commit(bar(ACCF + b));
            }
            // every MMA issued has completed before the teardown frees tensor memory
            if (issued_any) {
                mma_commit(bar(DRAIN));
                mbar_drain(bar(DRAIN), 0);
            }
        }
        __syncwarp();
    } else {
        // ---- drain warps
        const int q = warp & 3;
        const int dc = nb / 2;                                // columns a drain warp takes
        const int col0 = ((warp - WS_DRAIN_WARP0) >> 2) * dc;
        const uint32_t lane_base = tmem + ((uint32_t)(32 * q) << 16);
        double acc[WS_MAX_DC];
#pragma unroll
        for (int i = 0; i < WS_MAX_DC; ++i) acc[i] = 0.0;
        const auto add_cols = [&](uint32_t col) {
#pragma unroll
            for (int j = 0; j < WS_MAX_DC / 8; ++j) {
                if (8 * j < dc) {
                    float v[8];
                    tmem_ld8(lane_base + col + (uint32_t)(col0 + 8 * j), v);
#pragma unroll
                    for (int i = 0; i < 8; ++i) acc[8 * j + i] += (double)v[i];
                }
            }
        };
        // two k-tiles' main products (buffers at columns c0 and c1): their FP32 sum, rounded to
        // nearest once (unbiased, 2^-24 of the pair against the TF32x3 parts' 2^-22 of each
        // product), goes into the FP64 sums -- half the conversions and waits of one by one
        const auto add_pair = [&](uint32_t c0, uint32_t c1) {
#pragma unroll
            for (int j = 0; j < WS_MAX_DC / 8; ++j) {
                if (8 * j < dc) {
                    uint32_t r[16];
                    tmem_ld8_issue(lane_base + c0 + (uint32_t)(col0 + 8 * j), r);
                    tmem_ld8_issue(lane_base + c1 + (uint32_t)(col0 + 8 * j), r + 8);
                    tmem_wait_ld16(r);
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                        acc[8 * j + i] += (double)(__uint_as_float(r[i]) + __uint_as_float(r[8 + i]));
                }
            }
        };
#pragma unroll 1
        for (int t = 0; t < nt; t += 2) {
            const bool pair = t + 1 < nt;
            const int b0 = t % WS_NACC, b1 = (t + 1) % WS_NACC;
            bool got = mbar_wait(bar(ACCF + b0), (uint32_t)((t / WS_NACC) & 1), abort_flag);
            if (got && pair) got = mbar_wait(bar(ACCF + b1), (uint32_t)(((t + 1) / WS_NACC) & 1), abort_flag);
            if (!__all_sync(0xffffffffu, got)) {
                ok = false;
                break;
            }
            fence_after();
            if (pair)
                add_pair((uint32_t)(b0 * BN), (uint32_t)(b1 * BN));
            else
                add_cols((uint32_t)(b0 * BN));
            fence_before();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(bar(ACCE + b0));
                if (pair) mbar_arrive(bar(ACCE + b1));
            }
        }
        if (ok) {
            // the correction accumulator is complete with the last k-tile's commit
            fence_after();
            add_cols((uint32_t)(WS_NACC * BN));
            const int R = m0 + 32 * q + lane;
            const int l = R >> 1, pa = R & 1;
            if (l < g.nl) {
#pragma unroll
                for (int j = 0; j < WS_MAX_DC; ++j) {
                    const int Cg = n0 + col0 + j;
                    const int r = Cg >> 1, pc = Cg & 1;
                    if (j < dc && r < g.nr) {
                        const int qi = (pa == pc) ? pa : 2 + pa;  // ac, bd, ad, bc
                        atomicAdd(g.out4 + ((long long)l * g.nr + r) * 4 + qi, acc[j]);
                    }
                }
            }
        }
    }

    fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && *abort_flag)
        *reinterpret_cast<volatile int*>(g.out4 + (long long)4 * g.nl * g.nr) = 1;
    if (warp == 0) {
        __syncwarp();
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

}  // namespace tc
}  // namespace clk
