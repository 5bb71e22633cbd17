// Launchers of the register-FFT passes (rfft.cuh) for every compiled variant, and of the
// fused xy plane passes (plane_rf.cuh).
//
// A variant picks the radix split of the line length (the balanced split, or its two factors
// swapped), the lines per block (the default -- 16 for FP32, 8 for FP64 -- or half) and, for
// the forward x pass, the layout of its tile.  The autotuner in engine.cu times the variants
// of each pass on the request's own shapes and keeps the fastest, then times the fused plane
// passes (where compiled) against the separate passes they replace.  Each launcher returns
// false (nothing launched) when the length has no compiled kernel; launch errors surface
// through cudaGetLastError.
//
// The launchers are instantiated in passes_xfwd.cu, passes_xinv.cu, passes_yfwd.cu,
// passes_yinv.cu, passes_z.cu and passes_xy.cu (one translation unit per pass, compiled in
// parallel).
#pragma once

#include <cuda_runtime.h>

#include "fft.cuh"
#include "kernels.cuh"

namespace clk {
struct SlMix;
}

namespace clp {

using clk::cx;

struct Variant {
    int split = 0;  // 0: the balanced split; 1: its factors swapped
    int half = 0;   // 1: half the default lines (rows) per block (FP32 only)
    int pad = 0;    // forward x pass, FP32: 1 pads its tile one point in four
    bool operator==(const Variant& o) const { return split == o.split && half == o.half && pad == o.pad; }
};

// kXYFwd / kXYInv: the fused plane passes in place of x+y forward / y+x inverse (tuned
// choice: Variant::split = 1 uses them).
enum Pass { kXFwd = 0, kYFwd = 1, kZConv = 2, kYInv = 3, kXInv = 4, kXYFwd = 5, kXYInv = 6, kNumPasses = 7 };

// Number of distinct split variants compiled for a line length: 0 (no register pass), 1
// (square split) or 2.
int split_variants(int n);

// Density groups of a launch (gridDim.y): enough blocks to fill every SM several times over,
// while each block still reuses its per-block setup for a run of densities.
unsigned density_groups(long long blocks, int cnt);

// z pass: forward FFT along z, x Khat, inverse FFT along z (in place).
template <typename T>
bool zconv(cudaStream_t s, Variant v, cx<T>* buf, long long M, const cx<T>* tw, const T* kh, long long nxy, int nz,
           int cnt);

// y pass of direction S (in place); row_ptr (or nullptr) marks the rows without atoms.
template <int S, typename T>
bool ycol(cudaStream_t s, Variant v, cx<T>* buf, long long M, const cx<T>* tw, int nx, int ny, int nz, int cnt,
          const int* row_ptr);

// forward x pass: scatter of the atoms x conj(phase), FFT along x, rows stored; the pair
// densities rho are in the pass precision.
template <typename T>
bool xfwd(cudaStream_t s, Variant v, const cx<T>* rho, long long rho_stride, const int* row_ptr,
          const int* cell, cx<T>* buf, long long M, const cx<T>* tw, const clk::RoundPhase& rp, int nx, int ny,
          int nrows, int cnt, int skip_empty);

// inverse x pass: inverse FFT along x, the round's values at the atoms written to out.
template <typename T>
bool xinv(cudaStream_t s, Variant v, cx<T>* buf, long long M, const cx<T>* tw, const int* row_ptr,
          const int* cell, cx<T>* out, long long o_stride, int nx, int nrows, int cnt);

// Fused xy passes on whole planes (plane_rf.cuh), for the square plane shapes compiled there
// (false otherwise, nothing launched).  Forward: the atoms' pair densities x conj(phase) are
// transformed along x and y and every plane is stored; inverse: planes are transformed back
// along y and x and the round's values at the atoms are written to out.
bool plane_supported(bool fp32, int nx, int ny);
// Quadrant forward plane pass (plane_q.cuh): FP32 128 x 128 sub-lattice planes, atoms in
// [0, 64)^2.
bool quadrant_supported(bool fp32, int nx, int ny);
bool qfwd(cudaStream_t s, const cx<float>* rho, long long rho_stride, const int* row_ptr, const int* cell,
          cx<float>* buf, long long M, const cx<float>* tw, int nz, int cnt);
template <typename T>
bool xyfwd(cudaStream_t s, const cx<T>* rho, long long rho_stride, const int* row_ptr, const int* cell, cx<T>* buf,
           long long M, const cx<T>* tw, const clk::RoundPhase& rp, int nx, int ny, int nz, int cnt);
template <typename T>
bool xyinv(cudaStream_t s, cx<T>* buf, long long M, const cx<T>* tw, const int* row_ptr, const int* cell,
           cx<T>* out, long long o_stride, int nx, int ny, int nz, int cnt);

// z pass of the sub-lattice forms (sublattice.cuh): for every (kx, ky) column of the virtual
// grid and every class, forward FFT along z of nz = 2s points (the s stored planes, the rest zero
// padding), class mixing with the residue kernels H and the phases, inverse FFT, the s stored
// planes written back.  zb selects the compiled zinc-blende mixing table.
bool zmix_supported(int nz);
template <typename T>
bool zmix(cudaStream_t s, cx<T>* buf, long long stride, const cx<T>* tw, const cx<T>* H, const cx<T>* phxy,
          const cx<T>* phz, const clk::SlMix& mix, bool zb, long long nxy, int nz, int cnt);

}  // namespace clp
