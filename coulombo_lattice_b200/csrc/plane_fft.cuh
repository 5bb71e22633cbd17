// Line lengths with a compiled in-place chain for the fused xy-plane kernels.  FP32 chains
// use register codelets up to radix 16, FP64 chains up to radix 8 (register budget of a
// 512-thread block).  Any other length uses the separate x and y passes.
#pragma once

#include "fft.cuh"

namespace clk {

inline bool plane_size_supported(int n) {
    static const int sizes[] = {32, 36, 40, 45, 48, 60, 64, 72, 80, 90, 96, 100, 108, 120, 128, 144, 150, 160};
    for (int s : sizes)
        if (s == n) return true;
    return false;
}

// Transforms `lines` lines of length n in place (buf[line*ls + idx*is]).
template <int S, int VALS, typename T>
__device__ __forceinline__ void plane_axis(cx<T>* buf, const cx<T>* __restrict__ tw, int n, int lines, int ls,
                                           int is) {
    if constexpr (sizeof(T) == 4) {
        switch (n) {
            case 32: axis_ct<S, VALS, T, 16, 2>(buf, tw, lines, ls, is); break;
            case 36: axis_ct<S, VALS, T, 12, 3>(buf, tw, lines, ls, is); break;
            case 40: axis_ct<S, VALS, T, 8, 5>(buf, tw, lines, ls, is); break;
            case 45: axis_ct<S, VALS, T, 3, 3, 5>(buf, tw, lines, ls, is); break;
            case 48: axis_ct<S, VALS, T, 16, 3>(buf, tw, lines, ls, is); break;
            case 60: axis_ct<S, VALS, T, 12, 5>(buf, tw, lines, ls, is); break;
            case 64: axis_ct<S, VALS, T, 16, 4>(buf, tw, lines, ls, is); break;
            case 72: axis_ct<S, VALS, T, 8, 3, 3>(buf, tw, lines, ls, is); break;
            case 80: axis_ct<S, VALS, T, 16, 5>(buf, tw, lines, ls, is); break;
            case 90: axis_ct<S, VALS, T, 10, 3, 3>(buf, tw, lines, ls, is); break;
            case 96: axis_ct<S, VALS, T, 16, 6>(buf, tw, lines, ls, is); break;
            case 100: axis_ct<S, VALS, T, 4, 5, 5>(buf, tw, lines, ls, is); break;
            case 108: axis_ct<S, VALS, T, 12, 3, 3>(buf, tw, lines, ls, is); break;
            case 120: axis_ct<S, VALS, T, 8, 3, 5>(buf, tw, lines, ls, is); break;
            case 128: axis_ct<S, VALS, T, 16, 8>(buf, tw, lines, ls, is); break;
            case 144: axis_ct<S, VALS, T, 16, 3, 3>(buf, tw, lines, ls, is); break;
            case 150: axis_ct<S, VALS, T, 6, 5, 5>(buf, tw, lines, ls, is); break;
            case 160: axis_ct<S, VALS, T, 16, 10>(buf, tw, lines, ls, is); break;
            default: break;
        }
    } else {
        switch (n) {
            case 32: axis_ct<S, VALS, T, 8, 4>(buf, tw, lines, ls, is); break;
            case 36: axis_ct<S, VALS, T, 4, 3, 3>(buf, tw, lines, ls, is); break;
            case 40: axis_ct<S, VALS, T, 8, 5>(buf, tw, lines, ls, is); break;
            case 45: axis_ct<S, VALS, T, 3, 3, 5>(buf, tw, lines, ls, is); break;
            case 48: axis_ct<S, VALS, T, 8, 6>(buf, tw, lines, ls, is); break;
            case 60: axis_ct<S, VALS, T, 4, 3, 5>(buf, tw, lines, ls, is); break;
            case 64: axis_ct<S, VALS, T, 8, 8>(buf, tw, lines, ls, is); break;
            case 72: axis_ct<S, VALS, T, 8, 3, 3>(buf, tw, lines, ls, is); break;
            case 80: axis_ct<S, VALS, T, 8, 10>(buf, tw, lines, ls, is); break;
            case 90: axis_ct<S, VALS, T, 6, 3, 5>(buf, tw, lines, ls, is); break;
            case 96: axis_ct<S, VALS, T, 8, 4, 3>(buf, tw, lines, ls, is); break;
            case 100: axis_ct<S, VALS, T, 4, 5, 5>(buf, tw, lines, ls, is); break;
            case 108: axis_ct<S, VALS, T, 4, 3, 3, 3>(buf, tw, lines, ls, is); break;
            case 120: axis_ct<S, VALS, T, 8, 3, 5>(buf, tw, lines, ls, is); break;
            case 128: axis_ct<S, VALS, T, 8, 4, 4>(buf, tw, lines, ls, is); break;
            case 144: axis_ct<S, VALS, T, 8, 6, 3>(buf, tw, lines, ls, is); break;
            case 150: axis_ct<S, VALS, T, 6, 5, 5>(buf, tw, lines, ls, is); break;
            case 160: axis_ct<S, VALS, T, 8, 4, 5>(buf, tw, lines, ls, is); break;
            default: break;
        }
    }
}

}  // namespace clk
