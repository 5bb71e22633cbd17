// Template bodies of the pass launchers declared in passes.hpp; included only by the
// translation units that instantiate them (passes_xfwd.cu, passes_xinv.cu, passes_yfwd.cu,
// passes_yinv.cu, passes_z.cu).
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

#include "passes.hpp"
#include "rfft.cuh"

namespace clp {

template <typename T>
constexpr int default_lines() {
    return sizeof(T) == 4 ? 16 : 8;
}

template <typename K>
void set_smem(K kernel, size_t bytes) {
    // an oversized request makes the launch itself fail, which the caller reports
    if (bytes <= 227 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Calls f(std::integral_constant<int, L>) with the variant's lines per block (the half-width
// variant is compiled for FP32 only; FP64 always uses the default).
template <typename T, typename F>
void with_lines(const Variant& v, F&& f) {
    constexpr int L = default_lines<T>();
    if constexpr (sizeof(T) == 4) {
        if (v.half) {
            f(std::integral_constant<int, L / 2>{});
            return;
        }
    }
    f(std::integral_constant<int, L>{});
}

template <typename T>
bool zconv(cudaStream_t s, Variant v, cx<T>* buf, long long M, const cx<T>* tw, const T* kh, long long nxy, int nz,
           int cnt) {
    return clk::with_split2(
        nz,
        [&](auto tag) {
            using Tag = decltype(tag);
            with_lines<T>(v, [&](auto lines) {
                constexpr int L = decltype(lines)::value;
                constexpr int P = clk::ColShape<Tag::r1, Tag::r2>::P;
                auto kern = clk::k_zconv_rf<T, Tag::r1, Tag::r2, L>;
                const size_t smem = clk::ZconvLayout<T, Tag::r1, Tag::r2, L>::smem;
                set_smem(kern, smem);
                const long long blocks = (nxy + L - 1) / L;
                kern<<<dim3((unsigned)blocks, density_groups(blocks, cnt)), L * P, smem, s>>>(buf, M, tw, kh, nxy,
                                                                                              cnt);
            });
        },
        v.split);
}

template <int S, typename T>
bool ycol(cudaStream_t s, Variant v, cx<T>* buf, long long M, const cx<T>* tw, int nx, int ny, int nz, int cnt,
          const int* row_ptr) {
    return clk::with_split2(
        ny,
        [&](auto tag) {
            using Tag = decltype(tag);
            with_lines<T>(v, [&](auto lines) {
                constexpr int L = decltype(lines)::value;
                constexpr int P = clk::ColShape<Tag::r1, Tag::r2>::P;
                auto kern = clk::k_ycol_rf<S, T, Tag::r1, Tag::r2, L>;
                const size_t smem = clk::YcolLayout<T, Tag::r1, Tag::r2, L>::smem;
                set_smem(kern, smem);
                const int xchunks = (nx + L - 1) / L;
                const long long blocks = (long long)xchunks * nz;
                kern<<<dim3((unsigned)blocks, density_groups(blocks, cnt)), L * P, smem, s>>>(buf, M, tw, nx, ny,
                                                                                              xchunks, cnt, row_ptr);
            });
        },
        v.split);
}

template <typename T>
bool xfwd(cudaStream_t s, Variant v, const cx<T>* rho, long long rho_stride, const int* row_ptr,
          const int* cell, cx<T>* buf, long long M, const cx<T>* tw, const clk::RoundPhase& rp, int nx, int ny,
          int nrows, int cnt, int skip_empty) {
    return clk::with_split2(
        nx,
        [&](auto tag) {
            using Tag = decltype(tag);
            with_lines<T>(v, [&](auto lines) {
                const auto launch = [&](auto pad) {
                    constexpr int LR = decltype(lines)::value;
                    constexpr bool PAD = decltype(pad)::value;
                    constexpr int Q = Tag::r1 > Tag::r2 ? Tag::r1 : Tag::r2;
                    auto kern = clk::k_xfwd_rf<T, Tag::r1, Tag::r2, LR, PAD>;
                    const size_t smem =
                        sizeof(cx<T>) * clk::XfwdPitch<Tag::r1, Tag::r2, LR, PAD, sizeof(cx<T>)>::elems;
                    set_smem(kern, smem);
                    const long long blocks = (nrows + LR - 1) / LR;
                    kern<<<dim3((unsigned)blocks, density_groups(blocks, cnt)), LR * Q, smem, s>>>(
                        rho, rho_stride, row_ptr, cell, buf, M, tw, rp, ny, nrows, cnt, skip_empty);
                };
                if constexpr (sizeof(T) == 4) {
                    if (v.pad) {
                        launch(std::true_type{});
                        return;
                    }
                }
                launch(std::false_type{});
            });
        },
        v.split);
}

template <typename T>
bool xinv(cudaStream_t s, Variant v, cx<T>* buf, long long M, const cx<T>* tw, const int* row_ptr,
          const int* cell, cx<T>* out, long long o_stride, int nx, int nrows, int cnt) {
    return clk::with_split2(
        nx,
        [&](auto tag) {
            using Tag = decltype(tag);
            with_lines<T>(v, [&](auto lines) {
                constexpr int LR = decltype(lines)::value;
                constexpr int N = Tag::r1 * Tag::r2;
                constexpr int Q = Tag::r1 > Tag::r2 ? Tag::r1 : Tag::r2;
                auto kern = clk::k_xinv_rf<T, Tag::r1, Tag::r2, LR>;
                using Pitch = clk::XinvPitch<Tag::r1, Tag::r2, LR, sizeof(cx<T>)>;
                const size_t smem = sizeof(cx<T>) * ((size_t)N + (size_t)LR * Pitch::PP + (size_t)LR * Pitch::NP);
                set_smem(kern, smem);
                const long long blocks = (nrows + LR - 1) / LR;
                kern<<<dim3((unsigned)blocks, density_groups(blocks, cnt)), LR * Q, smem, s>>>(
                    buf, M, tw, row_ptr, cell, out, o_stride, nrows, cnt);
            });
        },
        v.split);
}

}  // namespace clp
