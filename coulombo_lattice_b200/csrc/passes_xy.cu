// Launchers of the fused xy plane passes (plane_rf.cuh).
#include <algorithm>

#include "passes_impl.cuh"
#include "plane_q.cuh"
#include "plane_rf.cuh"

namespace clp {

namespace {

// Density groups (gridDim.y) of a plane launch: the group count whose modelled span -- waves
// of blocks over the resident slots, times the densities a block runs plus its setup (about
// half a density) -- is shortest.
unsigned plane_groups(int nz, int cnt, int min_blocks) {
    const long long slots = 148LL * std::max(1, min_blocks);
    unsigned best = 1;
    double best_t = 1e300;
    for (int g = 1; g <= cnt; ++g) {
        const long long per = (cnt + g - 1) / g;
        if ((long long)(g - 1) * per >= cnt) continue;  // a group would be empty
        const long long waves = ((long long)nz * g + slots - 1) / slots;
        const double t = (double)waves * ((double)per + 0.5);
        if (t < best_t) {
            best_t = t;
            best = (unsigned)g;
        }
    }
    return best;
}

}  // namespace

bool plane_supported(bool fp32, int nx, int ny) {
    return fp32 ? clk::with_plane<float>(nx, ny, [](auto, auto, auto) {})
                : clk::with_plane<double>(nx, ny, [](auto, auto, auto) {});
}

template <typename T>
bool xyfwd(cudaStream_t s, const cx<T>* rho, long long rho_stride, const int* row_ptr, const int* cell, cx<T>* buf,
           long long M, const cx<T>* tw, const clk::RoundPhase& rp, int nx, int ny, int nz, int cnt) {
    return clk::with_plane<T>(nx, ny, [&](auto tag, auto threads, auto minb) {
        using Tag = decltype(tag);
        constexpr int TH = decltype(threads)::value, MB = decltype(minb)::value;
        auto kern = clk::k_xyfwd_plane<T, Tag::r1, Tag::r2, TH, MB>;
        const size_t smem = clk::PlaneSmem<T, Tag::r1, Tag::r2, TH, true, MB>::bytes;
        set_smem(kern, smem);
        kern<<<dim3((unsigned)nz, plane_groups(nz, cnt, MB)), TH, smem, s>>>(rho, rho_stride, row_ptr, cell, buf, M,
                                                                             tw, rp, cnt);
    });
}

template <typename T>
bool xyinv(cudaStream_t s, cx<T>* buf, long long M, const cx<T>* tw, const int* row_ptr, const int* cell,
           cx<T>* out, long long o_stride, int nx, int ny, int nz, int cnt) {
    return clk::with_plane<T>(nx, ny, [&](auto tag, auto threads, auto minb) {
        using Tag = decltype(tag);
        constexpr int TH = decltype(threads)::value, MB = decltype(minb)::value;
        auto kern = clk::k_xyinv_plane<T, Tag::r1, Tag::r2, TH, MB>;
        const size_t smem = clk::PlaneSmem<T, Tag::r1, Tag::r2, TH, false>::bytes;
        set_smem(kern, smem);
        kern<<<dim3((unsigned)nz, plane_groups(nz, cnt, MB)), TH, smem, s>>>(buf, M, tw, row_ptr, cell, out,
                                                                             o_stride, cnt);
    });
}

bool quadrant_supported(bool fp32, int nx, int ny) { return fp32 && nx == clk::qp::N && ny == clk::qp::N; }

bool qfwd(cudaStream_t s, const cx<float>* rho, long long rho_stride, const int* row_ptr, const int* cell,
          cx<float>* buf, long long M, const cx<float>* tw, int nz, int cnt) {
    set_smem(clk::qp::k_qfwd, clk::qp::SMEM);
    clk::qp::k_qfwd<<<dim3((unsigned)nz, plane_groups(nz, cnt, 2)), clk::qp::THREADS, clk::qp::SMEM, s>>>(
        rho, rho_stride, row_ptr, cell, buf, M, tw, cnt);
    return true;
}

template bool xyfwd<float>(cudaStream_t, const cx<float>*, long long, const int*, const int*, cx<float>*, long long,
                           const cx<float>*, const clk::RoundPhase&, int, int, int, int);
template bool xyfwd<double>(cudaStream_t, const cx<double>*, long long, const int*, const int*, cx<double>*,
                            long long, const cx<double>*, const clk::RoundPhase&, int, int, int, int);
template bool xyinv<float>(cudaStream_t, cx<float>*, long long, const cx<float>*, const int*, const int*,
                           cx<float>*, long long, int, int, int, int);
template bool xyinv<double>(cudaStream_t, cx<double>*, long long, const cx<double>*, const int*, const int*,
                            cx<double>*, long long, int, int, int, int);

}  // namespace clp
