// Launchers of the sub-lattice z pass (sublattice.cuh): z transforms and class mixing.
#include <algorithm>

#include "passes_impl.cuh"
#include "sublattice.cuh"

namespace clp {

namespace {

// Columns per block: the largest of 8, 4, 2 whose block has at most 512 threads and whose
// shared memory fits one SM.
template <typename T, int R1, int R2>
constexpr int zmix_lines() {
    constexpr int P = clk::ColShape<R1, R2>::P;
    if (clk::kSlMaxClasses * 8 * P <= 512 && clk::ZmixLayout<T, R1, R2, 8>::smem <= 227 * 1024) return 8;
    if (clk::kSlMaxClasses * 4 * P <= 512 && clk::ZmixLayout<T, R1, R2, 4>::smem <= 227 * 1024) return 4;
    return 2;
}

}  // namespace

bool zmix_supported(int nz) {
    return clk::with_zmix_split(nz, [](auto) {});
}

template <typename T>
bool zmix(cudaStream_t s, cx<T>* buf, long long stride, const cx<T>* tw, const cx<T>* H, const cx<T>* phxy,
          const cx<T>* phz, const clk::SlMix& mix, bool zb, long long nxy, int nz, int cnt) {
    return clk::with_zmix_split(nz, [&](auto tag) {
        using Tag = decltype(tag);
        constexpr int R1 = Tag::r1, R2 = Tag::r2;
        constexpr int L = zmix_lines<T, R1, R2>();
        constexpr int NT = clk::kSlMaxClasses * L * clk::ColShape<R1, R2>::P;
        const size_t smem = clk::ZmixLayout<T, R1, R2, L>::smem;
        const long long blocks = (nxy + L - 1) / L;
        const unsigned groups = density_groups(blocks, cnt);
        if (zb) {
            auto kern = clk::k_zmix_rf<T, R1, R2, L, true>;
            set_smem(kern, smem);
            kern<<<dim3((unsigned)blocks, groups), NT, smem, s>>>(buf, stride, tw, H, phxy, phz, mix, nxy, cnt);
        } else {
            auto kern = clk::k_zmix_rf<T, R1, R2, L, false>;
            set_smem(kern, smem);
            kern<<<dim3((unsigned)blocks, groups), NT, smem, s>>>(buf, stride, tw, H, phxy, phz, mix, nxy, cnt);
        }
    });
}

template bool zmix<float>(cudaStream_t, cx<float>*, long long, const cx<float>*, const cx<float>*,
                          const cx<float>*, const cx<float>*, const clk::SlMix&, bool, long long, int, int);
template bool zmix<double>(cudaStream_t, cx<double>*, long long, const cx<double>*, const cx<double>*,
                           const cx<double>*, const cx<double>*, const clk::SlMix&, bool, long long, int, int);

}  // namespace clp
