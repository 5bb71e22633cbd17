// z-pass launchers (passes.hpp) and the variant helpers.
#include <algorithm>

#include "passes_impl.cuh"

namespace clp {

int split_variants(int n) {
    int k = 0;
    if (!clk::with_split2(n, [&](auto tag) { k = decltype(tag)::r1 == decltype(tag)::r2 ? 1 : 2; })) return 0;
    return k;
}

unsigned density_groups(long long blocks, int cnt) {
    const long long target = 148LL * 16;
    const long long g = (target + blocks - 1) / blocks;
    return (unsigned)std::max(1LL, std::min<long long>(g, cnt));
}

template bool zconv<float>(cudaStream_t, Variant, cx<float>*, long long, const cx<float>*, const float*, long long,
                           int, int);
template bool zconv<double>(cudaStream_t, Variant, cx<double>*, long long, const cx<double>*, const double*,
                            long long, int, int);

}  // namespace clp
