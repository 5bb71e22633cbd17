// Inverse x-pass launchers (passes.hpp).
#include "passes_impl.cuh"

namespace clp {
template bool xinv<float>(cudaStream_t, Variant, cx<float>*, long long, const cx<float>*, const int*, const int*,
                          cx<float>*, long long, int, int, int);
template bool xinv<double>(cudaStream_t, Variant, cx<double>*, long long, const cx<double>*, const int*, const int*,
                           cx<double>*, long long, int, int, int);
}  // namespace clp
