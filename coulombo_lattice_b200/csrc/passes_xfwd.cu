// Forward x-pass launchers (passes.hpp).
#include "passes_impl.cuh"

namespace clp {
template bool xfwd<float>(cudaStream_t, Variant, const cx<float>*, long long, const int*, const int*, cx<float>*,
                          long long, const cx<float>*, const clk::RoundPhase&, int, int, int, int, int);
template bool xfwd<double>(cudaStream_t, Variant, const cx<double>*, long long, const int*, const int*, cx<double>*,
                           long long, const cx<double>*, const clk::RoundPhase&, int, int, int, int, int);
}  // namespace clp
