// Forward y-pass launchers (passes.hpp).
#include "passes_impl.cuh"

namespace clp {
template bool ycol<-1, float>(cudaStream_t, Variant, cx<float>*, long long, const cx<float>*, int, int, int, int,
                              const int*);
template bool ycol<-1, double>(cudaStream_t, Variant, cx<double>*, long long, const cx<double>*, int, int, int, int,
                               const int*);
}  // namespace clp
