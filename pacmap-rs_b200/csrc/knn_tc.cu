// Tensor-core (tcgen05) distance-GEMM filter for the exact kNN.
#include "knn_tc.cuh"

namespace pacmap {
bool knn_tc_supported(uint64_t, uint64_t, uint64_t) { return false; }
bool knn_tc_device(Ctx&, const float*, uint64_t, uint64_t, uint64_t, bool, uint32_t*, float*) { return false; }
}  // namespace pacmap
