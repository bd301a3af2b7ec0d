// Tensor-core (tcgen05) distance-GEMM filter for the exact kNN.
#pragma once
#include "engine.cuh"

namespace pacmap {
// True when the tcgen05 filter handles this shape.
bool knn_tc_supported(uint64_t n, uint64_t d, uint64_t kp);
// Exact kNN through the tensor-core filter + FP32 re-rank; false when it declined the problem.
// nprobe in 1..255: approximate -- each row block searches only the nprobe pivot cells nearest its own.
bool knn_tc_device(Ctx& c, const float* d_x, uint64_t n, uint64_t d, uint64_t kp, bool bf16, uint32_t* d_idx,
                   float* d_dist, const KnnShard& shard = KnnShard(), int nprobe = 0);
// Rows of the last tensor-core kNN on this thread that needed the exact SIMT recomputation.
uint64_t& last_tc_fallback_rows();
// Device time (ms) of the last filter kernel launch on this thread (CUDA events on its stream).
double& last_tc_filter_ms();
}  // namespace pacmap
