// Tensor-core (tcgen05) distance-GEMM filter for the exact kNN.
#pragma once
#include "engine.cuh"

namespace pacmap {
// True when the tcgen05 filter handles this shape.
bool knn_tc_supported(uint64_t n, uint64_t d, uint64_t kp);
// Exact kNN through the tensor-core filter + FP32 re-rank; false when it declined the problem.
// nprobe in 1..255: approximate -- each row block searches only the nprobe pivot cells nearest its own.
// prune (exact mode, large n): column tiles that provably hold no neighbour of a row block are skipped
// (knn_prune.cu); the result is the same.
bool knn_tc_device(Ctx& c, const float* d_x, uint64_t n, uint64_t d, uint64_t kp, bool bf16, uint32_t* d_idx,
                   float* d_dist, const KnnShard& shard = KnnShard(), int nprobe = 0, bool prune = true);
// Counters of the last tensor-core kNN on this thread.
struct KnnTcStats {
  double filter_ms = 0.0;       // device time of the filter launch that produced the candidates
  double bound_ms = 0.0;        // device time of the pruning's bound pass, statistics and tile lists
  uint64_t fallback_rows = 0;   // rows recomputed by the exact SIMT kernel
  uint64_t tiles_full = 0;      // (row block, column tile) pairs of the full sweep
  uint64_t tiles_visited = 0;   // pairs the filter computed
  uint64_t tiles_bound = 0;     // pairs the bound pass computed
  uint64_t insertions = 0;      // candidate entries the filter passes wrote (all rows)
  uint64_t compactions = 0;     // row compactions inside the filter passes
  uint64_t band_entries = 0;    // candidates left for the exact re-rank (all rows)
  uint64_t rows = 0;            // rows of the problem
};
KnnTcStats& last_tc_stats();
}  // namespace pacmap
