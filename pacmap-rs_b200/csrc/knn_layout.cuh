// Layout constants shared by the tensor-core kNN filter (knn_tc.cu) and its tile pruning (knn_prune.cu).
#pragma once
#include <cstdint>

namespace pacmap {

constexpr int TC_BM = 256;  // rows per filter block (two M = 128 accumulators)
constexpr int TC_BN = 128;  // columns per tile (MMA N)
constexpr int PIV = 256;    // pivots (cells) of the locality order

// Column tile visited at step t by row block b: first the window of SWEEP_W tiles around the block's own
// rows, then every other tile in ascending order (all blocks of a wave advance through the same region,
// which keeps the B operand in L2).
constexpr int SWEEP_W = 16;
__host__ __device__ __forceinline__ int sweep_tile(int t, int b, int ntiles) {
  if (ntiles <= SWEEP_W) return t;
  int w0 = 2 * b - SWEEP_W / 2 + 1;
  w0 = w0 < 0 ? 0 : (w0 > ntiles - SWEEP_W ? ntiles - SWEEP_W : w0);
  if (t < SWEEP_W) return w0 + t;
  const int r = t - SWEEP_W;
  return r < w0 ? r : r + SWEEP_W;
}

}  // namespace pacmap
