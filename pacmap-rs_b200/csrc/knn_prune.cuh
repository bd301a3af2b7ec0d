// Pivots of the kNN locality order and certified tile pruning for the exact tensor-core kNN.
#pragma once
#include "engine.cuh"

namespace pacmap {

// PIV pivot rows of d_x (n x d) by k-means++ seeding in batches on a fixed subsample; deterministic.
void select_pivots(Ctx& c, const float* d_x, uint64_t n, uint64_t d, uint32_t* d_piv_rows);

// Inputs of the tile test, all on the device and in the locality order unless noted:
//   perm        position r -> original row
//   cell        original row -> pivot cell
//   score       original row o -> |p|^2 - 2 x_o . p for every pivot p (n x PIV, f32, fused multiply-add sums)
//   pnorm       |p|^2 of every pivot (f32)
//   rownorm     position r -> |x s|^2 (f32; s the filter's power-of-two scale)
//   ub          position r -> an upper bound of the squared distance (scaled by s^2) to the row's k'-th
//               neighbour; +inf when unknown
struct PruneInputs {
  const uint32_t* perm = nullptr;
  const uint32_t* cell = nullptr;
  const float* score = nullptr;
  const float* pnorm = nullptr;
  const float* rownorm = nullptr;
  const float* ub = nullptr;
  uint64_t n = 0, n_pad = 0, d = 0;
  float inv_s = 1.0f;  // 1 / s (exact)
  uint64_t blk0 = 0, blk1 = 0;  // the row blocks to plan (a shard's range)
  // tiles already computed for each row block (CSR, may be null): left out of the lists
  const uint32_t* skip_ptr = nullptr;
  const uint32_t* skip_list = nullptr;
};

// Per row block in [blk0, blk1): the column tiles of its own pivot cells, then those of the probe - 1
// cells nearest each own cell (pivot-to-pivot distance) that holds fewer than min_cell points (all of them
// for min_cell = UINT32_MAX), as a CSR list (ptr: n_pad / 256 + 1 offsets, list); d_cstart: the PIV cell
// starts of the locality order. Returns the number of (block, tile) pairs. Needs n_pad / 128 <= 131,072
// column tiles.
uint64_t build_probe_tile_lists(Ctx& c, const float* d_x, uint64_t d, const uint32_t* d_piv_rows,
                                const uint32_t* d_cstart, uint64_t n, uint64_t n_pad, int probe, uint32_t min_cell,
                                uint64_t blk0, uint64_t blk1, DevBuf<uint32_t>& ptr, DevBuf<uint32_t>& list);

// Per row block in [blk0, blk1): the column tiles that may hold one of its rows' k' nearest points and are
// not in its skip list, in the filter's sweep order, as a CSR list (ptr: n_pad / 256 + 1 offsets, list).
// Returns the number of (block, tile) pairs kept.
uint64_t build_pruned_tile_lists(Ctx& c, const PruneInputs& in, DevBuf<uint32_t>& ptr, DevBuf<uint32_t>& list);

}  // namespace pacmap
