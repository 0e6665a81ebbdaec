// Device view of a packed random forest and the block walk shared by the
// classifier kernels.
//
// Layout (cbmv_b200/forest.py, FlatForest.pack): every tree is cut into
// two-level blocks of 32 bytes (one L2 sector), numbered breadth-first per
// tree:
//   words 0-2  float32 thresholds of nodes 0 (block root), 1, 2 (its
//              children); t32 = the largest float32 <= sklearn's float64
//              threshold, so `x <= t32` branches as sklearn's
//              `float32(x) <= threshold` does (sklearn/tree/_tree.pyx,
//              Tree._apply_dense)
//   word 3     features of nodes 0, 1, 2 in bytes 0-2; 0xFF marks a leaf
//   words 4-7  node 1's left/right and node 2's left/right child: bit 31
//              set = leaf index, clear = block rooted at that child.  A leaf
//              at node 0 or 1 keeps its leaf index in word 4, at node 2 in
//              word 6.
// One walk step reads one block (two 16-byte loads of the same sector) and
// descends two levels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cbmv.h"

namespace cbmv {

constexpr uint32_t kLeafFlag = 1u << 31;
constexpr uint32_t kLeafFeature = 0xFFu;

struct RfView {
  const uint4* blocks;        // [2 * n_blocks]: words 0-3, words 4-7
  const double2* leaf_value;  // {class-0 fraction, class-1 fraction}
  const double* leaf_p0;      // class-0 fraction alone
  const int32_t* offsets;     // [n_trees + 1] first block of each tree
  int n_trees;
  int n_features;
  int64_t n_blocks;
  int64_t n_leaves;
};

const RfView* forest_view(const cbmv_forest* f);

struct RfBlock {
  uint4 a, b;
};

// Descends the two levels of block `blk` for the sample whose feature k is
// x[k * stride].  Returns the next block index, or the leaf index with
// kLeafFlag set.
// Branch-free: leaves read feature 0 as a dummy and the result is selected.
__device__ __forceinline__ uint32_t rf_step(const RfBlock& blk, const float* x, int stride) {
  const uint32_t feats = blk.a.w;
  const uint32_t f0 = feats & 0xFFu;
  const bool leaf0 = f0 == kLeafFeature;
  const bool right = !(x[(leaf0 ? 0u : f0) * stride] <= __uint_as_float(blk.a.x));
  const uint32_t fn = __byte_perm(feats, 0, right ? 0x4442u : 0x4441u);
  const bool leafn = fn == kLeafFeature;
  const float tn = __uint_as_float(right ? blk.a.z : blk.a.y);
  const bool right2 = !(x[(leafn ? 0u : fn) * stride] <= tn);
  const uint32_t cl = right ? blk.b.z : blk.b.x;
  const uint32_t cr = right ? blk.b.w : blk.b.y;
  const uint32_t c = right2 ? cr : cl;
  return leaf0 ? (blk.b.x | kLeafFlag) : (leafn ? (cl | kLeafFlag) : c);
}

}  // namespace cbmv
