// Device view of a packed random forest (see rf.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cbmv.h"

namespace cbmv {

constexpr uint32_t kLeafFlag = 1u << 31;
constexpr uint32_t kChildMask = (1u << 26) - 1;

struct RfView {
  const uint2* nodes;         // {float32 threshold bits, word}
  const double2* leaf_value;  // {class-0 fraction, class-1 fraction}
  const int32_t* offsets;     // [n_trees + 1]
  int n_trees;
  int n_features;
  int64_t n_nodes;
  int64_t n_leaves;
};

const RfView* forest_view(const cbmv_forest* f);

}  // namespace cbmv
