// Random-forest classifier: the walk of sklearn's RandomForestClassifier
// (sklearn/tree/_tree.pyx Tree._apply_dense; averaging in
// sklearn/ensemble/_forest.py ForestClassifier.predict_proba) over a packed
// forest (cbmv_b200/forest.py):
//   node = {float32 t32, uint32 word}; word bit 31 = leaf, bits 0-4 =
//   feature, bits 5-30 = left child (right child = left + 1); a leaf's word
//   holds its index into leaf_value (float64 class-0 / class-1 fractions).
// sklearn tests float32(x) <= float64 threshold; t32 is the largest float32
// not above the threshold, so `x <= t32` takes the same branch for every
// float32 x.  The class fractions are summed in float64 in tree order and
// divided by the tree count, as predict_proba does with one job.
#include "common.cuh"
#include "rf.cuh"

namespace cbmv {
namespace {

constexpr int kBlock = 128;

__global__ void rf_predict_kernel(RfView f, const float* __restrict__ X, int64_t N,
                                  double* __restrict__ proba, int32_t* __restrict__ leaves) {
  extern __shared__ float xs[];  // [F][blockDim.x]
  const int tid = threadIdx.x;
  for (int64_t n0 = (int64_t)blockIdx.x * blockDim.x; n0 < N; n0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t n = n0 + tid;
    __syncthreads();
    // stage the block's feature rows, coalesced, transposed to [F][block]
    for (int k = tid; k < f.n_features * (int)blockDim.x; k += blockDim.x) {
      const int r = k / f.n_features, c = k - r * f.n_features;
      const int64_t row = n0 + r;
      xs[c * blockDim.x + r] = row < N ? X[row * f.n_features + c] : 0.0f;
    }
    __syncthreads();
    if (n >= N) continue;
    double p0 = 0.0, p1 = 0.0;
    for (int t = 0; t < f.n_trees; t++) {
      uint32_t idx = (uint32_t)f.offsets[t];
      uint2 node = __ldg(f.nodes + idx);
      while (!(node.y & kLeafFlag)) {
        const float x = xs[(node.y & 31u) * blockDim.x + tid];
        idx = ((node.y >> 5) & kChildMask) + (x <= __uint_as_float(node.x) ? 0u : 1u);
        node = __ldg(f.nodes + idx);
      }
      const double2 v = __ldg(f.leaf_value + (node.y & ~kLeafFlag));
      p0 += v.x;
      p1 += v.y;
      if (leaves) leaves[n * f.n_trees + t] = (int32_t)(idx - (uint32_t)f.offsets[t]);
    }
    if (proba) {
      proba[2 * n] = p0 / f.n_trees;
      proba[2 * n + 1] = p1 / f.n_trees;
    }
  }
}

}  // namespace
}  // namespace cbmv

using namespace cbmv;

struct cbmv_forest {
  RfView view;
  void* mem;
};

extern "C" int cbmv_forest_create(const uint32_t* nodes, int64_t n_nodes, const double* leaf_value,
                                  int64_t n_leaves, const int32_t* tree_offsets, int n_trees,
                                  int n_features, cbmv_forest** out) {
  CBMV_REQUIRE(nodes && leaf_value && tree_offsets && out, CBMV_EINVAL, "null pointer argument");
  CBMV_REQUIRE(n_nodes > 0 && n_leaves > 0 && n_trees > 0, CBMV_EINVAL, "empty forest");
  CBMV_REQUIRE(n_features > 0 && n_features <= 32, CBMV_EINVAL, "n_features %d not in 1..32",
               n_features);
  CBMV_REQUIRE(n_nodes <= (int64_t)kChildMask, CBMV_ERANGE, "forest has too many nodes");
  CBMV_REQUIRE(tree_offsets[0] == 0 && tree_offsets[n_trees] == n_nodes, CBMV_EINVAL,
               "tree offsets do not cover the node array");
  // validate the packed structure on the host: every index stays in range,
  // so the device walk never reads outside the arrays
  for (int t = 0; t < n_trees; t++) {
    CBMV_REQUIRE(tree_offsets[t] < tree_offsets[t + 1], CBMV_EINVAL, "empty tree %d", t);
    for (int64_t k = tree_offsets[t]; k < tree_offsets[t + 1]; k++) {
      const uint32_t w = nodes[2 * k + 1];
      if (w & kLeafFlag) {
        CBMV_REQUIRE((int64_t)(w & ~kLeafFlag) < n_leaves, CBMV_EINVAL, "leaf index out of range");
      } else {
        const int64_t c = (w >> 5) & kChildMask;
        CBMV_REQUIRE((int)(w & 31u) < n_features, CBMV_EINVAL, "feature out of range");
        CBMV_REQUIRE(c > k && c + 1 < tree_offsets[t + 1], CBMV_EINVAL,
                     "child of node %lld outside its tree", (long long)k);
      }
    }
  }
  cbmv_forest* f = new cbmv_forest();
  // each array starts on a 256-byte boundary (leaf values are 16-byte double2)
  auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t nb = up((size_t)n_nodes * sizeof(uint2)), lb = up((size_t)n_leaves * sizeof(double2)),
               ob = (size_t)(n_trees + 1) * sizeof(int32_t);
  cudaError_t e = cudaMalloc(&f->mem, nb + lb + ob);
  if (e != cudaSuccess) {
    delete f;
    return set_error(CBMV_ENOMEM, "forest upload: %s", cudaGetErrorString(e));
  }
  char* base = (char*)f->mem;
  f->view.nodes = (const uint2*)base;
  f->view.leaf_value = (const double2*)(base + nb);
  f->view.offsets = (const int32_t*)(base + nb + lb);
  f->view.n_trees = n_trees;
  f->view.n_features = n_features;
  f->view.n_nodes = n_nodes;
  f->view.n_leaves = n_leaves;
  if (cudaMemcpy(base, nodes, (size_t)n_nodes * sizeof(uint2), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(base + nb, leaf_value, (size_t)n_leaves * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(base + nb + lb, tree_offsets, ob, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(f->mem);
    delete f;
    return set_error(CBMV_ECUDA, "forest upload failed");
  }
  *out = f;
  return CBMV_OK;
}

extern "C" int cbmv_forest_info(const cbmv_forest* f, int* n_trees, int64_t* n_nodes,
                                int64_t* n_leaves) {
  CBMV_REQUIRE(f, CBMV_EINVAL, "null forest");
  if (n_trees) *n_trees = f->view.n_trees;
  if (n_nodes) *n_nodes = f->view.n_nodes;
  if (n_leaves) *n_leaves = f->view.n_leaves;
  return CBMV_OK;
}

extern "C" int cbmv_forest_destroy(cbmv_forest* f) {
  if (!f) return CBMV_OK;
  cudaFree(f->mem);
  delete f;
  return CBMV_OK;
}

namespace cbmv {
const RfView* forest_view(const cbmv_forest* f) { return &f->view; }
}  // namespace cbmv

extern "C" int cbmv_forest_predict(const cbmv_forest* f, const float* X, int64_t N, double* proba,
                                   int32_t* leaves, void* stream) {
  CBMV_REQUIRE(f && X, CBMV_EINVAL, "null pointer argument");
  CBMV_REQUIRE(N > 0, CBMV_EINVAL, "N must be positive");
  const size_t smem = (size_t)f->view.n_features * kBlock * sizeof(float);
  rf_predict_kernel<<<grid_for(N, kBlock), kBlock, smem, as_stream(stream)>>>(f->view, X, N, proba,
                                                                             leaves);
  return check_launch("forest_predict");
}
