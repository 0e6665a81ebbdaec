// Random-forest classifier: sklearn's RandomForestClassifier.predict_proba
// (sklearn/ensemble/_forest.py; tree walk sklearn/tree/_tree.pyx
// Tree._apply_dense) over the packed two-level-block forest of rf.cuh.
// The class fractions of the leaves are summed in float64 in tree order and
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
    const float* x = xs + tid;
    double p0 = 0.0, p1 = 0.0;
    for (int t = 0; t < f.n_trees; t++) {
      uint32_t b = (uint32_t)f.offsets[t];
      for (;;) {
        RfBlock blk;
        blk.a = __ldg(f.blocks + 2 * (size_t)b);
        blk.b = __ldg(f.blocks + 2 * (size_t)b + 1);
        b = rf_step(blk, x, blockDim.x);
        if (b & kLeafFlag) break;
      }
      const uint32_t leaf = b & ~kLeafFlag;
      const double2 v = __ldg(f.leaf_value + leaf);
      p0 += v.x;
      p1 += v.y;
      if (leaves) leaves[n * f.n_trees + t] = (int32_t)leaf;
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

extern "C" int cbmv_forest_create(const uint32_t* blocks, int64_t n_blocks, const double* leaf_value,
                                  int64_t n_leaves, const int32_t* tree_offsets, int n_trees,
                                  int n_features, cbmv_forest** out) {
  CBMV_REQUIRE(blocks && leaf_value && tree_offsets && out, CBMV_EINVAL, "null pointer argument");
  CBMV_REQUIRE(n_blocks > 0 && n_leaves > 0 && n_trees > 0, CBMV_EINVAL, "empty forest");
  CBMV_REQUIRE(n_features > 0 && n_features <= 32, CBMV_EINVAL, "n_features %d not in 1..32",
               n_features);
  CBMV_REQUIRE(n_blocks < (int64_t)kLeafFlag && n_leaves < (int64_t)kLeafFlag, CBMV_ERANGE,
               "forest too large for 31-bit indices");
  CBMV_REQUIRE(tree_offsets[0] == 0 && tree_offsets[n_trees] == n_blocks, CBMV_EINVAL,
               "tree offsets do not cover the block array");
  // Validate the structure on the host, so the device walk never reads
  // outside the arrays and always ends: every feature is in range, every
  // leaf index exists, every child block lies later in the same tree.
  for (int t = 0; t < n_trees; t++) {
    CBMV_REQUIRE(tree_offsets[t] < tree_offsets[t + 1], CBMV_EINVAL, "empty tree %d", t);
    for (int64_t k = tree_offsets[t]; k < tree_offsets[t + 1]; k++) {
      const uint32_t* w = blocks + 8 * k;
      const uint32_t f0 = w[3] & 0xFFu, f1 = (w[3] >> 8) & 0xFFu, f2 = (w[3] >> 16) & 0xFFu;
      auto leaf_ok = [&](uint32_t v) { return (int64_t)(v & ~kLeafFlag) < n_leaves; };
      auto feat_ok = [&](uint32_t f) { return f == kLeafFeature || (int)f < n_features; };
      CBMV_REQUIRE(feat_ok(f0) && feat_ok(f1) && feat_ok(f2), CBMV_EINVAL,
                   "block %lld: feature out of range", (long long)k);
      if (f0 == kLeafFeature) {
        CBMV_REQUIRE(leaf_ok(w[4]), CBMV_EINVAL, "block %lld: leaf index out of range", (long long)k);
        continue;
      }
      for (int n = 1; n <= 2; n++) {
        const uint32_t fn = n == 1 ? f1 : f2;
        const int slot = 4 + 2 * (n - 1);
        if (fn == kLeafFeature) {
          CBMV_REQUIRE(leaf_ok(w[slot]), CBMV_EINVAL, "block %lld: leaf index out of range",
                       (long long)k);
          continue;
        }
        for (int j = 0; j < 2; j++) {
          const uint32_t c = w[slot + j];
          if (c & kLeafFlag) {
            CBMV_REQUIRE(leaf_ok(c), CBMV_EINVAL, "block %lld: leaf index out of range",
                         (long long)k);
          } else {
            CBMV_REQUIRE((int64_t)c > k && (int64_t)c < tree_offsets[t + 1], CBMV_EINVAL,
                         "block %lld: child block outside its tree", (long long)k);
          }
        }
      }
    }
  }
  cbmv_forest* f = new cbmv_forest();
  auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t bb = up((size_t)n_blocks * 32), lb = up((size_t)n_leaves * sizeof(double2)),
               pb = up((size_t)n_leaves * sizeof(double)), ob = (size_t)(n_trees + 1) * sizeof(int32_t);
  cudaError_t e = cudaMalloc(&f->mem, bb + lb + pb + ob);
  if (e != cudaSuccess) {
    delete f;
    return set_error(CBMV_ENOMEM, "forest upload: %s", cudaGetErrorString(e));
  }
  char* base = (char*)f->mem;
  f->view.blocks = (const uint4*)base;
  f->view.leaf_value = (const double2*)(base + bb);
  f->view.leaf_p0 = (const double*)(base + bb + lb);
  f->view.offsets = (const int32_t*)(base + bb + lb + pb);
  f->view.n_trees = n_trees;
  f->view.n_features = n_features;
  f->view.n_blocks = n_blocks;
  f->view.n_leaves = n_leaves;
  if (cudaMemcpy(base, blocks, (size_t)n_blocks * 32, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(base + bb, leaf_value, (size_t)n_leaves * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy2D(base + bb + lb, sizeof(double), leaf_value, 2 * sizeof(double), sizeof(double),
                   (size_t)n_leaves, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(base + bb + lb + pb, tree_offsets, ob, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(f->mem);
    delete f;
    return set_error(CBMV_ECUDA, "forest upload failed");
  }
  *out = f;
  return CBMV_OK;
}

namespace cbmv {
const RfView* forest_view(const cbmv_forest* f) { return &f->view; }
}  // namespace cbmv

extern "C" int cbmv_forest_info(const cbmv_forest* f, int* n_trees, int64_t* n_blocks,
                                int64_t* n_leaves) {
  CBMV_REQUIRE(f, CBMV_EINVAL, "null forest");
  if (n_trees) *n_trees = f->view.n_trees;
  if (n_blocks) *n_blocks = f->view.n_blocks;
  if (n_leaves) *n_leaves = f->view.n_leaves;
  return CBMV_OK;
}

extern "C" int cbmv_forest_destroy(cbmv_forest* f) {
  if (!f) return CBMV_OK;
  cudaDeviceSynchronize();
  cudaFree(f->mem);
  delete f;
  return CBMV_OK;
}

extern "C" int cbmv_forest_predict(const cbmv_forest* f, const float* X, int64_t N, double* proba,
                                   int32_t* leaves, void* stream) {
  CBMV_REQUIRE(f && X, CBMV_EINVAL, "null pointer argument");
  CBMV_REQUIRE(N > 0, CBMV_EINVAL, "N must be positive");
  const size_t smem = (size_t)f->view.n_features * kBlock * sizeof(float);
  rf_predict_kernel<<<grid_for(N, kBlock), kBlock, smem, as_stream(stream)>>>(f->view, X, N, proba,
                                                                             leaves);
  return check_launch("forest_predict");
}
