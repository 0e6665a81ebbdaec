// Fused classifier kernels: the 20 CBMV features of every (pixel, d) built in
// shared memory and classified in place, so the [H*W*D, 20] feature matrix
// of the reference (test.py:541-595, handed to predict_proba at test.py:620)
// never exists in HBM.  Output: P(class 0), float32 [H,W,D], the matching
// cost the post-processing consumes (test.py:144-145).
//
// Random-forest walk (features_rf_tiled):
//  - one persistent CTA of 512 threads per SM; shared memory holds only the
//    feature tile (40 KB), leaving the rest of the SM's 256 KB to L1, which
//    keeps the hot upper levels of the trees (staging them in shared memory
//    explicitly measured slower: the extra address checks cost more than the
//    L1 misses they saved);
//  - each walk step reads one 32-byte block (one L2 sector) and descends two
//    tree levels, halving the chain of dependent loads;
//  - a warp covers 8 pixels x 4 disparities: neighbouring pixels at nearby
//    disparities have similar features and walk similar paths, so a warp's
//    requests touch fewer distinct sectors than 32 disparities of one pixel;
//  - each thread walks ILP trees at once (independent loads in flight) and
//    adds the leaf fractions in tree order, as predict_proba does.
#include "common.cuh"
#include "features.cuh"
#include "pipeline.cuh"
#include "rf.cuh"

namespace cbmv {
namespace {

constexpr int kRfBlock = 512;        // threads per CTA
constexpr int kRfWarpsX = 4;         // warps along x in a CTA tile (8 px each)
constexpr int kRfTileX = kRfWarpsX * 8;                    // 32 px
constexpr int kRfTileD = (kRfBlock / 32 / kRfWarpsX) * 4;  // 16 disparities
constexpr int kRfIlp = 4;

template <int ILP>
__global__ void __launch_bounds__(kRfBlock, 1)
    features_rf_tiled(FeatVols fv, const double* __restrict__ stats, int64_t H, int64_t W, int D,
                      RfView f, float* __restrict__ prob0) {
  extern __shared__ float xs[];  // [20][kRfBlock]: one feature column per thread
  const int T = f.n_trees;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int wx = warp % kRfWarpsX, wd = warp / kRfWarpsX;
  const int64_t ntx = (W + kRfTileX - 1) / kRfTileX;
  const int64_t ntd = (D + kRfTileD - 1) / kRfTileD;
  const int64_t tiles = H * ntx * ntd;
  const int64_t HW = H * W;
  float* col = xs + tid;

  for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int64_t td = tile % ntd;
    const int64_t tx = (tile / ntd) % ntx;
    const int64_t y = tile / (ntd * ntx);
    const int64_t x = tx * kRfTileX + wx * 8 + (lane & 7);
    const int d = (int)(td * kRfTileD + wd * 4 + (lane >> 3));
    if (x >= W || d >= D) continue;
    const int64_t p = y * W + x;
    features_store(fv.v, stats, HW, D, p, x, d, col, kRfBlock);

    double acc = 0.0;
    for (int t = 0; t < T; t += ILP) {
      uint32_t b[ILP];
#pragma unroll
      for (int k = 0; k < ILP; k++) b[k] = t + k < T ? (uint32_t)__ldg(f.offsets + t + k) : kLeafFlag;
      for (;;) {
        bool live = false;
#pragma unroll
        for (int k = 0; k < ILP; k++) live |= !(b[k] & kLeafFlag);
        if (!live) break;
        RfBlock blk[ILP];
#pragma unroll
        for (int k = 0; k < ILP; k++) {
          // a finished walk steps through a leaf-only block (reads feature 0)
          blk[k].a = make_uint4(0u, 0u, 0u, 0xFFFFFFFFu);
          blk[k].b = make_uint4(0u, 0u, 0u, 0u);
          if (!(b[k] & kLeafFlag)) {
            blk[k].a = __ldg(f.blocks + 2 * (size_t)b[k]);
            blk[k].b = __ldg(f.blocks + 2 * (size_t)b[k] + 1);
          }
        }
#pragma unroll
        for (int k = 0; k < ILP; k++) {
          const uint32_t nb = rf_step(blk[k], col, kRfBlock);
          b[k] = (b[k] & kLeafFlag) ? b[k] : nb;
        }
      }
#pragma unroll
      for (int k = 0; k < ILP; k++)
        if (t + k < T) acc += __ldg(f.leaf_p0 + (b[k] & ~kLeafFlag));
    }
    prob0[p * D + d] = (float)(acc / T);
  }
}

}  // namespace

int launch_features_rf(const double* const* vols, const double* stats, int64_t H, int64_t W,
                       int D, const cbmv_forest* forest, float* prob0, cudaStream_t st) {
  const RfView& f = *forest_view(forest);
  CBMV_REQUIRE(f.n_features == 20, CBMV_EINVAL, "the forest must take the 20 CBMV features");
  int dev = 0, sms = 0;
  CBMV_CUDA(cudaGetDevice(&dev));
  CBMV_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const size_t smem = (size_t)20 * kRfBlock * sizeof(float);
  FeatVols fv = {{vols[0], vols[1], vols[2], vols[3]}};
  features_rf_tiled<kRfIlp><<<sms, kRfBlock, smem, st>>>(fv, stats, H, W, D, f, prob0);
  return check_launch("features_rf_tiled");
}

}  // namespace cbmv
