// The fused test path for one rectified pair: the work of main.py:53-70
// (Testing.test_model, test.py:597-626, then Testing.eval_prob with the
// default `_mem` post-processing, test.py:143-149 and 341-449) as one
// sequence of device launches on one stream, with every intermediate
// resident in HBM:
//
//   1. per-pixel terms: census descriptors, NCC window sums, ZSAD means,
//      Sobel responses (both images)
//   2. the four [H,W,D] float64 cost volumes (census, ncc, sadsob, zsad)
//   3. per-pixel row minimum and likelihood denominator of every volume, for
//      the left and the right reference view
//   4. features + random forest fused -> P(class 0), float32 [H,W,D]
//   5. post: image normalisation, cross arms, SGM x sgm_i, CBCA x cbca_i2,
//      winner-take-all + subpixel, median, thresholded Gaussian.
//
// The reference's per-row batching of the classifier (test.py:608-623) only
// bounds its host memory; every feature is row-local, so one launch covers
// the whole image with identical results.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "pipeline.cuh"
#include "post.cuh"

using namespace cbmv;

extern "C" void cbmv_params_default(cbmv_params* p) {
  // Testing.__init__ defaults, test.py:44-47; SAD-on-Sobel window test.py:131
  p->censw = 11;
  p->nccw = 3;
  p->sadw = 5;
  p->sobw = 5;
  p->pi1 = 1.3f;
  p->pi2 = 10.0f;
  p->sgm_q1 = 2.2f;
  p->sgm_q2 = 3.0f;
  p->alpha1 = 1.4f;
  p->tau_so = 0.12f;
  p->sgm_i = 2;
  p->L1 = 6;
  p->tau1 = 0.07f;
  p->cbca_i1 = 0;
  p->cbca_i2 = 4;
  p->median_i = 1;
  p->median_w = 3;
  p->blur_sigma = 2.2f;
  p->blur_t = 1.3f;
  p->direction = -1;  // test.py:501
  p->exact_cbca = 0;
  p->mlp_ctas = 0;
  p->cbca_rows = 0;
  p->sgm_prefetch = 0;
  p->interpolate = 0;  // main.py:70 runs the _mem post
}

struct cbmv_ctx {
  cudaStream_t stream = nullptr;
  // a second stream for work that overlaps the main one inside a call (the
  // CBCA support build runs beside the SGM), ordered by the two events
  cudaStream_t side = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr, prep_ev = nullptr;
  void* ws = nullptr;
  size_t ws_bytes = 0;
  cudaEvent_t ev[6] = {};
  float ms[5] = {};
  float* gauss = nullptr;  // device copy of the mean2d kernel
  int gauss_ks = 0;
  float gauss_sigma = -1.0f;
  void* io = nullptr;  // device copies of a host-buffer call's images and disparity
  size_t io_bytes = 0;
};

namespace {

// Testing.__gaussian, test.py:108-118 (centre offset by one, as written).
std::vector<float> gaussian_kernel(double sigma, int* ks_out) {
  const int kr = (int)ceil(sigma * 3);
  const int ks = kr * 2 + 1;
  std::vector<float> k((size_t)ks * ks);
  for (int i = 0; i < ks; i++)
    for (int j = 0; j < ks; j++) {
      const double y = (i - 1) - kr, x = (j - 1) - kr;
      k[(size_t)i * ks + j] = (float)exp(-(x * x + y * y) / (2 * sigma * sigma));
    }
  *ks_out = ks;
  return k;
}

struct Carve {
  char* base;
  size_t off = 0;
  template <class T>
  T* take(size_t n) {
    off = (off + 255) & ~(size_t)255;
    T* p = (T*)(base ? base + off : nullptr);
    off += n * sizeof(T);
    return p;
  }
};

struct Work {
  ulonglong2 *descL, *descR;
  uint32_t *AL, *AR;
  double *CL, *CR, *muL, *muR;
  int32_t *sobL, *sobR;
  double* vol[4];
  bool f32;  // matcher volumes in float32
  double* stats;
  float2* statsf;  // (min, 1/den) in float32 for the classifier network
  float *volA, *volB;
  float* volC;  // the right view's cost of the _interp post (else null)
  float *imL, *imR, *crossL, *crossR, *dtmp, *dtmp2, *dright, *outlier;
  float* grad;  // SGM neighbour differences: left h/v, right h/v
  uint32_t* masks;  // CBCA support words, 4 B per (p,d), live beside the SGM volumes
  bool prepped = false;  // the post's image terms were launched on the side stream (prep_ev)
  double* mom;
};

// f32: the four matcher volumes hold float32 (4 B per (p,d) each) instead of
// float64; the four SGM direction volumes then alias them one to one.
// interp: one more float32 volume for the right view of the _interp post.
Work carve(void* base, int64_t H, int64_t W, int D, size_t* bytes, bool f32, bool interp) {
  Carve c{(char*)base};
  Work w;
  const size_t HW = (size_t)H * W, V = HW * (size_t)D;
  w.descL = c.take<ulonglong2>(HW);
  w.descR = c.take<ulonglong2>(HW);
  w.AL = c.take<uint32_t>(HW);
  w.AR = c.take<uint32_t>(HW);
  w.CL = c.take<double>(HW);
  w.CR = c.take<double>(HW);
  w.muL = c.take<double>(HW);
  w.muR = c.take<double>(HW);
  w.sobL = c.take<int32_t>(HW);
  w.sobR = c.take<int32_t>(HW);
  for (int m = 0; m < 4; m++) w.vol[m] = f32 ? (double*)c.take<float>(V) : c.take<double>(V);
  w.f32 = f32;
  w.stats = c.take<double>(16 * HW);
  w.statsf = c.take<float2>(8 * HW);
  w.volA = c.take<float>(V);
  w.volB = c.take<float>(V);
  w.volC = interp ? c.take<float>(V) : nullptr;
  w.imL = c.take<float>(HW);
  w.imR = c.take<float>(HW);
  w.crossL = c.take<float>(4 * HW);
  w.crossR = c.take<float>(4 * HW);
  w.dtmp = c.take<float>(HW);
  w.dtmp2 = c.take<float>(HW);
  w.dright = c.take<float>(HW);
  w.outlier = c.take<float>(HW);
  w.grad = c.take<float>(4 * HW);
  // the support words: their own volume on the float32 path (the SGM's four
  // direction volumes take all four matcher volumes), the third float64
  // matcher volume otherwise (the SGM uses only the first two)
  w.masks = f32 ? c.take<uint32_t>(V) : reinterpret_cast<uint32_t*>(w.vol[2]);
  w.mom = c.take<double>(4);
  *bytes = c.off + 256;
  return w;
}

int check_params(const cbmv_params* p) {
  CBMV_REQUIRE(p->censw == 11 && p->nccw >= 1 && p->nccw <= 15 && (p->nccw & 1) && p->sadw >= 1 &&
                   p->sadw <= 15 && (p->sadw & 1) && p->sobw >= 1 && p->sobw <= 15 && (p->sobw & 1),
               CBMV_EINVAL, "unsupported matcher windows");
  CBMV_REQUIRE(p->sgm_i >= 0 && p->cbca_i1 >= 0 && p->cbca_i2 >= 0 && p->median_i >= 0,
               CBMV_EINVAL, "negative iteration count");
  CBMV_REQUIRE(p->median_w >= 1 && p->median_w <= 11 && (p->median_w & 1), CBMV_EINVAL,
               "median window must be odd <= 11");
  CBMV_REQUIRE(p->blur_sigma > 0 && p->blur_sigma <= 5.0f, CBMV_EINVAL, "blur_sigma not in (0, 5]");
  CBMV_REQUIRE(p->direction == 1 || p->direction == -1, CBMV_EINVAL, "direction must be +-1");
  CBMV_REQUIRE(p->cbca_rows == 0 || p->cbca_rows == 16 || p->cbca_rows == 32, CBMV_EINVAL,
               "cbca_rows must be 0, 16 or 32");
  CBMV_REQUIRE(p->sgm_prefetch == 0 || p->sgm_prefetch == 1 || p->sgm_prefetch == 2 || p->sgm_prefetch == 4,
               CBMV_EINVAL, "sgm_prefetch must be 0, 1, 2 or 4");
  CBMV_REQUIRE(p->mlp_ctas >= 0, CBMV_EINVAL, "mlp_ctas must be >= 0");
  CBMV_REQUIRE(p->interpolate == 0 || p->interpolate == 1, CBMV_EINVAL, "interpolate must be 0 or 1");
  return CBMV_OK;
}

}  // namespace

extern "C" int cbmv_ctx_create(void* stream, cbmv_ctx** out) {
  CBMV_REQUIRE(out, CBMV_EINVAL, "null pointer argument");
  cbmv_ctx* c = new cbmv_ctx();
  c->stream = as_stream(stream);
  for (int i = 0; i < 6; i++) {
    if (cudaEventCreate(&c->ev[i]) != cudaSuccess) {
      for (int j = 0; j < i; j++) cudaEventDestroy(c->ev[j]);
      delete c;
      return set_error(CBMV_ECUDA, "cudaEventCreate failed");
    }
  }
  if (cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->join_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->prep_ev, cudaEventDisableTiming) != cudaSuccess) {
    cbmv_ctx_destroy(c);
    return set_error(CBMV_ECUDA, "cudaStreamCreate / cudaEventCreate failed");
  }
  *out = c;
  return CBMV_OK;
}

extern "C" int cbmv_ctx_destroy(cbmv_ctx* c) {
  if (!c) return CBMV_OK;
  cudaStreamSynchronize(c->stream);
  if (c->side) cudaStreamSynchronize(c->side);
  if (c->ws) cudaFree(c->ws);
  if (c->gauss) cudaFree(c->gauss);
  if (c->io) cudaFree(c->io);
  for (int i = 0; i < 6; i++)
    if (c->ev[i]) cudaEventDestroy(c->ev[i]);
  if (c->fork_ev) cudaEventDestroy(c->fork_ev);
  if (c->join_ev) cudaEventDestroy(c->join_ev);
  if (c->prep_ev) cudaEventDestroy(c->prep_ev);
  if (c->side) cudaStreamDestroy(c->side);
  delete c;
  return CBMV_OK;
}

extern "C" int cbmv_ctx_timings(cbmv_ctx* c, float* ms5) {
  CBMV_REQUIRE(c && ms5, CBMV_EINVAL, "null pointer argument");
  const int pairs[5][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 4}, {0, 4}};
  for (int k = 0; k < 5; k++) CBMV_CUDA(cudaEventElapsedTime(&ms5[k], c->ev[pairs[k][0]], c->ev[pairs[k][1]]));
  return CBMV_OK;
}

static int ensure_workspace(cbmv_ctx* c, size_t bytes) {
  if (c->ws_bytes >= bytes) return CBMV_OK;
  CBMV_CUDA(cudaStreamSynchronize(c->stream));
  CBMV_CUDA(cudaStreamSynchronize(c->side));
  if (c->ws) cudaFree(c->ws);
  c->ws = nullptr;
  c->ws_bytes = 0;
  void* fresh = nullptr;
  cudaError_t e = cudaMalloc(&fresh, bytes);
  if (e != cudaSuccess)
    return set_error(CBMV_ENOMEM, "workspace of %zu bytes: %s", bytes, cudaGetErrorString(e));
  c->ws = fresh;
  c->ws_bytes = bytes;
  return CBMV_OK;
}

static int ensure_gaussian(cbmv_ctx* c, float sigma) {
  if (c->gauss && c->gauss_sigma == sigma) return CBMV_OK;
  int ks = 0;
  std::vector<float> k = gaussian_kernel(sigma, &ks);
  if (c->gauss) {
    CBMV_CUDA(cudaStreamSynchronize(c->stream));
    cudaFree(c->gauss);
    c->gauss = nullptr;
  }
  float* fresh = nullptr;
  CBMV_CUDA(cudaMalloc(&fresh, k.size() * sizeof(float)));
  c->gauss = fresh;
  c->gauss_sigma = -1.0f;  // valid once the copy below succeeded
  CBMV_CUDA(cudaMemcpy(c->gauss, k.data(), k.size() * sizeof(float), cudaMemcpyHostToDevice));
  c->gauss_ks = ks;
  c->gauss_sigma = sigma;
  return CBMV_OK;
}

#define RC(x)                 \
  do {                        \
    int rc_ = (x);            \
    if (rc_) return rc_;      \
  } while (0)

// The cost-optimisation chain of Testing.__postprocessing_mem
// (test.py:355-405) on one float32 [H,W,D] cost volume held in `cur`:
// cbca_i1 CBCA passes, sgm_i SGM iterations (each the mean of the four
// scan directions, test.py:378-383), cbca_i2 CBCA passes.  crossA / crossB
// are the arms of the volume's own view and of the matching view: the left
// view's chain passes (left, right, direction); the right view's chain of
// the _interp post (test.py:176-251) passes (right, left, -direction), and
// its SGM keeps the images in their order (test.py:203-207).  `oth` is a
// second volume; *result receives the buffer holding the result.
static int cost_chain(cbmv_ctx* c, const cbmv_params* p, Work& w, int64_t H, int64_t W, int D,
                      const float* crossA, const float* crossB, int direction, float* cur, float* oth,
                      float** result) {
  cudaStream_t st = c->stream;
  const int64_t HW = H * W;
  // the separable form's supports, built once for all the chain's passes
  // (they depend on the arms only); when every pass follows the SGM, the
  // build runs on the side stream beside it (the SGM keeps most of the GPU
  // idle: one warp per scan line) and the main stream waits for it before
  // the first pass
  const bool masked = !p->exact_cbca && p->L1 - 1 <= kCbcaMaskMaxHalo;
  uint32_t* masks = w.masks;
  const bool beside = masked && p->cbca_i1 == 0 && p->cbca_i2 > 0 && p->sgm_i > 0;
  if (beside) {
    CBMV_CUDA(cudaEventRecord(c->fork_ev, st));
    CBMV_CUDA(cudaStreamWaitEvent(c->side, c->fork_ev, 0));
    RC(launch_cbca_mask_build(crossA, crossB, H, W, D, direction, masks, c->side));
    CBMV_CUDA(cudaEventRecord(c->join_ev, c->side));
  } else if (masked && p->cbca_i1 + p->cbca_i2 > 0) {
    RC(launch_cbca_mask_build(crossA, crossB, H, W, D, direction, masks, st));
  }
  auto cbca = [&](const float* in, float* out) {
    const int rows = p->cbca_rows == 16 ? 16 : 32;
    if (p->exact_cbca)
      return launch_cbca(crossA, crossB, in, H, W, D, CBMV_HWD, direction, out, st, p->L1 - 1);
    if (masked) return launch_cbca_masked(masks, in, H, W, D, out, st, rows);
    return launch_cbca_sep(crossA, crossB, in, H, W, D, direction, out, st, p->L1 - 1, rows);
  };
  for (int i = 0; i < p->cbca_i1; i++) {
    RC(cbca(cur, oth));
    float* t = cur; cur = oth; oth = t;
  }
  SgmParams sp{p->pi1, p->pi2, p->tau_so, p->alpha1, p->sgm_q1, p->sgm_q2, direction};
  SgmGrad g{w.grad, w.grad + HW, w.grad + 2 * HW, w.grad + 3 * HW};
  // the four direction volumes reuse the cost volumes, dead by now
  const int64_t V = HW * D;
  SgmOut so = w.f32 ? SgmOut{{(float*)w.vol[0], (float*)w.vol[1], (float*)w.vol[2], (float*)w.vol[3]}}
                    : SgmOut{{(float*)w.vol[0], (float*)w.vol[0] + V, (float*)w.vol[1], (float*)w.vol[1] + V}};
  for (int i = 0; i < p->sgm_i; i++) {
    // out = ((L0 + L1 + L2) + L3) / 4   (test.py:379-383)
    RC(launch_sgm4(g, cur, H, W, D, sp, so, st, p->sgm_prefetch));
    RC(launch_sgm_combine(so, V, nullptr, 0.25f, oth, st));
    float* t = cur; cur = oth; oth = t;
  }
  if (beside) CBMV_CUDA(cudaStreamWaitEvent(st, c->join_ev, 0));
  for (int i = 0; i < p->cbca_i2; i++) {
    RC(cbca(cur, oth));
    float* t = cur; cur = oth; oth = t;
  }
  *result = cur;
  return CBMV_OK;
}

// Step 5 of the header comment on the float32 volume in w.volA; the
// disparity lands in `disp`.  p->interpolate = 0: the _mem post
// (test.py:341-449); 1: the _interp post (test.py:153-338), which first runs
// the right view's chain on get_right_cost of the cost (its winner-take-all
// is the right disparity) and after the left view's subpixel step marks
// occlusions and mismatches (left-right check) and fills them
// (interpolate_mismatch, then interpolate_occlusion) before the median.
// The post's image terms (do_post's normalisation, test.py:485-504; the
// cross arms; the SGM's neighbour differences): they depend on the images
// only, so the fused paths launch them on the side stream at the start of
// the call, beside the matchers.
static int post_prep(const cbmv_params* p, const uint8_t* L, const uint8_t* R, int64_t H, int64_t W, Work& w,
                     cudaStream_t s) {
  const int64_t HW = H * W;
  RC(launch_normalise(L, HW, w.mom, w.imL, s));
  RC(launch_normalise(R, HW, w.mom + 2, w.imR, s));
  RC(launch_cross(w.imL, H, W, p->L1, p->tau1, w.crossL, s));
  RC(launch_cross(w.imR, H, W, p->L1, p->tau1, w.crossR, s));
  SgmGrad g{w.grad, w.grad + HW, w.grad + 2 * HW, w.grad + 3 * HW};
  if (p->sgm_i > 0) RC(launch_sgm_grad(w.imL, w.imR, H, W, &g, s));
  return CBMV_OK;
}

static int run_post(cbmv_ctx* c, const cbmv_params* p, const uint8_t* L, const uint8_t* R,
                    int64_t H, int64_t W, int D, Work& w, float* disp) {
  cudaStream_t st = c->stream;
  RC(ensure_gaussian(c, p->blur_sigma));
  if (w.prepped)
    CBMV_CUDA(cudaStreamWaitEvent(st, c->prep_ev, 0));
  else
    RC(post_prep(p, L, R, H, W, w, st));
  float* res = nullptr;
  if (p->interpolate) {
    // right view (test.py:154, 176-255): its cost, its chain, its argmin
    RC(launch_right_cost_f32(w.volA, H, W, D, w.volC, st));
    RC(cost_chain(c, p, w, H, W, D, w.crossR, w.crossL, -p->direction, w.volC, w.volB, &res));
    RC(launch_wta_subpixel(res, H, W, D, w.dright, nullptr, st));
  }
  RC(cost_chain(c, p, w, H, W, D, w.crossL, w.crossR, p->direction, w.volA, w.volB, &res));
  float* d0 = w.dtmp;
  float* d1 = w.dtmp2;
  if (p->interpolate) {
    // The _interp chain checks and fills the integer winner-take-all
    // disparity: its subpixel step writes disp_temp (test.py:293), the
    // left-right check reads disp_d, still the argmin (test.py:297), and
    // interpolate_mismatch then overwrites every pixel of disp_temp
    // (test.py:299, post.cu:757-827), so the subpixel result never reaches
    // the output and is not formed here.
    RC(launch_wta_subpixel(res, H, W, D, d0, nullptr, st));
  } else {
    RC(launch_wta_subpixel(res, H, W, D, nullptr, d0, st));
  }
  if (p->interpolate) {
    // left-right check and fills (test.py:295-303, post.cu:717-869)
    RC(launch_outlier(d0, w.dright, H, W, D, w.outlier, st));
    RC(launch_mismatch(d0, w.outlier, H, W, d1, st));
    RC(launch_occlusion(d1, w.outlier, H, W, d0, st));
  }
  for (int i = 0; i < p->median_i; i++) {
    RC(launch_median(d0, H, W, p->median_w, d1, st));
    float* t = d0; d0 = d1; d1 = t;
  }
  RC(launch_mean2d(d0, H, W, c->gauss, c->gauss_ks, p->blur_t, disp, st));
  return CBMV_OK;
}

// Steps 1-3 of the header comment: the four cost volumes and their
// per-pixel statistics in the context's workspace.  f32 = false: float64
// volumes and float64 statistics (the exact features of the random forest
// and of the training samples); f32 = true: float32 volumes (in the first
// half of each float64 buffer) and float32 statistics only, for the network.
static int run_front(cbmv_ctx* c, const cbmv_params* p, const uint8_t* L, const uint8_t* R,
                     int64_t H, int64_t W, int D, Work* wout, bool f32 = false, bool prep = false) {
  RC(check_params(p));
  CBMV_REQUIRE(H > p->censw && W > p->censw, CBMV_EINVAL, "image %lldx%lld smaller than the census window",
               (long long)W, (long long)H);
  CBMV_REQUIRE(H <= 65535 && D >= 1 && D <= 1024, CBMV_ERANGE, "H must be <= 65535 and D in 1..1024");
  size_t bytes = 0;
  carve(nullptr, H, W, D, &bytes, f32, p->interpolate != 0);
  RC(ensure_workspace(c, bytes));
  Work w = carve(c->ws, H, W, D, &bytes, f32, p->interpolate != 0);
  cudaStream_t st = c->stream;
  CBMV_CUDA(cudaEventRecord(c->ev[0], st));
  if (prep) {  // the post's image terms beside the matchers; run_post waits for prep_ev
    RC(ensure_gaussian(c, p->blur_sigma));
    CBMV_CUDA(cudaEventRecord(c->fork_ev, st));
    CBMV_CUDA(cudaStreamWaitEvent(c->side, c->fork_ev, 0));
    RC(post_prep(p, L, R, H, W, w, c->side));
    CBMV_CUDA(cudaEventRecord(c->prep_ev, c->side));
    w.prepped = true;
  }
  RC(launch_census_desc(L, H, W, p->censw, w.descL, st));
  RC(launch_census_desc(R, H, W, p->censw, w.descR, st));
  RC(launch_ncc_stats(L, H, W, p->nccw, w.AL, w.CL, st));
  RC(launch_ncc_stats(R, H, W, p->nccw, w.AR, w.CR, st));
  // the learned path's ZSAD strip kernel (window 5) forms the window means
  // itself, from the column sums it holds anyway
  if (!(f32 && p->sadw == 5)) {
    RC(launch_zsad_means(L, H, W, p->sadw, w.muL, st));
    RC(launch_zsad_means(R, H, W, p->sadw, w.muR, st));
  }
  RC(launch_sobel_i32(L, H, W, w.sobL, st));
  RC(launch_sobel_i32(R, H, W, w.sobR, st));
  if (f32) {
    float* v[4] = {(float*)w.vol[0], (float*)w.vol[1], (float*)w.vol[2], (float*)w.vol[3]};
    RC(launch_census_cost<float>(w.descL, w.descR, H, W, D, p->censw, CBMV_HWD, v[0], st));
    RC(launch_ncc_cost_f32(L, R, w.AL, w.AR, w.CL, w.CR, H, W, D, p->nccw, v[1], st));
    RC(launch_sadsob_cost_f32(w.sobL, w.sobR, H, W, D, p->sobw, v[2], st));
    RC(launch_zsad_cost_f32(L, R, w.muL, w.muR, H, W, D, p->sadw, v[3], st));
    CBMV_CUDA(cudaEventRecord(c->ev[1], st));
    const float* vf[4] = {v[0], v[1], v[2], v[3]};
    RC(launch_feature_stats_f32(vf, H, W, D, w.statsf, st));
    CBMV_CUDA(cudaEventRecord(c->ev[2], st));
    *wout = w;
    return CBMV_OK;
  }
  RC(launch_census_cost<double>(w.descL, w.descR, H, W, D, p->censw, CBMV_HWD, w.vol[0], st));
  RC(launch_ncc_cost<double>(L, R, w.AL, w.AR, w.CL, w.CR, H, W, D, p->nccw, CBMV_HWD, w.vol[1], st));
  RC(launch_sadsob_cost<double>(w.sobL, w.sobR, H, W, D, p->sobw, CBMV_HWD, w.vol[2], st));
  RC(launch_zsad_cost<double>(L, R, w.muL, w.muR, H, W, D, p->sadw, CBMV_HWD, w.vol[3], st));
  CBMV_CUDA(cudaEventRecord(c->ev[1], st));
  const double* vols[4] = {w.vol[0], w.vol[1], w.vol[2], w.vol[3]};
  RC(launch_feature_stats(vols, H, W, D, w.stats, st));
  CBMV_CUDA(cudaEventRecord(c->ev[2], st));
  *wout = w;
  return CBMV_OK;
}

static const cbmv_params* params_or_default(const cbmv_params* p, cbmv_params* def) {
  if (p) return p;
  cbmv_params_default(def);
  return def;
}

extern "C" int cbmv_run_rf(cbmv_ctx* c, const cbmv_forest* f, const cbmv_params* p,
                           const uint8_t* L, const uint8_t* R, int64_t H, int64_t W, int D,
                           float* disp, float* prob0) {
  CBMV_REQUIRE(c && f && L && R && disp, CBMV_EINVAL, "null pointer argument");
  cbmv_params def;
  p = params_or_default(p, &def);
  CBMV_REQUIRE(forest_view(f)->n_features == 20, CBMV_EINVAL, "the forest must take the 20 CBMV features");
  Work w;
  RC(run_front(c, p, L, R, H, W, D, &w, false, true));
  cudaStream_t st = c->stream;
  const double* vols[4] = {w.vol[0], w.vol[1], w.vol[2], w.vol[3]};
  RC(launch_features_rf(vols, w.stats, H, W, D, f, w.volA, st));
  if (prob0)
    CBMV_CUDA(cudaMemcpyAsync(prob0, w.volA, sizeof(float) * H * W * D, cudaMemcpyDeviceToDevice, st));
  CBMV_CUDA(cudaEventRecord(c->ev[3], st));
  RC(run_post(c, p, L, R, H, W, D, w, disp));
  CBMV_CUDA(cudaEventRecord(c->ev[4], st));
  return CBMV_OK;
}

extern "C" int cbmv_run_mlp(cbmv_ctx* c, const cbmv_mlp* m, const cbmv_params* p, const uint8_t* L,
                            const uint8_t* R, int64_t H, int64_t W, int D, float* disp, float* prob0) {
  CBMV_REQUIRE(c && m && L && R && disp, CBMV_EINVAL, "null pointer argument");
  cbmv_params def;
  p = params_or_default(p, &def);
  Work w;
  RC(run_front(c, p, L, R, H, W, D, &w, true, true));
  cudaStream_t st = c->stream;
  const float* vols[4] = {(float*)w.vol[0], (float*)w.vol[1], (float*)w.vol[2], (float*)w.vol[3]};
  RC(launch_features_mlp(vols, w.statsf, H, W, D, m, w.volA, st, p->mlp_ctas));
  if (prob0)
    CBMV_CUDA(cudaMemcpyAsync(prob0, w.volA, sizeof(float) * H * W * D, cudaMemcpyDeviceToDevice, st));
  CBMV_CUDA(cudaEventRecord(c->ev[3], st));
  RC(run_post(c, p, L, R, H, W, D, w, disp));
  CBMV_CUDA(cudaEventRecord(c->ev[4], st));
  return CBMV_OK;
}

// The host-buffer forms: the images are copied into the context's device
// buffers (grown on demand; the previous host-buffer call synchronised the
// stream, so nothing still uses them), the path runs on the context's
// stream, the disparity is copied back and the stream synchronised.
template <class Run>
static int run_host_buffers(cbmv_ctx* c, const uint8_t* L, const uint8_t* R, int64_t H, int64_t W, float* disp,
                            Run run) {
  CBMV_REQUIRE(c && L && R && disp, CBMV_EINVAL, "null pointer argument");
  CBMV_REQUIRE(H > 0 && W > 0, CBMV_EINVAL, "bad size H=%lld W=%lld", (long long)H, (long long)W);
  CBMV_REQUIRE(H <= 65535 && W <= (int64_t(1) << 24), CBMV_ERANGE, "image %lldx%lld: W must be <= 2^24 and H <= 65535",
               (long long)W, (long long)H);
  const size_t HW = (size_t)H * (size_t)W, img = (HW + 255) & ~(size_t)255;
  const size_t need = 2 * img + HW * sizeof(float);
  if (need > c->io_bytes) {
    void* old = c->io;  // forgotten first, so that no error path frees it twice
    c->io = nullptr;
    c->io_bytes = 0;
    if (old) CBMV_CUDA(cudaFree(old));
    void* fresh = nullptr;
    CBMV_CUDA(cudaMalloc(&fresh, need));
    c->io = fresh;
    c->io_bytes = need;
  }
  uint8_t* dL = static_cast<uint8_t*>(c->io);
  uint8_t* dR = dL + img;
  float* dD = reinterpret_cast<float*>(dR + img);
  cudaStream_t st = c->stream;
  CBMV_CUDA(cudaMemcpyAsync(dL, L, HW, cudaMemcpyHostToDevice, st));
  CBMV_CUDA(cudaMemcpyAsync(dR, R, HW, cudaMemcpyHostToDevice, st));
  const int rc = run(dL, dR, dD);
  if (rc == CBMV_OK) CBMV_CUDA(cudaMemcpyAsync(disp, dD, HW * sizeof(float), cudaMemcpyDeviceToHost, st));
  CBMV_CUDA(cudaStreamSynchronize(st));
  return rc;
}

extern "C" int cbmv_run_rf_host(cbmv_ctx* c, const cbmv_forest* f, const cbmv_params* p, const uint8_t* L,
                                const uint8_t* R, int64_t H, int64_t W, int D, float* disp) {
  CBMV_REQUIRE(f, CBMV_EINVAL, "null pointer argument");
  return run_host_buffers(c, L, R, H, W, disp, [&](const uint8_t* dL, const uint8_t* dR, float* dD) {
    return cbmv_run_rf(c, f, p, dL, dR, H, W, D, dD, nullptr);
  });
}

extern "C" int cbmv_run_mlp_host(cbmv_ctx* c, const cbmv_mlp* m, const cbmv_params* p, const uint8_t* L,
                                 const uint8_t* R, int64_t H, int64_t W, int D, float* disp) {
  CBMV_REQUIRE(m, CBMV_EINVAL, "null pointer argument");
  return run_host_buffers(c, L, R, H, W, disp, [&](const uint8_t* dL, const uint8_t* dR, float* dD) {
    return cbmv_run_mlp(c, m, p, dL, dR, H, W, D, dD, nullptr);
  });
}

extern "C" int cbmv_run_post(cbmv_ctx* c, const cbmv_params* p, const uint8_t* L, const uint8_t* R, int64_t H,
                             int64_t W, int D, const float* cost, float* disp) {
  CBMV_REQUIRE(c && L && R && cost && disp, CBMV_EINVAL, "null pointer argument");
  cbmv_params def;
  p = params_or_default(p, &def);
  RC(check_params(p));
  CBMV_REQUIRE(H > p->censw && W > p->censw, CBMV_EINVAL, "image %lldx%lld smaller than the census window",
               (long long)W, (long long)H);
  CBMV_REQUIRE(H <= 65535 && D >= 1 && D <= 1024, CBMV_ERANGE, "H must be <= 65535 and D in 1..1024");
  size_t bytes = 0;
  carve(nullptr, H, W, D, &bytes, true, p->interpolate != 0);
  RC(ensure_workspace(c, bytes));
  Work w = carve(c->ws, H, W, D, &bytes, true, p->interpolate != 0);
  cudaStream_t st = c->stream;
  for (int i = 0; i < 4; i++) CBMV_CUDA(cudaEventRecord(c->ev[i], st));
  CBMV_CUDA(cudaMemcpyAsync(w.volA, cost, sizeof(float) * H * W * D, cudaMemcpyDeviceToDevice, st));
  RC(run_post(c, p, L, R, H, W, D, w, disp));
  CBMV_CUDA(cudaEventRecord(c->ev[4], st));
  return CBMV_OK;
}

extern "C" int cbmv_ctx_volumes_f32(cbmv_ctx* c, const cbmv_params* p, const uint8_t* L, const uint8_t* R,
                                    int64_t H, int64_t W, int D, float* out) {
  CBMV_REQUIRE(c && L && R && out, CBMV_EINVAL, "null pointer argument");
  cbmv_params def;
  p = params_or_default(p, &def);
  Work w;
  RC(run_front(c, p, L, R, H, W, D, &w, true));
  const size_t V = (size_t)H * W * D;
  for (int m = 0; m < 4; m++)
    CBMV_CUDA(cudaMemcpyAsync(out + m * V, w.vol[m], sizeof(float) * V, cudaMemcpyDeviceToDevice, c->stream));
  return CBMV_OK;
}

extern "C" int cbmv_ctx_features_at(cbmv_ctx* c, const cbmv_params* p, const uint8_t* L,
                                    const uint8_t* R, int64_t H, int64_t W, int D, const int64_t* idx,
                                    int64_t n, float* out) {
  CBMV_REQUIRE(c && L && R && idx && out, CBMV_EINVAL, "null pointer argument");
  CBMV_REQUIRE(n > 0, CBMV_EINVAL, "n must be positive");
  cbmv_params def;
  p = params_or_default(p, &def);
  Work w;
  RC(run_front(c, p, L, R, H, W, D, &w));
  const double* vols[4] = {w.vol[0], w.vol[1], w.vol[2], w.vol[3]};
  return launch_features_gather(vols, w.stats, H, W, D, idx, n, out, c->stream);
}

extern "C" int cbmv_ctx_features_f32_at(cbmv_ctx* c, const cbmv_params* p, const uint8_t* L,
                                        const uint8_t* R, int64_t H, int64_t W, int D, const int64_t* idx,
                                        int64_t n, float* out) {
  CBMV_REQUIRE(c && L && R && idx && out, CBMV_EINVAL, "null pointer argument");
  CBMV_REQUIRE(n > 0, CBMV_EINVAL, "n must be positive");
  cbmv_params def;
  p = params_or_default(p, &def);
  Work w;
  RC(run_front(c, p, L, R, H, W, D, &w, true));
  const float* vols[4] = {(float*)w.vol[0], (float*)w.vol[1], (float*)w.vol[2], (float*)w.vol[3]};
  return launch_features_f32_gather(vols, w.statsf, H, W, D, idx, n, out, c->stream);
}

// ====================================================================
// Batches: many pairs of uneven size in one CUDA graph launch.
// ====================================================================
struct cbmv_batch {
  int n = 0;
  std::vector<int64_t> H, W;
  std::vector<int> D;
  std::vector<std::vector<int>> order;  // context -> its pairs, in run order
  std::vector<cudaStream_t> streams;
  std::vector<cbmv_ctx*> ctx;
  cudaEvent_t fork = nullptr, t0 = nullptr;
  std::vector<cudaEvent_t> ev_start, ev_end, join;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // what the graph was captured with
  std::vector<const uint8_t*> L, R;
  std::vector<float*> disp;
  const cbmv_mlp* net = nullptr;
  cbmv_params params{};
  // the graph is captured on and launched into the batch's own stream (the
  // caller's may be the legacy default stream, which cannot be captured),
  // ordered after and before the caller's stream by events
  cudaStream_t origin = nullptr;
  cudaEvent_t in_ev = nullptr, out_ev = nullptr;
};

static void batch_free(cbmv_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (cbmv_ctx* c : b->ctx) cbmv_ctx_destroy(c);
  for (cudaStream_t s : b->streams) cudaStreamDestroy(s);
  for (cudaEvent_t e : b->ev_start) cudaEventDestroy(e);
  for (cudaEvent_t e : b->ev_end) cudaEventDestroy(e);
  for (cudaEvent_t e : b->join) cudaEventDestroy(e);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->t0) cudaEventDestroy(b->t0);
  if (b->in_ev) cudaEventDestroy(b->in_ev);
  if (b->out_ev) cudaEventDestroy(b->out_ev);
  if (b->origin) cudaStreamDestroy(b->origin);
  delete b;
}

extern "C" int cbmv_batch_create(int n, const int64_t* H, const int64_t* W, const int* D, int streams,
                                 cbmv_batch** out) {
  CBMV_REQUIRE(out && H && W && D, CBMV_EINVAL, "null pointer argument");
  CBMV_REQUIRE(n >= 1 && n <= 4096, CBMV_EINVAL, "batch of %d pairs (1..4096)", n);
  CBMV_REQUIRE(streams >= 1 && streams <= 32, CBMV_EINVAL, "streams must be in 1..32");
  for (int i = 0; i < n; i++)
    CBMV_REQUIRE(H[i] > 11 && W[i] > 11 && H[i] <= 65535 && D[i] >= 1 && D[i] <= 1024, CBMV_EINVAL,
                 "pair %d: bad shape %lldx%lld, D=%d", i, (long long)W[i], (long long)H[i], D[i]);
  cbmv_batch* b = new cbmv_batch();
  b->n = n;
  b->H.assign(H, H + n);
  b->W.assign(W, W + n);
  b->D.assign(D, D + n);
  const int K = std::min(streams, n);
  // longest first onto the least-loaded context
  std::vector<int> idx(n);
  for (int i = 0; i < n; i++) idx[i] = i;
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int c) {
    return H[a] * W[a] * D[a] > H[c] * W[c] * D[c];
  });
  std::vector<double> load(K, 0.0);
  b->order.resize(K);
  for (int i : idx) {
    const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    b->order[k].push_back(i);
    load[k] += (double)H[i] * W[i] * D[i];
  }
  int rc = CBMV_OK;
  auto fail = [&](int code) {
    batch_free(b);
    return code;
  };
  for (int k = 0; k < K; k++) {
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
      return fail(set_error(CBMV_ECUDA, "cudaStreamCreate failed"));
    b->streams.push_back(s);
    cbmv_ctx* c = nullptr;
    if ((rc = cbmv_ctx_create(s, &c))) return fail(rc);
    b->ctx.push_back(c);
    size_t need = 0;
    for (int i : b->order[k]) {
      size_t bytes = 0;
      carve(nullptr, H[i], W[i], D[i], &bytes, true, false);
      need = std::max(need, bytes);
    }
    if ((rc = ensure_workspace(c, need))) return fail(rc);
  }
  b->ev_start.resize(n);
  b->ev_end.resize(n);
  b->join.resize(K);
  bool ok = cudaEventCreate(&b->fork) == cudaSuccess && cudaEventCreate(&b->t0) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->in_ev, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->out_ev, cudaEventDisableTiming) == cudaSuccess &&
            cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking) == cudaSuccess;
  for (int i = 0; i < n && ok; i++)
    ok = cudaEventCreate(&b->ev_start[i]) == cudaSuccess && cudaEventCreate(&b->ev_end[i]) == cudaSuccess;
  for (int k = 0; k < K && ok; k++) ok = cudaEventCreate(&b->join[k]) == cudaSuccess;
  if (!ok) return fail(set_error(CBMV_ECUDA, "cudaEventCreate failed"));
  *out = b;
  return CBMV_OK;
}

extern "C" int cbmv_batch_destroy(cbmv_batch* b) {
  if (!b) return CBMV_OK;
  if (b->origin) cudaStreamSynchronize(b->origin);
  for (cudaStream_t s : b->streams) cudaStreamSynchronize(s);
  batch_free(b);
  return CBMV_OK;
}

static int batch_capture(cbmv_batch* b, const cbmv_mlp* m, const cbmv_params* p) {
  const int K = (int)b->ctx.size();
  cudaStream_t origin = b->origin;
  for (int k = 0; k < K; k++) RC(ensure_gaussian(b->ctx[k], p->blur_sigma));  // may allocate: before capture
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (b->graph) {
    cudaGraphDestroy(b->graph);
    b->graph = nullptr;
  }
  CBMV_CUDA(cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal));
  int rc = CBMV_OK;
  cudaError_t e = cudaEventRecord(b->fork, origin);
  if (e == cudaSuccess) e = cudaEventRecordWithFlags(b->t0, origin, cudaEventRecordExternal);
  for (int k = 0; k < K && e == cudaSuccess; k++) e = cudaStreamWaitEvent(b->streams[k], b->fork, 0);
  for (int k = 0; k < K && e == cudaSuccess && rc == CBMV_OK; k++) {
    for (int i : b->order[k]) {
      e = cudaEventRecordWithFlags(b->ev_start[i], b->streams[k], cudaEventRecordExternal);
      if (e != cudaSuccess) break;
      rc = cbmv_run_mlp(b->ctx[k], m, p, b->L[i], b->R[i], b->H[i], b->W[i], b->D[i], b->disp[i], nullptr);
      if (rc != CBMV_OK) break;
      e = cudaEventRecordWithFlags(b->ev_end[i], b->streams[k], cudaEventRecordExternal);
      if (e != cudaSuccess) break;
    }
    if (e == cudaSuccess && rc == CBMV_OK) e = cudaEventRecord(b->join[k], b->streams[k]);
    if (e == cudaSuccess && rc == CBMV_OK) e = cudaStreamWaitEvent(origin, b->join[k], 0);
  }
  cudaGraph_t g = nullptr;
  const cudaError_t e_end = cudaStreamEndCapture(origin, &g);  // always end, so the stream is usable again
  if (rc != CBMV_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess || e_end != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return set_error(CBMV_ECUDA, "batch graph capture: %s",
                     cudaGetErrorString(e != cudaSuccess ? e : e_end));
  }
  b->graph = g;
  CBMV_CUDA(cudaGraphInstantiate(&b->exec, g, 0));
  b->net = m;
  b->params = *p;
  return CBMV_OK;
}

extern "C" int cbmv_batch_run_mlp(cbmv_batch* b, const cbmv_mlp* m, const cbmv_params* p, const uint8_t* const* L,
                                  const uint8_t* const* R, float* const* disp, void* stream) {
  CBMV_REQUIRE(b && m && L && R && disp, CBMV_EINVAL, "null pointer argument");
  cbmv_params def;
  p = params_or_default(p, &def);
  RC(check_params(p));
  CBMV_REQUIRE(p->interpolate == 0, CBMV_EINVAL, "batches run the _mem post (interpolate = 0)");
  for (int i = 0; i < b->n; i++) CBMV_REQUIRE(L[i] && R[i] && disp[i], CBMV_EINVAL, "pair %d: null pointer", i);
  cudaStream_t user = as_stream(stream);
  bool same = b->exec && b->net == m && memcmp(&b->params, p, sizeof(cbmv_params)) == 0;
  for (int i = 0; i < b->n && same; i++) same = b->L[i] == L[i] && b->R[i] == R[i] && b->disp[i] == disp[i];
  if (!same) {
    b->L.assign(L, L + b->n);
    b->R.assign(R, R + b->n);
    b->disp.assign(disp, disp + b->n);
    RC(batch_capture(b, m, p));
  }
  CBMV_CUDA(cudaEventRecord(b->in_ev, user));
  CBMV_CUDA(cudaStreamWaitEvent(b->origin, b->in_ev, 0));
  CBMV_CUDA(cudaGraphLaunch(b->exec, b->origin));
  CBMV_CUDA(cudaEventRecord(b->out_ev, b->origin));
  CBMV_CUDA(cudaStreamWaitEvent(user, b->out_ev, 0));
  return CBMV_OK;
}

extern "C" int cbmv_batch_timings(cbmv_batch* b, float* pair_ms, float* done_ms, float* total_ms) {
  CBMV_REQUIRE(b && pair_ms && done_ms && total_ms, CBMV_EINVAL, "null pointer argument");
  CBMV_REQUIRE(b->exec, CBMV_ESTATE, "the batch has not run");
  float total = 0.0f;
  for (int i = 0; i < b->n; i++) {
    CBMV_CUDA(cudaEventSynchronize(b->ev_end[i]));
    CBMV_CUDA(cudaEventElapsedTime(&pair_ms[i], b->ev_start[i], b->ev_end[i]));
    CBMV_CUDA(cudaEventElapsedTime(&done_ms[i], b->t0, b->ev_end[i]));
    total = std::max(total, done_ms[i]);
  }
  *total_ms = total;
  return CBMV_OK;
}
