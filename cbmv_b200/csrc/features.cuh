// Device-side construction of the 20 CBMV features of one (pixel, d), shared
// by the feature kernels (featextract.cu) and the fused classifier kernels
// (classify.cu).
#pragma once
#include "common.cuh"

namespace cbmv {

// Per-matcher constants of the reference's feature extraction:
// ratio epsilon (test.py:548-551) and likelihood sigma (test.py:71-73).
static __constant__ double kEps[4] = {0.01, 1.01, 0.01, 0.01};
static __constant__ double kSigma[4] = {2.0 * 8 * 8, 0.02, 2.0 * 100 * 100, 2.0 * 100 * 100};
static const double hSigma[4] = {2.0 * 8 * 8, 0.02, 2.0 * 100 * 100, 2.0 * 100 * 100};

// ratio / likelihood of cost c against the statistics (min, den) of its row
// (featextract.cpp:333, :440).
__device__ __forceinline__ void confidences(double c, double mn, double den, double e, double sigma,
                                            float* ratio, float* lik) {
  if (mn == kRandMax) {
    *ratio = 0.0f;
    *lik = 0.0f;
  } else {
    *ratio = (float)((mn + e) / (c + e));
    const double t = c - mn;
    *lik = (float)(exp(-((t * t) / sigma)) / den);
  }
}

// The 20 features of (p, d) in the reference's column order.  The right-
// reference confidences at left (x, d) are those of right pixel x - d at
// disparity d, whose cost is C[p, d] itself; for x < d get_left_cost fills
// with the first element of the right-view feature volume, which is 0 (the
// right view's pixel (row, 0) has only sentinel costs).
__device__ __forceinline__ void features_at(const double* const* vols, const double* stats,
                                            int64_t HW, int64_t W, int D, int64_t p, int64_t x,
                                            int d, float* f) {
#pragma unroll
  for (int m = 0; m < 4; m++) {
    const double c = vols[m][p * D + d];
    f[m] = (float)c;
    const double* sl = stats + ((int64_t)(m * 2 + 0) * HW + p) * 2;
    confidences(c, sl[0], sl[1], kEps[m], kSigma[m], &f[4 + m], &f[8 + m]);
    if (x >= d) {
      const double* sr = stats + ((int64_t)(m * 2 + 1) * HW + (p - d)) * 2;
      confidences(c, sr[0], sr[1], kEps[m], kSigma[m], &f[12 + m], &f[16 + m]);
    } else {
      f[12 + m] = 0.0f;
      f[16 + m] = 0.0f;
    }
  }
}

// The same features written to f[k * stride] (a thread's column of a
// shared-memory feature tile); the matcher loop is kept rolled so the float64
// temporaries of one matcher are live at a time.
__device__ __forceinline__ void features_store(const double* const* vols, const double* stats,
                                               int64_t HW, int D, int64_t p, int64_t x, int d,
                                               float* f, int stride) {
#pragma unroll 1
  for (int m = 0; m < 4; m++) {
    const double c = vols[m][p * D + d];
    float r, l;
    f[m * stride] = (float)c;
    const double* sl = stats + ((int64_t)(m * 2 + 0) * HW + p) * 2;
    confidences(c, sl[0], sl[1], kEps[m], kSigma[m], &r, &l);
    f[(4 + m) * stride] = r;
    f[(8 + m) * stride] = l;
    if (x >= d) {
      const double* sr = stats + ((int64_t)(m * 2 + 1) * HW + (p - d)) * 2;
      confidences(c, sr[0], sr[1], kEps[m], kSigma[m], &r, &l);
    } else {
      r = 0.0f;
      l = 0.0f;
    }
    f[(12 + m) * stride] = r;
    f[(16 + m) * stride] = l;
  }
}

// The features of matchers m0 and m0+1 only: f[2g + i] is feature group g
// (0 cost, 1 ratio, 2 likelihood, 3 right ratio, 4 right likelihood) of
// matcher m0 + i, i.e. reference column 4g + m0 + i.
__device__ __forceinline__ void features_pair(const double* const* vols, const double* stats,
                                              int64_t HW, int D, int64_t p, int64_t x, int d, int m0,
                                              float* f) {
#pragma unroll
  for (int i = 0; i < 2; i++) {
    const int m = m0 + i;
    const double c = vols[m][p * D + d];
    float r, l;
    f[i] = (float)c;
    const double* sl = stats + ((int64_t)(m * 2 + 0) * HW + p) * 2;
    confidences(c, sl[0], sl[1], kEps[m], kSigma[m], &r, &l);
    f[2 + i] = r;
    f[4 + i] = l;
    if (x >= d) {
      const double* sr = stats + ((int64_t)(m * 2 + 1) * HW + (p - d)) * 2;
      confidences(c, sr[0], sr[1], kEps[m], kSigma[m], &r, &l);
    } else {
      r = 0.0f;
      l = 0.0f;
    }
    f[6 + i] = r;
    f[8 + i] = l;
  }
}

struct FeatVols {
  const double* v[4];
};


}  // namespace cbmv
