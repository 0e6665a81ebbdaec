/*
 * oracle.c -- CPU restatement of the CBMV cost-volume path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the CUDA path is
 * compared against (tests/, __graft_entry__.smoke(), bench.py's CPU leg); it
 * is never linked into the product.  Each function restates one reference
 * function, named in its comment by file:line, with the same loop bounds,
 * sentinels, and floating-point types and operation order, so that its
 * results equal the reference's bit for bit.  That claim is itself checked
 * against the reference compiled unmodified (oracle/_ref, tests/golden).
 *
 * Conventions: images are row-major [H,W]; "HWD" volumes are [H,W,D] with d
 * fastest, "DHW" volumes are [D,H,W].  Every parallel loop writes disjoint
 * outputs with a sequential inner loop, so results do not depend on the
 * thread count.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define RAND_MAX_D 2147483647.0 /* glibc RAND_MAX, the reference's sentinel */

typedef long long i64;

/* ------------------------------------------------------------------ */
/* matchers (cpp/matchers/matchers.cpp)                                */
/* ------------------------------------------------------------------ */

/* census: matchers.cpp:209-350.  Descriptor bit k of pixel p is
 * (center < neighbour_k) over the w*w window in row-major order (int16
 * compare, _mm_cmplt_epi16 at :292-293); descriptors exist for rows/cols
 * (i+wc, j+wc), i < H-w, j < W-w.  Cost = number of differing bits for
 * d < min(D, j+1) (:315), stored at (i+wc, j+wc, d) of an [H,W,D] volume
 * prefilled with RAND_MAX (:229). */
void orc_census(const uint8_t* L, const uint8_t* R, i64 H, i64 W, int D, int w, double* out) {
  const int wc = w / 2;
  const i64 n = H * W * (i64)D;
  for (i64 k = 0; k < n; k++) out[k] = RAND_MAX_D;
  if (H <= w || W <= w) return;
#pragma omp parallel for schedule(static)
  for (i64 i = 0; i < H - w; i++) {
    for (i64 j = 0; j < W - w; j++) {
      const int end = D < (int)(j + 1) ? D : (int)(j + 1);
      const int cl = L[(i + wc) * W + (j + wc)];
      for (int d = 0; d < end; d++) {
        const int cr = R[(i + wc) * W + (j - d + wc)];
        int diff = 0;
        for (int wh = 0; wh < w; wh++)
          for (int ww = 0; ww < w; ww++) {
            const int bl = cl < L[(i + wh) * W + (j + ww)];
            const int br = cr < R[(i + wh) * W + (j - d + ww)];
            diff += bl != br;
          }
        out[((i + wc) * W + (j + wc)) * D + d] = (double)diff;
      }
    }
  }
}

/* nccNister: matchers.cpp:24-205.  With A = sum I, B = sum I^2 over the
 * w*w window (exact integers, :121-124), C = 1/sqrt(w^2 B - A^2) in double
 * (:127-128) and S = sum L*R(j-d) (an exact integer; the reference gets it
 * from a double integral image, :137-176):
 *   cost = -(double)(w^2 S - A_L A_R) * C_L * C_R        (:179)
 * or 1 when either C is not finite (flat window, :181).  Valid at rows i+wc,
 * i < H-w, cols j+wc, d <= j < W-w; elsewhere RAND_MAX.  Output [D,H,W]. */
void orc_ncc(const uint8_t* L, const uint8_t* R, i64 H, i64 W, int D, int w, double* out) {
  const int wc = w / 2;
  const int sq = w * w;
  const i64 HW = H * W;
  for (i64 k = 0; k < HW * D; k++) out[k] = RAND_MAX_D;
  if (H <= w || W <= w) return;
  uint64_t* Al = (uint64_t*)calloc(HW, sizeof(uint64_t));
  uint64_t* Ar = (uint64_t*)calloc(HW, sizeof(uint64_t));
  double* Cl = (double*)calloc(HW, sizeof(double));
  double* Cr = (double*)calloc(HW, sizeof(double));
#pragma omp parallel for schedule(static)
  for (i64 i = 0; i < H - w; i++) {
    for (i64 j = 0; j < W - w; j++) {
      uint64_t al = 0, ar = 0, bl = 0, br = 0;
      for (int wh = 0; wh < w; wh++)
        for (int ww = 0; ww < w; ww++) {
          const uint64_t l = L[(i + wh) * W + j + ww], r = R[(i + wh) * W + j + ww];
          al += l; ar += r; bl += l * l; br += r * r;
        }
      const i64 p = (i + wc) * W + (j + wc);
      Al[p] = al; Ar[p] = ar;
      Cl[p] = 1 / (sqrt(sq * bl - (double)(al) * (al)));
      Cr[p] = 1 / (sqrt(sq * br - (double)(ar) * (ar)));
    }
  }
#pragma omp parallel for schedule(static)
  for (int d = 0; d < D; d++) {
    for (i64 i = 0; i < H - w; i++) {
      const i64 row = (i + wc) * W;
      for (i64 j = d; j < W - w; j++) {
        uint64_t s = 0;
        for (int wh = 0; wh < w; wh++)
          for (int ww = 0; ww < w; ww++)
            s += (uint64_t)L[(i + wh) * W + j + ww] * R[(i + wh) * W + j + ww - d];
        const double lD = (double)s;
        const i64 pl = row + j + wc, pr = row + (j - d + wc);
        double v;
        if (isfinite(Cl[pl]) && isfinite(Cr[pr]))
          v = -(double)(sq * lD - Al[pl] * Ar[pr]) * Cl[pl] * Cr[pr];
        else
          v = 1;
        out[(i64)d * HW + pl] = v;
      }
    }
  }
  free(Al); free(Ar); free(Cl); free(Cr);
}

/* sobel: matchers.cpp:515-555.  Horizontal kernel [-1 0 1; -2 0 2; -1 0 1]
 * in int arithmetic, written at (i+1, j+1) for i < H-3, j < W-3 (so the last
 * two rows and columns stay 0). */
void orc_sobel(const uint8_t* I, i64 H, i64 W, double* out) {
  for (i64 k = 0; k < H * W; k++) out[k] = 0;
#pragma omp parallel for schedule(static)
  for (i64 i = 0; i < H - 3; i++)
    for (i64 j = 0; j < W - 3; j++) {
      const uint8_t* a = I + i * W + j;
      const int v = -a[0] + a[2] - 2 * a[W] + 2 * a[W + 2] - a[2 * W] + a[2 * W + 2];
      out[(i + 1) * W + (j + 1)] = (double)v;
    }
}

/* sadsob: matchers.cpp:353-436.  Per d, the w*w box sum of |SL(j) - SR(j-d)|
 * for box columns j >= d (the reference's integral image holds exact
 * integers, :389-421), stored at (i+wc, j+wc) for i < H-w, d <= j < W-w of a
 * [D,H,W] volume prefilled with RAND_MAX (:374).  Inputs are the Sobel
 * responses (doubles holding integers). */
void orc_sadsob(const double* SL, const double* SR, i64 H, i64 W, int D, int w, double* out) {
  const int wc = w / 2;
  const i64 HW = H * W;
  for (i64 k = 0; k < HW * D; k++) out[k] = RAND_MAX_D;
  if (H <= w || W <= w) return;
#pragma omp parallel for schedule(static)
  for (int d = 0; d < D; d++)
    for (i64 i = 0; i < H - w; i++)
      for (i64 j = d; j < W - w; j++) {
        double s = 0;
        for (int wh = 0; wh < w; wh++)
          for (int ww = 0; ww < w; ww++)
            s += fabs(SL[(i + wh) * W + j + ww] - SR[(i + wh) * W + j + ww - d]);
        out[(i64)d * HW + (i + wc) * W + (j + wc)] = s;
      }
}

/* zsad: matchers.cpp:440-512.  Window means in double (:474-482), then
 * cost = sum_{wh,ww} fabs(L - muL - R(j-d) + muR(j-d)), accumulated in
 * double in wh-major order (:499-505), for i < H-w, d <= j < W-w; output
 * [D,H,W] prefilled with RAND_MAX (:460). */
void orc_zsad(const uint8_t* L, const uint8_t* R, i64 H, i64 W, int D, int w, double* out) {
  const int wc = w / 2;
  const int sq = w * w;
  const i64 HW = H * W;
  for (i64 k = 0; k < HW * D; k++) out[k] = RAND_MAX_D;
  if (H <= w || W <= w) return;
  double* ml = (double*)calloc(HW, sizeof(double));
  double* mr = (double*)calloc(HW, sizeof(double));
#pragma omp parallel for schedule(static)
  for (i64 i = 0; i < H - w; i++)
    for (i64 j = 0; j < W - w; j++) {
      double a = 0, b = 0;
      for (int wh = 0; wh < w; wh++)
        for (int ww = 0; ww < w; ww++) {
          a += L[(i + wh) * W + (j + ww)];
          b += R[(i + wh) * W + (j + ww)];
        }
      ml[(i + wc) * W + (j + wc)] = a / sq;
      mr[(i + wc) * W + (j + wc)] = b / sq;
    }
#pragma omp parallel for schedule(static)
  for (int d = 0; d < D; d++)
    for (i64 i = 0; i < H - w; i++)
      for (i64 j = d; j < W - w; j++) {
        const double mul = ml[(i + wc) * W + (j + wc)];
        const double mur = mr[(i + wc) * W + (j - d + wc)];
        double s = 0;
        for (int wh = 0; wh < w; wh++)
          for (int ww = 0; ww < w; ww++)
            s += fabs(L[(i + wh) * W + (j + ww)] - mul - R[(i + wh) * W + (j - d + ww)] + mur);
        out[(i64)d * HW + (i + wc) * W + (j + wc)] = s;
      }
  free(ml); free(mr);
}

/* ------------------------------------------------------------------ */
/* feature extraction (cpp/featextract/featextract.cpp)                */
/* ------------------------------------------------------------------ */

/* swap_axes: featextract.cpp:24-53, [D,H,W] -> [H,W,D]. */
void orc_swap_axes(const double* in, i64 D, i64 H, i64 W, double* out) {
#pragma omp parallel for schedule(static)
  for (i64 p = 0; p < H * W; p++)
    for (i64 d = 0; d < D; d++) out[p * D + d] = in[d * H * W + p];
}

/* swap_axes_back: featextract.cpp:55-83, [H,W,D] -> [D,H,W]. */
void orc_swap_axes_back(const double* in, i64 H, i64 W, i64 D, double* out) {
#pragma omp parallel for schedule(static)
  for (i64 p = 0; p < H * W; p++)
    for (i64 d = 0; d < D; d++) out[d * H * W + p] = in[p * D + d];
}

/* get_cost: featextract.cpp:85-113, [H,W,D,K] -> [H,W,D] taking k = 0. */
void orc_get_cost(const double* in, i64 H, i64 W, i64 D, i64 K, double* out) {
#pragma omp parallel for schedule(static)
  for (i64 p = 0; p < H * W; p++)
    for (i64 d = 0; d < D; d++) out[p * D + d] = in[(p * D + d) * K];
}

/* get_right_cost: featextract.cpp:115-152.  R[i,j,d] = C[i,j+d,d] for
 * j < W-d, else C[0,0,0] (:130). */
void orc_get_right_cost(const double* C, i64 H, i64 W, i64 D, double* out) {
  const double fill = C[0];
#pragma omp parallel for schedule(static)
  for (i64 i = 0; i < H; i++)
    for (i64 j = 0; j < W; j++)
      for (i64 d = 0; d < D; d++)
        out[(i * W + j) * D + d] = (j < W - d) ? C[(i * W + j + d) * D + d] : fill;
}

/* get_left_cost_from_right: featextract.cpp:452-488.  L[i,j,d] = R[i,j-d,d]
 * for j >= d, else R[0,0,0] (:467). */
void orc_get_left_cost(const double* Rv, i64 H, i64 W, i64 D, double* out) {
  const double fill = Rv[0];
#pragma omp parallel for schedule(static)
  for (i64 i = 0; i < H; i++)
    for (i64 j = 0; j < W; j++)
      for (i64 d = 0; d < D; d++)
        out[(i * W + j) * D + d] = (j >= d) ? Rv[(i * W + j - d) * D + d] : fill;
}

/* Row minimum as in featextract.cpp:322-329: start at RAND_MAX, strict <. */
static double row_min(const double* v, i64 n) {
  double m = RAND_MAX_D;
  for (i64 k = 0; k < n; k++)
    if (v[k] < m) m = v[k];
  return m;
}

/* extract_pkrn_test: featextract.cpp:303-342.  Per row of an [N,D] volume,
 * r = (m+e)/(c+e) with m the row minimum; 0 when m == RAND_MAX. */
void orc_extract_ratio(const double* v, i64 N, i64 D, double e, double* out) {
#pragma omp parallel for schedule(static)
  for (i64 i = 0; i < N; i++) {
    const double* r = v + i * D;
    const double m = row_min(r, D);
    for (i64 j = 0; j < D; j++) out[i * D + j] = (m == RAND_MAX_D) ? 0.0 : (m + e) / (r[j] + e);
  }
}

/* extract_aml_testing: featextract.cpp:402-450.  Per row,
 * exp(-(c-m)^2/s) / sum_k exp(-(c_k-m)^2/s), the sum taken in k order
 * (:432-435); 0 when m == RAND_MAX. */
void orc_extract_likelihood(const double* v, i64 N, i64 D, double sigma, double* out) {
#pragma omp parallel for schedule(static)
  for (i64 i = 0; i < N; i++) {
    const double* r = v + i * D;
    const double m = row_min(r, D);
    double denom = 0, num = 0;
    for (i64 k = 0; k < D; k++) {
      num = r[k] - m;
      denom += exp(-(num * num) / sigma);
    }
    for (i64 j = 0; j < D; j++) {
      const double t = r[j] - m;
      out[i * D + j] = (m == RAND_MAX_D) ? 0.0 : exp(-((t * t) / sigma)) / denom;
    }
  }
}

/* extract_pkrn (training form): featextract.cpp:254-300.  Rows of an [N,D]
 * volume, three sampled disparities per row (samples [N,3] int32). */
void orc_extract_ratio_samples(const double* v, i64 N, i64 D, const int32_t* s, double e,
                               double* out) {
#pragma omp parallel for schedule(static)
  for (i64 i = 0; i < N; i++) {
    const double* r = v + i * D;
    const double m = row_min(r, D);
    for (int k = 0; k < 3; k++)
      out[3 * i + k] = (m == RAND_MAX_D) ? 0.0 : (m + e) / (r[s[3 * i + k]] + e);
  }
}

/* extract_aml (training form): featextract.cpp:345-399. */
void orc_extract_likelihood_samples(const double* v, i64 N, i64 D, const int32_t* s, double sigma,
                                    double* out) {
#pragma omp parallel for schedule(static)
  for (i64 i = 0; i < N; i++) {
    const double* r = v + i * D;
    const double m = row_min(r, D);
    double denom = 0, num = 0;
    for (i64 k = 0; k < D; k++) {
      num = r[k] - m;
      denom += exp(-(num * num) / sigma);
    }
    for (int k = 0; k < 3; k++) {
      const double t = r[s[3 * i + k]] - m;
      out[3 * i + k] = (m == RAND_MAX_D) ? 0.0 : exp(-((t * t) / sigma)) / denom;
    }
  }
}

/* get_samples: featextract.cpp:217-252. */
void orc_get_samples(const double* v, i64 N, i64 D, const int32_t* s, double* out) {
#pragma omp parallel for schedule(static)
  for (i64 i = 0; i < N; i++)
    for (int k = 0; k < 3; k++) out[3 * i + k] = v[i * D + s[3 * i + k]];
}

/* generate_labels: featextract.cpp:490-516, [1,0,0] per sample row. */
void orc_generate_labels(i64 N, int32_t* out) {
  for (i64 i = 0; i < N; i++) {
    out[3 * i] = 1; out[3 * i + 1] = 0; out[3 * i + 2] = 0;
  }
}

/* Counter-based draw in [0, n): splitmix64 of (seed, sample, slot). */
static uint32_t draw(uint64_t seed, i64 s, int slot, uint32_t n) {
  uint64_t z = seed * 0x9E3779B97F4A7C15ull + (uint64_t)s * 3ull + (uint64_t)slot + 1;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (uint32_t)(z % n);
}

/* generate_d_indices: featextract.cpp:154-215.  Per sample: the ground
 * truth, then two negatives, each drawn below gt-thr when gt-thr > 0 and
 * otherwise above gt+thr (and the mirror for the second draw), with the same
 * ranges as :187-206.  The reference draws with rand() inside an OpenMP loop,
 * which is not reproducible; this restatement draws from a counter-based
 * generator keyed by (seed, sample, slot), which the CUDA sampler shares.
 * Returns -1 when a range is empty (the reference would divide by zero,
 * :199/:202, when gt+thr+1 >= maxd and gt-thr <= 0). */
int orc_generate_d_indices(const int32_t* gt, i64 N, int maxd, int thr, uint64_t seed, int32_t* out) {
  int bad = 0;
  for (i64 s = 0; s < N; s++) {
    const int g = gt[s];
    const int low = !(g - thr <= 0);
    const int high = !(g + thr >= maxd);
    const int lo_n = g - thr;
    const int hi_n = maxd - (g + thr + 1);
    int d1, d2;
    if (low) d1 = lo_n > 0 ? (int)draw(seed, s, 0, (uint32_t)lo_n) : 0;
    else d1 = hi_n > 0 ? (int)draw(seed, s, 0, (uint32_t)hi_n) + (g + thr + 1) : (bad = 1, 0);
    if (high) d2 = hi_n > 0 ? (int)draw(seed, s, 1, (uint32_t)hi_n) + (g + thr + 1) : (bad = 1, 0);
    else d2 = lo_n > 0 ? (int)draw(seed, s, 1, (uint32_t)lo_n) : (bad = 1, 0);
    out[3 * s] = g; out[3 * s + 1] = d1; out[3 * s + 2] = d2;
  }
  return bad ? -1 : 0;
}

/* ------------------------------------------------------------------ */
/* random forest (sklearn RandomForestClassifier.predict_proba, called */
/* at test.py:620; tree walk sklearn/tree/_tree.pyx:954-996)           */
/* ------------------------------------------------------------------ */

/* Flat forest: node k of tree t at offset roots[t]+k; left[] < 0 marks a
 * leaf.  X is float32 [N,F] (sklearn casts to float32 before the walk);
 * the test is x <= threshold with threshold in double, as in _tree.pyx:989.
 * p0[n] = (sum over trees, in tree order, of the leaf's class-0 fraction)
 * / T, accumulated in double (forest.py:951-962 with one job).  leaves, if
 * not NULL, receives the local leaf index per (sample, tree). */
void orc_rf_predict(const int32_t* roots, int T, const int32_t* feature, const double* threshold,
                    const int32_t* left, const int32_t* right, const double* value0,
                    const float* X, i64 N, int F, double* p0, int32_t* leaves) {
#pragma omp parallel for schedule(static)
  for (i64 n = 0; n < N; n++) {
    const float* x = X + n * F;
    double acc = 0.0;
    for (int t = 0; t < T; t++) {
      const i64 base = roots[t];
      i64 k = 0;
      while (left[base + k] >= 0) {
        const float v = x[feature[base + k]];
        k = ((double)v <= threshold[base + k]) ? left[base + k] : right[base + k];
      }
      acc += value0[base + k];
      if (leaves) leaves[n * T + t] = (int32_t)k;
    }
    p0[n] = acc / T;
  }
}

/* ------------------------------------------------------------------ */
/* cost optimisation (cpp/post/post.cu), restated on the CPU in the    */
/* reference kernels' own mixed float/double arithmetic                */
/* ------------------------------------------------------------------ */

/* cross: post.cu:336-396.  out [4,H,W] float: arm end coordinate for
 * directions -x, +x, -y, +y. */
void orc_cross(const float* x0, i64 H, i64 W, int L1, float tau1, float* out) {
#pragma omp parallel for schedule(static)
  for (i64 id = 0; id < 4 * H * W; id++) {
    const i64 x = id % W, y = (id / W) % H, dir = id / (W * H);
    const int dx = dir == 0 ? -1 : dir == 1 ? 1 : 0;
    const int dy = dir == 2 ? -1 : dir == 3 ? 1 : 0;
    const i64 ind1 = y * W + x;
    i64 xx = x + dx, yy = y + dy;
    for (;; xx += dx, yy += dy) {
      if (xx < 0 || xx >= W || yy < 0 || yy >= H) break;
      const i64 ax = llabs(xx - x), ay = llabs(yy - y);
      const i64 dist = ax > ay ? ax : ay;
      if (dist == 1) continue;
      const i64 ind2 = yy * W + xx;
      if (fabsf(x0[ind1] - x0[ind2]) >= tau1) break;
      if (dist >= L1) break;
    }
    out[id] = (float)(dir <= 1 ? xx : yy);
  }
}

static inline int imaxf_(float a, float b) { return (int)(a > b ? a : b); }
static inline int iminf_(float a, float b) { return (int)(a < b ? a : b); }

/* cbca: post.cu:399-450 over a [D,H,W] volume.  Pixels whose match
 * x + d*direction falls outside the image are copied; others get the float
 * mean over the intersected cross support, summed rows then columns. */
void orc_cbca(const float* x0c, const float* x1c, const double* vol, i64 D, i64 H, i64 W,
              int direction, double* out) {
  const i64 n = D * H * W;
#pragma omp parallel for schedule(static)
  for (i64 id = 0; id < n; id++) {
    const i64 x = id % W, y = (id / W) % H, d = id / (W * H);
    const i64 xm = x + d * direction;
    if (xm < 0 || xm >= W) {
      out[id] = vol[id];
      continue;
    }
    float sum = 0;
    int cnt = 0;
    const int yy_s = imaxf_(x0c[(2 * H + y) * W + x], x1c[(2 * H + y) * W + xm]);
    const int yy_t = iminf_(x0c[(3 * H + y) * W + x], x1c[(3 * H + y) * W + xm]);
    for (int yy = yy_s + 1; yy < yy_t; yy++) {
      const int xx_s = imaxf_(x0c[(0 * H + yy) * W + x], x1c[(0 * H + yy) * W + xm] - d * direction);
      const int xx_t = iminf_(x0c[(1 * H + yy) * W + x], x1c[(1 * H + yy) * W + xm] - d * direction);
      for (int xx = xx_s + 1; xx < xx_t; xx++) {
        const float val = (float)vol[(d * H + yy) * W + xx];
        sum += val;
        cnt++;
      }
    }
    out[id] = sum / cnt;
  }
}

/* sgm2 / sgm_w: post.cu:178-333 on an [H,W,D] volume.  Directions 0..3
 * (right, left, down, up) run one after another; within a direction the
 * scan steps are sequential and the scan lines independent.  The previous
 * step's values are read back as float (:219), the transition is computed
 * in float (:229-256), and the new value in double (:258), which is added
 * to `out` (double) and kept for the next step.  `out` must be zero on
 * entry (test.py:379).  As in the reference, direction 2 divides P1 by
 * alpha1 on the d-1 term and direction 3 on the d+1 term. */
void orc_sgm(const float* x0, const float* x1, const double* in, i64 H, i64 W, int D, float pi1,
             float pi2, float tau_so, float alpha1, float q1, float q2, int direction, double* out) {
  for (int sd = 0; sd < 4; sd++) {
    const int nlines = sd <= 1 ? (int)H : (int)W;
    const int nsteps = sd <= 1 ? (int)W : (int)H;
#pragma omp parallel for schedule(static)
    for (int line = 0; line < nlines; line++) {
      double* tmp = (double*)malloc(sizeof(double) * D);
      float* s = (float*)malloc(sizeof(float) * D);
      for (int step = 0; step < nsteps; step++) {
        int x, y, dx, dy;
        if (sd == 0) { x = step; y = line; dx = 1; dy = 0; }
        else if (sd == 1) { x = (int)W - 1 - step; y = line; dx = -1; dy = 0; }
        else if (sd == 2) { x = line; y = step; dx = 0; dy = 1; }
        else { x = line; y = (int)H - 1 - step; dx = 0; dy = -1; }
        const i64 base = ((i64)y * W + x) * D;
        if (y - dy < 0 || y - dy >= H || x - dx < 0 || x - dx >= W) {
          for (int d = 0; d < D; d++) {
            const float val = (float)in[base + d];
            out[base + d] += val;
            tmp[d] = val;
          }
          continue;
        }
        float mn = 0;
        for (int d = 0; d < D; d++) {
          s[d] = (float)tmp[d];
          if (d == 0 || s[d] < mn) mn = s[d];
        }
        const i64 ind2 = (i64)y * W + x;
        const float D1 = fabsf(x0[ind2] - x0[ind2 - dy * W - dx]);
        for (int d = 0; d < D; d++) {
          float D2;
          const i64 xx = x + (i64)d * direction;
          if (xx < 0 || xx >= W || xx - dx < 0 || xx - dx >= W)
            D2 = 10;
          else
            D2 = fabsf(x1[ind2 + d * direction] - x1[ind2 + d * direction - dy * W - dx]);
          float P1, P2;
          if (D1 < tau_so && D2 < tau_so) {
            P1 = pi1; P2 = pi2;
          } else if (D1 > tau_so && D2 > tau_so) {
            P1 = pi1 / (q1 * q2); P2 = pi2 / (q1 * q2);
          } else {
            P1 = pi1 / q1; P2 = pi2 / q1;
          }
          float cost = fminf(s[d], mn + P2);
          if (d - 1 >= 0) cost = fminf(cost, s[d - 1] + (sd == 2 ? P1 / alpha1 : P1));
          if (d + 1 < D) cost = fminf(cost, s[d + 1] + (sd == 3 ? P1 / alpha1 : P1));
          const double val = (in[base + d] + cost - mn);
          out[base + d] += val;
          tmp[d] = val;
        }
      }
      free(tmp);
      free(s);
    }
  }
}

/* np.argmin(cost, axis=0) over [D,H,W] (test.py:408-409): first minimum. */
void orc_wta(const double* c, i64 D, i64 H, i64 W, float* disp) {
#pragma omp parallel for schedule(static)
  for (i64 p = 0; p < H * W; p++) {
    i64 best = 0;
    double bv = c[p];
    for (i64 d = 1; d < D; d++)
      if (c[d * H * W + p] < bv) { bv = c[d * H * W + p]; best = d; }
    disp[p] = (float)best;
  }
}

/* subpixel_enchancement: post.cu:453-483 ([D,H,W] cost). */
void orc_subpixel(const float* d0, const double* c2, i64 H, i64 W, int D, float* out) {
  const i64 n = H * W;
#pragma omp parallel for schedule(static)
  for (i64 id = 0; id < n; id++) {
    const int d = (int)d0[id];
    out[id] = (float)d;
    if (1 <= d && d < D - 1) {
      const float cn = (float)c2[(i64)(d - 1) * n + id];
      const float cz = (float)c2[(i64)d * n + id];
      const float cp = (float)c2[(i64)(d + 1) * n + id];
      const float denom = 2 * (cp + cn - 2 * cz);
      if (denom > 1e-5) {
        const double q = (double)((cp - cn) / denom);
        const double cl = q < -1.0 ? -1.0 : q;
        out[id] = (float)(d - (cl > 1.0 ? 1.0 : cl));
      }
    }
  }
}

static void sortf(float* x, int n) {
  for (int i = 0; i < n - 1; i++) {
    int mn = i;
    for (int j = i + 1; j < n; j++)
      if (x[j] < x[mn]) mn = j;
    const float t = x[mn];
    x[mn] = x[i];
    x[i] = t;
  }
}

/* median2d: post.cu:486-518 (k x k window clipped at the borders). */
void orc_median2d(const float* img, i64 H, i64 W, int k, float* out) {
  const int r = k / 2;
#pragma omp parallel for schedule(static)
  for (i64 id = 0; id < H * W; id++) {
    const i64 x = id % W, y = id / W;
    float xs[11 * 11];
    int n = 0;
    for (i64 xx = x - r; xx <= x + r; xx++)
      for (i64 yy = y - r; yy <= y + r; yy++)
        if (0 <= xx && xx < W && 0 <= yy && yy < H) xs[n++] = img[yy * W + xx];
    sortf(xs, n);
    out[id] = xs[n / 2];
  }
}

/* mean2d: post.cu:520-566.  Gaussian-weighted mean over neighbours with
 * |I(q) - I(p)| < alpha2; the kernel is indexed xx-major (:530-535).  The
 * CUDA compiler contracts `sum += v * k` into a fused multiply-add, so the
 * restatement uses fmaf to match the reference's device arithmetic. */
void orc_mean2d(const float* img, i64 H, i64 W, const float* kernel, int ks, float alpha2,
                float* out) {
  const int r = ks / 2;
#pragma omp parallel for schedule(static)
  for (i64 id = 0; id < H * W; id++) {
    const i64 x = id % W, y = id / W;
    float sum = 0, cnt = 0;
    int i = 0;
    for (i64 xx = x - r; xx <= x + r; xx++)
      for (i64 yy = y - r; yy <= y + r; yy++, i++)
        if (0 <= xx && xx < W && 0 <= yy && yy < H && fabsf(img[yy * W + xx] - img[y * W + x]) < alpha2) {
          sum = fmaf(img[yy * W + xx], kernel[i], sum);
          cnt += kernel[i];
        }
    out[id] = sum / cnt;
  }
}

/* outlier_detection: post.cu:717-754.  0 match, 1 occlusion, 2 mismatch. */
void orc_outlier_detection(const float* d0, const float* d1, i64 H, i64 W, int disp_max, float* out) {
#pragma omp parallel for schedule(static)
  for (i64 id = 0; id < H * W; id++) {
    const i64 x = id % W;
    const int d0i = (int)d0[id];
    if (x - d0i < 0) {
      out[id] = 1;
    } else if (fabsf(d0[id] - d1[id - d0i]) < 1.1) {
      out[id] = 0;
    } else {
      out[id] = 1;
      for (int d = 0; d < disp_max; d++)
        if (x - d >= 0 && fabsf(d - d1[id - d]) < 1.1) {
          out[id] = 2;
          break;
        }
    }
  }
}

/* interpolate_mismatch: post.cu:757-827.  Median of the first non-mismatch
 * pixel along 16 directions. */
void orc_interpolate_mismatch(const float* d0, const float* outlier, i64 H, i64 W, float* out) {
  static const float dir[32] = {0, 1, -0.5f, 1, -1, 1, -1, 0.5f, -1, 0, -1, -0.5f, -1, -1,
                                -0.5f, -1, 0, -1, 0.5f, -1, 1, -1, 1, -0.5f, 1, 0, 1, 0.5f,
                                1, 1, 0.5f, 1};
#pragma omp parallel for schedule(static)
  for (i64 id = 0; id < H * W; id++) {
    if (outlier[id] != 2) {
      out[id] = d0[id];
      continue;
    }
    float vals[16];
    int n = 0;
    const i64 x = id % W, y = id / W;
    for (int d = 0; d < 16; d++) {
      const float dx = dir[2 * d], dy = dir[2 * d + 1];
      float xx = (float)x, yy = (float)y;
      i64 xi = (i64)roundf(xx), yi = (i64)roundf(yy);
      while (0 <= yi && yi < H && 0 <= xi && xi < W && outlier[yi * W + xi] == 2) {
        xx += dx;
        yy += dy;
        xi = (i64)roundf(xx);
        yi = (i64)roundf(yy);
      }
      if (0 <= yi && yi < H && 0 <= xi && xi < W) vals[n++] = d0[yi * W + xi];
    }
    if (n == 0) {
      out[id] = d0[id];  /* the reference asserts n > 0 here (post.cu:810) */
      continue;
    }
    sortf(vals, n);
    out[id] = vals[n / 2];
  }
}

/* interpolate_occlusion: post.cu:829-869.  Nearest match (outlier == 0) to
 * the left, else to the right. */
void orc_interpolate_occlusion(const float* d0, const float* outlier, i64 H, i64 W, float* out) {
#pragma omp parallel for schedule(static)
  for (i64 id = 0; id < H * W; id++) {
    if (outlier[id] != 1) {
      out[id] = d0[id];
      continue;
    }
    const i64 x = id % W;
    i64 dx = 0;
    while (x + dx >= 0 && outlier[id + dx] != 0) dx--;
    if (x + dx < 0) {
      dx = 0;
      while (x + dx < W && outlier[id + dx] != 0) dx++;
    }
    out[id] = (x + dx < W) ? d0[id + dx] : d0[id];
  }
}
