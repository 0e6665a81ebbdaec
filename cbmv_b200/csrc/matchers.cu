// Matching-cost kernels: census, NCC, Sobel, SAD-on-Sobel, zero-mean SAD.
//
// Each kernel reproduces the reference's valid region, sentinel and
// arithmetic (cpp/matchers/matchers.cpp), so the float64 outputs equal the
// reference's bit for bit:
//   - census and SAD-on-Sobel are integer counts / sums;
//   - NCC's window sums are exact integers and the final
//     -(w^2 S - A_L A_R) * C_L * C_R is evaluated in float64 in the
//     reference's order (matchers.cpp:179);
//   - ZSAD accumulates fabs(L - muL - R + muR) in float64 in the reference's
//     wh-major order (matchers.cpp:499-505).
// Outputs are float32 or float64, in [H,W,D] or [D,H,W] layout.
//
// Thread mapping: for [H,W,D] outputs consecutive threads take consecutive
// d of a pixel (coalesced stores); for [D,H,W] they take consecutive x.
#include <type_traits>

#include "common.cuh"

namespace cbmv {
namespace {

constexpr int kBlock = 128;

// Decodes the (y, x, d) a thread owns from a launch over (row-slab, y[, d]).
struct VolCoord {
  int64_t y, x;
  int d;
  bool in;
};

__device__ __forceinline__ VolCoord vol_coord(int layout, int64_t W, int D) {
  VolCoord c;
  c.y = blockIdx.y;
  if (layout == CBMV_HWD) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    c.in = idx < W * D;
    c.x = idx / D;
    c.d = (int)(idx - c.x * D);
  } else {
    c.x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    c.d = blockIdx.z;
    c.in = c.x < W;
  }
  return c;
}

inline dim3 vol_grid(int layout, int64_t H, int64_t W, int D) {
  if (layout == CBMV_HWD) return dim3((unsigned)((W * D + kBlock - 1) / kBlock), (unsigned)H, 1);
  return dim3((unsigned)((W + kBlock - 1) / kBlock), (unsigned)H, (unsigned)D);
}

// ---------------------------------------------------------------- census
// Descriptor of pixel (i+wc, j+wc), i < H-w, j < W-w: bit k set when the
// window's centre is below its k-th pixel in row-major order
// (_mm_cmplt_epi16(centre, neighbour), matchers.cpp:286-294).
__global__ void census_desc_kernel(const uint8_t* __restrict__ img, int64_t H, int64_t W, int w,
                                   ulonglong2* __restrict__ desc) {
  const int64_t n = (H - w) * (W - w);
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / (W - w), j = t - i * (W - w);
    const int wc = w / 2;
    const int c = img[(i + wc) * W + j + wc];
    unsigned long long b0 = 0, b1 = 0;
    int k = 0;
    for (int wh = 0; wh < w; wh++) {
      const uint8_t* row = img + (i + wh) * W + j;
      for (int ww = 0; ww < w; ww++, k++) {
        const unsigned long long bit = c < row[ww] ? 1ull : 0ull;
        if (k < 64) b0 |= bit << k;
        else b1 |= bit << (k - 64);
      }
    }
    desc[(i + wc) * W + j + wc] = make_ulonglong2(b0, b1);
  }
}

template <class T>
__global__ void census_cost_kernel(const ulonglong2* __restrict__ dl,
                                   const ulonglong2* __restrict__ dr, int64_t H, int64_t W, int D,
                                   int w, int layout, T* __restrict__ out) {
  const VolCoord c = vol_coord(layout, W, D);
  if (!c.in) return;
  const int wc = w / 2;
  const int64_t i = c.y - wc, j = c.x - wc;
  double v = kRandMax;
  // matchers.cpp:312-316: rows i < H-w, cols j < W-w, d < min(D, j+1)
  if (i >= 0 && i < H - w && j >= 0 && j < W - w && c.d <= j) {
    const ulonglong2 a = dl[c.y * W + c.x];
    const ulonglong2 b = dr[c.y * W + c.x - c.d];
    v = (double)(__popcll(a.x ^ b.x) + __popcll(a.y ^ b.y));
  }
  out[vol_index(layout, c.y, c.x, c.d, H, W, D)] = cvt_out<T>(v);
}

// The float32 [H,W,D] census volume of the learned path, without a
// division per element: a CTA owns 16 columns of one row and 128
// disparities (lane = d), so the left descriptor is one broadcast load per
// column and the right one a coalesced run along d.  Same values and
// sentinels as census_cost_kernel (the popcount sum is exact in float32).
__global__ void __launch_bounds__(128) census_cost_hwd_f32_kernel(const ulonglong2* __restrict__ dl,
                                                                  const ulonglong2* __restrict__ dr, int64_t H,
                                                                  int64_t W, int D, int w, float* __restrict__ out) {
  const int64_t y = blockIdx.y;
  const int64_t x0 = (int64_t)blockIdx.x * 16;
  const int d = blockIdx.z * 128 + threadIdx.x;
  if (d >= D) return;
  const int wc = w / 2;
  const int64_t i = y - wc;
  const bool row_ok = i >= 0 && i < H - w;
#pragma unroll 4
  for (int s = 0; s < 16; s++) {
    const int64_t x = x0 + s;
    if (x >= W) break;
    const int64_t j = x - wc;
    float v = kRandMaxF;
    // matchers.cpp:312-316: rows i < H-w, cols j < W-w, d < min(D, j+1)
    if (row_ok && j >= 0 && j < W - w && d <= j) {
      const ulonglong2 a = dl[y * W + x];
      const ulonglong2 b = dr[y * W + x - d];
      v = (float)(__popcll(a.x ^ b.x) + __popcll(a.y ^ b.y));
    }
    out[(y * W + x) * D + d] = v;
  }
}

// ------------------------------------------------------------------- NCC
// Window sum A and 1/sqrt(w^2 B - A^2) (matchers.cpp:115-131); B is exact.
__global__ void ncc_stats_kernel(const uint8_t* __restrict__ img, int64_t H, int64_t W, int w,
                                 uint32_t* __restrict__ A, double* __restrict__ C) {
  const int64_t n = (H - w) * (W - w);
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / (W - w), j = t - i * (W - w);
    const int wc = w / 2;
    unsigned long long a = 0, b = 0;
    for (int wh = 0; wh < w; wh++)
      for (int ww = 0; ww < w; ww++) {
        const unsigned long long v = img[(i + wh) * W + j + ww];
        a += v;
        b += v * v;
      }
    const int64_t p = (i + wc) * W + j + wc;
    A[p] = (uint32_t)a;
    C[p] = 1.0 / sqrt((double)((unsigned long long)(w * w) * b) - (double)a * (double)a);
  }
}

template <class T>
__global__ void ncc_cost_kernel(const uint8_t* __restrict__ L, const uint8_t* __restrict__ R,
                                const uint32_t* __restrict__ Al, const uint32_t* __restrict__ Ar,
                                const double* __restrict__ Cl, const double* __restrict__ Cr,
                                int64_t H, int64_t W, int D, int w, int layout,
                                T* __restrict__ out) {
  const VolCoord c = vol_coord(layout, W, D);
  if (!c.in) return;
  const int wc = w / 2;
  const int64_t i = c.y - wc, j = c.x - wc;
  double v = kRandMax;
  // matchers.cpp:168-172: rows i < H-w, cols d <= j < W-w
  if (i >= 0 && i < H - w && j >= c.d && j < W - w) {
    unsigned long long s = 0;
    for (int wh = 0; wh < w; wh++) {
      const uint8_t* lr = L + (i + wh) * W + j;
      const uint8_t* rr = R + (i + wh) * W + j - c.d;
      for (int ww = 0; ww < w; ww++) s += (unsigned)lr[ww] * (unsigned)rr[ww];
    }
    const int64_t pl = c.y * W + c.x, pr = pl - c.d;
    const double cl = Cl[pl], cr = Cr[pr];
    if (isfinite(cl) && isfinite(cr)) {
      const double lD = (double)s;
      const unsigned long long aa = (unsigned long long)Al[pl] * (unsigned long long)Ar[pr];
      const double num = (double)(w * w) * lD - (double)aa;  // exact: integers < 2^53
      v = -num * cl * cr;                                      // matchers.cpp:179
    } else {
      v = 1.0;                                                 // matchers.cpp:181
    }
  }
  out[vol_index(layout, c.y, c.x, c.d, H, W, D)] = cvt_out<T>(v);
}

// ----------------------------------------------------------------- Sobel
template <class T>
__global__ void sobel_kernel(const uint8_t* __restrict__ img, int64_t H, int64_t W,
                             T* __restrict__ out) {
  const int64_t n = H * W;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t y = p / W, x = p - y * W;
    int v = 0;
    // matchers.cpp:539-548: written at (i+1, j+1) for i < H-3, j < W-3
    if (y >= 1 && y - 1 < H - 3 && x >= 1 && x - 1 < W - 3) {
      const uint8_t* a = img + (y - 1) * W + (x - 1);
      v = -(int)a[0] + (int)a[2] - 2 * (int)a[W] + 2 * (int)a[W + 2] - (int)a[2 * W] +
          (int)a[2 * W + 2];
    }
    out[p] = (T)v;
  }
}

template <class S>
__global__ void to_int_kernel(const S* __restrict__ in, int64_t n, int32_t* __restrict__ out) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x)
    out[p] = (int32_t)in[p];
}

// ---------------------------------------------------------- SAD on Sobel
template <class T>
__global__ void sadsob_cost_kernel(const int32_t* __restrict__ SL, const int32_t* __restrict__ SR,
                                   int64_t H, int64_t W, int D, int w, int layout,
                                   T* __restrict__ out) {
  const VolCoord c = vol_coord(layout, W, D);
  if (!c.in) return;
  const int wc = w / 2;
  const int64_t i = c.y - wc, j = c.x - wc;
  double v = kRandMax;
  // matchers.cpp:412-423: rows i < H-w, cols d <= j < W-w
  if (i >= 0 && i < H - w && j >= c.d && j < W - w) {
    int s = 0;
    for (int wh = 0; wh < w; wh++) {
      const int32_t* lr = SL + (i + wh) * W + j;
      const int32_t* rr = SR + (i + wh) * W + j - c.d;
      for (int ww = 0; ww < w; ww++) s += abs(lr[ww] - rr[ww]);
    }
    v = (double)s;
  }
  out[vol_index(layout, c.y, c.x, c.d, H, W, D)] = cvt_out<T>(v);
}

// ------------------------------------------------------------------ ZSAD
// Window means: exact integer sum, one float64 division (matchers.cpp:474-482).
__global__ void zsad_means_kernel(const uint8_t* __restrict__ img, int64_t H, int64_t W, int w,
                                  double* __restrict__ mean) {
  const int64_t n = (H - w) * (W - w);
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / (W - w), j = t - i * (W - w);
    const int wc = w / 2;
    int s = 0;
    for (int wh = 0; wh < w; wh++)
      for (int ww = 0; ww < w; ww++) s += img[(i + wh) * W + j + ww];
    mean[(i + wc) * W + j + wc] = (double)s / (double)(w * w);
  }
}

template <class T>
__global__ void zsad_cost_kernel(const uint8_t* __restrict__ L, const uint8_t* __restrict__ R,
                                 const double* __restrict__ ml, const double* __restrict__ mr,
                                 int64_t H, int64_t W, int D, int w, int layout,
                                 T* __restrict__ out) {
  const VolCoord c = vol_coord(layout, W, D);
  if (!c.in) return;
  const int wc = w / 2;
  const int64_t i = c.y - wc, j = c.x - wc;
  double v = kRandMax;
  // matchers.cpp:495-505: rows i < H-w, cols d <= j < W-w
  if (i >= 0 && i < H - w && j >= c.d && j < W - w) {
    const double mul = ml[c.y * W + c.x];
    const double mur = mr[c.y * W + c.x - c.d];
    double s = 0.0;
    for (int wh = 0; wh < w; wh++) {
      const uint8_t* lr = L + (i + wh) * W + j;
      const uint8_t* rr = R + (i + wh) * W + j - c.d;
      for (int ww = 0; ww < w; ww++) {
        // ((L - muL) - R) + muR, each step rounded as in the reference
        const double t = __dadd_rn(__dadd_rn(__dsub_rn((double)lr[ww], mul), -(double)rr[ww]), mur);
        s = __dadd_rn(s, fabs(t));
      }
    }
    v = s;
  }
  out[vol_index(layout, c.y, c.x, c.d, H, W, D)] = cvt_out<T>(v);
}

// ------------------------------------------- float32 strip matchers
// The three window matchers for the learned classifier's float32 volumes
// ([H,W,D]): a warp owns 32 disparities (lane = d) of one row and walks a
// strip of SX columns; the window's L and R columns sit in a register ring,
// so each step loads one new column of each (L uniform across the warp, R
// at x - d per lane).  Window sums are exact integers (SAD of Sobel
// responses, sum of L*R, ZSAD as sum |25 (L - R) - (sum L - sum R)| / 25), so
// the float32 result equals the rounding of the reference's value (its
// float64 ZSAD chain differs from the exact quotient by ~1e-15 relative).
// Validity and sentinels as in the reference kernels above.
enum StripMode { kStripNcc = 0, kStripSadSob = 1, kStripZsad = 2 };
constexpr int kStripX = 16;

template <int MODE, int WIN>
__global__ void __launch_bounds__(128) matcher_strip_kernel(
    const void* __restrict__ Lp, const void* __restrict__ Rp, const uint32_t* __restrict__ Al,
    const uint32_t* __restrict__ Ar, const double* __restrict__ Cl, const double* __restrict__ Cr,
    const double* __restrict__ ml, const double* __restrict__ mr, int64_t H, int64_t W, int D,
    float* __restrict__ out) {
  using Px = typename std::conditional<MODE == kStripSadSob, int32_t, uint8_t>::type;
  const Px* L = static_cast<const Px*>(Lp);
  const Px* R = static_cast<const Px*>(Rp);
  constexpr int r = WIN / 2;
  const int64_t y = blockIdx.y;
  const int64_t x0 = (int64_t)blockIdx.x * kStripX;
  const int d = blockIdx.z * 128 + threadIdx.x;
  if (d >= D) return;
  // window rows, clamped into the image (values of clamped rows are never used)
  int64_t rowoff[WIN];
#pragma unroll
  for (int wh = 0; wh < WIN; wh++) {
    int64_t yy = y - r + wh;
    yy = yy < 0 ? 0 : (yy >= H ? H - 1 : yy);
    rowoff[wh] = yy * W;
  }
  // ring slot contents, computed when the column is loaded: SAD and NCC
  // keep the column's sum (of |SL - SR|, of L * R), ZSAD keeps 25 (L - R)
  // per window row
  int col[WIN];
  int dif[MODE == kStripZsad ? WIN : 1][WIN];
  // ZSAD: the column's sum of L minus its sum of R (the window's sum of
  // these is sum L - sum R, exact: 25 x its mean difference)
  int cdm[MODE == kStripZsad ? WIN : 1];
  auto load_col = [&](int slot, int64_t c) {
    const int64_t cl = c < 0 ? 0 : (c >= W ? W - 1 : c);
    int64_t cr = c - d;
    cr = cr < 0 ? 0 : (cr >= W ? W - 1 : cr);
    int sum = 0;
#pragma unroll
    for (int wh = 0; wh < WIN; wh++) {
      const int a = (int)__ldg(L + rowoff[wh] + cl), b = (int)__ldg(R + rowoff[wh] + cr);
      if (MODE == kStripSadSob) sum += abs(a - b);
      else if (MODE == kStripNcc) sum += a * b;
      else {
        dif[MODE == kStripZsad ? slot : 0][wh] = (WIN * WIN) * (a - b);
        sum += a - b;
      }
    }
    if (MODE == kStripZsad) cdm[MODE == kStripZsad ? slot : 0] = sum;
    col[slot] = sum;
  };
#pragma unroll
  for (int j = 0; j < WIN - 1; j++) load_col(j, x0 - r + j);
  const bool row_ok = y >= r && y < H - WIN + r;
#pragma unroll
  for (int s = 0; s < kStripX; s++) {
    const int64_t x = x0 + s;
    if (x >= W) break;
    load_col((s + WIN - 1) % WIN, x + r);
    // ring slot (s + k) % WIN holds column x - r + k
    float v = kRandMaxF;
    if (row_ok && x >= d + r && x < W - WIN + r) {
      if (MODE == kStripSadSob) {
        int acc = 0;
#pragma unroll
        for (int k = 0; k < WIN; k++) acc += col[(s + k) % WIN];
        v = (float)acc;
      } else if (MODE == kStripZsad) {
        // 25 x (mean L - mean R) over the window, exactly (the window lies
        // inside both images here, so no column or row was clamped)
        int m = 0;
#pragma unroll
        for (int k = 0; k < WIN; k++) m += cdm[MODE == kStripZsad ? (s + k) % WIN : 0];
        unsigned acc = 0;
#pragma unroll
        for (int k = 0; k < WIN; k++)
#pragma unroll
          for (int wh = 0; wh < WIN; wh++) acc = __sad(dif[MODE == kStripZsad ? (s + k) % WIN : 0][wh], m, acc);
        // acc < 2^24 (WIN^2 terms of at most 2 WIN^2 255) is exact in
        // float32, and acc / WIN^2 is either an integer or more than 2^-29
        // (relative) away from every float32 rounding midpoint, so one
        // correctly rounded float32 division gives the float32 rounding of
        // the exact quotient -- what rounding a float64 quotient would give
        static_assert(WIN * WIN * WIN * WIN * 510 < (1 << 24), "ZSAD window sum exact in float32");
        v = __fdiv_rn((float)acc, (float)(WIN * WIN));
      } else {
        const int64_t pl = y * W + x, pr = pl - d;
        unsigned acc = 0;
#pragma unroll
        for (int k = 0; k < WIN; k++) acc += (unsigned)col[(s + k) % WIN];
        const double cl = Cl[pl], cr = Cr[pr];
        if (isfinite(cl) && isfinite(cr)) {
          const unsigned long long aa = (unsigned long long)Al[pl] * (unsigned long long)Ar[pr];
          const double num = (double)(WIN * WIN) * (double)acc - (double)aa;
          v = (float)(-num * cl * cr);
        } else {
          v = 1.0f;
        }
      }
    }
    out[(y * W + x) * D + d] = v;
  }
}

}  // namespace

// Argument checks shared by the matcher entry points (also cbmv_census_static).
int check_common(const void* a, const void* b, const void* out, int64_t H, int64_t W, int D, int w,
                 int dtype, int layout, int wmax) {
  CBMV_REQUIRE(a && b && out, CBMV_EINVAL, "null pointer argument");
  CBMV_REQUIRE(H > 0 && W > 0 && D > 0, CBMV_EINVAL, "bad size H=%lld W=%lld D=%d",
               (long long)H, (long long)W, D);
  CBMV_REQUIRE(H <= 65535, CBMV_ERANGE, "H=%lld exceeds 65535", (long long)H);
  CBMV_REQUIRE(D <= 65535, CBMV_ERANGE, "D=%d exceeds 65535", D);
  CBMV_REQUIRE(w >= 1 && (w & 1) && w <= wmax, CBMV_EINVAL, "window %d must be odd and <= %d", w,
               wmax);
  CBMV_REQUIRE(dtype == CBMV_F32 || dtype == CBMV_F64, CBMV_EINVAL, "bad dtype %d", dtype);
  CBMV_REQUIRE(layout == CBMV_HWD || layout == CBMV_DHW, CBMV_EINVAL, "bad layout %d", layout);
  return CBMV_OK;
}

namespace {

// Scratch allocation for the stand-alone matcher entry points (the fused
// pipeline keeps its scratch in its context instead).
struct Scratch {
  void* p = nullptr;
  ~Scratch() {
    if (p) cudaFree(p);
  }
};

}  // namespace

// Fills a volume with the sentinel where the valid region is empty.
template <class T>
__global__ void fill_kernel(T* out, int64_t n, T v) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x)
    out[p] = v;
}

int launch_census_desc(const uint8_t* img, int64_t H, int64_t W, int w, ulonglong2* desc,
                       cudaStream_t st) {
  if (H <= w || W <= w) return CBMV_OK;
  const int64_t n = (H - w) * (W - w);
  census_desc_kernel<<<grid_for(n, kBlock), kBlock, 0, st>>>(img, H, W, w, desc);
  return check_launch("census_desc");
}

template <class T>
int launch_census_cost(const ulonglong2* dl, const ulonglong2* dr, int64_t H, int64_t W, int D,
                       int w, int layout, T* out, cudaStream_t st) {
  if (std::is_same<T, float>::value && layout == CBMV_HWD) {
    const dim3 grid((unsigned)((W + 15) / 16), (unsigned)H, (unsigned)((D + 127) / 128));
    census_cost_hwd_f32_kernel<<<grid, 128, 0, st>>>(dl, dr, H, W, D, w, reinterpret_cast<float*>(out));
    return check_launch("census_cost");
  }
  census_cost_kernel<T><<<vol_grid(layout, H, W, D), kBlock, 0, st>>>(dl, dr, H, W, D, w, layout, out);
  return check_launch("census_cost");
}

int launch_ncc_stats(const uint8_t* img, int64_t H, int64_t W, int w, uint32_t* A, double* C,
                     cudaStream_t st) {
  if (H <= w || W <= w) return CBMV_OK;
  const int64_t n = (H - w) * (W - w);
  ncc_stats_kernel<<<grid_for(n, kBlock), kBlock, 0, st>>>(img, H, W, w, A, C);
  return check_launch("ncc_stats");
}

template <class T>
int launch_ncc_cost(const uint8_t* L, const uint8_t* R, const uint32_t* Al, const uint32_t* Ar,
                    const double* Cl, const double* Cr, int64_t H, int64_t W, int D, int w,
                    int layout, T* out, cudaStream_t st) {
  ncc_cost_kernel<T><<<vol_grid(layout, H, W, D), kBlock, 0, st>>>(L, R, Al, Ar, Cl, Cr, H, W, D, w,
                                                                   layout, out);
  return check_launch("ncc_cost");
}

int launch_sobel_i32(const uint8_t* img, int64_t H, int64_t W, int32_t* out, cudaStream_t st) {
  sobel_kernel<int32_t><<<grid_for(H * W, kBlock), kBlock, 0, st>>>(img, H, W, out);
  return check_launch("sobel");
}

template <class T>
int launch_sadsob_cost(const int32_t* SL, const int32_t* SR, int64_t H, int64_t W, int D, int w,
                       int layout, T* out, cudaStream_t st) {
  sadsob_cost_kernel<T><<<vol_grid(layout, H, W, D), kBlock, 0, st>>>(SL, SR, H, W, D, w, layout, out);
  return check_launch("sadsob_cost");
}

int launch_zsad_means(const uint8_t* img, int64_t H, int64_t W, int w, double* mean,
                      cudaStream_t st) {
  if (H <= w || W <= w) return CBMV_OK;
  const int64_t n = (H - w) * (W - w);
  zsad_means_kernel<<<grid_for(n, kBlock), kBlock, 0, st>>>(img, H, W, w, mean);
  return check_launch("zsad_means");
}

template <class T>
int launch_zsad_cost(const uint8_t* L, const uint8_t* R, const double* ml, const double* mr,
                     int64_t H, int64_t W, int D, int w, int layout, T* out, cudaStream_t st) {
  zsad_cost_kernel<T><<<vol_grid(layout, H, W, D), kBlock, 0, st>>>(L, R, ml, mr, H, W, D, w, layout,
                                                                    out);
  return check_launch("zsad_cost");
}

template <int MODE, int WIN>
static int launch_strip(const void* L, const void* R, const uint32_t* Al, const uint32_t* Ar, const double* Cl,
                        const double* Cr, const double* ml, const double* mr, int64_t H, int64_t W, int D,
                        float* out, cudaStream_t st) {
  const dim3 grid((unsigned)((W + kStripX - 1) / kStripX), (unsigned)H, (unsigned)((D + 127) / 128));
  matcher_strip_kernel<MODE, WIN><<<grid, 128, 0, st>>>(L, R, Al, Ar, Cl, Cr, ml, mr, H, W, D, out);
  return check_launch("matcher_strip");
}

// float32 [H,W,D] matchers of the learned path: the strip kernels for the
// default windows, the general kernels otherwise
int launch_ncc_cost_f32(const uint8_t* L, const uint8_t* R, const uint32_t* Al, const uint32_t* Ar,
                        const double* Cl, const double* Cr, int64_t H, int64_t W, int D, int w, float* out,
                        cudaStream_t st) {
  if (w == 3 && H <= 65535)
    return launch_strip<kStripNcc, 3>(L, R, Al, Ar, Cl, Cr, nullptr, nullptr, H, W, D, out, st);
  return launch_ncc_cost<float>(L, R, Al, Ar, Cl, Cr, H, W, D, w, CBMV_HWD, out, st);
}
int launch_sadsob_cost_f32(const int32_t* SL, const int32_t* SR, int64_t H, int64_t W, int D, int w, float* out,
                           cudaStream_t st) {
  if (w == 5 && H <= 65535)
    return launch_strip<kStripSadSob, 5>(SL, SR, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, H, W, D,
                                         out, st);
  return launch_sadsob_cost<float>(SL, SR, H, W, D, w, CBMV_HWD, out, st);
}
int launch_zsad_cost_f32(const uint8_t* L, const uint8_t* R, const double* ml, const double* mr, int64_t H,
                         int64_t W, int D, int w, float* out, cudaStream_t st) {
  if (w == 5 && H <= 65535)
    return launch_strip<kStripZsad, 5>(L, R, nullptr, nullptr, nullptr, nullptr, ml, mr, H, W, D, out, st);
  return launch_zsad_cost<float>(L, R, ml, mr, H, W, D, w, CBMV_HWD, out, st);
}

template int launch_census_cost<double>(const ulonglong2*, const ulonglong2*, int64_t, int64_t, int,
                                        int, int, double*, cudaStream_t);
template int launch_census_cost<float>(const ulonglong2*, const ulonglong2*, int64_t, int64_t, int,
                                       int, int, float*, cudaStream_t);
template int launch_ncc_cost<double>(const uint8_t*, const uint8_t*, const uint32_t*,
                                     const uint32_t*, const double*, const double*, int64_t,
                                     int64_t, int, int, int, double*, cudaStream_t);
template int launch_sadsob_cost<double>(const int32_t*, const int32_t*, int64_t, int64_t, int, int,
                                        int, double*, cudaStream_t);
template int launch_zsad_cost<double>(const uint8_t*, const uint8_t*, const double*, const double*,
                                      int64_t, int64_t, int, int, int, double*, cudaStream_t);
template int launch_ncc_cost<float>(const uint8_t*, const uint8_t*, const uint32_t*, const uint32_t*,
                                    const double*, const double*, int64_t, int64_t, int, int, int, float*,
                                    cudaStream_t);
template int launch_sadsob_cost<float>(const int32_t*, const int32_t*, int64_t, int64_t, int, int, int,
                                       float*, cudaStream_t);
template int launch_zsad_cost<float>(const uint8_t*, const uint8_t*, const double*, const double*,
                                     int64_t, int64_t, int, int, int, float*, cudaStream_t);

}  // namespace cbmv

using namespace cbmv;

extern "C" int cbmv_census(const uint8_t* L, const uint8_t* R, int64_t H, int64_t W, int D,
                           int wsize, void* out, int dtype, int layout, void* stream) {
  int rc = check_common(L, R, out, H, W, D, wsize, dtype, layout, 11);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  Scratch s;
  CBMV_CUDA(cudaMallocAsync(&s.p, (size_t)H * W * sizeof(ulonglong2) * 2, st));
  ulonglong2* dl = (ulonglong2*)s.p;
  ulonglong2* dr = dl + H * W;
  if ((rc = launch_census_desc(L, H, W, wsize, dl, st))) return rc;
  if ((rc = launch_census_desc(R, H, W, wsize, dr, st))) return rc;
  rc = dtype == CBMV_F64 ? launch_census_cost(dl, dr, H, W, D, wsize, layout, (double*)out, st)
                         : launch_census_cost(dl, dr, H, W, D, wsize, layout, (float*)out, st);
  CBMV_CUDA(cudaFreeAsync(s.p, st));
  s.p = nullptr;
  return rc;
}

extern "C" int cbmv_ncc(const uint8_t* L, const uint8_t* R, int64_t H, int64_t W, int D, int wsize,
                        void* out, int dtype, int layout, void* stream) {
  int rc = check_common(L, R, out, H, W, D, wsize, dtype, layout, 15);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  Scratch s;
  const size_t n = (size_t)H * W;
  CBMV_CUDA(cudaMallocAsync(&s.p, n * (2 * sizeof(uint32_t) + 2 * sizeof(double)), st));
  double* Cl = (double*)s.p;
  double* Cr = Cl + n;
  uint32_t* Al = (uint32_t*)(Cr + n);
  uint32_t* Ar = Al + n;
  if ((rc = launch_ncc_stats(L, H, W, wsize, Al, Cl, st))) return rc;
  if ((rc = launch_ncc_stats(R, H, W, wsize, Ar, Cr, st))) return rc;
  rc = dtype == CBMV_F64
           ? launch_ncc_cost(L, R, Al, Ar, Cl, Cr, H, W, D, wsize, layout, (double*)out, st)
           : launch_ncc_cost(L, R, Al, Ar, Cl, Cr, H, W, D, wsize, layout, (float*)out, st);
  CBMV_CUDA(cudaFreeAsync(s.p, st));
  s.p = nullptr;
  return rc;
}

extern "C" int cbmv_sobel(const uint8_t* img, int64_t H, int64_t W, void* out, int dtype,
                          void* stream) {
  CBMV_REQUIRE(img && out, CBMV_EINVAL, "null pointer argument");
  CBMV_REQUIRE(H > 0 && W > 0, CBMV_EINVAL, "bad size");
  CBMV_REQUIRE(dtype == CBMV_F32 || dtype == CBMV_F64, CBMV_EINVAL, "bad dtype %d", dtype);
  cudaStream_t st = as_stream(stream);
  if (dtype == CBMV_F64)
    sobel_kernel<double><<<grid_for(H * W, kBlock), kBlock, 0, st>>>(img, H, W, (double*)out);
  else
    sobel_kernel<float><<<grid_for(H * W, kBlock), kBlock, 0, st>>>(img, H, W, (float*)out);
  return check_launch("sobel");
}

extern "C" int cbmv_sadsob(const void* SL, const void* SR, int sob_dtype, int64_t H, int64_t W,
                           int D, int wsize, void* out, int dtype, int layout, void* stream) {
  int rc = check_common(SL, SR, out, H, W, D, wsize, dtype, layout, 15);
  if (rc) return rc;
  CBMV_REQUIRE(sob_dtype == CBMV_F32 || sob_dtype == CBMV_F64, CBMV_EINVAL, "bad sobel dtype");
  cudaStream_t st = as_stream(stream);
  Scratch s;
  const int64_t n = H * W;
  CBMV_CUDA(cudaMallocAsync(&s.p, (size_t)n * 2 * sizeof(int32_t), st));
  int32_t* il = (int32_t*)s.p;
  int32_t* ir = il + n;
  if (sob_dtype == CBMV_F64) {
    to_int_kernel<double><<<grid_for(n, kBlock), kBlock, 0, st>>>((const double*)SL, n, il);
    to_int_kernel<double><<<grid_for(n, kBlock), kBlock, 0, st>>>((const double*)SR, n, ir);
  } else {
    to_int_kernel<float><<<grid_for(n, kBlock), kBlock, 0, st>>>((const float*)SL, n, il);
    to_int_kernel<float><<<grid_for(n, kBlock), kBlock, 0, st>>>((const float*)SR, n, ir);
  }
  if ((rc = check_launch("sadsob_convert"))) return rc;
  rc = dtype == CBMV_F64 ? launch_sadsob_cost(il, ir, H, W, D, wsize, layout, (double*)out, st)
                         : launch_sadsob_cost(il, ir, H, W, D, wsize, layout, (float*)out, st);
  CBMV_CUDA(cudaFreeAsync(s.p, st));
  s.p = nullptr;
  return rc;
}

extern "C" int cbmv_zsad(const uint8_t* L, const uint8_t* R, int64_t H, int64_t W, int D,
                         int wsize, void* out, int dtype, int layout, void* stream) {
  int rc = check_common(L, R, out, H, W, D, wsize, dtype, layout, 15);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  Scratch s;
  const size_t n = (size_t)H * W;
  CBMV_CUDA(cudaMallocAsync(&s.p, n * 2 * sizeof(double), st));
  double* ml = (double*)s.p;
  double* mr = ml + n;
  if ((rc = launch_zsad_means(L, H, W, wsize, ml, st))) return rc;
  if ((rc = launch_zsad_means(R, H, W, wsize, mr, st))) return rc;
  rc = dtype == CBMV_F64
           ? launch_zsad_cost(L, R, ml, mr, H, W, D, wsize, layout, (double*)out, st)
           : launch_zsad_cost(L, R, ml, mr, H, W, D, wsize, layout, (float*)out, st);
  CBMV_CUDA(cudaFreeAsync(s.p, st));
  s.p = nullptr;
  return rc;
}
