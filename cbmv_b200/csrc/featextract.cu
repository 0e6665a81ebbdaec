// Feature extraction: the reference's layout helpers and confidence
// measures (cpp/featextract/featextract.cpp) and the fused 20-feature kernel
// that replaces Testing.__extract_features_lr (test.py:521-595).
//
// Every confidence is computed in float64 with the reference's operation
// order, so the features equal the reference's float64 values (and so their
// float32 roundings, which is what the random forest compares).  The one
// freedom taken is the order of the likelihood denominator's sum over d,
// which only moves it by an ulp of float64.
#include "common.cuh"
#include "features.cuh"

namespace cbmv {
namespace {

constexpr int kBlock = 256;

#define GRID_STRIDE(i, n) \
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

__global__ void swap_axes_kernel(const double* __restrict__ in, int64_t D, int64_t HW,
                                 double* __restrict__ out) {
  GRID_STRIDE(t, D * HW) {
    const int64_t p = t / D, d = t - p * D;
    out[t] = in[d * HW + p];
  }
}

__global__ void swap_axes_back_kernel(const double* __restrict__ in, int64_t HW, int64_t D,
                                      double* __restrict__ out) {
  GRID_STRIDE(t, D * HW) {
    const int64_t d = t / HW, p = t - d * HW;
    out[t] = in[p * D + d];
  }
}

__global__ void get_cost_kernel(const double* __restrict__ in, int64_t n, int64_t K,
                                double* __restrict__ out) {
  GRID_STRIDE(t, n) out[t] = in[t * K];
}

// dir = +1: R[i,j,d] = C[i,j+d,d] for j < W-d (featextract.cpp:136-145)
// dir = -1: L[i,j,d] = R[i,j-d,d] for j >= d (featextract.cpp:473-481)
// otherwise the volume's first element (:130, :467).
__global__ void shift_kernel(const double* __restrict__ in, int64_t H, int64_t W, int64_t D,
                             int dir, double* __restrict__ out) {
  const double fill = in[0];
  GRID_STRIDE(t, H * W * D) {
    const int64_t d = t % D;
    const int64_t p = t / D;
    const int64_t j = p % W;
    const int64_t js = j + dir * d;
    out[t] = (js >= 0 && js < W) ? in[(p + dir * d) * D + d] : fill;
  }
}

// Row minimum as featextract.cpp:322-329 (start at RAND_MAX, strict <),
// one warp per row.
__device__ __forceinline__ double warp_row_min(const double* r, int64_t D) {
  double m = kRandMax;
  for (int64_t k = threadIdx.x & 31; k < D; k += 32) m = fmin(m, r[k]);
  for (int o = 16; o; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
  return m;
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double lik_term(double c, double m, double sigma) {
  const double num = c - m;
  return exp(-(num * num) / sigma);  // featextract.cpp:433-434
}

__global__ void ratio_kernel(const double* __restrict__ v, int64_t N, int64_t D, double e,
                             double* __restrict__ out) {
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x / 32);
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32; i < N; i += warps) {
    const double* r = v + i * D;
    const double m = warp_row_min(r, D);
    for (int64_t k = threadIdx.x & 31; k < D; k += 32)
      out[i * D + k] = (m == kRandMax) ? 0.0 : (m + e) / (r[k] + e);
  }
}

__global__ void likelihood_kernel(const double* __restrict__ v, int64_t N, int64_t D, double sigma,
                                  double* __restrict__ out) {
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x / 32);
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32; i < N; i += warps) {
    const double* r = v + i * D;
    const double m = warp_row_min(r, D);
    double den = 0.0;
    for (int64_t k = threadIdx.x & 31; k < D; k += 32) den += lik_term(r[k], m, sigma);
    den = warp_sum(den);
    for (int64_t k = threadIdx.x & 31; k < D; k += 32) {
      const double t = r[k] - m;
      out[i * D + k] = (m == kRandMax) ? 0.0 : exp(-((t * t) / sigma)) / den;
    }
  }
}

__global__ void ratio_samples_kernel(const double* __restrict__ v, int64_t N, int64_t D,
                                     const int32_t* __restrict__ s, double e,
                                     double* __restrict__ out) {
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x / 32);
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32; i < N; i += warps) {
    const double* r = v + i * D;
    const double m = warp_row_min(r, D);
    const int k = threadIdx.x & 31;
    if (k < 3) out[3 * i + k] = (m == kRandMax) ? 0.0 : (m + e) / (r[s[3 * i + k]] + e);
  }
}

__global__ void likelihood_samples_kernel(const double* __restrict__ v, int64_t N, int64_t D,
                                          const int32_t* __restrict__ s, double sigma,
                                          double* __restrict__ out) {
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x / 32);
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32; i < N; i += warps) {
    const double* r = v + i * D;
    const double m = warp_row_min(r, D);
    double den = 0.0;
    for (int64_t k = threadIdx.x & 31; k < D; k += 32) den += lik_term(r[k], m, sigma);
    den = warp_sum(den);
    const int k = threadIdx.x & 31;
    if (k < 3) {
      const double t = r[s[3 * i + k]] - m;
      out[3 * i + k] = (m == kRandMax) ? 0.0 : exp(-((t * t) / sigma)) / den;
    }
  }
}

__global__ void get_samples_kernel(const double* __restrict__ v, int64_t N, int64_t D,
                                   const int32_t* __restrict__ s, double* __restrict__ out) {
  GRID_STRIDE(t, 3 * N) out[t] = v[(t / 3) * D + s[t]];
}

__global__ void labels_kernel(int64_t N, int32_t* __restrict__ out) {
  GRID_STRIDE(t, 3 * N) out[t] = (t % 3) == 0 ? 1 : 0;
}

__device__ __forceinline__ uint32_t draw(uint64_t seed, int64_t s, int slot, uint32_t n) {
  uint64_t z = seed * 0x9E3779B97F4A7C15ull + (uint64_t)s * 3ull + (uint64_t)slot + 1;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (uint32_t)(z % n);
}

__global__ void d_indices_kernel(const int32_t* __restrict__ gt, int64_t N, int maxd, int thr,
                                 uint64_t seed, int32_t* __restrict__ out, int* __restrict__ bad) {
  GRID_STRIDE(s, N) {
    const int g = gt[s];
    const bool low = !(g - thr <= 0), high = !(g + thr >= maxd);
    const int lo_n = g - thr, hi_n = maxd - (g + thr + 1);
    int d1 = 0, d2 = 0;
    bool ok = g >= 0 && g <= maxd;
    if (low) d1 = (int)draw(seed, s, 0, (uint32_t)lo_n);
    else if (hi_n > 0) d1 = (int)draw(seed, s, 0, (uint32_t)hi_n) + (g + thr + 1);
    else ok = false;
    if (high && hi_n > 0) d2 = (int)draw(seed, s, 1, (uint32_t)hi_n) + (g + thr + 1);
    else if (!high && lo_n > 0) d2 = (int)draw(seed, s, 1, (uint32_t)lo_n);
    else ok = false;
    out[3 * s] = g;
    out[3 * s + 1] = d1;
    out[3 * s + 2] = d2;
    if (!ok) atomicExch(bad, 1);
  }
}

}  // namespace

// ------------------------------------------------------ fused features
// Per-pixel statistics of one matcher volume for both reference views:
// stats[((m*2 + view)*HW + p)*2 + {0,1}] = {row minimum, likelihood
// denominator}; view 0 = left reference (row p of the volume), view 1 =
// right reference (right pixel p: entries C[p + d, d], RAND_MAX when
// x + d >= W, featextract.cpp:115-152).  One warp per (pixel, view).
// Row statistics of matcher m: (min, den) in float64 for the exact features
// and, when statsf is given, (min, 1/den) in float32 for the classifier
// network (min = 2^31 and 1/den = 0 where the row has only sentinels).
__global__ void feature_stats_kernel(const double* __restrict__ vol, int m, int64_t H, int64_t W,
                                     int D, double sigma, double* __restrict__ stats,
                                     float2* __restrict__ statsf) {
  const int64_t HW = H * W;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x / 32);
  const int lane = threadIdx.x & 31;
  for (int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32; t < 2 * HW; t += nwarps) {
    const int view = (int)(t / HW);
    const int64_t p = t - view * HW;
    const int64_t x = p % W;
    const double fill = vol[0];  // get_right_cost's fill, featextract.cpp:130
    double mn = kRandMax;
    if (view == 0) {
      const double* r = vol + p * D;
      for (int d = lane; d < D; d += 32) mn = fmin(mn, r[d]);
    } else {
      for (int d = lane; d < D; d += 32) mn = fmin(mn, x + d < W ? vol[(p + d) * D + d] : fill);
    }
    for (int o = 16; o; o >>= 1) mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    double den = 0.0;
    if (view == 0) {
      const double* r = vol + p * D;
      for (int d = lane; d < D; d += 32) den += lik_term(r[d], mn, sigma);
    } else {
      for (int d = lane; d < D; d += 32)
        den += lik_term(x + d < W ? vol[(p + d) * D + d] : fill, mn, sigma);
    }
    den = warp_sum(den);
    if (lane == 0) {
      double* o = stats + ((int64_t)(m * 2 + view) * HW + p) * 2;
      o[0] = mn;
      o[1] = den;
      if (statsf)
        statsf[(int64_t)(m * 2 + view) * HW + p] =
            mn == kRandMax ? make_float2(kRandMaxF, 0.0f) : make_float2((float)mn, (float)(1.0 / den));
    }
  }
}

__global__ void features_kernel(FeatVols fv, const double* __restrict__ stats, int64_t H, int64_t W,
                                int D, float* __restrict__ out) {
  const int64_t HW = H * W;
  GRID_STRIDE(t, HW * D) {
    const int64_t p = t / D;
    const int d = (int)(t - p * D);
    float f[20];
    features_at(fv.v, stats, HW, W, D, p, p % W, d, f);
#pragma unroll
    for (int k = 0; k < 20; k++) out[t * 20 + k] = f[k];
  }
}

__global__ void features_gather_kernel(FeatVols fv, const double* __restrict__ stats, int64_t H,
                                       int64_t W, int D, const int64_t* __restrict__ idx, int64_t n,
                                       float* __restrict__ out) {
  const int64_t HW = H * W, N = HW * D;
  GRID_STRIDE(i, n) {
    int64_t t = idx[i];
    t = t < 0 ? 0 : (t >= N ? N - 1 : t);  // indices are validated on the host; clamp anyway
    const int64_t p = t / D;
    const int d = (int)(t - p * D);
    features_store(fv.v, stats, HW, D, p, p % W, d, out + i * 20, 1);
  }
}

int launch_features_gather(const double* const* vols, const double* stats, int64_t H, int64_t W,
                           int D, const int64_t* idx, int64_t n, float* out, cudaStream_t st) {
  FeatVols fv = {{vols[0], vols[1], vols[2], vols[3]}};
  features_gather_kernel<<<grid_for(n, kBlock), kBlock, 0, st>>>(fv, stats, H, W, D, idx, n, out);
  return check_launch("features_gather");
}

// ---------------------------------------------- float32 row statistics
// The classifier network's row statistics (min, 1/den) in float32 from
// float32 volumes (the learned path never needs the float64 features):
// statsf[(m*2 + view)*HW + p], min = 2^31 and 1/den = 0 where the row holds
// only sentinels.  All four matchers in one launch (blockIdx.y = matcher).
struct VolsF {
  const float* v[4];
};
static __constant__ float kInvSigmaF32[4] = {(float)(1.0 / (2.0 * 8 * 8)), (float)(1.0 / 0.02),
                                             (float)(1.0 / (2.0 * 100 * 100)), (float)(1.0 / (2.0 * 100 * 100))};

__device__ __forceinline__ float2 stats_pair(float mn, float den) {
  return mn == kRandMaxF ? make_float2(kRandMaxF, 0.0f) : make_float2(mn, 1.0f / den);
}

// view 0: one warp per pixel, the pixel's D costs are contiguous
__global__ void stats_f32_left_kernel(VolsF vols, int64_t HW, int D, float2* __restrict__ statsf) {
  const int m = blockIdx.y;
  const float* __restrict__ vol = vols.v[m];
  const float inv_sigma = kInvSigmaF32[m];
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
  const bool vec = (D & 3) == 0 && D <= 512;  // the row as <= 4 float4 per lane, kept in registers
  for (int64_t p = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < HW; p += nw) {
    const float* r = vol + p * D;
    float mn = kRandMaxF, den = 0.0f;
    if (vec) {
      float4 v[4];
      const int nq = D >> 2;
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const int q = lane + 32 * k;
        v[k] = q < nq ? __ldg(reinterpret_cast<const float4*>(r) + q) : make_float4(kRandMaxF, kRandMaxF, kRandMaxF, kRandMaxF);
        mn = fminf(mn, fminf(fminf(v[k].x, v[k].y), fminf(v[k].z, v[k].w)));
      }
      for (int o = 16; o; o >>= 1) mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
#pragma unroll
      for (int k = 0; k < 4; k++) {
        if (lane + 32 * k < nq) {
          const float tx = v[k].x - mn, ty = v[k].y - mn, tz = v[k].z - mn, tw = v[k].w - mn;
          den += (__expf(-(tx * tx) * inv_sigma) + __expf(-(ty * ty) * inv_sigma)) +
                 (__expf(-(tz * tz) * inv_sigma) + __expf(-(tw * tw) * inv_sigma));
        }
      }
    } else {
      for (int d = lane; d < D; d += 32) mn = fminf(mn, __ldg(r + d));
      for (int o = 16; o; o >>= 1) mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
      for (int d = lane; d < D; d += 32) {
        const float t = __ldg(r + d) - mn;
        den += __expf(-(t * t) * inv_sigma);
      }
    }
    for (int o = 16; o; o >>= 1) den += __shfl_xor_sync(0xffffffffu, den, o);
    if (lane == 0) statsf[(int64_t)(m * 2) * HW + p] = stats_pair(mn, den);
  }
}

// view 1: right pixel x' of row y sees C[y, x' + d, d] (the fill C[0,0,0]
// where x' + d >= W, featextract.cpp:115-152).  A CTA owns RS_PIX right
// pixels of one row; for each 32-wide disparity chunk it stages the
// (RS_PIX + 32) x 32 block of the volume the chunk's diagonals cross
// (coalesced along d) and each thread walks its diagonal in shared memory.
constexpr int RS_PIX = 256;

__global__ void __launch_bounds__(RS_PIX) stats_f32_right_kernel(VolsF vols, int64_t H, int64_t W, int D,
                                                                 float2* __restrict__ statsf) {
  __shared__ float tile[(RS_PIX + 32) * 33];
  const int m = blockIdx.y;
  const float* __restrict__ vol = vols.v[m];
  const float fill = __ldg(vol);
  const float inv_sigma = kInvSigmaF32[m];
  const int64_t nxb = (W + RS_PIX - 1) / RS_PIX;
  const int64_t y = blockIdx.x / nxb;
  const int64_t X0 = (blockIdx.x % nxb) * RS_PIX;
  const int tid = threadIdx.x;
  const int64_t xr = X0 + tid;
  float mn = kRandMaxF, den = 0.0f;
  for (int pass = 0; pass < 2; pass++) {
    for (int d0 = 0; d0 < D; d0 += 32) {
      __syncthreads();
      for (int q = tid; q < (RS_PIX + 32) * 32; q += RS_PIX) {
        const int i = q >> 5, j = q & 31;
        const int64_t x = X0 + d0 + i;
        const int d = d0 + j;
        float v = fill;
        if (x < W && d < D) v = __ldg(vol + (y * W + x) * D + d);
        tile[i * 33 + j] = v;
      }
      __syncthreads();
      if (xr < W) {
        const int nj = D - d0 < 32 ? D - d0 : 32;
        if (pass == 0) {
          for (int j = 0; j < nj; j++) mn = fminf(mn, tile[(tid + j) * 33 + j]);
        } else {
          for (int j = 0; j < nj; j++) {
            const float t = tile[(tid + j) * 33 + j] - mn;
            den += __expf(-(t * t) * inv_sigma);
          }
        }
      }
    }
  }
  if (xr < W) statsf[(int64_t)(m * 2 + 1) * H * W + y * W + xr] = stats_pair(mn, den);
}

// view 0 for D a multiple of 4 up to 128: a pixel's row is one float4 per
// lane, the minimum one `redux.sync.min.f32`, and each warp works on two
// pixels at a time; the per-lane sum and the shuffle tree are those of
// stats_f32_left_kernel, so the results are the same bit for bit.
__global__ void __launch_bounds__(256) stats_f32_left_q_kernel(VolsF vols, int64_t HW, int D,
                                                               float2* __restrict__ statsf) {
  const int m = blockIdx.y;
  const float inv_sigma = kInvSigmaF32[m];
  const int lane = threadIdx.x & 31;
  const int nq = D >> 2;  // float4s per row, <= 32
  const bool on = lane < nq;
  const float4* __restrict__ rows = reinterpret_cast<const float4*>(vols.v[m]) + lane;
  float2* __restrict__ out = statsf + (int64_t)(m * 2) * HW;
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
  const float4 big = make_float4(kRandMaxF, kRandMaxF, kRandMaxF, kRandMaxF);
  auto den4 = [&](float4 v, float mn) {
    const float tx = v.x - mn, ty = v.y - mn, tz = v.z - mn, tw = v.w - mn;
    return (__expf(-(tx * tx) * inv_sigma) + __expf(-(ty * ty) * inv_sigma)) +
           (__expf(-(tz * tz) * inv_sigma) + __expf(-(tw * tw) * inv_sigma));
  };
  for (int64_t p = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < HW; p += 2 * nw) {
    const int64_t p2 = p + nw;
    const bool two = p2 < HW;
    const float4 va = on ? __ldg(rows + p * nq) : big;
    const float4 vb = on && two ? __ldg(rows + p2 * nq) : big;
    float ma = fminf(fminf(va.x, va.y), fminf(va.z, va.w));
    float mb = fminf(fminf(vb.x, vb.y), fminf(vb.z, vb.w));
    asm volatile("redux.sync.min.f32 %0, %0, 0xffffffff;" : "+f"(ma));
    asm volatile("redux.sync.min.f32 %0, %0, 0xffffffff;" : "+f"(mb));
    float da = on ? den4(va, ma) : 0.0f, db = on ? den4(vb, mb) : 0.0f;
    for (int o = 16; o; o >>= 1) {
      da += __shfl_xor_sync(0xffffffffu, da, o);
      db += __shfl_xor_sync(0xffffffffu, db, o);
    }
    if (lane == 0) out[p] = stats_pair(ma, da);
    if (lane == 1 && two) out[p2] = stats_pair(mb, db);
  }
}

// view 0 for D = 128 exactly (the headline's disparity count): eight lanes
// per pixel, four pixels per warp at a time, each lane four float4 of its
// pixel's row; the minimum and the denominator reduce over the eight lanes
// in three shuffle steps.  (Its denominator adds in another order than
// stats_f32_left_q_kernel: the same value to float32 rounding.)
__global__ void __launch_bounds__(256) stats_f32_left_g8_kernel(VolsF vols, int64_t HW,
                                                                float2* __restrict__ statsf) {
  const int m = blockIdx.y;
  const float inv_sigma = kInvSigmaF32[m];
  const int lane = threadIdx.x & 31, gi = lane >> 3, li = lane & 7;
  const float4* __restrict__ rows = reinterpret_cast<const float4*>(vols.v[m]);
  float2* __restrict__ out = statsf + (int64_t)(m * 2) * HW;
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t p0 = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 4; p0 < HW; p0 += 4 * nw) {
    const int64_t p = p0 + gi;
    const bool on = p < HW;
    float4 v[4];
#pragma unroll
    for (int k = 0; k < 4; k++)
      v[k] = on ? __ldg(rows + p * 32 + li + 8 * k) : make_float4(kRandMaxF, kRandMaxF, kRandMaxF, kRandMaxF);
    float mn = kRandMaxF;
#pragma unroll
    for (int k = 0; k < 4; k++) mn = fminf(mn, fminf(fminf(v[k].x, v[k].y), fminf(v[k].z, v[k].w)));
#pragma unroll
    for (int o = 4; o; o >>= 1) mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    float den = 0.0f;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const float tx = v[k].x - mn, ty = v[k].y - mn, tz = v[k].z - mn, tw = v[k].w - mn;
      den += (__expf(-(tx * tx) * inv_sigma) + __expf(-(ty * ty) * inv_sigma)) +
             (__expf(-(tz * tz) * inv_sigma) + __expf(-(tw * tw) * inv_sigma));
    }
#pragma unroll
    for (int o = 4; o; o >>= 1) den += __shfl_xor_sync(0xffffffffu, den, o);
    if (li == 0 && on) out[p] = stats_pair(mn, den);
  }
}

// view 1 for D a multiple of 4: as stats_f32_right_kernel, the staging
// loads one float4 (4 disparities) per thread and step with 32-bit row
// offsets; the diagonal walk, and so the order of the sums, is unchanged.
__global__ void __launch_bounds__(RS_PIX) stats_f32_right_q_kernel(VolsF vols, int64_t H, int64_t W, int D,
                                                                   float2* __restrict__ statsf) {
  __shared__ float tile[(RS_PIX + 32) * 33];
  const int m = blockIdx.y;
  const float* __restrict__ vol = vols.v[m];
  const float fill = __ldg(vol);
  const float inv_sigma = kInvSigmaF32[m];
  const int64_t nxb = (W + RS_PIX - 1) / RS_PIX;
  const int64_t y = blockIdx.x / nxb;
  const int X0 = (int)((blockIdx.x % nxb) * RS_PIX);
  const int Wi = (int)W;
  const float* __restrict__ rowp = vol + y * W * D;  // C[y, 0, 0]
  const int tid = threadIdx.x;
  const int xr = X0 + tid;
  float mn = kRandMaxF, den = 0.0f;
  for (int pass = 0; pass < 2; pass++) {
    for (int d0 = 0; d0 < D; d0 += 32) {
      __syncthreads();
#pragma unroll
      for (int it = 0; it < (RS_PIX + 32) * 8 / RS_PIX; it++) {
        const int q = tid + it * RS_PIX;
        const int i = q >> 3, j4 = (q & 7) * 4;
        const int x = X0 + d0 + i;
        float4 v = make_float4(fill, fill, fill, fill);
        if (x < Wi && d0 + j4 < D) v = __ldg(reinterpret_cast<const float4*>(rowp + (int64_t)x * D + d0 + j4));
        float* t = tile + i * 33 + j4;
        t[0] = v.x;
        t[1] = v.y;
        t[2] = v.z;
        t[3] = v.w;
      }
      __syncthreads();
      if (xr < Wi) {
        const int nj = D - d0 < 32 ? D - d0 : 32;
        if (pass == 0) {
          for (int j = 0; j < nj; j++) mn = fminf(mn, tile[(tid + j) * 33 + j]);
        } else {
          for (int j = 0; j < nj; j++) {
            const float t = tile[(tid + j) * 33 + j] - mn;
            den += __expf(-(t * t) * inv_sigma);
          }
        }
      }
    }
  }
  if (xr < Wi) statsf[(int64_t)(m * 2 + 1) * H * W + y * W + xr] = stats_pair(mn, den);
}

int launch_feature_stats_f32(const float* const* vols, int64_t H, int64_t W, int D, float2* statsf,
                             cudaStream_t st) {
  const VolsF v = {{vols[0], vols[1], vols[2], vols[3]}};
  const int64_t HW = H * W;
  const int64_t lblocks = (HW + 7) / 8;  // 8 warps per block, one pixel each
  const bool q = D % 4 == 0 && ((uintptr_t)vols[0] | (uintptr_t)vols[1] | (uintptr_t)vols[2] | (uintptr_t)vols[3]) % 16 == 0;
  if (q && D == 128) {
    const int64_t gblocks = (HW + 31) / 32;  // 8 warps per block, four pixels each
    stats_f32_left_g8_kernel<<<dim3((unsigned)(gblocks < 65535 * 16 ? gblocks : 65535 * 16), 4), 256, 0, st>>>(
        v, HW, statsf);
  } else if (q && D <= 128) {
    const int64_t qblocks = (HW + 15) / 16;  // 8 warps per block, two pixels each
    stats_f32_left_q_kernel<<<dim3((unsigned)(qblocks < 65535 * 16 ? qblocks : 65535 * 16), 4), 256, 0, st>>>(
        v, HW, D, statsf);
  } else {
    stats_f32_left_kernel<<<dim3((unsigned)(lblocks < 65535 * 16 ? lblocks : 65535 * 16), 4), 256, 0, st>>>(
        v, HW, D, statsf);
  }
  const int64_t rblocks = H * ((W + RS_PIX - 1) / RS_PIX);
  CBMV_REQUIRE(rblocks < ((int64_t)1 << 31), CBMV_ERANGE, "image too large for the statistics grid");
  if (q && W < ((int64_t)1 << 30))
    stats_f32_right_q_kernel<<<dim3((unsigned)rblocks, 4), RS_PIX, 0, st>>>(v, H, W, D, statsf);
  else
    stats_f32_right_kernel<<<dim3((unsigned)rblocks, 4), RS_PIX, 0, st>>>(v, H, W, D, statsf);
  return check_launch("feature_stats_f32");
}

int launch_feature_stats(const double* const* vols, int64_t H, int64_t W, int D, double* stats,
                         cudaStream_t st, float2* statsf) {
  const int64_t warps = 2 * H * W;
  for (int m = 0; m < 4; m++)
    feature_stats_kernel<<<grid_for(warps * 32, kBlock), kBlock, 0, st>>>(vols[m], m, H, W, D,
                                                                          hSigma[m], stats, statsf);
  return check_launch("feature_stats");
}

}  // namespace cbmv

using namespace cbmv;

#define CHECK_VOL(p, q) CBMV_REQUIRE((p) && (q), CBMV_EINVAL, "null pointer argument")

extern "C" int cbmv_swap_axes(const double* in, int64_t D, int64_t H, int64_t W, double* out,
                              void* stream) {
  CHECK_VOL(in, out);
  CBMV_REQUIRE(D > 0 && H > 0 && W > 0, CBMV_EINVAL, "bad size");
  swap_axes_kernel<<<grid_for(D * H * W, kBlock), kBlock, 0, as_stream(stream)>>>(in, D, H * W, out);
  return check_launch("swap_axes");
}

extern "C" int cbmv_swap_axes_back(const double* in, int64_t H, int64_t W, int64_t D, double* out,
                                   void* stream) {
  CHECK_VOL(in, out);
  CBMV_REQUIRE(D > 0 && H > 0 && W > 0, CBMV_EINVAL, "bad size");
  swap_axes_back_kernel<<<grid_for(D * H * W, kBlock), kBlock, 0, as_stream(stream)>>>(in, H * W, D,
                                                                                      out);
  return check_launch("swap_axes_back");
}

extern "C" int cbmv_get_cost(const double* in, int64_t H, int64_t W, int64_t D, int64_t K,
                             double* out, void* stream) {
  CHECK_VOL(in, out);
  CBMV_REQUIRE(D > 0 && H > 0 && W > 0 && K > 0, CBMV_EINVAL, "bad size");
  get_cost_kernel<<<grid_for(H * W * D, kBlock), kBlock, 0, as_stream(stream)>>>(in, H * W * D, K, out);
  return check_launch("get_cost");
}

extern "C" int cbmv_get_right_cost(const double* C, int64_t H, int64_t W, int64_t D, double* out,
                                   void* stream) {
  CHECK_VOL(C, out);
  CBMV_REQUIRE(D > 0 && H > 0 && W > 0 && C != out, CBMV_EINVAL, "bad size or in-place call");
  shift_kernel<<<grid_for(H * W * D, kBlock), kBlock, 0, as_stream(stream)>>>(C, H, W, D, 1, out);
  return check_launch("get_right_cost");
}

extern "C" int cbmv_get_left_cost(const double* Rv, int64_t H, int64_t W, int64_t D, double* out,
                                  void* stream) {
  CHECK_VOL(Rv, out);
  CBMV_REQUIRE(D > 0 && H > 0 && W > 0 && Rv != out, CBMV_EINVAL, "bad size or in-place call");
  shift_kernel<<<grid_for(H * W * D, kBlock), kBlock, 0, as_stream(stream)>>>(Rv, H, W, D, -1, out);
  return check_launch("get_left_cost");
}

extern "C" int cbmv_extract_ratio(const double* vol, int64_t N, int64_t D, double e, double* out,
                                  void* stream) {
  CHECK_VOL(vol, out);
  CBMV_REQUIRE(N > 0 && D > 0, CBMV_EINVAL, "bad size");
  ratio_kernel<<<grid_for(N * 32, kBlock), kBlock, 0, as_stream(stream)>>>(vol, N, D, e, out);
  return check_launch("extract_ratio");
}

extern "C" int cbmv_extract_likelihood(const double* vol, int64_t N, int64_t D, double sigma,
                                       double* out, void* stream) {
  CHECK_VOL(vol, out);
  CBMV_REQUIRE(N > 0 && D > 0 && sigma > 0, CBMV_EINVAL, "bad size or sigma");
  likelihood_kernel<<<grid_for(N * 32, kBlock), kBlock, 0, as_stream(stream)>>>(vol, N, D, sigma, out);
  return check_launch("extract_likelihood");
}

extern "C" int cbmv_extract_ratio_samples(const double* vol, int64_t N, int64_t D,
                                          const int32_t* samples, double e, double* out,
                                          void* stream) {
  CHECK_VOL(vol, out);
  CBMV_REQUIRE(samples && N > 0 && D > 0, CBMV_EINVAL, "bad argument");
  ratio_samples_kernel<<<grid_for(N * 32, kBlock), kBlock, 0, as_stream(stream)>>>(vol, N, D, samples,
                                                                                  e, out);
  return check_launch("extract_ratio_samples");
}

extern "C" int cbmv_extract_likelihood_samples(const double* vol, int64_t N, int64_t D,
                                               const int32_t* samples, double sigma, double* out,
                                               void* stream) {
  CHECK_VOL(vol, out);
  CBMV_REQUIRE(samples && N > 0 && D > 0 && sigma > 0, CBMV_EINVAL, "bad argument");
  likelihood_samples_kernel<<<grid_for(N * 32, kBlock), kBlock, 0, as_stream(stream)>>>(
      vol, N, D, samples, sigma, out);
  return check_launch("extract_likelihood_samples");
}

extern "C" int cbmv_get_samples(const double* vol, int64_t N, int64_t D, const int32_t* samples,
                                double* out, void* stream) {
  CHECK_VOL(vol, out);
  CBMV_REQUIRE(samples && N > 0 && D > 0, CBMV_EINVAL, "bad argument");
  get_samples_kernel<<<grid_for(3 * N, kBlock), kBlock, 0, as_stream(stream)>>>(vol, N, D, samples, out);
  return check_launch("get_samples");
}

extern "C" int cbmv_generate_labels(int64_t N, int32_t* out, void* stream) {
  CBMV_REQUIRE(out && N > 0, CBMV_EINVAL, "bad argument");
  labels_kernel<<<grid_for(3 * N, kBlock), kBlock, 0, as_stream(stream)>>>(N, out);
  return check_launch("generate_labels");
}

extern "C" int cbmv_generate_d_indices(const int32_t* gt, int64_t N, int maxd, int thr,
                                       uint64_t seed, int32_t* out, void* stream) {
  CBMV_REQUIRE(gt && out && N > 0 && maxd > 0 && thr >= 0, CBMV_EINVAL, "bad argument");
  cudaStream_t st = as_stream(stream);
  int* bad = nullptr;
  CBMV_CUDA(cudaMallocAsync(&bad, sizeof(int), st));
  CBMV_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), st));
  d_indices_kernel<<<grid_for(N, kBlock), kBlock, 0, st>>>(gt, N, maxd, thr, seed, out, bad);
  int rc = check_launch("generate_d_indices");
  int hbad = 0;
  CBMV_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
  CBMV_CUDA(cudaFreeAsync(bad, st));
  CBMV_CUDA(cudaStreamSynchronize(st));
  if (rc) return rc;
  CBMV_REQUIRE(!hbad, CBMV_EINVAL,
               "generate_d_indices: a ground-truth value is outside [0, maxd] or leaves an empty "
               "negative range (gt = maxd - thr - 1)");
  return CBMV_OK;
}

extern "C" int cbmv_features(const double* census, const double* ncc, const double* sob,
                             const double* sad, int64_t H, int64_t W, int D, float* out,
                             void* stream) {
  CBMV_REQUIRE(census && ncc && sob && sad && out, CBMV_EINVAL, "null pointer argument");
  CBMV_REQUIRE(H > 0 && W > 0 && D > 0, CBMV_EINVAL, "bad size");
  cudaStream_t st = as_stream(stream);
  double* stats = nullptr;
  CBMV_CUDA(cudaMallocAsync(&stats, sizeof(double) * 16 * H * W, st));
  const double* vols[4] = {census, ncc, sob, sad};
  int rc = launch_feature_stats(vols, H, W, D, stats, st, nullptr);
  if (!rc) {
    FeatVols fv = {{census, ncc, sob, sad}};
    features_kernel<<<grid_for(H * W * D, kBlock), kBlock, 0, st>>>(fv, stats, H, W, D, out);
    rc = check_launch("features");
  }
  CBMV_CUDA(cudaFreeAsync(stats, st));
  return rc;
}
