// MC-CNN cost optimisation ("post", cpp/post/post.cu), float32 on the device.
//
// The reference keeps its volumes in float64 and does most arithmetic in
// float32; these kernels keep the volumes in float32 and do the same float32
// arithmetic as the reference kernels (comparisons, arm bounds, transition
// penalties, CBCA summation order, subpixel parabola, median, thresholded
// Gaussian).  Where the reference accumulates in float64 (the SGM path
// values and their sum over the four directions) the sums here are float32.
//
// SGM runs one scan direction per launch with one warp per scan line and the
// scan inside the kernel (the reference launches one kernel per scan step,
// 2(W+H) launches per call, post.cu:273-330); each lane holds D/32 path
// values in registers, the minimum over d is a warp-shuffle reduction, and
// the next step's costs are loaded one step ahead.
#include "common.cuh"
#include "post.cuh"

namespace cbmv {
namespace {

constexpr int kBlock = 128;

#define GRID_STRIDE(i, n) \
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

__device__ __forceinline__ void decode(int layout, int64_t t, int64_t H, int64_t W, int64_t D,
                                       int64_t* y, int64_t* x, int64_t* d) {
  if (layout == CBMV_HWD) {
    *d = t % D;
    const int64_t p = t / D;
    *x = p % W;
    *y = p / W;
  } else {
    *x = t % W;
    const int64_t q = t / W;
    *y = q % H;
    *d = q / H;
  }
}

// cross (post.cu:336-396)
__global__ void cross_kernel(const float* __restrict__ x0, int64_t H, int64_t W, int L1, float tau1,
                             float* __restrict__ out) {
  GRID_STRIDE(id, 4 * H * W) {
    const int64_t x = id % W, y = (id / W) % H;
    const int dir = (int)(id / (W * H));
    const int dx = dir == 0 ? -1 : dir == 1 ? 1 : 0;
    const int dy = dir == 2 ? -1 : dir == 3 ? 1 : 0;
    const float c = x0[y * W + x];
    int64_t xx = x + dx, yy = y + dy;
    for (;; xx += dx, yy += dy) {
      if (xx < 0 || xx >= W || yy < 0 || yy >= H) break;
      const int64_t dist = max(llabs(xx - x), llabs(yy - y));
      if (dist == 1) continue;
      if (fabsf(c - x0[yy * W + xx]) >= tau1) break;  // rule 1
      if (dist >= L1) break;                          // rule 2
    }
    out[id] = (float)(dir <= 1 ? xx : yy);
  }
}

// Absolute differences of neighbouring pixels of a normalised image:
// gh[y][x] = |I[y][x] - I[y][x-1]|, gv[y][x] = |I[y][x] - I[y-1][x]| (0 on
// the first column / row).  SGM's image terms D1 and D2 (post.cu:230-237)
// are exactly these values (|a - b| == |b - a| in IEEE arithmetic).
__global__ void grad_kernel(const float* __restrict__ img, int64_t H, int64_t W,
                            float* __restrict__ gh, float* __restrict__ gv) {
  GRID_STRIDE(p, H * W) {
    const int64_t y = p / W, x = p - y * W;
    const float c = img[p];
    gh[p] = x > 0 ? fabsf(c - img[p - 1]) : 0.0f;
    gv[p] = y > 0 ? fabsf(c - img[p - W]) : 0.0f;
  }
}

// sgm2 (post.cu:178-261) for all four scan directions in one launch (one
// scan routine, the direction a run-time argument: a single copy of the
// code keeps the instruction cache warm across the four directions): one
// warp per scan line (the 2H horizontal and 2W vertical lines run
// concurrently, each direction writing its path costs to its own volume),
// lane = d (mod 32), KPL disparities per lane.  The scan runs inside the
// kernel; the step's costs, D1 and the per-d D2 do not depend on the
// recursion and are loaded PF steps ahead from a register ring.
template <int KPL, int PF, bool FULL>
__device__ __noinline__ void sgm_scan(const SgmGrad& g, const float* __restrict__ in, int H, int W, int D,
                                      const SgmParams& sp, int line, float* __restrict__ out, const int DIR) {
  const int lane = threadIdx.x & 31;
  const int nsteps = DIR <= 1 ? W : H;
  const int dx = DIR == 0 ? 1 : DIR == 1 ? -1 : 0;
  const float inf = __int_as_float(0x7f800000);
  // penalties of post.cu:239-248; the alpha1 split of :252/:255 applies to
  // the d-1 term in direction 2 and to the d+1 term in direction 3
  const float p1[3] = {sp.pi1, sp.pi1 / (sp.q1 * sp.q2), sp.pi1 / sp.q1};
  const float p2[3] = {sp.pi2, sp.pi2 / (sp.q1 * sp.q2), sp.pi2 / sp.q1};
  float p1lo[3], p1hi[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    p1lo[c] = DIR == 2 ? p1[c] / sp.alpha1 : p1[c];
    p1hi[c] = DIR == 3 ? p1[c] / sp.alpha1 : p1[c];
  }
  const float* gl = DIR <= 1 ? g.lh : g.lv;
  const float* gr = DIR <= 1 ? g.rh : g.rv;
  // the difference to the previous pixel of the scan sits at the later of
  // the two pixels in the neighbour-difference images
  const int gshift = DIR == 1 ? 1 : DIR == 3 ? W : 0;
  // step s visits pixel p0 + s * pstep, column x0 + s * dx
  const int64_t p0 = DIR == 0 ? (int64_t)line * W
                   : DIR == 1 ? (int64_t)line * W + W - 1
                   : DIR == 2 ? (int64_t)line
                              : (int64_t)(H - 1) * W + line;
  const int64_t pstep = DIR == 0 ? 1 : DIR == 1 ? -1 : DIR == 2 ? (int64_t)W : -(int64_t)W;
  const int x0 = DIR == 0 ? 0 : DIR == 1 ? W - 1 : line;
  // post.cu:232-237: D2 = 10 when the matching pixel xx = x + d*direction
  // or its predecessor xx - dx leaves the image, i.e. unless
  // max(0, dx) <= xx < min(W, W + dx)
  const int s = sp.direction;
  const int xlo = max(0, dx);
  const unsigned xspan = (unsigned)(min(W, W + dx) - xlo);

  struct Step {
    float cost[KPL], d2[KPL];
    float d1;
  };
  auto load = [&](int step, Step& st) {
    const int64_t ind2 = p0 + step * pstep;
    const int xl = x0 + step * dx + lane * s - xlo;  // xx - xlo of this lane's d = lane
    const float* src = in + ind2 * D + lane;
    const float* grp = gr + ind2 + gshift + lane * s;
    st.d1 = step > 0 ? gl[ind2 + gshift] : 0.0f;
#pragma unroll
    for (int k = 0; k < KPL; k++) {
      const bool dk = FULL || lane + 32 * k < D;
      st.cost[k] = dk ? src[32 * k] : inf;
      const bool inside = (unsigned)(xl + 32 * k * s) < xspan;
      st.d2[k] = (step > 0 && dk && inside) ? grp[32 * k * s] : 10.0f;
    }
  };
  float prev[KPL];
  Step ring[PF];
#pragma unroll
  for (int i = 0; i < PF; i++)
    if (i < nsteps) load(i, ring[i]);
  for (int s0 = 0; s0 < nsteps; s0 += PF) {
#pragma unroll
    for (int i = 0; i < PF; i++) {
      const int step = s0 + i;
      if (step >= nsteps) break;
      const Step cur = ring[i];
      if (step + PF < nsteps) load(step + PF, ring[i]);
      float L[KPL];
      if (step == 0) {
#pragma unroll
        for (int k = 0; k < KPL; k++) L[k] = cur.cost[k];
      } else {
        float mn = prev[0];
#pragma unroll
        for (int k = 1; k < KPL; k++) mn = fminf(mn, prev[k]);
#pragma unroll
        for (int o = 16; o; o >>= 1) mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        const bool d1lo = cur.d1 < sp.tau_so, d1hi = cur.d1 > sp.tau_so;
        // class 0 (both gradients below tau) or 1 (both above) when the step's
        // D1 allows it and D2 agrees, else class 2
        const float a2 = d1lo ? p2[0] : p2[1], a1lo = d1lo ? p1lo[0] : p1lo[1],
                    a1hi = d1lo ? p1hi[0] : p1hi[1];
#pragma unroll
        for (int k = 0; k < KPL; k++) {
          const int d = lane + 32 * k;
          // neighbours d-1 and d+1 of the previous step: lane 31 hands lane 0
          // its value of the previous disparity block, lane 0 hands lane 31
          // its value of the next one
          const float up = lane == 31 ? prev[k > 0 ? k - 1 : 0] : prev[k];
          const float dn = lane == 0 ? prev[k + 1 < KPL ? k + 1 : k] : prev[k];
          const float lo = __shfl_sync(0xffffffffu, up, (lane + 31) & 31);
          const float hi = __shfl_sync(0xffffffffu, dn, (lane + 1) & 31);
          const float D2 = cur.d2[k];
          const bool ca = d1lo ? D2 < sp.tau_so : (d1hi && D2 > sp.tau_so);
          float cost = fminf(prev[k], mn + (ca ? a2 : p2[2]));
          if (d - 1 >= 0) cost = fminf(cost, lo + (ca ? a1lo : p1lo[2]));
          if (d + 1 < D) cost = fminf(cost, hi + (ca ? a1hi : p1hi[2]));
          L[k] = (FULL || d < D) ? cur.cost[k] + cost - mn : inf;
        }
      }
      float* dst = out + (p0 + step * pstep) * D + lane;
#pragma unroll
      for (int k = 0; k < KPL; k++) {
        if (FULL || lane + 32 * k < D) dst[32 * k] = L[k];
        prev[k] = L[k];
      }
    }
  }
}

// The same scan with each lane holding KPL CONSECUTIVE disparities, d =
// KPL * lane + k (KPL a multiple of 4, D a multiple of 4): a step's path
// costs are KPL/4 float4 loads and stores per lane, the d-1 / d+1
// neighbours are in the lane's own registers except at its two ends (two
// shuffles per step instead of two per register), and the minimum over d
// is one `redux.sync.min.f32`.  The matching direction S (+-1) and FULL
// (D == 32 * KPL) are compile-time, the step's addresses advance by
// constant strides, and step 0 (whose path cost is its cost) loads no
// image terms.  Per element the arithmetic and its order are those of
// sgm_scan, so the results are the same bit for bit.
template <int KPL, int PF, bool FULL, int S>
__device__ __noinline__ void sgm_scan_c(const SgmGrad& g, const float* __restrict__ in, int H, int W, int D,
                                        const SgmParams& sp, int line, float* __restrict__ out, const int DIR) {
  static_assert(KPL % 4 == 0, "float4 path costs");
  constexpr int NV = KPL / 4;
  const int lane = threadIdx.x & 31;
  const int nsteps = DIR <= 1 ? W : H;
  const int dx = DIR == 0 ? 1 : DIR == 1 ? -1 : 0;
  const float inf = __int_as_float(0x7f800000);
  const float p1[3] = {sp.pi1, sp.pi1 / (sp.q1 * sp.q2), sp.pi1 / sp.q1};
  const float p2[3] = {sp.pi2, sp.pi2 / (sp.q1 * sp.q2), sp.pi2 / sp.q1};
  float p1lo[3], p1hi[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    p1lo[c] = DIR == 2 ? p1[c] / sp.alpha1 : p1[c];
    p1hi[c] = DIR == 3 ? p1[c] / sp.alpha1 : p1[c];
  }
  const float* gl = DIR <= 1 ? g.lh : g.lv;
  const float* gr = DIR <= 1 ? g.rh : g.rv;
  const int gshift = DIR == 1 ? 1 : DIR == 3 ? W : 0;
  const int64_t p0 = DIR == 0 ? (int64_t)line * W
                   : DIR == 1 ? (int64_t)line * W + W - 1
                   : DIR == 2 ? (int64_t)line
                              : (int64_t)(H - 1) * W + line;
  const int64_t pstep = DIR == 0 ? 1 : DIR == 1 ? -1 : DIR == 2 ? (int64_t)W : -(int64_t)W;
  const int x0 = DIR == 0 ? 0 : DIR == 1 ? W - 1 : line;
  const int xlo = max(0, dx);
  const unsigned xspan = (unsigned)(min(W, W + dx) - xlo);
  const int d0 = KPL * lane;  // this lane's first disparity
  const bool lane_on = FULL || d0 < D;  // D % 4 == 0: a float4 is all in or all out

  struct Step {
    float cost[KPL], d2[KPL];
    float d1;
  };
  // the next step to load: its pixel's path-cost row, its image terms
  // (D1 at gl[.], D2 at gr[. + d*S]) and the matching column of its first
  // disparity relative to the span where D2 exists
  const float* lsrc = in + p0 * D + d0;
  const float* lgl = gl + p0 + gshift;
  const float* lgr = gr + p0 + gshift + d0 * S;
  int lxl = x0 + d0 * S - xlo;
  const int64_t vstride = pstep * D;
  auto load_costs = [&](Step& st) {
    const float4* src = reinterpret_cast<const float4*>(lsrc);
#pragma unroll
    for (int v = 0; v < NV; v++) {
      const bool on = lane_on && (FULL || d0 + 4 * v < D);
      const float4 c = on ? src[v] : make_float4(inf, inf, inf, inf);
      st.cost[4 * v] = c.x;
      st.cost[4 * v + 1] = c.y;
      st.cost[4 * v + 2] = c.z;
      st.cost[4 * v + 3] = c.w;
    }
    lsrc += vstride;
  };
  // a step >= 1: costs, D1 and the per-d D2 (10 where the matching pixel
  // or its predecessor leaves the image, post.cu:232-237)
  auto load = [&](Step& st) {
    load_costs(st);
    st.d1 = *lgl;
#pragma unroll
    for (int k = 0; k < KPL; k++) {
      const bool inside = (FULL || d0 + k < D) && (unsigned)(lxl + k * S) < xspan;
      st.d2[k] = inside ? lgr[k * S] : 10.0f;
    }
    lgl += pstep;
    lgr += pstep;
    lxl += dx;
  };
  float prev[KPL];
  Step ring[PF];
  {
    // step 0: the path cost is the cost
    Step st0;
    load_costs(st0);
    lgl += pstep;
    lgr += pstep;
    lxl += dx;
#pragma unroll
    for (int k = 0; k < KPL; k++) prev[k] = st0.cost[k];
    float4* dst = reinterpret_cast<float4*>(out + p0 * D + d0);
#pragma unroll
    for (int v = 0; v < NV; v++)
      if (lane_on && (FULL || d0 + 4 * v < D))
        dst[v] = make_float4(prev[4 * v], prev[4 * v + 1], prev[4 * v + 2], prev[4 * v + 3]);
  }
#pragma unroll
  for (int i = 0; i < PF; i++)
    if (1 + i < nsteps) load(ring[i]);
  float* ldst = out + (p0 + pstep) * D + d0;
  for (int s0 = 1; s0 < nsteps; s0 += PF) {
#pragma unroll
    for (int i = 0; i < PF; i++) {
      const int step = s0 + i;
      if (step >= nsteps) break;
      const Step cur = ring[i];
      if (step + PF < nsteps) load(ring[i]);
      float m = fminf(fminf(prev[0], prev[1]), fminf(prev[2], prev[3]));
#pragma unroll
      for (int k = 4; k < KPL; k++) m = fminf(m, prev[k]);
      float mn;
      asm volatile("redux.sync.min.f32 %0, %1, 0xffffffff;" : "=f"(mn) : "f"(m));
      // the neighbours across the lane's ends: d0 - 1 from the previous
      // lane's last register, d0 + KPL from the next lane's first
      const float lo0 = __shfl_up_sync(0xffffffffu, prev[KPL - 1], 1);
      const float hiL = __shfl_down_sync(0xffffffffu, prev[0], 1);
      const bool d1lo = cur.d1 < sp.tau_so, d1hi = cur.d1 > sp.tau_so;
      const float a2 = d1lo ? p2[0] : p2[1], a1lo = d1lo ? p1lo[0] : p1lo[1], a1hi = d1lo ? p1hi[0] : p1hi[1];
      float L[KPL];
#pragma unroll
      for (int k = 0; k < KPL; k++) {
        const int d = d0 + k;
        const float lo = k > 0 ? prev[k - 1] : lo0;
        const float hi = k + 1 < KPL ? prev[k + 1] : hiL;
        const float D2 = cur.d2[k];
        const bool ca = d1lo ? D2 < sp.tau_so : (d1hi && D2 > sp.tau_so);
        float cost = fminf(prev[k], mn + (ca ? a2 : p2[2]));
        if (k > 0 || d - 1 >= 0) cost = fminf(cost, lo + (ca ? a1lo : p1lo[2]));
        if (FULL ? (k + 1 < KPL || lane < 31) : d + 1 < D) cost = fminf(cost, hi + (ca ? a1hi : p1hi[2]));
        L[k] = (FULL || d < D) ? cur.cost[k] + cost - mn : inf;
      }
      float4* dst = reinterpret_cast<float4*>(ldst);
#pragma unroll
      for (int v = 0; v < NV; v++)
        if (lane_on && (FULL || d0 + 4 * v < D)) dst[v] = make_float4(L[4 * v], L[4 * v + 1], L[4 * v + 2], L[4 * v + 3]);
      ldst += vstride;
#pragma unroll
      for (int k = 0; k < KPL; k++) prev[k] = L[k];
    }
  }
}

template <int KPL, int PF, bool FULL, int S>
__global__ void __launch_bounds__(128) sgm4c_kernel(SgmGrad g, const float* __restrict__ in, int H, int W,
                                                    int D, SgmParams sp, SgmOut o) {
  const int warp = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  int dir = -1, line = 0;
  if (warp < H) {
    dir = 0;
    line = warp;
  } else if (warp < 2 * H) {
    dir = 1;
    line = warp - H;
  } else if (warp < 2 * H + W) {
    dir = 2;
    line = warp - 2 * H;
  } else if (warp < 2 * H + 2 * W) {
    dir = 3;
    line = warp - 2 * H - W;
  }
  if (dir >= 0) sgm_scan_c<KPL, PF, FULL, S>(g, in, H, W, D, sp, line, o.dir[dir], dir);
}

template <int KPL, int PF, bool FULL>
__global__ void __launch_bounds__(128) sgm4_kernel(SgmGrad g, const float* __restrict__ in, int H,
                                                   int W, int D, SgmParams sp, SgmOut o) {
  const int warp = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  int dir = -1, line = 0;
  if (warp < H) {
    dir = 0;
    line = warp;
  } else if (warp < 2 * H) {
    dir = 1;
    line = warp - H;
  } else if (warp < 2 * H + W) {
    dir = 2;
    line = warp - 2 * H;
  } else if (warp < 2 * H + 2 * W) {
    dir = 3;
    line = warp - 2 * H - W;
  }
  if (dir >= 0) sgm_scan<KPL, PF, FULL>(g, in, H, W, D, sp, line, o.dir[dir], dir);
}

// out = base + (((L0 + L1) + L2) + L3) * scale over n elements (base may be
// out itself, or null for 0): the four directions summed as post.cu
// sgm_w adds them (directions in order 0..3).
__global__ void sgm_combine_kernel(SgmOut o, int64_t n, const float* base, float scale,
                                   float* out) {
  GRID_STRIDE(i, n) {
    const float s = ((o.dir[0][i] + o.dir[1][i]) + o.dir[2][i]) + o.dir[3][i];
    out[i] = base ? base[i] + s * scale : s * scale;
  }
}

// cbca (post.cu:399-450), any layout.
__global__ void cbca_kernel(const float* __restrict__ lc, const float* __restrict__ rc,
                            const float* __restrict__ in, int64_t H, int64_t W, int64_t D,
                            int layout, int direction, float* __restrict__ out) {
  GRID_STRIDE(id, H * W * D) {
    int64_t y, x, d;
    decode(layout, id, H, W, D, &y, &x, &d);
    const int64_t xm = x + d * direction;
    if (xm < 0 || xm >= W) {
      out[id] = in[id];
      continue;
    }
    const int yy_s = (int)fmaxf(lc[(2 * H + y) * W + x], rc[(2 * H + y) * W + xm]);
    const int yy_t = (int)fminf(lc[(3 * H + y) * W + x], rc[(3 * H + y) * W + xm]);
    const float dd = (float)(d * direction);
    float sum = 0.0f;
    int cnt = 0;
    for (int yy = yy_s + 1; yy < yy_t; yy++) {
      const int xx_s = (int)fmaxf(lc[(0 * H + yy) * W + x], rc[(0 * H + yy) * W + xm] - dd);
      const int xx_t = (int)fminf(lc[(1 * H + yy) * W + x], rc[(1 * H + yy) * W + xm] - dd);
      for (int xx = xx_s + 1; xx < xx_t; xx++) {
        sum += in[vol_index(layout, yy, xx, d, H, W, D)];
        cnt++;
      }
    }
    out[id] = sum / (float)cnt;
  }
}

// cbca on [H,W,D] volumes, tiled: a CTA owns CB_TY x CB_TX pixels x 32
// disparities.  Shared memory holds the input tile with a `halo`-pixel
// border (a pixel's support never reaches beyond its cross arms' interior,
// L1 - 1 pixels) and the tile's cross arms as int16: the left arms of the
// tile columns, and the right arms of every column x + d*direction the tile
// matches against.  Lane = disparity, so the running sums read consecutive
// banks.  Each output is the float sum over its support in the reference's
// order (rows ascending, then columns ascending, from 0; post.cu:415-429)
// divided by the count; a support row that reaches outside the staged tile
// (arms longer than the halo) is summed from global memory instead.
constexpr int CB_TX = 16, CB_TY = 16, CB_TD = 32;

__host__ __device__ constexpr int cbca_rw() { return CB_TX + CB_TD - 1; }

__host__ __device__ inline size_t cbca_smem_bytes(int halo) {
  const int SW = CB_TX + 2 * halo, SH = CB_TY + 2 * halo;
  return (size_t)SW * SH * CB_TD * sizeof(float) +
         (size_t)4 * SH * (CB_TX + cbca_rw()) * sizeof(int16_t);
}

__global__ void __launch_bounds__(256) cbca_hwd_tiled_kernel(
    const float* __restrict__ lc, const float* __restrict__ rc, const float* __restrict__ in,
    int H, int W, int D, int direction, int halo, float* __restrict__ out) {
  extern __shared__ float tile[];  // [SH*SW][CB_TD], then int16 arms
  const int SW = CB_TX + 2 * halo, SH = CB_TY + 2 * halo;
  const int RW = cbca_rw();
  int16_t* sl = reinterpret_cast<int16_t*>(tile + (size_t)SW * SH * CB_TD);  // [4][SH][CB_TX]
  int16_t* sr = sl + 4 * SH * CB_TX;                                         // [4][SH][RW]
  const int ntx = (W + CB_TX - 1) / CB_TX, nty = (H + CB_TY - 1) / CB_TY;
  const int ntd = (D + CB_TD - 1) / CB_TD;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int64_t HW = (int64_t)H * W;
  for (int64_t t = blockIdx.x; t < (int64_t)ntx * nty * ntd; t += gridDim.x) {
    const int td = (int)(t % ntd), tx = (int)((t / ntd) % ntx), ty = (int)(t / ((int64_t)ntd * ntx));
    const int X0 = tx * CB_TX, Y0 = ty * CB_TY, d0 = td * CB_TD;
    const int x0 = X0 - halo, y0 = Y0 - halo;
    // first matched column of the tile: x + d*direction over the tile
    const int xr0 = direction < 0 ? X0 - d0 - (CB_TD - 1) : X0 + d0;
    __syncthreads();
    for (int q = warp; q < SW * SH; q += nwarp) {
      const int yy = y0 + q / SW, xx = x0 + q % SW, d = d0 + lane;
      float v = 0.0f;
      if (yy >= 0 && yy < H && xx >= 0 && xx < W && d < D) v = __ldg(in + ((int64_t)yy * W + xx) * D + d);
      tile[q * CB_TD + lane] = v;
    }
    for (int q = threadIdx.x; q < 4 * SH * CB_TX; q += blockDim.x) {
      const int a = q / (SH * CB_TX), r = (q / CB_TX) % SH, c = q % CB_TX;
      const int yy = y0 + r, xx = X0 + c;
      sl[q] = (yy >= 0 && yy < H && xx < W) ? (int16_t)__ldg(lc + a * HW + (int64_t)yy * W + xx) : 0;
    }
    for (int q = threadIdx.x; q < 4 * SH * RW; q += blockDim.x) {
      const int a = q / (SH * RW), r = (q / RW) % SH, c = q % RW;
      const int yy = y0 + r, xx = xr0 + c;
      sr[q] = (yy >= 0 && yy < H && xx >= 0 && xx < W) ? (int16_t)__ldg(rc + a * HW + (int64_t)yy * W + xx) : 0;
    }
    __syncthreads();
    const int d = d0 + lane;
    const int dd = d * direction;
    for (int q = warp; q < CB_TX * CB_TY; q += nwarp) {
      const int cy = q / CB_TX, cx = q % CB_TX;
      const int y = Y0 + cy, x = X0 + cx;
      if (y >= H || x >= W || d >= D) continue;
      const int64_t id = ((int64_t)y * W + x) * D + d;
      const int xm = x + dd;
      if (xm < 0 || xm >= W) {
        out[id] = in[id];
        continue;
      }
      const int cm = xm - xr0;  // column of xm in the staged right arms
      const int ry = cy + halo;
      const int yy_s = max((int)sl[(2 * SH + ry) * CB_TX + cx], (int)sr[(2 * SH + ry) * RW + cm]);
      const int yy_t = min((int)sl[(3 * SH + ry) * CB_TX + cx], (int)sr[(3 * SH + ry) * RW + cm]);
      float sum = 0.0f;
      int cnt = 0;
      for (int yy = yy_s + 1; yy < yy_t; yy++) {
        const int r = yy - y0;
        int xx_s, xx_t;
        const bool row_in = r >= 0 && r < SH;
        if (row_in) {
          xx_s = max((int)sl[r * CB_TX + cx], (int)sr[r * RW + cm] - dd);
          xx_t = min((int)sl[(SH + r) * CB_TX + cx], (int)sr[(SH + r) * RW + cm] - dd);
        } else {
          xx_s = (int)fmaxf(lc[(int64_t)yy * W + x], rc[(int64_t)yy * W + xm] - (float)dd);
          xx_t = (int)fminf(lc[HW + (int64_t)yy * W + x], rc[HW + (int64_t)yy * W + xm] - (float)dd);
        }
        if (row_in && xx_s + 1 >= x0 && xx_t - 1 < x0 + SW) {
          const float* rowp = tile + ((size_t)r * SW - x0) * CB_TD + lane;
          for (int xx = xx_s + 1; xx < xx_t; xx++) sum += rowp[xx * CB_TD];
        } else {
          for (int xx = xx_s + 1; xx < xx_t; xx++) sum += in[((int64_t)yy * W + xx) * D + d];
        }
        cnt += max(xx_t - xx_s - 1, 0);
      }
      out[id] = sum / (float)cnt;
    }
  }
}

// cbca on [H,W,D] volumes in separable form, the row-then-column
// decomposition of integral-image aggregation: the support row of row yy
// for (x, d) is the same interval for every centre row y (it depends on the
// arms of (yy, x) and (yy, x + d*direction) only), so
//   R(yy, x, d) = sum of the support row,   C(yy, x, d) = its length,
//   out(y, x, d) = sum over the support rows yy of R / sum of C.
// A CTA owns CS_TY x CS_TX pixels x 32 disparities (lane = disparity): it
// forms R and C for its rows and HALO rows above and below into shared
// memory, then the column sums.  Both sums run over fixed 2*HALO+1 taps,
// masked to the support, in ascending order, from register windows (a tile
// row's inputs; a column's R and C); with arms of at most
// HALO = L1 - 1 pixels every support element is within the taps.  The
// result differs from the reference's single running float sum
// (post.cu:415-429) by rounding only.
constexpr int CS_TX = 8, CS_TD = 32;

template <int HALO, int CS_TY>
constexpr size_t cbca_sep_smem_bytes() {
  return (size_t)(CS_TY + 2 * HALO) * CS_TX * CS_TD * (sizeof(float) + sizeof(uint8_t));
}

template <int HALO, int CS_TY>
__global__ void __launch_bounds__(256, 4) cbca_hwd_sep_kernel(
    const float* __restrict__ lc, const float* __restrict__ rc, const float* __restrict__ in, int H, int W,
    int D, int direction, float* __restrict__ out) {
  constexpr int SR = CS_TY + 2 * HALO;   // rows of R: the tile's and HALO above and below
  constexpr int NV = CS_TX + 2 * HALO;   // input columns a tile row needs
  constexpr int G = 8;                   // output rows per column-sum window
  static_assert(CS_TX == 8 && CS_TY % G == 0, "one warp per tile column");
  extern __shared__ float sR[];                                       // [SR][CS_TX][CS_TD]
  uint8_t* sC = reinterpret_cast<uint8_t*>(sR + SR * CS_TX * CS_TD);  // [SR][CS_TX][CS_TD]
  const int ntd = (D + CS_TD - 1) / CS_TD, ntx = (W + CS_TX - 1) / CS_TX;
  const int64_t t = blockIdx.x;
  const int td = (int)(t % ntd), tx = (int)((t / ntd) % ntx), ty = (int)(t / ((int64_t)ntd * ntx));
  const int X0 = tx * CS_TX, Y0 = ty * CS_TY;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int d = td * CS_TD + lane, dd = d * direction;
  const bool dok = d < D;
  const int64_t HW = (int64_t)H * W;
  // 1. row sums: warp w forms R and C of tile rows w, w + 8, ... for all CS_TX columns
  //    from the NV input values of its row, held in registers
  for (int r = warp; r < SR; r += 8) {
    const int yy = Y0 - HALO + r;
    const bool rok = yy >= 0 && yy < H && dok;
    float v[NV];
    const int64_t o = (int64_t)(rok ? yy : 0) * W;
    const float* row = in + o * D + d;
#pragma unroll
    for (int j = 0; j < NV; j++) {
      const int xx = X0 - HALO + j;
      v[j] = (rok && xx >= 0 && xx < W) ? __ldg(row + (int64_t)xx * D) : 0.0f;
    }
#pragma unroll
    for (int c = 0; c < CS_TX; c++) {
      const int x = X0 + c, xm = x + dd;
      float sum = 0.0f;
      int cnt = 0;
      if (rok && x < W && xm >= 0 && xm < W) {
        // support row of (yy, x, d) in tap coordinates: ks < k < kt
        const int ks = max((int)__ldg(lc + o + x), (int)__ldg(rc + o + xm) - dd) - x;
        const int kt = min((int)__ldg(lc + HW + o + x), (int)__ldg(rc + HW + o + xm) - dd) - x;
#pragma unroll
        for (int k = -HALO; k <= HALO; k++)
          if (k > ks && k < kt) sum += v[c + HALO + k];
        cnt = max(kt - ks - 1, 0);
      }
      sR[(r * CS_TX + c) * CS_TD + lane] = sum;
      sC[(r * CS_TX + c) * CS_TD + lane] = (uint8_t)cnt;
    }
  }
  __syncthreads();
  // 2. column sums: warp c owns tile column c; G output rows at a time from a
  //    register window of G + 2*HALO rows of R and C
  const int c = warp, x = X0 + c, xm = x + dd;
  if (x >= W || !dok) return;
  const bool xok = xm >= 0 && xm < W;
#pragma unroll 1
  for (int g0 = 0; g0 < CS_TY; g0 += G) {
    float wr[G + 2 * HALO];
    int wc[G + 2 * HALO];
#pragma unroll
    for (int j = 0; j < G + 2 * HALO; j++) {
      const int i = ((g0 + j) * CS_TX + c) * CS_TD + lane;
      wr[j] = sR[i];
      wc[j] = sC[i];
    }
#pragma unroll
    for (int cy = 0; cy < G; cy++) {
      const int y = Y0 + g0 + cy;
      if (y >= H) break;
      const int64_t o = (int64_t)y * W;
      const int64_t id = (o + x) * D + d;
      if (!xok) {
        out[id] = __ldg(in + id);
        continue;
      }
      const int ks = max((int)__ldg(lc + 2 * HW + o + x), (int)__ldg(rc + 2 * HW + o + xm)) - y;
      const int kt = min((int)__ldg(lc + 3 * HW + o + x), (int)__ldg(rc + 3 * HW + o + xm)) - y;
      float sum = 0.0f;
      int cnt = 0;
#pragma unroll
      for (int k = -HALO; k <= HALO; k++)
        if (k > ks && k < kt) {
          sum += wr[cy + HALO + k];
          cnt += wc[cy + HALO + k];
        }
      out[id] = sum / (float)cnt;
    }
  }
}

template <int HALO, int TY>
int launch_cbca_sep_ht(const float* lc, const float* rc, const float* in, int64_t H, int64_t W, int D,
                       int direction, float* out, cudaStream_t st) {
  constexpr size_t smem = cbca_sep_smem_bytes<HALO, TY>();
  CBMV_CUDA(cudaFuncSetAttribute(cbca_hwd_sep_kernel<HALO, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  const int64_t tiles = (int64_t)((W + CS_TX - 1) / CS_TX) * ((H + TY - 1) / TY) * ((D + CS_TD - 1) / CS_TD);
  cbca_hwd_sep_kernel<HALO, TY><<<(unsigned)tiles, 256, smem, st>>>(lc, rc, in, (int)H, (int)W, D, direction, out);
  return check_launch("cbca_sep");
}

// tile rows 16 or 32 (the results do not depend on them)
template <int HALO>
int launch_cbca_sep_h(const float* lc, const float* rc, const float* in, int64_t H, int64_t W, int D,
                      int direction, float* out, cudaStream_t st, int rows) {
  if (rows == 16) return launch_cbca_sep_ht<HALO, 16>(lc, rc, in, H, W, D, direction, out, st);
  return launch_cbca_sep_ht<HALO, 32>(lc, rc, in, H, W, D, direction, out, st);
}

// The separable CBCA with its supports precomputed: the support of every
// (y, x, d) depends on the cross arms only, so the cbca_i2 passes of one
// post share it.  One 32-bit word per (y, x, d), for arms of at most
// kMaskHalo pixels:
//   bits  0..10  taps k = -5..5 of its support row (bit k + 5),
//   bits 11..21  taps of its support column,
//   bits 22..28  the number of pixels in its support (at most 121),
//   bit  31      x + d*direction is outside the image (the input is copied).
// The passes then sum the same taps in the same ascending order as
// cbca_hwd_sep_kernel, so the results are bit-identical to it.
constexpr int kMaskHalo = kCbcaMaskMaxHalo;
constexpr uint32_t kMaskCopy = 1u << 31;

// Relative arms of one pixel packed as four int8: arm a minus the pixel's
// x (arms 0, 1) or y (arms 2, 3).  cross_kernel's arms lie within L1 of
// their pixel; anything beyond 127 is clamped (the taps stop at +-5 anyway).
__device__ __forceinline__ int clamp_i8(int v) { return min(max(v, -128), 127); }
__device__ __forceinline__ uint32_t pack_rel_arms(const float* __restrict__ c, int64_t HW, int64_t o, int x, int y) {
  const int a0 = clamp_i8((int)__ldg(c + o) - x), a1 = clamp_i8((int)__ldg(c + HW + o) - x);
  const int a2 = clamp_i8((int)__ldg(c + 2 * HW + o) - y), a3 = clamp_i8((int)__ldg(c + 3 * HW + o) - y);
  return (uint32_t)(a0 & 0xFF) | ((uint32_t)(a1 & 0xFF) << 8) | ((uint32_t)(a2 & 0xFF) << 16) |
         ((uint32_t)(a3 & 0xFF) << 24);
}
template <int B>
__device__ __forceinline__ int rel_arm(uint32_t w) {
  return (int)((int32_t)(w << (24 - 8 * B)) >> 24);
}

template <int CS_TY>
__global__ void __launch_bounds__(256) cbca_mask_build_kernel(const float* __restrict__ lc,
                                                              const float* __restrict__ rc, int H, int W, int D,
                                                              int direction, uint32_t* __restrict__ mask) {
  constexpr int HALO = kMaskHalo;
  constexpr int SR = CS_TY + 2 * HALO;
  constexpr int NXM = CS_TX + CS_TD - 1;  // matching columns x + d * direction of the tile
  // support-row lengths of rows 0..SR-1 in sP[1..SR], then (in place)
  // their prefix sums over the rows: sP[r] = lengths of rows 0..r-1
  __shared__ uint16_t sP[SR + 1][CS_TX][CS_TD];
  __shared__ uint16_t sH[CS_TY][CS_TX][CS_TD];  // support-row taps of the tile's own rows
  __shared__ uint32_t sAL[SR][CS_TX];           // packed relative arms, left view at (yy, x)
  __shared__ uint32_t sAR[SR][NXM];             // right view at (yy, xm)
  const int ntd = (D + CS_TD - 1) / CS_TD, ntx = (W + CS_TX - 1) / CS_TX;
  const int64_t t = blockIdx.x;
  const int td = (int)(t % ntd), tx = (int)((t / ntd) % ntx), ty = (int)(t / ((int64_t)ntd * ntx));
  const int X0 = tx * CS_TX, Y0 = ty * CS_TY;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int d = td * CS_TD + lane, dd = d * direction;
  const bool dok = d < D;
  const int64_t HW = (int64_t)H * W;
  // the tile's matching columns: X0 + d * direction over its disparities
  const int xm_lo = direction > 0 ? X0 + td * CS_TD : X0 - (td * CS_TD + CS_TD - 1);
  // 0. the arms the tile needs, converted once per pixel (rows and columns
  //    outside the image are never read back)
  for (int q = threadIdx.x; q < SR * (CS_TX + NXM); q += blockDim.x) {
    const int r = q / (CS_TX + NXM), j = q - r * (CS_TX + NXM);
    const int yy = Y0 - HALO + r;
    if (yy < 0 || yy >= H) continue;
    if (j < CS_TX) {
      const int x = X0 + j;
      if (x < W) sAL[r][j] = pack_rel_arms(lc, HW, (int64_t)yy * W + x, x, yy);
    } else {
      const int xm = xm_lo + (j - CS_TX);
      if (xm >= 0 && xm < W) sAR[r][j - CS_TX] = pack_rel_arms(rc, HW, (int64_t)yy * W + xm, xm, yy);
    }
  }
  __syncthreads();
  // 1. support rows of the tile's rows and HALO rows above and below
  for (int r = warp; r < SR; r += 8) {
    const int yy = Y0 - HALO + r;
    const bool rok = yy >= 0 && yy < H && dok;
#pragma unroll
    for (int c = 0; c < CS_TX; c++) {
      const int x = X0 + c, xm = x + dd;
      int cnt = 0;
      uint32_t hm = 0;
      if (rok && x < W && xm >= 0 && xm < W) {
        const uint32_t wl = sAL[r][c], wr = sAR[r][xm - xm_lo];
        // max(lc0[x], rc0[xm] - dd) - x and min(lc1[x], rc1[xm] - dd) - x
        const int ks = max(rel_arm<0>(wl), rel_arm<0>(wr));
        const int kt = min(rel_arm<1>(wl), rel_arm<1>(wr));
        cnt = max(kt - ks - 1, 0);
        const int lo = max(ks + 1, -HALO), hi = min(kt - 1, HALO);
        if (hi >= lo) hm = ((1u << (hi - lo + 1)) - 1u) << (lo + HALO);
      }
      sP[r + 1][c][lane] = (uint16_t)cnt;
      if (r >= HALO && r < HALO + CS_TY) sH[r - HALO][c][lane] = (uint16_t)hm;
    }
  }
  __syncthreads();
  // 2. support columns: warp c owns tile column c; the thread first forms
  //    the prefix sums of its (column, disparity)'s support-row lengths, so
  //    a support of rows lo..hi counts sP[hi + 1] - sP[lo] pixels (exact
  //    integers, the same count as adding them row by row)
  const int c = warp, x = X0 + c, xm = x + dd;
  {
    uint32_t run = 0;
    sP[0][c][lane] = 0;
    for (int r = 1; r <= SR; r++) {
      run += sP[r][c][lane];
      sP[r][c][lane] = (uint16_t)run;
    }
  }
  if (x >= W || !dok) return;
  const bool xok = xm >= 0 && xm < W;
  for (int cy = 0; cy < CS_TY; cy++) {
    const int y = Y0 + cy;
    if (y >= H) break;
    const int64_t id = ((int64_t)y * W + x) * D + d;
    if (!xok) {
      mask[id] = kMaskCopy;
      continue;
    }
    const uint32_t wl = sAL[cy + HALO][c], wr = sAR[cy + HALO][xm - xm_lo];
    // max(lc2[x], rc2[xm]) - y and min(lc3[x], rc3[xm]) - y: the support
    // rows are the taps k with ks < k < kt, within +-HALO
    const int ks = max(rel_arm<2>(wl), rel_arm<2>(wr));
    const int kt = min(rel_arm<3>(wl), rel_arm<3>(wr));
    const int lo = max(ks + 1, -HALO), hi = min(kt - 1, HALO);
    uint32_t vm = 0, cnt = 0;
    if (hi >= lo) {
      vm = ((1u << (hi - lo + 1)) - 1u) << (lo + HALO);
      cnt = (uint32_t)sP[cy + HALO + hi + 1][c][lane] - (uint32_t)sP[cy + HALO + lo][c][lane];
    }
    mask[id] = (uint32_t)sH[cy][c][lane] | (vm << 11) | ((cnt & 0x7Fu) << 22);
  }
}

// One CBCA pass from the precomputed supports (same tiling and summation
// order as cbca_hwd_sep_kernel<kMaskHalo>).
template <int CS_TY>
__global__ void __launch_bounds__(256, 4) cbca_hwd_mask_kernel(const uint32_t* __restrict__ mask,
                                                               const float* __restrict__ in, int H, int W,
                                                               int D, float* __restrict__ out) {
  constexpr int HALO = kMaskHalo;
  constexpr int SR = CS_TY + 2 * HALO;
  constexpr int NV = CS_TX + 2 * HALO;
  constexpr int G = 8;
  static_assert(CS_TX == 8 && CS_TY % G == 0, "one warp per tile column");
  extern __shared__ float sR[];  // [SR][CS_TX][CS_TD]
  const int ntd = (D + CS_TD - 1) / CS_TD, ntx = (W + CS_TX - 1) / CS_TX;
  const int64_t t = blockIdx.x;
  const int td = (int)(t % ntd), tx = (int)((t / ntd) % ntx), ty = (int)(t / ((int64_t)ntd * ntx));
  const int X0 = tx * CS_TX, Y0 = ty * CS_TY;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int d = td * CS_TD + lane;
  const bool dok = d < D;
  // 1. row sums over each (yy, x, d)'s support-row taps
  for (int r = warp; r < SR; r += 8) {
    const int yy = Y0 - HALO + r;
    const bool rok = yy >= 0 && yy < H && dok;
    const int64_t o = (int64_t)(rok ? yy : 0) * W;
    const float* row = in + o * D + d;
    const uint32_t* mrow = mask + o * D + d;
    float v[NV];
#pragma unroll
    for (int j = 0; j < NV; j++) {
      const int xx = X0 - HALO + j;
      v[j] = (rok && xx >= 0 && xx < W) ? __ldg(row + (int64_t)xx * D) : 0.0f;
    }
#pragma unroll
    for (int c = 0; c < CS_TX; c++) {
      const int x = X0 + c;
      const uint32_t hm = (rok && x < W) ? __ldg(mrow + (int64_t)x * D) : 0u;
      float sum = 0.0f;
#pragma unroll
      for (int k = -HALO; k <= HALO; k++)
        if (hm & (1u << (k + HALO))) sum += v[c + HALO + k];
      sR[(r * CS_TX + c) * CS_TD + lane] = sum;
    }
  }
  __syncthreads();
  // 2. column sums: warp c owns tile column c; G output rows at a time from
  //    a register window of G + 2*HALO row sums
  const int c = warp, x = X0 + c;
  if (x >= W || !dok) return;
#pragma unroll 1
  for (int g0 = 0; g0 < CS_TY; g0 += G) {
    float wr[G + 2 * HALO];
#pragma unroll
    for (int j = 0; j < G + 2 * HALO; j++) wr[j] = sR[((g0 + j) * CS_TX + c) * CS_TD + lane];
#pragma unroll
    for (int cy = 0; cy < G; cy++) {
      const int y = Y0 + g0 + cy;
      if (y >= H) break;
      const int64_t id = ((int64_t)y * W + x) * D + d;
      const uint32_t w = __ldg(mask + id);
      if (w & kMaskCopy) {
        out[id] = __ldg(in + id);
        continue;
      }
      float sum = 0.0f;
#pragma unroll
      for (int k = -HALO; k <= HALO; k++)
        if (w & (1u << (k + HALO + 11))) sum += wr[cy + HALO + k];
      out[id] = sum / (float)((w >> 22) & 0x7Fu);
    }
  }
}

template <int TY>
int launch_cbca_masked_t(const uint32_t* mask, const float* in, int64_t H, int64_t W, int D, float* out,
                         cudaStream_t st) {
  constexpr size_t smem = (size_t)(TY + 2 * kMaskHalo) * CS_TX * CS_TD * sizeof(float);
  const int64_t tiles = (int64_t)((W + CS_TX - 1) / CS_TX) * ((H + TY - 1) / TY) * ((D + CS_TD - 1) / CS_TD);
  cbca_hwd_mask_kernel<TY><<<(unsigned)tiles, 256, smem, st>>>(mask, in, (int)H, (int)W, D, out);
  return check_launch("cbca_masked");
}


// Winner-take-all (first minimum, as np.argmin) and the subpixel parabola
// (post.cu:453-483).  One warp per pixel on [H,W,D] volumes.
__global__ void wta_subpixel_hwd_kernel(const float* __restrict__ c, int64_t HW, int D,
                                        float* __restrict__ disp_int, float* __restrict__ disp) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t p = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < HW; p += nw) {
    const float* r = c + p * D;
    int bd = 0x7fffffff;
    if (D <= 128) {
      // the minimum over d (NaN ignored), then the first d that holds it;
      // as in the loop below, +inf is never a winner
      float v[4];
#pragma unroll
      for (int k = 0; k < 4; k++) v[k] = lane + 32 * k < D ? r[lane + 32 * k] : __int_as_float(0x7fc00000);
      float mn = fminf(fminf(v[0], v[1]), fminf(v[2], v[3]));
      asm volatile("redux.sync.min.f32 %0, %0, 0xffffffff;" : "+f"(mn));
      unsigned first = 0x7fffffffu;
#pragma unroll
      for (int k = 3; k >= 0; k--)
        if (v[k] == mn && mn < __int_as_float(0x7f800000)) first = (unsigned)(lane + 32 * k);
      bd = (int)__reduce_min_sync(0xffffffffu, first);
    } else {
      float bv = __int_as_float(0x7f800000);
      for (int d = lane; d < D; d += 32) {
        const float v = r[d];
        if (v < bv) { bv = v; bd = d; }
      }
      for (int o = 16; o; o >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
        const int od = __shfl_xor_sync(0xffffffffu, bd, o);
        if (ov < bv || (ov == bv && od < bd)) { bv = ov; bd = od; }
      }
    }
    if (bd == 0x7fffffff) bd = 0;  // all NaN: np.argmin would return 0 for a NaN at 0
    if (lane == 0) {
      if (disp_int) disp_int[p] = (float)bd;
      if (disp) {
        float o = (float)bd;
        if (1 <= bd && bd < D - 1) {
          const float cn = r[bd - 1], cz = r[bd], cp = r[bd + 1];
          const float denom = 2 * (cp + cn - 2 * cz);
          if (denom > 1e-5) {
            const double q = (double)((cp - cn) / denom);
            o = (float)(bd - fmin(1.0, fmax(-1.0, q)));
          }
        }
        disp[p] = o;
      }
    }
  }
}

__global__ void wta_dhw_kernel(const float* __restrict__ c, int64_t HW, int D,
                               float* __restrict__ disp) {
  GRID_STRIDE(p, HW) {
    float bv = c[p];
    int bd = 0;
    for (int d = 1; d < D; d++) {
      const float v = c[(int64_t)d * HW + p];
      if (v < bv) { bv = v; bd = d; }
    }
    disp[p] = (float)bd;
  }
}

__global__ void subpixel_kernel(const float* __restrict__ d0, const float* __restrict__ c,
                                int64_t H, int64_t W, int D, int layout, float* __restrict__ out) {
  GRID_STRIDE(id, H * W) {
    const int d = (int)d0[id];
    float o = (float)d;
    if (1 <= d && d < D - 1) {
      const int64_t y = id / W, x = id - y * W;
      const float cn = c[vol_index(layout, y, x, d - 1, H, W, D)];
      const float cz = c[vol_index(layout, y, x, d, H, W, D)];
      const float cp = c[vol_index(layout, y, x, d + 1, H, W, D)];
      const float denom = 2 * (cp + cn - 2 * cz);
      if (denom > 1e-5) {
        const double q = (double)((cp - cn) / denom);
        o = (float)(d - fmin(1.0, fmax(-1.0, q)));
      }
    }
    out[id] = o;
  }
}

__device__ void sort_small(float* x, int n) {
  for (int i = 0; i < n - 1; i++) {
    int mn = i;
    for (int j = i + 1; j < n; j++)
      if (x[j] < x[mn]) mn = j;
    const float t = x[mn];
    x[mn] = x[i];
    x[i] = t;
  }
}

// median2d (post.cu:486-518)
__global__ void median_kernel(const float* __restrict__ img, int64_t H, int64_t W, int r,
                              float* __restrict__ out) {
  GRID_STRIDE(id, H * W) {
    const int64_t x = id % W, y = id / W;
    float xs[11 * 11];
    int n = 0;
    for (int64_t xx = x - r; xx <= x + r; xx++)
      for (int64_t yy = y - r; yy <= y + r; yy++)
        if (0 <= xx && xx < W && 0 <= yy && yy < H) xs[n++] = img[yy * W + xx];
    sort_small(xs, n);
    out[id] = xs[n / 2];
  }
}

// mean2d (post.cu:520-566): kernel indexed xx-major as the reference.
__global__ void mean2d_kernel(const float* __restrict__ img, int64_t H, int64_t W,
                              const float* __restrict__ kernel, int r, float alpha2,
                              float* __restrict__ out) {
  GRID_STRIDE(id, H * W) {
    const int64_t x = id % W, y = id / W;
    const float c = img[id];
    float sum = 0.0f, cnt = 0.0f;
    int i = 0;
    for (int64_t xx = x - r; xx <= x + r; xx++)
      for (int64_t yy = y - r; yy <= y + r; yy++, i++)
        if (0 <= xx && xx < W && 0 <= yy && yy < H) {
          const float v = img[yy * W + xx];
          if (fabsf(v - c) < alpha2) {
            sum = fmaf(v, kernel[i], sum);
            cnt += kernel[i];
          }
        }
    out[id] = sum / cnt;
  }
}

// mean2d for kernels up to 15 x 15 (the pipeline's: blur_sigma <= 2.33):
// a 16 x 16 block of pixels stages its (16 + 2r)^2 window of the image in
// shared memory, pixels outside the image as NaN (so the |v - c| < alpha2
// test drops them, as mean2d_kernel's bounds test does), and the weights;
// the taps run in mean2d_kernel's order (xx outer, yy inner) with the same
// fused multiply-add, so the results are the same bit for bit.
constexpr int kMeanTile = 16, kMeanMaxR = 7;
__global__ void __launch_bounds__(kMeanTile * kMeanTile) mean2d_tiled_kernel(const float* __restrict__ img, int H,
                                                                           int W, const float* __restrict__ kernel,
                                                                           int r, float alpha2, float* __restrict__ out) {
  constexpr int TS = kMeanTile + 2 * kMeanMaxR;
  __shared__ float tile[TS][TS + 1];
  __shared__ float kw[(2 * kMeanMaxR + 1) * (2 * kMeanMaxR + 1)];
  const int ks = 2 * r + 1, span = kMeanTile + 2 * r;
  const int X0 = blockIdx.x * kMeanTile, Y0 = blockIdx.y * kMeanTile;
  const int tx = threadIdx.x % kMeanTile, ty = threadIdx.x / kMeanTile;
  for (int q = threadIdx.x; q < ks * ks; q += blockDim.x) kw[q] = kernel[q];
  const float nan = __int_as_float(0x7fc00000);
  for (int q = threadIdx.x; q < span * span; q += blockDim.x) {
    const int ry = q / span, rx = q - ry * span;
    const int yy = Y0 - r + ry, xx = X0 - r + rx;
    tile[ry][rx] = (yy >= 0 && yy < H && xx >= 0 && xx < W) ? img[(int64_t)yy * W + xx] : nan;
  }
  __syncthreads();
  const int x = X0 + tx, y = Y0 + ty;
  if (x >= W || y >= H) return;
  const float c = tile[ty + r][tx + r];
  float sum = 0.0f, cnt = 0.0f;
  int i = 0;
  for (int xo = 0; xo < ks; xo++)
    for (int yo = 0; yo < ks; yo++, i++) {
      const float v = tile[ty + yo][tx + xo];
      if (fabsf(v - c) < alpha2) {
        sum = fmaf(v, kw[i], sum);
        cnt += kw[i];
      }
    }
  out[(int64_t)y * W + x] = sum / cnt;
}

// outlier_detection (post.cu:717-754)
__global__ void outlier_kernel(const float* __restrict__ d0, const float* __restrict__ d1,
                               int64_t H, int64_t W, int disp_max, float* __restrict__ out) {
  GRID_STRIDE(id, H * W) {
    const int64_t x = id % W;
    const int d0i = (int)d0[id];
    float o;
    if (x - d0i < 0 || x - d0i >= W) {  // (>= W only for negative input, where the reference reads out of bounds)
      o = 1;
    } else if (fabsf(d0[id] - d1[id - d0i]) < 1.1) {
      o = 0;
    } else {
      o = 1;
      for (int d = 0; d < disp_max; d++)
        if (x - d >= 0 && fabsf((float)d - d1[id - d]) < 1.1) {
          o = 2;
          break;
        }
    }
    out[id] = o;
  }
}

// interpolate_mismatch (post.cu:757-827).  Where every direction leaves the
// image before meeting a non-mismatch pixel the reference asserts; here the
// pixel keeps its disparity.
__global__ void mismatch_kernel(const float* __restrict__ d0, const float* __restrict__ outlier,
                                int64_t H, int64_t W, float* __restrict__ out) {
  const float dir[32] = {0, 1, -0.5f, 1, -1, 1, -1, 0.5f, -1, 0, -1, -0.5f, -1, -1, -0.5f, -1,
                         0, -1, 0.5f, -1, 1, -1, 1, -0.5f, 1, 0, 1, 0.5f, 1, 1, 0.5f, 1};
  GRID_STRIDE(id, H * W) {
    if (outlier[id] != 2) {
      out[id] = d0[id];
      continue;
    }
    float vals[16];
    int n = 0;
    const int64_t x = id % W, y = id / W;
    for (int k = 0; k < 16; k++) {
      const float dx = dir[2 * k], dy = dir[2 * k + 1];
      float xx = (float)x, yy = (float)y;
      int64_t xi = (int64_t)roundf(xx), yi = (int64_t)roundf(yy);
      while (0 <= yi && yi < H && 0 <= xi && xi < W && outlier[yi * W + xi] == 2) {
        xx += dx;
        yy += dy;
        xi = (int64_t)roundf(xx);
        yi = (int64_t)roundf(yy);
      }
      if (0 <= yi && yi < H && 0 <= xi && xi < W) vals[n++] = d0[yi * W + xi];
    }
    if (n == 0) {
      out[id] = d0[id];
      continue;
    }
    sort_small(vals, n);
    out[id] = vals[n / 2];
  }
}

// interpolate_occlusion (post.cu:829-869)
__global__ void occlusion_kernel(const float* __restrict__ d0, const float* __restrict__ outlier,
                                 int64_t H, int64_t W, float* __restrict__ out) {
  GRID_STRIDE(id, H * W) {
    if (outlier[id] != 1) {
      out[id] = d0[id];
      continue;
    }
    const int64_t x = id % W;
    int64_t dx = 0;
    while (x + dx >= 0 && outlier[id + dx] != 0) dx--;
    if (x + dx < 0) {
      dx = 0;
      while (x + dx < W && outlier[id + dx] != 0) dx++;
    }
    out[id] = (x + dx < W) ? d0[id + dx] : d0[id];
  }
}

// [H*W, D] <-> [D, H*W] tiled transpose of float32.
__global__ void transpose_kernel(const float* __restrict__ in, int64_t rows, int64_t cols,
                                 float* __restrict__ out) {
  __shared__ float tile[32][33];
  const int64_t c0 = (int64_t)blockIdx.x * 32, r0 = (int64_t)blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int64_t r = r0 + k, c = c0 + threadIdx.x;
    if (r < rows && c < cols) tile[k][threadIdx.x] = in[r * cols + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int64_t c = c0 + k, r = r0 + threadIdx.x;
    if (r < rows && c < cols) out[c * rows + r] = tile[threadIdx.x][k];
  }
}

__global__ void scale_kernel(float* a, int64_t n, float mul) {
  GRID_STRIDE(i, n) a[i] *= mul;
}

__global__ void f64_to_f32_kernel(const double* __restrict__ in, int64_t n, float* __restrict__ out) {
  GRID_STRIDE(i, n) out[i] = (float)in[i];
}

__global__ void f32_to_f64_kernel(const float* __restrict__ in, int64_t n, double* __restrict__ out) {
  GRID_STRIDE(i, n) out[i] = (double)in[i];
}

// Sums of an image and of its squares in float64 (one block).
// Sum and sum of squares of the image as exact 64-bit integers (so the
// result does not depend on the order of the additions), accumulated by
// every block into mom[0..1] with integer atomics; mom is zeroed first.
__global__ void moments_kernel(const uint8_t* __restrict__ img, int64_t n,
                               unsigned long long* __restrict__ mom) {
  unsigned long long a = 0, b = 0;
  GRID_STRIDE(i, n) {
    const unsigned v = img[i];
    a += v;
    b += v * v;
  }
  for (int o = 16; o; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(mom, a);
    atomicAdd(mom + 1, b);
  }
}

// (I - mean) / std in float32 with float32 mean and population std, as
// test.py:489-492 does with numpy on the float32 image.
__global__ void normalise_kernel(const uint8_t* __restrict__ img, int64_t n,
                                 const unsigned long long* __restrict__ mom, float* __restrict__ out) {
  const double mean = (double)mom[0] / (double)n;
  const double var = fmax((double)mom[1] / (double)n - mean * mean, 0.0);
  const float m = (float)mean, s = (float)sqrt(var);
  GRID_STRIDE(i, n) out[i] = ((float)img[i] - m) / s;
}

}  // namespace

int launch_cross(const float* img, int64_t H, int64_t W, int L1, float tau1, float* out,
                 cudaStream_t st) {
  cross_kernel<<<grid_for(4 * H * W, kBlock), kBlock, 0, st>>>(img, H, W, L1, tau1, out);
  return check_launch("cross");
}

int launch_sgm_grad(const float* imL, const float* imR, int64_t H, int64_t W, SgmGrad* g,
                    cudaStream_t st) {
  grad_kernel<<<grid_for(H * W, 256), 256, 0, st>>>(imL, H, W, g->lh, g->lv);
  grad_kernel<<<grid_for(H * W, 256), 256, 0, st>>>(imR, H, W, g->rh, g->rv);
  return check_launch("sgm_grad");
}

// prefetch: steps loaded ahead (1, 2 or 4; 0 = the default: shallow
// prefetch keeps the scan at ~80 registers, measured faster than deeper
// rings, whose registers cost more occupancy than they hide latency).
// The results do not depend on it.
template <int KPL>
static void sgm4_launch(const SgmGrad& g, const float* in, int H, int W, int D, const SgmParams& sp,
                        const SgmOut& o, cudaStream_t st, int prefetch) {
  const int lines = 2 * H + 2 * W;
  const int blocks = (lines * 32 + 127) / 128;
  constexpr int PF0 = KPL <= 2 ? 4 : KPL <= 8 ? 2 : 1;
  const int pf = prefetch > 0 && KPL <= 8 ? prefetch : PF0;
  if (D == 32 * KPL) {  // every lane's disparities exist: no bounds tests on d
    if (pf >= 4) sgm4_kernel<KPL, KPL <= 8 ? 4 : 1, true><<<blocks, 128, 0, st>>>(g, in, H, W, D, sp, o);
    else if (pf >= 2) sgm4_kernel<KPL, KPL <= 8 ? 2 : 1, true><<<blocks, 128, 0, st>>>(g, in, H, W, D, sp, o);
    else sgm4_kernel<KPL, 1, true><<<blocks, 128, 0, st>>>(g, in, H, W, D, sp, o);
  } else {
    if (pf >= 4) sgm4_kernel<KPL, KPL <= 8 ? 4 : 1, false><<<blocks, 128, 0, st>>>(g, in, H, W, D, sp, o);
    else if (pf >= 2) sgm4_kernel<KPL, KPL <= 8 ? 2 : 1, false><<<blocks, 128, 0, st>>>(g, in, H, W, D, sp, o);
    else sgm4_kernel<KPL, 1, false><<<blocks, 128, 0, st>>>(g, in, H, W, D, sp, o);
  }
}

// The consecutive-disparity scan (sgm_scan_c) for D a multiple of 4 in
// (64, 512] with 16-byte aligned volumes; 2 steps loaded ahead (default,
// measured faster at 694x554 D=128: post 2.74 against 2.88 ms) or 1.
template <int KPL>
static void sgm4c_launch(const SgmGrad& g, const float* in, int H, int W, int D, const SgmParams& sp,
                         const SgmOut& o, cudaStream_t st, int prefetch) {
  const int lines = 2 * H + 2 * W;
  const int blocks = (lines * 32 + 127) / 128;
  const bool full = D == 32 * KPL;
#define SGM4C(PF_, FULL_, S_) sgm4c_kernel<KPL, PF_, FULL_, S_><<<blocks, 128, 0, st>>>(g, in, H, W, D, sp, o)
  if (sp.direction > 0) {
    if (prefetch == 1) { if (full) SGM4C(1, true, 1); else SGM4C(1, false, 1); }
    else { if (full) SGM4C(2, true, 1); else SGM4C(2, false, 1); }
  } else {
    if (prefetch == 1) { if (full) SGM4C(1, true, -1); else SGM4C(1, false, -1); }
    else { if (full) SGM4C(2, true, -1); else SGM4C(2, false, -1); }
  }
#undef SGM4C
}

static bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

int launch_sgm4(const SgmGrad& g, const float* in, int64_t H, int64_t W, int D, const SgmParams& sp,
                const SgmOut& o, cudaStream_t st, int prefetch) {
  const int kpl = (D + 31) / 32;
  const int h = (int)H, w = (int)W;
  const bool vec = D % 4 == 0 && D > 64 && D <= 512 && aligned16(in) && aligned16(o.dir[0]) &&
                   aligned16(o.dir[1]) && aligned16(o.dir[2]) && aligned16(o.dir[3]);
  if (vec) {
    if (D <= 128) sgm4c_launch<4>(g, in, h, w, D, sp, o, st, prefetch);
    else if (D <= 256) sgm4c_launch<8>(g, in, h, w, D, sp, o, st, prefetch);
    else sgm4c_launch<16>(g, in, h, w, D, sp, o, st, prefetch);
    return check_launch("sgm4");
  }
  if (kpl <= 1) sgm4_launch<1>(g, in, h, w, D, sp, o, st, prefetch);
  else if (kpl <= 2) sgm4_launch<2>(g, in, h, w, D, sp, o, st, prefetch);
  else if (kpl <= 4) sgm4_launch<4>(g, in, h, w, D, sp, o, st, prefetch);
  else if (kpl <= 8) sgm4_launch<8>(g, in, h, w, D, sp, o, st, prefetch);
  else if (kpl <= 16) sgm4_launch<16>(g, in, h, w, D, sp, o, st, prefetch);
  else sgm4_launch<32>(g, in, h, w, D, sp, o, st, prefetch);
  return check_launch("sgm4");
}

int launch_sgm_combine(const SgmOut& o, int64_t n, const float* base, float scale, float* out,
                       cudaStream_t st) {
  sgm_combine_kernel<<<grid_for(n, 256), 256, 0, st>>>(o, n, base, scale, out);
  return check_launch("sgm_combine");
}

int launch_cbca(const float* lc, const float* rc, const float* in, int64_t H, int64_t W, int D,
                int layout, int direction, float* out, cudaStream_t st, int halo) {
  if (layout == CBMV_HWD && halo >= 0 && halo <= 8 && H < 32767 && W < 32767) {
    const size_t smem = cbca_smem_bytes(halo);
    CBMV_CUDA(cudaFuncSetAttribute(cbca_hwd_tiled_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)cbca_smem_bytes(8)));
    const int64_t tiles = (int64_t)((W + CB_TX - 1) / CB_TX) * ((H + CB_TY - 1) / CB_TY) *
                          ((D + CB_TD - 1) / CB_TD);
    const unsigned grid = (unsigned)(tiles < (int64_t)1 << 30 ? tiles : (int64_t)1 << 30);
    cbca_hwd_tiled_kernel<<<grid, 256, smem, st>>>(lc, rc, in, (int)H, (int)W, D, direction, halo,
                                                   out);
    return check_launch("cbca_tiled");
  }
  cbca_kernel<<<grid_for(H * W * D, kBlock), kBlock, 0, st>>>(lc, rc, in, H, W, D, layout, direction,
                                                             out);
  return check_launch("cbca");
}

int launch_cbca_sep(const float* lc, const float* rc, const float* in, int64_t H, int64_t W, int D,
                    int direction, float* out, cudaStream_t st, int halo, int rows) {
  CBMV_REQUIRE(H < (1 << 30) && W < (1 << 30) && (int64_t)((W + CS_TX - 1) / CS_TX) * ((H + 15) / 16) *
                   ((D + CS_TD - 1) / CS_TD) < ((int64_t)1 << 31),
               CBMV_ERANGE, "cbca: volume too large");
  switch (halo) {
    case 1: return launch_cbca_sep_h<1>(lc, rc, in, H, W, D, direction, out, st, rows);
    case 2: return launch_cbca_sep_h<2>(lc, rc, in, H, W, D, direction, out, st, rows);
    case 3: return launch_cbca_sep_h<3>(lc, rc, in, H, W, D, direction, out, st, rows);
    case 4: return launch_cbca_sep_h<4>(lc, rc, in, H, W, D, direction, out, st, rows);
    case 5: return launch_cbca_sep_h<5>(lc, rc, in, H, W, D, direction, out, st, rows);
    case 6: return launch_cbca_sep_h<6>(lc, rc, in, H, W, D, direction, out, st, rows);
    case 7: return launch_cbca_sep_h<7>(lc, rc, in, H, W, D, direction, out, st, rows);
    case 8: return launch_cbca_sep_h<8>(lc, rc, in, H, W, D, direction, out, st, rows);
    default: return launch_cbca(lc, rc, in, H, W, D, CBMV_HWD, direction, out, st, halo);
  }
}

int launch_cbca_mask_build(const float* lc, const float* rc, int64_t H, int64_t W, int D, int direction,
                           uint32_t* mask, cudaStream_t st) {
  CBMV_REQUIRE(H < (1 << 30) && W < (1 << 30) &&
                   (int64_t)((W + CS_TX - 1) / CS_TX) * ((H + 15) / 16) * ((D + CS_TD - 1) / CS_TD) <
                       ((int64_t)1 << 31),
               CBMV_ERANGE, "cbca: volume too large");
  constexpr int TY = 32;
  const int64_t tiles = (int64_t)((W + CS_TX - 1) / CS_TX) * ((H + TY - 1) / TY) * ((D + CS_TD - 1) / CS_TD);
  cbca_mask_build_kernel<TY><<<(unsigned)tiles, 256, 0, st>>>(lc, rc, (int)H, (int)W, D, direction, mask);
  return check_launch("cbca_mask_build");
}

// tile rows 16 or 32 (the results do not depend on them)
int launch_cbca_masked(const uint32_t* mask, const float* in, int64_t H, int64_t W, int D, float* out,
                       cudaStream_t st, int rows) {
  CBMV_REQUIRE(H < (1 << 30) && W < (1 << 30) &&
                   (int64_t)((W + CS_TX - 1) / CS_TX) * ((H + 15) / 16) * ((D + CS_TD - 1) / CS_TD) <
                       ((int64_t)1 << 31),
               CBMV_ERANGE, "cbca: volume too large");
  if (rows == 16) return launch_cbca_masked_t<16>(mask, in, H, W, D, out, st);
  return launch_cbca_masked_t<32>(mask, in, H, W, D, out, st);
}

int launch_wta_subpixel(const float* cost, int64_t H, int64_t W, int D, float* disp_int,
                        float* disp, cudaStream_t st) {
  wta_subpixel_hwd_kernel<<<grid_for(H * W * 32, 256), 256, 0, st>>>(cost, H * W, D, disp_int, disp);
  return check_launch("wta_subpixel");
}

int launch_median(const float* in, int64_t H, int64_t W, int k, float* out, cudaStream_t st) {
  median_kernel<<<grid_for(H * W, kBlock), kBlock, 0, st>>>(in, H, W, k / 2, out);
  return check_launch("median2d");
}

int launch_mean2d(const float* in, int64_t H, int64_t W, const float* kernel, int ks, float alpha2,
                  float* out, cudaStream_t st) {
  if (ks / 2 <= kMeanMaxR && H < 65536 * kMeanTile && W < ((int64_t)1 << 30)) {
    const dim3 grid((unsigned)((W + kMeanTile - 1) / kMeanTile), (unsigned)((H + kMeanTile - 1) / kMeanTile));
    mean2d_tiled_kernel<<<grid, kMeanTile * kMeanTile, 0, st>>>(in, (int)H, (int)W, kernel, ks / 2, alpha2, out);
    return check_launch("mean2d");
  }
  mean2d_kernel<<<grid_for(H * W, kBlock), kBlock, 0, st>>>(in, H, W, kernel, ks / 2, alpha2, out);
  return check_launch("mean2d");
}

int launch_normalise(const uint8_t* img, int64_t n, double* mom, float* out, cudaStream_t st) {
  unsigned long long* m = reinterpret_cast<unsigned long long*>(mom);
  CBMV_CUDA(cudaMemsetAsync(m, 0, 2 * sizeof(unsigned long long), st));
  moments_kernel<<<grid_for(n, 256), 256, 0, st>>>(img, n, m);
  normalise_kernel<<<grid_for(n, 256), 256, 0, st>>>(img, n, m, out);
  return check_launch("normalise");
}

// get_right_cost (featextract.cpp:115-152) of a float32 [H,W,D] volume:
// R[y,x,d] = C[y,x+d,d] where x + d < W, else C[0,0,0] (test.py:154)
__global__ void right_cost_f32_kernel(const float* __restrict__ in, int64_t H, int64_t W, int64_t D,
                                      float* __restrict__ out) {
  const float fill = in[0];
  GRID_STRIDE(t, H * W * D) {
    const int64_t d = t % D;
    const int64_t p = t / D;
    const int64_t x = p % W;
    out[t] = x + d < W ? in[(p + d) * D + d] : fill;
  }
}

int launch_right_cost_f32(const float* in, int64_t H, int64_t W, int D, float* out, cudaStream_t st) {
  right_cost_f32_kernel<<<grid_for(H * W * D, kBlock), kBlock, 0, st>>>(in, H, W, D, out);
  return check_launch("right_cost_f32");
}

int launch_outlier(const float* d0, const float* d1, int64_t H, int64_t W, int disp_max, float* out,
                   cudaStream_t st) {
  outlier_kernel<<<grid_for(H * W, kBlock), kBlock, 0, st>>>(d0, d1, H, W, disp_max, out);
  return check_launch("outlier_detection");
}

int launch_mismatch(const float* d0, const float* o, int64_t H, int64_t W, float* out,
                    cudaStream_t st) {
  mismatch_kernel<<<grid_for(H * W, kBlock), kBlock, 0, st>>>(d0, o, H, W, out);
  return check_launch("interpolate_mismatch");
}

int launch_occlusion(const float* d0, const float* o, int64_t H, int64_t W, float* out,
                     cudaStream_t st) {
  occlusion_kernel<<<grid_for(H * W, kBlock), kBlock, 0, st>>>(d0, o, H, W, out);
  return check_launch("interpolate_occlusion");
}

}  // namespace cbmv

using namespace cbmv;

#define REQ_PTR(...) CBMV_REQUIRE(__VA_ARGS__, CBMV_EINVAL, "null pointer argument")
#define REQ_HW(H, W) \
  CBMV_REQUIRE((H) > 0 && (W) > 0 && (H) <= (1 << 30) && (W) <= (1 << 30), CBMV_EINVAL, "bad size")

extern "C" int cbmv_cross(const float* img, int64_t H, int64_t W, int L1, float tau1, float* out,
                          void* stream) {
  REQ_PTR(img && out);
  REQ_HW(H, W);
  return launch_cross(img, H, W, L1, tau1, out, as_stream(stream));
}

extern "C" int cbmv_sgm(const float* imL, const float* imR, const float* in, int64_t H, int64_t W,
                        int D, float pi1, float pi2, float tau_so, float alpha1, float q1, float q2,
                        int direction, float* out, void* stream) {
  REQ_PTR(imL && imR && in && out);
  REQ_HW(H, W);
  CBMV_REQUIRE(D > 0 && D <= 1024, CBMV_ERANGE, "D=%d not in 1..1024", D);
  CBMV_REQUIRE(in != out, CBMV_EINVAL, "sgm: in and out must differ");
  CBMV_REQUIRE(direction == 1 || direction == -1, CBMV_EINVAL, "direction must be +-1");
  cudaStream_t st = as_stream(stream);
  const int64_t HW = H * W, V = HW * D;
  float* scratch = nullptr;
  CBMV_CUDA(cudaMallocAsync(&scratch, sizeof(float) * (4 * HW + 4 * V), st));
  SgmGrad g{scratch, scratch + HW, scratch + 2 * HW, scratch + 3 * HW};
  SgmOut o{{scratch + 4 * HW, scratch + 4 * HW + V, scratch + 4 * HW + 2 * V, scratch + 4 * HW + 3 * V}};
  SgmParams sp{pi1, pi2, tau_so, alpha1, q1, q2, direction};
  int rc = launch_sgm_grad(imL, imR, H, W, &g, st);
  if (!rc) rc = launch_sgm4(g, in, H, W, D, sp, o, st);
  if (!rc) rc = launch_sgm_combine(o, V, out, 1.0f, out, st);
  CBMV_CUDA(cudaFreeAsync(scratch, st));
  return rc;
}

extern "C" int cbmv_cbca(const float* crossL, const float* crossR, const float* in, int64_t H,
                         int64_t W, int D, int layout, int direction, float* out, void* stream) {
  REQ_PTR(crossL && crossR && in && out);
  REQ_HW(H, W);
  CBMV_REQUIRE(D > 0, CBMV_EINVAL, "bad D");
  CBMV_REQUIRE(in != out, CBMV_EINVAL, "cbca: in and out must differ");
  CBMV_REQUIRE(direction == 1 || direction == -1, CBMV_EINVAL, "direction must be +-1");
  CBMV_REQUIRE(layout == CBMV_HWD || layout == CBMV_DHW, CBMV_EINVAL, "bad layout");
  return launch_cbca(crossL, crossR, in, H, W, D, layout, direction, out, as_stream(stream));
}

extern "C" int cbmv_cbca_separable(const float* crossL, const float* crossR, const float* in, int64_t H,
                                   int64_t W, int D, int L1, int direction, float* out, void* stream) {
  REQ_PTR(crossL && crossR && in && out);
  REQ_HW(H, W);
  CBMV_REQUIRE(D > 0, CBMV_EINVAL, "bad D");
  CBMV_REQUIRE(in != out, CBMV_EINVAL, "cbca: in and out must differ");
  CBMV_REQUIRE(direction == 1 || direction == -1, CBMV_EINVAL, "direction must be +-1");
  CBMV_REQUIRE(L1 >= 2 && L1 <= 9, CBMV_EINVAL, "cbca_separable: L1 must be in 2..9");
  cudaStream_t st = as_stream(stream);
  if (L1 - 1 > kCbcaMaskMaxHalo) return launch_cbca_sep(crossL, crossR, in, H, W, D, direction, out, st, L1 - 1);
  // the pipeline's form: supports precomputed into a stream-ordered scratch buffer
  uint32_t* mask = nullptr;
  CBMV_CUDA(cudaMallocAsync(&mask, sizeof(uint32_t) * H * W * D, st));
  int rc = launch_cbca_mask_build(crossL, crossR, H, W, D, direction, mask, st);
  if (rc == CBMV_OK) rc = launch_cbca_masked(mask, in, H, W, D, out, st);
  CBMV_CUDA(cudaFreeAsync(mask, st));
  return rc;
}

extern "C" int cbmv_wta(const float* cost, int64_t H, int64_t W, int D, int layout, float* disp,
                        void* stream) {
  REQ_PTR(cost && disp);
  REQ_HW(H, W);
  CBMV_REQUIRE(D > 0, CBMV_EINVAL, "bad D");
  if (layout == CBMV_HWD) return launch_wta_subpixel(cost, H, W, D, disp, nullptr, as_stream(stream));
  wta_dhw_kernel<<<grid_for(H * W, kBlock), kBlock, 0, as_stream(stream)>>>(cost, H * W, D, disp);
  return check_launch("wta");
}

extern "C" int cbmv_subpixel(const float* disp, const float* cost, int64_t H, int64_t W, int D,
                             int layout, float* out, void* stream) {
  REQ_PTR(disp && cost && out);
  REQ_HW(H, W);
  CBMV_REQUIRE(D > 0, CBMV_EINVAL, "bad D");
  subpixel_kernel<<<grid_for(H * W, kBlock), kBlock, 0, as_stream(stream)>>>(disp, cost, H, W, D, layout,
                                                                            out);
  return check_launch("subpixel");
}

extern "C" int cbmv_median2d(const float* in, int64_t H, int64_t W, int k, float* out,
                             void* stream) {
  REQ_PTR(in && out);
  REQ_HW(H, W);
  CBMV_REQUIRE(k >= 1 && k <= 11 && (k & 1), CBMV_EINVAL, "median window %d must be odd <= 11", k);
  CBMV_REQUIRE(in != out, CBMV_EINVAL, "median2d: in and out must differ");
  return launch_median(in, H, W, k, out, as_stream(stream));
}

extern "C" int cbmv_mean2d(const float* in, int64_t H, int64_t W, const float* kernel, int ks,
                           float alpha2, float* out, void* stream) {
  REQ_PTR(in && out && kernel);
  REQ_HW(H, W);
  CBMV_REQUIRE(ks >= 1 && ks <= 31 && (ks & 1), CBMV_EINVAL, "kernel size %d must be odd <= 31", ks);
  CBMV_REQUIRE(in != out, CBMV_EINVAL, "mean2d: in and out must differ");
  return launch_mean2d(in, H, W, kernel, ks, alpha2, out, as_stream(stream));
}

extern "C" int cbmv_outlier_detection(const float* d0, const float* d1, int64_t H, int64_t W,
                                      int disp_max, float* out, void* stream) {
  REQ_PTR(d0 && d1 && out);
  REQ_HW(H, W);
  return launch_outlier(d0, d1, H, W, disp_max, out, as_stream(stream));
}

extern "C" int cbmv_interpolate_mismatch(const float* d0, const float* outlier, int64_t H,
                                         int64_t W, float* out, void* stream) {
  REQ_PTR(d0 && outlier && out);
  REQ_HW(H, W);
  CBMV_REQUIRE(d0 != out, CBMV_EINVAL, "in and out must differ");
  return launch_mismatch(d0, outlier, H, W, out, as_stream(stream));
}

extern "C" int cbmv_interpolate_occlusion(const float* d0, const float* outlier, int64_t H,
                                          int64_t W, float* out, void* stream) {
  REQ_PTR(d0 && outlier && out);
  REQ_HW(H, W);
  CBMV_REQUIRE(d0 != out, CBMV_EINVAL, "in and out must differ");
  return launch_occlusion(d0, outlier, H, W, out, as_stream(stream));
}

extern "C" int cbmv_transpose_f32(const float* in, int64_t H, int64_t W, int64_t D, int to_layout,
                                  float* out, void* stream) {
  REQ_PTR(in && out);
  CBMV_REQUIRE(H > 0 && W > 0 && D > 0 && in != out, CBMV_EINVAL, "bad argument");
  const int64_t rows = to_layout == CBMV_DHW ? H * W : D;
  const int64_t cols = to_layout == CBMV_DHW ? D : H * W;
  CBMV_REQUIRE((rows + 31) / 32 <= 65535, CBMV_ERANGE, "volume too large for the transpose grid");
  dim3 grid((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32));
  transpose_kernel<<<grid, dim3(32, 8), 0, as_stream(stream)>>>(in, rows, cols, out);
  return check_launch("transpose");
}

extern "C" int cbmv_scale_f32(float* a, int64_t n, float mul, void* stream) {
  REQ_PTR(a);
  CBMV_REQUIRE(n >= 0, CBMV_EINVAL, "bad size");
  if (n == 0) return CBMV_OK;
  scale_kernel<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(a, n, mul);
  return check_launch("scale");
}

extern "C" int cbmv_f64_to_f32(const double* in, int64_t n, float* out, void* stream) {
  REQ_PTR(in && out);
  if (n <= 0) return n == 0 ? CBMV_OK : set_error(CBMV_EINVAL, "bad size");
  f64_to_f32_kernel<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(in, n, out);
  return check_launch("f64_to_f32");
}

extern "C" int cbmv_f32_to_f64(const float* in, int64_t n, double* out, void* stream) {
  REQ_PTR(in && out);
  if (n <= 0) return n == 0 ? CBMV_OK : set_error(CBMV_EINVAL, "bad size");
  f32_to_f64_kernel<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(in, n, out);
  return check_launch("f32_to_f64");
}
