// The fused inference kernel of the learned classifier, instantiated once
// per hidden-layer activation in its own translation unit
// (mlp_infer_relu.cu, mlp_infer_gelu.cu), so that neither instantiation
// changes how the compiler allocates the other's registers.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "features.cuh"
#include "mlp_net.cuh"
#include "pipeline.cuh"
#include "umma.cuh"

// ====================================================================
// Fused inference: features of 128 consecutive (pixel, d) samples -> the
// network on the tensor cores -> matching cost 1 - P(correct), float32.
//
// One persistent CTA per SM, four independent groups of 128 threads; each
// group owns a 128-row tile in flight (its activation buffer in shared
// memory and 128 tensor-memory columns), so while one group's MMAs run the
// others compute features or epilogues.  Thread r of a group owns row r of
// its tile: it forms the 20 features of sample r (their inputs for the
// next tile are loaded while this one runs through the network), then
// that row's columns in each epilogue.  The group's first thread issues
// its MMAs, commits them to the group's mbarrier and alone polls it; the
// others wait on the group's named barrier (no issue slots spent
// spinning), which also hands them the poll's result.
//
// Arithmetic, per layer (the float32 accumulator in tensor memory), with
// 16-bit operands of the network's precision (f16 by default, bf16 on
// request; "16-bit" below); every bias enters as 16-bit high + low parts
// multiplied by constant ones:
//   layer 1  K = 32: 20 normalised features, two constant-one columns whose
//            weights are b1's parts, zeros;
//   layers 2, 3: a first K = 16 MMA of a constant tile (ones in columns 0
//            and 1) against b2's / b3's parts (stored in the unused K
//            columns 32..63 of layer 1's weight tile) initialises the
//            accumulator, the layer's MMAs accumulate onto it;
//   hidden activations: ReLU and the 16-bit rounding in one instruction
//            per pair of columns, or the GELU in packed 16-bit arithmetic
//            (six instructions per pair in f16, seven in bf16);
//   output   layer 4 is an MMA too: N = 16, rows 0 and 1 of its weight tile
//            are the high and low 16-bit parts of w4, z = D[0] + D[1] + b4,
//            cost = 1 - sigmoid(z) = 1 / (1 + exp(z)).
// The features themselves are formed in float32 (they enter the network in
// 16 bits), from float32 cost volumes and float32 row statistics (min, 1/den),
// with one reciprocal 1/(c + e) shared by the left and right ratio.
// ====================================================================

namespace cbmv {
namespace {

struct FeatVolsF {
  const float* v[4];
};

constexpr int kGroups = 4;                        // tiles in flight per CTA
constexpr int kGroupThreads = 128;               // one thread per tile row
constexpr int kInfThreads = kGroupThreads * kGroups;
constexpr size_t kSmW1i = 128 * 128;      // [128 x 64] SW128, K = 32 used
constexpr size_t kSmW2i = 2 * 128 * 128;  // [128 x 128]
constexpr size_t kSmW3i = 2 * 64 * 128;   // [64 x 128]
constexpr size_t kSmW4i = 16 * 128;       // [16 x 64]
constexpr size_t kSmOne = 128 * 128;      // [128 x 64], ones in columns 0 and 1
constexpr size_t kSmTile = 2 * 128 * 128; // a group's activation tile [128 x 128]
constexpr size_t kSmInf = 1024 + kSmW1i + kSmW2i + kSmW3i + kSmW4i + kSmOne + kGroups * kSmTile;
constexpr int kColB2 = 32, kColB3 = 48;  // K columns of layer 1's weight tile holding b2, b3

static __constant__ float kEpsF[4] = {0.01f, 1.01f, 0.01f, 0.01f};
static __constant__ float kInvSigmaF[4] = {(float)(1.0 / (2.0 * 8 * 8)), (float)(1.0 / 0.02),
                                           (float)(1.0 / (2.0 * 100 * 100)), (float)(1.0 / (2.0 * 100 * 100))};

__device__ __forceinline__ void group_sync(int g) {
  asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "n"(kGroupThreads) : "memory");
}
// barrier of the group that also ANDs a flag over its threads
__device__ __forceinline__ bool group_all(int g, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(g + 1), "n"(kGroupThreads)
      : "memory");
  return r != 0;
}

// The network's 16-bit operand type in the fused kernel (cbmv_mlp_set_precision):
// F16 = true, IEEE half (the default), F16 = false, bfloat16.  Per type: the
// packed conversion of two float32 values (low = a), round to nearest even
// (f16: saturated to +-65504); ReLU of two pre-activations in the same
// instruction; the GELU of two pre-activations; the bits of one value and
// its high + low split; the instruction descriptor of the MMAs.
template <bool F16>
struct Op16;

template <>
struct Op16<true> {
  static constexpr uint32_t kOneOne = 0x3C003C00u;  // two f16 ones
  static __device__ __forceinline__ uint32_t pack(float a, float b) {
    uint32_t r;
    asm("cvt.rn.satfinite.f16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(b), "f"(a));
    return r;
  }
  static __device__ __forceinline__ uint32_t relu(float a, float b) {
    uint32_t r;
    asm("cvt.rn.relu.satfinite.f16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(b), "f"(a));
    return r;
  }
  // gelu_t's f16 operations, both lanes per instruction: six instructions
  // per pair, the conversion included, the clamp of q to [0, 1] folded into
  // its FMA (`fma.rn.sat.f16x2`)
  static __device__ __forceinline__ uint32_t gelu(float a, float b) {
    const __half2 g0 = __half2half2(f16_bits(kG0Bits)), g1 = __half2half2(f16_bits(kG1Bits)),
                  g2 = __half2half2(f16_bits(kG2Bits));
    const __half2 half = __float2half2_rn(0.5f);
    const uint32_t xb = pack(a, b);
    const __half2 x = *reinterpret_cast<const __half2*>(&xb);
    const __half2 u = __hmul2(x, x);
    __half2 p = __hfma2(g2, u, g1);
    p = __hfma2(p, u, g0);
    const __half2 q = __hfma2_sat(x, p, half);
    const __half2 g = __hmul2(x, q);
    return *reinterpret_cast<const uint32_t*>(&g);
  }
  static __device__ __forceinline__ uint16_t bits(float x) { return to_f16(x); }
  static __device__ __forceinline__ void split(float x, float* hi, float* lo) {
    *hi = __half2float(__float2half_rn(fminf(fmaxf(x, -65504.0f), 65504.0f)));
    *lo = x - *hi;
  }
  static __host__ __device__ constexpr uint32_t idesc(int M, int N) { return umma::idesc_f16(M, N); }
};

template <>
struct Op16<false> {
  static constexpr uint32_t kOneOne = 0x3F803F80u;  // two bf16 ones
  static __device__ __forceinline__ uint32_t pack(float a, float b) {
    const __nv_bfloat162 x = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&x);
  }
  static __device__ __forceinline__ uint32_t relu(float a, float b) {
    uint32_t r;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(b), "f"(a));
    return r;
  }
  // the same polynomial form in bf16 operations with its own coefficients
  // (gelu_bf16_t): seven instructions per pair -- bf16 has no saturating
  // FMA, so the clamp is a `.relu` FMA and a min
  static __device__ __forceinline__ uint32_t gelu(float a, float b) {
    const __nv_bfloat162 g0 = __bfloat162bfloat162(bf16_bits(kGB0Bits)),
                         g1 = __bfloat162bfloat162(bf16_bits(kGB1Bits)),
                         g2 = __bfloat162bfloat162(bf16_bits(kGB2Bits));
    const __nv_bfloat162 half = __float2bfloat162_rn(0.5f), one = __float2bfloat162_rn(1.0f);
    const __nv_bfloat162 x = __floats2bfloat162_rn(a, b);
    const __nv_bfloat162 u = __hmul2(x, x);
    __nv_bfloat162 p = __hfma2(g2, u, g1);
    p = __hfma2(p, u, g0);
    __nv_bfloat162 q = __hfma2_relu(x, p, half);
    q = __hmin2(q, one);
    const __nv_bfloat162 g = __hmul2(x, q);
    return *reinterpret_cast<const uint32_t*>(&g);
  }
  static __device__ __forceinline__ uint16_t bits(float x) { return to_bf16(x); }
  static __device__ __forceinline__ void split(float x, float* hi, float* lo) {
    *hi = __bfloat162float(__float2bfloat16_rn(x));
    *lo = x - *hi;
  }
  static __host__ __device__ constexpr uint32_t idesc(int M, int N) { return umma::idesc_bf16(M, N); }
};

// ratio and likelihood of cost c (featextract.cpp:333 and :440) in float32
// against its row statistics st = (min, 1/den); inv_ce = 1 / (c + e).
// The approximate exponential (one multiply by log2(e) and the hardware
// exp2): its relative error, about |x| * 6e-8 from rounding x log2(e) plus
// two units of the exp2, stays below 5e-6 for every likelihood above
// exp(-80), the same order as the float32 rounding of the argument itself.
__device__ __forceinline__ void conf_f32(float c, float inv_ce, float2 st, float e, float inv_sigma,
                                         float* ratio, float* lik) {
  const float t = c - st.x;
  *ratio = st.x == kRandMaxF ? 0.0f : (st.x + e) * inv_ce;
  *lik = __expf(-(t * t) * inv_sigma) * st.y;  // 1/den = 0 on sentinel rows
}

// Stage the inference weights from the float32 parameter vector, and the
// constant tile of the bias MMAs.
template <bool F16>
__device__ __forceinline__ void stage_inference_weights(const float* __restrict__ P, unsigned char* sW1, unsigned char* sW2,
                                        unsigned char* sW3, unsigned char* sW4, unsigned char* sOne) {
  for (int q = threadIdx.x; q < 128 * 64; q += blockDim.x) {
    const int r = q >> 6, k = q & 63;
    float v = 0.0f, hi, lo;
    if (k < kF) {
      v = P[kOffW1 + r * kF + k];
    } else if (k == kF || k == kF + 1) {
      Op16<F16>::split(P[kOffB1 + r], &hi, &lo);
      v = k == kF ? hi : lo;
    } else if (k == kColB2 || k == kColB2 + 1) {
      Op16<F16>::split(P[kOffB2 + r], &hi, &lo);
      v = k == kColB2 ? hi : lo;
    } else if (r < kH3 && (k == kColB3 || k == kColB3 + 1)) {
      Op16<F16>::split(P[kOffB3 + r], &hi, &lo);
      v = k == kColB3 ? hi : lo;
    }
    *reinterpret_cast<uint16_t*>(sW1 + umma::sw128_offset(128, r, k)) = Op16<F16>::bits(v);
    *reinterpret_cast<uint16_t*>(sOne + umma::sw128_offset(128, r, k)) = Op16<F16>::bits(k < 2 ? 1.0f : 0.0f);
  }
  for (int q = threadIdx.x; q < 128 * 128; q += blockDim.x) {
    const int r = q >> 7, k = q & 127;
    *reinterpret_cast<uint16_t*>(sW2 + umma::sw128_offset(128, r, k)) = Op16<F16>::bits(P[kOffW2 + q]);
  }
  for (int q = threadIdx.x; q < 64 * 128; q += blockDim.x) {
    const int r = q >> 7, k = q & 127;
    *reinterpret_cast<uint16_t*>(sW3 + umma::sw128_offset(64, r, k)) = Op16<F16>::bits(P[kOffW3 + q]);
  }
  for (int q = threadIdx.x; q < 16 * 64; q += blockDim.x) {
    const int r = q >> 6, k = q & 63;
    float hi, lo;
    Op16<F16>::split(P[kOffW4 + k], &hi, &lo);
    *reinterpret_cast<uint16_t*>(sW4 + umma::sw128_offset(16, r, k)) = Op16<F16>::bits(r == 0 ? hi : r == 1 ? lo : 0.0f);
  }
}

// Row `row` of a K-major SW128 activation tile: 16-byte chunk j (columns
// 8j .. 8j+7 of a 64-column atom) of atom a sits at
// rowp + a * 128 * 128 + ((j << 4) ^ r7s), r7s = (row % 8) << 4.
__device__ __forceinline__ uint4* tile_chunk(unsigned char* rowp, int r7s, int a, int j) {
  return reinterpret_cast<uint4*>(rowp + a * 128 * 128 + ((j << 4) ^ r7s));
}

// The activation of 16 loaded accumulator columns c .. c+15 -> the
// activation tile (two 16-byte stores)
template <int ACT, bool F16>
__device__ __forceinline__ void act_store16(unsigned char* rowp, int r7s, int c, const uint32_t* v) {
  uint32_t h[8];
#pragma unroll
  for (int i = 0; i < 8; i++) {
    if constexpr (ACT == CBMV_ACT_GELU)
      h[i] = Op16<F16>::gelu(__uint_as_float(v[2 * i]), __uint_as_float(v[2 * i + 1]));
    else
      h[i] = Op16<F16>::relu(__uint_as_float(v[2 * i]), __uint_as_float(v[2 * i + 1]));
  }
#pragma unroll
  for (int q = 0; q < 2; q++)
    *tile_chunk(rowp, r7s, c >> 6, ((c & 63) >> 3) + q) = make_uint4(h[4 * q], h[4 * q + 1], h[4 * q + 2], h[4 * q + 3]);
}

// Columns C0 .. C0+NC-1 of the accumulator (tensor-memory columns and
// activation-tile columns alike; C0 a multiple of 64), 16 columns per
// tensor-memory load, the next load in flight while the current columns
// are computed.
template <int C0, int NC, int ACT, bool F16>
__device__ __forceinline__ void epilogue_hidden(uint32_t tlane, unsigned char* rowp, int r7s) {
  uint32_t ga[16], gb[16];
  umma::tmem_ld16_issue(tlane + C0, ga);
  umma::tmem_ld16_wait(ga);
#pragma unroll
  for (int c = C0; c < C0 + NC; c += 32) {
    umma::tmem_ld16_issue(tlane + c + 16, gb);
    act_store16<ACT, F16>(rowp, r7s, c, ga);
    umma::tmem_ld16_wait(gb);
    if (c + 32 < C0 + NC) umma::tmem_ld16_issue(tlane + c + 32, ga);
    act_store16<ACT, F16>(rowp, r7s, c + 16, gb);
    if (c + 32 < C0 + NC) umma::tmem_ld16_wait(ga);
  }
}

// Inputs of the four matchers' features of one sample: its costs and the
// row statistics (min, 1/den) of its left and right views.
struct FeatIn {
  float c[4];
  float2 sl[4], sr[4];
};

__device__ __forceinline__ void load_feat_in(const FeatVolsF& fv, const float2* __restrict__ statsf, int64_t HW,
                                             int64_t N, int64_t t, int64_t p, int d, int64_t x, FeatIn& in) {
  const bool valid = t < N;
  const int64_t tv = valid ? t : 0, pv = valid ? p : 0;
  const int dv = valid ? d : 0;
  const bool has_right = valid && x >= d;
#pragma unroll
  for (int m = 0; m < 4; m++) {
    in.c[m] = __ldg(fv.v[m] + tv);
    in.sl[m] = __ldg(statsf + (int64_t)(2 * m) * HW + pv);
    in.sr[m] = has_right ? __ldg(statsf + (int64_t)(2 * m + 1) * HW + pv - dv) : make_float2(kRandMaxF, 0.0f);
  }
}

// The 20 features of one sample in the reference's column order
// (test.py:521-595): 0-3 the costs, 4-7 ratio, 8-11 likelihood, 12-19 the
// same two of the right view warped to the left, all in float32.
__device__ __forceinline__ void features_f32(const FeatIn& in, float* f) {
#pragma unroll
  for (int m = 0; m < 4; m++) {
    const float c = in.c[m];
    const float inv_ce = __fdividef(1.0f, c + kEpsF[m]);
    f[m] = c;
    conf_f32(c, inv_ce, in.sl[m], kEpsF[m], kInvSigmaF[m], &f[4 + m], &f[8 + m]);
    conf_f32(c, inv_ce, in.sr[m], kEpsF[m], kInvSigmaF[m], &f[12 + m], &f[16 + m]);
  }
}

// The learned path's float32 features of the samples idx[i] = (y*W + x)*D + d,
// through the same code as the fused kernel below; out [n, 20].
__global__ void features_f32_gather_kernel(FeatVolsF fv, const float2* __restrict__ statsf, int64_t H, int64_t W,
                                           int D, const int64_t* __restrict__ idx, int64_t n, float* __restrict__ out) {
  const int64_t HW = H * W, N = HW * D;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t t = idx[i];
    const int64_t p = t / D;
    FeatIn in;
    load_feat_in(fv, statsf, HW, N, t, p, (int)(t - p * D), p % W, in);
    float f[20];
    features_f32(in, f);
#pragma unroll
    for (int k = 0; k < 20; k++) out[i * 20 + k] = f[k];
  }
}

template <int ACT, bool F16>
__global__ void __launch_bounds__(kInfThreads, 1)
    features_mlp_kernel(FeatVolsF fv, const float2* __restrict__ statsf, int64_t H, int64_t W, int D,
                        const float* __restrict__ P, float* __restrict__ prob0, int* __restrict__ status) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* sW1 = base;
  unsigned char* sW2 = sW1 + kSmW1i;
  unsigned char* sW3 = sW2 + kSmW2i;
  unsigned char* sW4 = sW3 + kSmW3i;
  unsigned char* sOne = sW4 + kSmW4i;
  unsigned char* sTiles = sOne + kSmOne;
  __shared__ float4 s_nrm[kF];  // per feature column: cap, mu, inv_sd
  __shared__ float s_b4;
  __shared__ uint64_t bars[kGroups];
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, g = tid / kGroupThreads, row = tid % kGroupThreads, wq = row >> 5;

  if (tid < 32) umma::tmem_alloc(&tmem_base, 128 * kGroups);
  if (tid < kGroups) umma::mbar_init(&bars[tid], 1);
  stage_inference_weights<F16>(P, sW1, sW2, sW3, sW4, sOne);
  for (int i = tid; i < kF; i += kInfThreads) s_nrm[i] = make_float4(P[i], P[kF + i], P[2 * kF + i], 0.0f);
  if (tid == 0) s_b4 = P[kOffB4];
  umma::fence_async_smem();
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();

  unsigned char* sA = sTiles + g * kSmTile;
  unsigned char* rowp = sA + (row >> 3) * 1024 + (row & 7) * 128;
  const int r7s = (row & 7) << 4;
  uint64_t* bar0 = &bars[g];
  const uint32_t tacc = tmem_base + (uint32_t)(g * 128);
  const uint32_t tlane = tacc + ((uint32_t)(wq * 32) << 16);
  const bool leader = row == 0;
  constexpr uint32_t id128 = Op16<F16>::idesc(128, 128), id64 = Op16<F16>::idesc(128, 64),
                     id16 = Op16<F16>::idesc(128, 16);
  // operand descriptors, formed where the leader issues (keeps them out of the other threads' registers)
#define DESC(ptr) umma::sw128_desc(umma::smem_u32(ptr))

  const int64_t HW = H * W, N = HW * D;
  const int64_t tiles = (N + 127) / 128;
  const int64_t tstride = (int64_t)gridDim.x * kGroups;
  // this thread's sample t = tile * 128 + row as (pixel p, disparity d, column x), advanced incrementally
  int64_t tile = (int64_t)blockIdx.x * kGroups + g;
  int64_t t = tile * 128 + row;
  int64_t p = t / D;
  int d = (int)(t - p * D);
  int64_t x = p % W;
  const int64_t step = tstride * 128;
  const int64_t sp = step / D;
  const int sd = (int)(step - sp * D);
  const int64_t sx = sp % W;
  // the group's MMAs are committed to bar0, one phase per layer
  uint32_t ph0 = 0;
  bool ok = true;
  // the leader polls, the group learns the result at its named barrier
  auto wait = [&](uint64_t* b, uint32_t& ph) {
    const bool r = group_all(g, leader ? umma::mbar_wait(b, ph, kWaitLimit) : true);
    ph ^= 1u;
    umma::tc_fence_after();
    return r;
  };
  auto handoff = [&]() {  // the group's shared-memory writes -> the next MMAs
    umma::fence_async_smem();
    umma::tc_fence_before();
    group_sync(g);
    umma::tc_fence_after();
  };

  FeatIn in;
  load_feat_in(fv, statsf, HW, N, t, p, d, x, in);
  for (; tile < tiles; tile += tstride) {
    // 1. the 20 features of sample t -> row of X0, in the tile's second
    //    atom: columns 0..19 in the reference's order, 20 and 21 the bias
    //    inputs, 22..31 zero
    {
      float f[20];
      features_f32(in, f);
      uint32_t u[10];
#pragma unroll
      for (int k = 0; k < 20; k += 2) {
        const float4 na = s_nrm[k], nb = s_nrm[k + 1];
        u[k >> 1] = Op16<F16>::pack((fminf(f[k], na.x) - na.y) * na.z, (fminf(f[k + 1], nb.x) - nb.y) * nb.z);
      }
      *tile_chunk(rowp, r7s, 1, 0) = make_uint4(u[0], u[1], u[2], u[3]);
      *tile_chunk(rowp, r7s, 1, 1) = make_uint4(u[4], u[5], u[6], u[7]);
      *tile_chunk(rowp, r7s, 1, 2) = make_uint4(u[8], u[9], Op16<F16>::kOneOne, 0u);
      *tile_chunk(rowp, r7s, 1, 3) = make_uint4(0u, 0u, 0u, 0u);
    }
    // advance to this thread's next sample (tile + tstride) and load its
    // inputs, in flight while this tile runs through the network
    const int64_t t_cur = t;
    t += step;
    p += sp;
    d += sd;
    x += sx;
    if (d >= D) {
      d -= D;
      p += 1;
      x += 1;
    }
    if (x >= W) x -= W;
    if (tile + tstride < tiles) load_feat_in(fv, statsf, HW, N, t, p, d, x, in);
    handoff();
    // 2. layer 1 (K = 32) -> accumulator columns 0..127
    if (leader) {
      const uint64_t dX = DESC(sA + 128 * 128), dW1 = DESC(sW1);
      umma::mma_f16(tacc, dX, dW1, id128, false);
      umma::mma_f16(tacc, dX + 2, dW1 + 2, id128, true);
      umma::mma_commit(bar0);
    }
    if (!(ok = wait(bar0, ph0))) break;
    epilogue_hidden<0, 128, ACT, F16>(tlane, rowp, r7s);
    handoff();
    // 3. layer 2 (K = 128) onto the bias b2
    if (leader) {
      const uint64_t dA0 = DESC(sA), dA1 = DESC(sA + 128 * 128), dW20 = DESC(sW2), dW21 = DESC(sW2 + 128 * 128);
      umma::mma_f16(tacc, DESC(sOne), DESC(sW1) + 2 * (kColB2 / 16), id128, false);
#pragma unroll
      for (int kk = 0; kk < 4; kk++) umma::mma_f16(tacc, dA0 + 2 * kk, dW20 + 2 * kk, id128, true);
#pragma unroll
      for (int kk = 0; kk < 4; kk++) umma::mma_f16(tacc, dA1 + 2 * kk, dW21 + 2 * kk, id128, true);
      umma::mma_commit(bar0);
    }
    if (!(ok = wait(bar0, ph0))) break;
    epilogue_hidden<0, 128, ACT, F16>(tlane, rowp, r7s);
    handoff();
    // 4. layer 3 (N = 64) onto the bias b3
    if (leader) {
      const uint64_t dA0 = DESC(sA), dA1 = DESC(sA + 128 * 128), dW30 = DESC(sW3), dW31 = DESC(sW3 + 64 * 128);
      umma::mma_f16(tacc, DESC(sOne), DESC(sW1) + 2 * (kColB3 / 16), id64, false);
#pragma unroll
      for (int kk = 0; kk < 4; kk++) umma::mma_f16(tacc, dA0 + 2 * kk, dW30 + 2 * kk, id64, true);
#pragma unroll
      for (int kk = 0; kk < 4; kk++) umma::mma_f16(tacc, dA1 + 2 * kk, dW31 + 2 * kk, id64, true);
      umma::mma_commit(bar0);
    }
    if (!(ok = wait(bar0, ph0))) break;
    epilogue_hidden<0, 64, ACT, F16>(tlane, rowp, r7s);
    handoff();
    // 5. output layer (N = 16, rows 0/1 = high/low parts of w4) -> columns 64..79
    if (leader) {
      const uint64_t dA0 = DESC(sA), dW4 = DESC(sW4);
#pragma unroll
      for (int kk = 0; kk < 4; kk++) umma::mma_f16(tacc + 64, dA0 + 2 * kk, dW4 + 2 * kk, id16, kk > 0);
      umma::mma_commit(bar0);
    }
    if (!(ok = wait(bar0, ph0))) break;
    {
      uint32_t z2[2];
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0,%1}, [%2];"
                   : "=r"(z2[0]), "=r"(z2[1])
                   : "r"(tlane + 64));
      asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(z2[0]), "+r"(z2[1]) : : "memory");
      const float z = (__uint_as_float(z2[0]) + __uint_as_float(z2[1])) + s_b4;
      if (t_cur < N) prob0[t_cur] = 1.0f / (1.0f + __expf(z));
    }
    umma::tc_fence_before();
  }
  if (!ok && leader) {
    // a wait gave up: record it, then let the group's MMAs still in flight
    // finish (bounded: the phase that was waited for) before the memory is
    // freed
    atomicExch(status, 1);
    umma::mbar_wait(bar0, ph0 ^ 1u, kWaitLimit);
  }
  umma::tc_fence_before();
  __syncthreads();
  if (tid < 32) umma::tmem_dealloc(tmem_base, 128 * kGroups);
#undef DESC
}

}  // namespace

// Launch shape of the fused kernel; returns the grid (CTAs).
inline int features_mlp_grid(int64_t H, int64_t W, int D, int max_ctas, int sms) {
  const int64_t tiles = (H * W * D + 127) / 128;
  const int64_t need = (tiles + kGroups - 1) / kGroups;
  const int cap = max_ctas > 0 && max_ctas < sms ? max_ctas : sms;
  return (int)(need < cap ? need : cap);
}

template <int ACT, bool F16>
int launch_features_mlp_act(const float* const* vols, const float2* statsf, int64_t H, int64_t W, int D,
                            const cbmv_mlp* m, float* prob0, cudaStream_t st, int max_ctas) {
  int dev = 0, sms = 0;
  CBMV_CUDA(cudaGetDevice(&dev));
  CBMV_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  CBMV_CUDA(cudaFuncSetAttribute(features_mlp_kernel<ACT, F16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kSmInf));
  CBMV_REQUIRE(((uintptr_t)statsf & 7) == 0, CBMV_EINVAL, "feature statistics must be 8-byte aligned");
  const int grid = features_mlp_grid(H, W, D, max_ctas, sms);
  FeatVolsF fv = {{vols[0], vols[1], vols[2], vols[3]}};
  features_mlp_kernel<ACT, F16><<<grid, kInfThreads, kSmInf, st>>>(fv, statsf, H, W, D, m->P, prob0, m->status);
  return check_launch("features_mlp");
}

}  // namespace cbmv
