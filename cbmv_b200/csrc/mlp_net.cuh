// Definitions shared by the learned classifier's training kernels (mlp.cu)
// and its fused inference kernels (mlp_infer_relu.cu, mlp_infer_gelu.cu):
// the parameter-vector layout, the hidden-layer activations and the device
// state of a network (struct cbmv_mlp).
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"

namespace cbmv {
namespace {

// polls of an mbarrier before a tensor-core wait gives up (and reports)
constexpr uint32_t kWaitLimit = 1u << 22;

constexpr int kF = 20, kK1 = 64, kH1 = 128, kH2 = 128, kH3 = 64;
constexpr int kNormN = 3 * kF;
constexpr int kOffW1 = kNormN, kOffB1 = kOffW1 + kH1 * kF, kOffW2 = kOffB1 + kH1,
              kOffB2 = kOffW2 + kH2 * kH1, kOffW3 = kOffB2 + kH2, kOffB3 = kOffW3 + kH3 * kH2,
              kOffW4 = kOffB3 + kH3, kOffB4 = kOffW4 + kH3, kNParams = kOffB4 + 1;

// ReLU and its derivative (0 at x = 0)
__device__ __forceinline__ float relu_t(float x, float* drelu) {
  if (drelu) *drelu = x > 0.0f ? 1.0f : 0.0f;
  return x > 0.0f ? x : 0.0f;
}

// The network's GELU, x * Phi(x) with Phi the standard normal CDF, computed
// in half-precision (binary16) arithmetic (the fused inference stores its
// activations as f16 anyway), on the packed half-precision FMA pipe,
// without the special-function unit:
//   x <- f16(x);  u = x * x;  p = G2 u + G1;  p = p u + G0;
//   q = sat(x p + 0.5) (clamped to [0, 1]);  gelu = x * q
// every operation one f16 rounding (round to nearest even), q ~ Phi(x).
// G0..G2 (f16) are a minimax fit of x * clamp(0.5 + x (G0 + G1 x^2 + G2 x^4),
// 0, 1) to x * Phi(x), then the f16 coefficients searched for the smallest
// error of this f16 evaluation: over every finite f16 x, |gelu(x) - x Phi(x)|
// <= 8.32e-3 (the polynomial itself is within 7.7e-3; rounding x Phi(x) to
// f16 costs up to 9.8e-4 below 8); the clamp makes it x for x >= 3.5 and 0
// (-0) for x <= -3.5; x is saturated to +-65504 when it is rounded to f16,
// and where x * x overflows q is 1 or 0, so the value stays finite (x or
// -0).  Training and the fused inference
// kernel (two lanes at a time, `fma.rn.sat.f16x2` for the clamp) evaluate
// it identically.
constexpr uint16_t kG0Bits = 0x35fe, kG1Bits = 0xa977, kG2Bits = 0x18a7;  // 0.37451171875, -0.042694091796875, 0.0022716522216796875

__device__ __forceinline__ __half f16_bits(uint16_t b) { return __ushort_as_half(b); }

// The same form evaluated in bfloat16 operations, for the fused inference
// with bf16 operands (cbmv_mlp_set_precision): x <- bf16(x); u = x * x;
// p = G2 u + G1; p = p u + G0; q = min(max(x p + 0.5, 0), 1); x * q, every
// operation one bf16 rounding, with coefficients searched for this bf16
// evaluation: within 1.21e-2 of x * Phi(x) on every bf16 x.
constexpr uint16_t kGB0Bits = 0x3ebf, kGB1Bits = 0xbd30, kGB2Bits = 0x3b1c;  // 0.373046875, -0.04296875, 0.00238037109375
__device__ __forceinline__ __nv_bfloat16 bf16_bits(uint16_t b) { return __ushort_as_bfloat16(b); }

// GELU of x (float32 in, its f16 rounding used) and, for the backward pass,
// the derivative of the smooth function it approximates at that point:
// q + x (p + 2 u p'(u)) where 0 < x p + 0.5 < 1, else q (0 or 1), in float32.
__device__ __forceinline__ float gelu_t(float x, float* dgelu) {
  const __half xh = __float2half_rn(fminf(fmaxf(x, -65504.0f), 65504.0f));  // saturated, as the fused kernel's cvt
  const __half u = __hmul(xh, xh);
  __half p = __hfma(f16_bits(kG2Bits), u, f16_bits(kG1Bits));
  p = __hfma(p, u, f16_bits(kG0Bits));
  const __half q = __hfma_sat(xh, p, __float2half_rn(0.5f));
  const float g = __half2float(__hmul(xh, q));
  if (dgelu) {
    const float xf = __half2float(xh), uf = xf * xf;
    const float g0 = __half2float(f16_bits(kG0Bits)), g1 = __half2float(f16_bits(kG1Bits)),
                g2 = __half2float(f16_bits(kG2Bits));
    const float pf = fmaf(fmaf(g2, uf, g1), uf, g0);
    const float qr = fmaf(xf, pf, 0.5f);
    const float dq = fmaf(2.0f * uf, fmaf(2.0f * g2, uf, g1), pf);  // d(x p(x^2))/dx
    *dgelu = qr <= 0.0f ? 0.0f : qr >= 1.0f ? 1.0f : fmaf(xf, dq, qr);
  }
  return g;
}

// the network's activation (cbmv_mlp_set_activation) and its derivative
__device__ __forceinline__ float act_t(int act, float x, float* d) {
  return act == CBMV_ACT_GELU ? gelu_t(x, d) : relu_t(x, d);
}

__device__ __forceinline__ uint16_t to_bf16(float x) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}
// float32 -> f16 bits, round to nearest even, saturated to +-65504
__device__ __forceinline__ uint16_t to_f16(float x) {
  return __half_as_ushort(__float2half_rn(fminf(fmaxf(x, -65504.0f), 65504.0f)));
}

}  // namespace
}  // namespace cbmv

struct cbmv_mlp {
  int B = 0;
  void* mem = nullptr;
  float *P, *m, *v, *g;                  // params, Adam moments, gathered grads
  uint16_t *W1b, *W1T, *W2b, *W2T, *W3b, *W3T;
  uint16_t *X0, *X0T, *A1, *A1T, *A2, *A2T, *dS3, *dS3T, *dS2, *dS2T, *dS1, *dS1T;
  float *Z, *S1, *S2, *S3, *A3f, *dA, *dSf, *loss_i, *dz, *dw4_i;
  float *dW1, *dW2, *dW3T, *db1, *db2, *db3, *dw4, *db4, *loss;
  int* status;
  int step = 0;
  int act = CBMV_ACT_RELU;    // hidden-layer activation
  int prec = CBMV_PREC_F16;   // 16-bit operand type of the fused inference
};
