// Definitions shared by the learned classifier's training kernels (mlp.cu)
// and its fused inference kernels (mlp_infer_relu.cu, mlp_infer_gelu.cu):
// the parameter-vector layout, the hidden-layer activations and the device
// state of a network (struct cbmv_mlp).
#pragma once
#include <cuda_bf16.h>

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
// without the special-function unit: Phi(x) ~ sat(0.5 + x * p(x^2)), sat =
// clamp to [0, 1], p(u) = G0 + G1 u + G2 u^2 + G3 u^3 + G4 u^4.  The
// coefficients are a minimax fit of x * (0.5 + x p(x^2)) to x * Phi(x) on
// [0, 3.45] by linear programming, constrained so that 0.5 + x p(x^2) >= 1
// for x >= 3.45 (where Phi > 0.9997) and, by symmetry, <= 0 for x <= -3.45:
// the saturation then makes the function exact to x (or 0) in the tails.
// In float32, in exactly the order below, |gelu(x) - x Phi(x)| <= 1.15e-3
// for every x (the activation is rounded to bf16 next, a relative 2^-9).
// Training and the fused inference kernel evaluate it identically (the
// inference kernel two lanes at a time with the packed float32 FMA).
constexpr float kG0 = 3.9385697e-01f, kG1 = -5.9378225e-02f, kG2 = 6.5808324e-03f,
                kG3 = -3.9975342e-04f, kG4 = 9.9452836e-06f;

__device__ __forceinline__ float fma_sat(float a, float b, float c) {
  float r;
  asm("fma.rn.sat.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}

// GELU and its derivative: Phi~ + x Phi~' where 0 < 0.5 + x p < 1, else Phi~
__device__ __forceinline__ float gelu_t(float x, float* dgelu) {
  const float u = x * x;
  const float p = fmaf(fmaf(fmaf(fmaf(kG4, u, kG3), u, kG2), u, kG1), u, kG0);
  const float q = fma_sat(x, p, 0.5f);
  if (dgelu) {
    const float qr = fmaf(x, p, 0.5f);
    const float dp = fmaf(fmaf(fmaf(4.0f * kG4, u, 3.0f * kG3), u, 2.0f * kG2), u, kG1);  // p'(u)
    const float dq = fmaf(2.0f * u, dp, p);                                                 // d(x p(x^2))/dx
    *dgelu = (qr > 0.0f && qr < 1.0f) ? fmaf(x, dq, q) : q;
  }
  return x * q;
}

// the network's activation (cbmv_mlp_set_activation) and its derivative
__device__ __forceinline__ float act_t(int act, float x, float* d) {
  return act == CBMV_ACT_GELU ? gelu_t(x, d) : relu_t(x, d);
}

__device__ __forceinline__ uint16_t to_bf16(float x) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(x));
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
  int act = CBMV_ACT_RELU;  // hidden-layer activation
};
