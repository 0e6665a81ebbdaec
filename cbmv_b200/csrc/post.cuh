// Launch helpers of the cost-optimisation kernels (post.cu), shared with the
// fused pipeline.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cbmv {

struct SgmParams {
  float pi1, pi2, tau_so, alpha1, q1, q2;
  int direction;
};

int launch_cross(const float* img, int64_t H, int64_t W, int L1, float tau1, float* out,
                 cudaStream_t st);
// Neighbour differences of both normalised images (see post.cu grad_kernel).
struct SgmGrad {
  float *lh, *lv, *rh, *rv;
};
int launch_sgm_grad(const float* imL, const float* imR, int64_t H, int64_t W, SgmGrad* g,
                    cudaStream_t st);
// Path costs of the four scan directions, one volume each.
struct SgmOut {
  float* dir[4];
};
int launch_sgm4(const SgmGrad& g, const float* in, int64_t H, int64_t W, int D, const SgmParams& sp,
                const SgmOut& o, cudaStream_t st, int prefetch = 0);
// out = base + (((L0 + L1) + L2) + L3) * scale; base may be null or out.
int launch_sgm_combine(const SgmOut& o, int64_t n, const float* base, float scale, float* out,
                       cudaStream_t st);
// halo: how far (pixels) the cross arms' interior reaches, L1 - 1; supports
// reaching further are still summed correctly, from global memory.
int launch_cbca(const float* lc, const float* rc, const float* in, int64_t H, int64_t W, int D,
                int layout, int direction, float* out, cudaStream_t st, int halo = 5);
// cbca on [H,W,D] in separable form (row sums, then column sums); arms of
// at most `halo` pixels (L1 - 1), halo 1..8 (larger: the reference-order kernel)
int launch_cbca_sep(const float* lc, const float* rc, const float* in, int64_t H, int64_t W, int D,
                    int direction, float* out, cudaStream_t st, int halo, int rows = 32);
// the separable cbca with its supports precomputed (arms of at most 5
// pixels, L1 <= 6): one 32-bit word per (p,d) in `mask`, built once per
// cross, then any number of passes; bit-identical to launch_cbca_sep
int launch_cbca_mask_build(const float* lc, const float* rc, int64_t H, int64_t W, int D, int direction,
                           uint32_t* mask, cudaStream_t st);
int launch_cbca_masked(const uint32_t* mask, const float* in, int64_t H, int64_t W, int D, float* out,
                       cudaStream_t st, int rows = 32);
constexpr int kCbcaMaskMaxHalo = 5;
int launch_wta_subpixel(const float* cost, int64_t H, int64_t W, int D, float* disp_int,
                        float* disp, cudaStream_t st);
int launch_median(const float* in, int64_t H, int64_t W, int k, float* out, cudaStream_t st);
int launch_mean2d(const float* in, int64_t H, int64_t W, const float* kernel, int ks, float alpha2,
                  float* out, cudaStream_t st);
int launch_normalise(const uint8_t* img, int64_t n, double* mom, float* out, cudaStream_t st);
// get_right_cost of a float32 [H,W,D] volume (the _interp post's right view)
int launch_right_cost_f32(const float* in, int64_t H, int64_t W, int D, float* out, cudaStream_t st);
int launch_outlier(const float* d0, const float* d1, int64_t H, int64_t W, int disp_max, float* out,
                   cudaStream_t st);
int launch_mismatch(const float* d0, const float* o, int64_t H, int64_t W, float* out,
                    cudaStream_t st);
int launch_occlusion(const float* d0, const float* o, int64_t H, int64_t W, float* out,
                     cudaStream_t st);

}  // namespace cbmv
