// Launch helpers shared by the fused pipeline (pipeline.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "rf.cuh"

namespace cbmv {

// Matcher arguments: non-null pointers, 0 < H <= 65535, 0 < D <= 65535
// (CBMV_ERANGE beyond), W > 0, window odd and <= wmax, dtype and layout.
int check_common(const void* a, const void* b, const void* out, int64_t H, int64_t W, int D, int w,
                 int dtype, int layout, int wmax);
int launch_census_desc(const uint8_t* img, int64_t H, int64_t W, int w, ulonglong2* desc,
                       cudaStream_t st);
template <class T>
int launch_census_cost(const ulonglong2* dl, const ulonglong2* dr, int64_t H, int64_t W, int D,
                       int w, int layout, T* out, cudaStream_t st);
int launch_ncc_stats(const uint8_t* img, int64_t H, int64_t W, int w, uint32_t* A, double* C,
                     cudaStream_t st);
template <class T>
int launch_ncc_cost(const uint8_t* L, const uint8_t* R, const uint32_t* Al, const uint32_t* Ar,
                    const double* Cl, const double* Cr, int64_t H, int64_t W, int D, int w,
                    int layout, T* out, cudaStream_t st);
int launch_sobel_i32(const uint8_t* img, int64_t H, int64_t W, int32_t* out, cudaStream_t st);
template <class T>
int launch_sadsob_cost(const int32_t* SL, const int32_t* SR, int64_t H, int64_t W, int D, int w,
                       int layout, T* out, cudaStream_t st);
int launch_zsad_means(const uint8_t* img, int64_t H, int64_t W, int w, double* mean,
                      cudaStream_t st);
template <class T>
int launch_zsad_cost(const uint8_t* L, const uint8_t* R, const double* ml, const double* mr,
                     int64_t H, int64_t W, int D, int w, int layout, T* out, cudaStream_t st);
// float32 [H,W,D] window matchers for the learned path (strip kernels)
int launch_ncc_cost_f32(const uint8_t* L, const uint8_t* R, const uint32_t* Al, const uint32_t* Ar,
                        const double* Cl, const double* Cr, int64_t H, int64_t W, int D, int w, float* out,
                        cudaStream_t st);
int launch_sadsob_cost_f32(const int32_t* SL, const int32_t* SR, int64_t H, int64_t W, int D, int w, float* out,
                           cudaStream_t st);
int launch_zsad_cost_f32(const uint8_t* L, const uint8_t* R, const double* ml, const double* mr, int64_t H,
                         int64_t W, int D, int w, float* out, cudaStream_t st);
int launch_feature_stats(const double* const* vols, int64_t H, int64_t W, int D, double* stats,
                         cudaStream_t st, float2* statsf = nullptr);
// (min, 1/den) in float32 of float32 volumes, both views, the four matchers
int launch_feature_stats_f32(const float* const* vols, int64_t H, int64_t W, int D, float2* statsf,
                             cudaStream_t st);
int launch_features_mlp(const float* const* vols, const float2* statsf, int64_t H, int64_t W, int D,
                        const cbmv_mlp* m, float* prob0, cudaStream_t st, int max_ctas = 0);
// The learned path's float32 features of the samples idx[i] = (y*W + x)*D + d
// (the fused network kernel's own feature code), out [n, 20].
int launch_features_f32_gather(const float* const* vols, const float2* statsf, int64_t H, int64_t W, int D,
                               const int64_t* idx, int64_t n, float* out, cudaStream_t st);
// The 20 features (float32) of the samples idx[i] = (y*W + x)*D + d.
int launch_features_gather(const double* const* vols, const double* stats, int64_t H, int64_t W,
                           int D, const int64_t* idx, int64_t n, float* out, cudaStream_t st);
int launch_features_rf(const double* const* vols, const double* stats, int64_t H, int64_t W,
                       int D, const cbmv_forest* forest, float* prob0, cudaStream_t st);

}  // namespace cbmv
