// Shared helpers of libcbmv: status codes, the per-thread error message,
// argument checks and small device utilities.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/cbmv.h"

namespace cbmv {

// The reference's invalid-cost sentinel, glibc RAND_MAX (matchers.cpp:42,
// 229, 374, 460 fill the volumes with it).
constexpr double kRandMax = 2147483647.0;
// The same sentinel once stored as float32.
constexpr float kRandMaxF = 2147483648.0f;

int set_error(int code, const char* fmt, ...);
int check_launch(const char* what);

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Grid size for a 1-D launch over n items with `block` threads per block,
// capped at a multiple of the SM count (grid-stride loops cover the rest).
unsigned grid_for(int64_t n, int block);

template <class T> struct dtype_of;
template <> struct dtype_of<float> { static constexpr int value = CBMV_F32; };
template <> struct dtype_of<double> { static constexpr int value = CBMV_F64; };

// Store a float64 value into a volume element of type T.
template <class T> __device__ __forceinline__ T cvt_out(double v) { return static_cast<T>(v); }

// Index of element (y, x, d) of an H x W x D volume in the given layout.
__device__ __forceinline__ int64_t vol_index(int layout, int64_t y, int64_t x, int64_t d,
                                             int64_t H, int64_t W, int64_t D) {
  return layout == CBMV_HWD ? (y * W + x) * D + d : (d * H + y) * W + x;
}

}  // namespace cbmv

#define CBMV_REQUIRE(cond, code, ...)                         \
  do {                                                        \
    if (!(cond)) return ::cbmv::set_error((code), __VA_ARGS__); \
  } while (0)

#define CBMV_CUDA(call)                                                                  \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return ::cbmv::set_error(CBMV_ECUDA, "%s: %s", #call, cudaGetErrorString(e_));     \
  } while (0)
