// BF16 tensor-core kernels of the learned matching-probability classifier
// (the MLP surrogate of the reference's random forest, test.py:603-620):
// a general C = A * B^T GEMM on tcgen05 used by the trainer.
//
// Every CTA computes a 128-row x N tile: the K dimension streams through
// shared memory in 64-wide, 128-byte-swizzled chunks (umma.cuh), one thread
// issues four 128xNx16 MMAs per chunk into a float32 accumulator in tensor
// memory, and the epilogue reads it back with tcgen05.ld (warp w owns rows
// 32w..32w+31).  Waits on the MMA-completion barrier are bounded: on a
// timeout the kernel records an error in `status` and returns.
#include <cuda_bf16.h>

#include "common.cuh"
#include "umma.cuh"

namespace cbmv {
namespace {

constexpr uint32_t kWaitLimit = 1u << 22;

template <int NT>
__global__ void __launch_bounds__(128) gemm_bf16_kernel(const uint16_t* __restrict__ A,
                                                         const uint16_t* __restrict__ B,
                                                         float* __restrict__ C, int M, int N, int K,
                                                         int* __restrict__ status) {
  constexpr int kTmemCols = NT < 32 ? 32 : NT;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte aligned operand tiles: A 128x64, B NTx64 bf16
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* sA = base;
  unsigned char* sB = base + 128 * 128;
  __shared__ uint64_t bar;
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int m0 = blockIdx.x * 128;
  const int n0 = blockIdx.y * NT;

  if (warp == 0) umma::tmem_alloc(&tmem_base, kTmemCols);
  if (tid == 0) umma::mbar_init(&bar, 1);
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = umma::idesc_bf16(128, NT);
  bool ok = true;
  uint32_t phase = 0;

  for (int k0 = 0; k0 < K && ok; k0 += 64) {
    // stage A[m0:m0+128, k0:k0+64] and B[n0:n0+NT, k0:k0+64], 16 B per thread-step
    for (int q = tid; q < 128 * 8; q += 128) {
      const int r = q >> 3, c = q & 7;
      const uint4 v = *reinterpret_cast<const uint4*>(A + (size_t)(m0 + r) * K + k0 + c * 8);
      *reinterpret_cast<uint4*>(sA + umma::sw128_offset(128, r, c * 8)) = v;
    }
    for (int q = tid; q < NT * 8; q += 128) {
      const int r = q >> 3, c = q & 7;
      const uint4 v = *reinterpret_cast<const uint4*>(B + (size_t)(n0 + r) * K + k0 + c * 8);
      *reinterpret_cast<uint4*>(sB + umma::sw128_offset(NT, r, c * 8)) = v;
    }
    umma::fence_async_smem();
    umma::tc_fence_before();
    __syncthreads();
    umma::tc_fence_after();
    if (tid == 0) {
      const uint64_t da = umma::sw128_desc(umma::smem_u32(sA));
      const uint64_t db = umma::sw128_desc(umma::smem_u32(sB));
#pragma unroll
      for (int kk = 0; kk < 4; kk++)  // 16-wide K steps: +32 B = +2 in descriptor units
        umma::mma_bf16(tmem, da + 2 * kk, db + 2 * kk, idesc, k0 > 0 || kk > 0);
      umma::mma_commit(&bar);
    }
    ok = umma::mbar_wait(&bar, phase, kWaitLimit);
    phase ^= 1u;
    umma::tc_fence_after();
  }
  if (!ok) {
    if (tid == 0) atomicExch(status, 1);
    // let the MMAs still in flight finish (bounded) before freeing their memory
    umma::mbar_wait(&bar, phase ^ 1u, kWaitLimit);
  } else {
    // epilogue: warp w reads rows 32w..32w+31, 16 columns at a time
    const int row = m0 + warp * 32 + (tid & 31);
    for (int c0 = 0; c0 < NT; c0 += 16) {
      float v[16];
      umma::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c0, v);
      float* dst = C + (size_t)row * N + n0 + c0;
#pragma unroll
      for (int i = 0; i < 16; i += 4) *reinterpret_cast<float4*>(dst + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
    }
  }
  umma::tc_fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, kTmemCols);
}

template <int NT>
int launch_gemm(const uint16_t* A, const uint16_t* B, float* C, int M, int N, int K, int* status,
                cudaStream_t st) {
  const size_t smem = 1024 + 128 * 128 + (size_t)NT * 128;
  CBMV_CUDA(cudaFuncSetAttribute(gemm_bf16_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid(M / 128, N / NT);
  gemm_bf16_kernel<NT><<<grid, 128, smem, st>>>(A, B, C, M, N, K, status);
  return check_launch("gemm_bf16");
}

}  // namespace

int launch_gemm_bf16(const uint16_t* A, const uint16_t* B, float* C, int M, int N, int K, int* status,
                     cudaStream_t st) {
  if (N % 128 == 0) return launch_gemm<128>(A, B, C, M, N, K, status, st);
  if (N % 64 == 0) return launch_gemm<64>(A, B, C, M, N, K, status, st);
  return launch_gemm<32>(A, B, C, M, N, K, status, st);
}

}  // namespace cbmv

using namespace cbmv;

extern "C" int cbmv_gemm_bf16(const uint16_t* A, const uint16_t* B, float* C, int64_t M, int64_t N,
                              int64_t K, int* status, void* stream) {
  CBMV_REQUIRE(A && B && C && status, CBMV_EINVAL, "null pointer argument");
  CBMV_REQUIRE(M > 0 && N > 0 && K > 0 && M % 128 == 0 && N % 32 == 0 && K % 64 == 0, CBMV_EINVAL,
               "gemm_bf16 needs M %% 128 == 0, N %% 32 == 0, K %% 64 == 0 (got %lld, %lld, %lld)",
               (long long)M, (long long)N, (long long)K);
  CBMV_REQUIRE(M < (1ll << 31) && N <= 65535 * 32 && K < (1 << 30), CBMV_ERANGE, "gemm too large");
  CBMV_REQUIRE(((uintptr_t)A & 15) == 0 && ((uintptr_t)B & 15) == 0 && ((uintptr_t)C & 15) == 0,
               CBMV_EINVAL, "gemm_bf16 operands must be 16-byte aligned");
  return launch_gemm_bf16(A, B, C, (int)M, (int)N, (int)K, status, as_stream(stream));
}

// ====================================================================
// MLP: 20 -> 128 -> 128 -> 64 -> 1, ReLU, sigmoid output.
// Parameter vector (float32, host order):
//   cap[20] mu[20] inv_sd[20]        input transform x' = (min(x,cap)-mu)*inv_sd
//   W1[128x20] b1[128] W2[128x128] b2[128] W3[64x128] b3[64] w4[64] b4[1]
// Training keeps float32 master weights (Adam) and bfloat16 copies for the
// tensor cores: W1b [128x64] (K zero-padded), W2b, W3b, and the transposes
// W1T [64x128], W2T, W3T [128x64] used by the input-gradient GEMMs.
// ====================================================================
namespace cbmv {
namespace {

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

__device__ __forceinline__ uint16_t to_bf16(float x) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}

#define GS(i, n) for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// raw features [B,20] -> normalised bf16 [B,64] (zero padded) and its transpose [64,B]
__global__ void mlp_prep_kernel(const float* __restrict__ X, int B, const float* __restrict__ P,
                                uint16_t* __restrict__ X0, uint16_t* __restrict__ X0T) {
  GS(t, (int64_t)B * kK1) {
    const int b = (int)(t / kK1), k = (int)(t % kK1);
    float v = 0.0f;
    if (k < kF) v = (fminf(X[(int64_t)b * kF + k], P[k]) - P[kF + k]) * P[2 * kF + k];
    const uint16_t h = to_bf16(v);
    X0[t] = h;
    X0T[(int64_t)k * B + b] = h;
  }
}

// S = Z + b; A = relu(S) as bf16 [B,N] and [N,B]; Af = relu(S) float (optional)
__global__ void mlp_bias_relu_kernel(const float* __restrict__ Z, const float* __restrict__ bias, int B,
                                     int N, float* __restrict__ S, uint16_t* __restrict__ A,
                                     uint16_t* __restrict__ AT, float* __restrict__ Af) {
  GS(t, (int64_t)B * N) {
    const int b = (int)(t / N), n = (int)(t % N);
    const float s = Z[t] + bias[n];
    S[t] = s;
    const float a = relu_t(s, nullptr);
    if (A) A[t] = to_bf16(a);
    if (AT) AT[(int64_t)n * B + b] = to_bf16(a);
    if (Af) Af[t] = a;
  }
}

// output layer, loss and the first backward step, one warp per sample:
// z = A3 . w4 + b4, p = sigmoid(z), loss_i = BCE; dz = (p - y) / B;
// dS3 = dz * w4 * relu'(S3) -> bf16 [B,64] and [64,B]; per-sample dz and
// dz*A3 kept for the (ordered) reductions of dw4 / db4.
__global__ void mlp_head_kernel(const float* __restrict__ A3f, const float* __restrict__ S3,
                                const float* __restrict__ y, const float* __restrict__ P, int B,
                                float* __restrict__ loss_i, float* __restrict__ dz,
                                float* __restrict__ dw4_i, uint16_t* __restrict__ dS3,
                                uint16_t* __restrict__ dS3T, float* __restrict__ dS3f) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < B; b += warps) {
    const float* a = A3f + (int64_t)b * kH3;
    float z = a[lane] * P[kOffW4 + lane] + a[lane + 32] * P[kOffW4 + lane + 32];
    for (int o = 16; o; o >>= 1) z += __shfl_xor_sync(0xffffffffu, z, o);
    z += P[kOffB4];
    const float p = 1.0f / (1.0f + expf(-z));
    const float yy = y[b];
    // BCE with logits, stable form
    const float l = fmaxf(z, 0.0f) - z * yy + log1pf(expf(-fabsf(z)));
    const float g = (p - yy) / (float)B;
    if (lane == 0) {
      loss_i[b] = l / (float)B;
      dz[b] = g;
    }
    for (int k = lane; k < kH3; k += 32) {
      float dg;
      relu_t(S3[(int64_t)b * kH3 + k], &dg);
      const float d = g * P[kOffW4 + k] * dg;
      dS3[(int64_t)b * kH3 + k] = to_bf16(d);
      dS3T[(int64_t)k * B + b] = to_bf16(d);
      dS3f[(int64_t)b * kH3 + k] = d;
      dw4_i[(int64_t)b * kH3 + k] = g * a[k];
    }
  }
}

// dS = dA * relu'(S) -> bf16 [B,N], [N,B] and float [B,N]
__global__ void mlp_drelu_kernel(const float* __restrict__ dA, const float* __restrict__ S, int B, int N,
                                 uint16_t* __restrict__ dS, uint16_t* __restrict__ dST,
                                 float* __restrict__ dSf) {
  GS(t, (int64_t)B * N) {
    const int b = (int)(t / N), n = (int)(t % N);
    float dg;
    relu_t(S[t], &dg);
    const float d = dA[t] * dg;
    dS[t] = to_bf16(d);
    dST[(int64_t)n * B + b] = to_bf16(d);
    dSf[t] = d;
  }
}

// column sums of a float [B,N] matrix in a fixed order (deterministic):
// out[n] = sum over b of M[b,n]; one thread per column, sequential over b
// in 8 interleaved partial sums added in order.
__global__ void mlp_colsum_kernel(const float* __restrict__ M, int B, int N, float* __restrict__ out) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int b = 0; b < B; b += 8)
#pragma unroll
    for (int j = 0; j < 8; j++)
      if (b + j < B) s[j] += M[(int64_t)(b + j) * N + n];
  out[n] = ((s[0] + s[1]) + (s[2] + s[3])) + ((s[4] + s[5]) + (s[6] + s[7]));
}

// Adam on float32 masters from the gathered gradient vector g (same order
// as the parameters, norm part excluded), then refresh the bf16 copies.
__global__ void mlp_adam_kernel(float* __restrict__ P, float* __restrict__ m, float* __restrict__ v,
                                const float* __restrict__ g, float lr, float b1, float b2, float eps,
                                float bc1, float bc2, float wd) {
  GS(i, (int64_t)(kNParams - kNormN)) {
    const int j = (int)i + kNormN;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const bool is_weight = (j >= kOffW1 && j < kOffB1) || (j >= kOffW2 && j < kOffB2) ||
                           (j >= kOffW3 && j < kOffB3) || (j >= kOffW4 && j < kOffB4);
    float p = P[j];
    if (is_weight) p -= lr * wd * p;
    P[j] = p - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  }
}

__global__ void mlp_pack_kernel(const float* __restrict__ P, uint16_t* __restrict__ W1b,
                                uint16_t* __restrict__ W1T, uint16_t* __restrict__ W2b,
                                uint16_t* __restrict__ W2T, uint16_t* __restrict__ W3b,
                                uint16_t* __restrict__ W3T) {
  GS(t, (int64_t)kH1 * kK1) {  // W1b [128,64], W1T [64,128]
    const int n = (int)(t / kK1), k = (int)(t % kK1);
    const uint16_t h = to_bf16(k < kF ? P[kOffW1 + n * kF + k] : 0.0f);
    W1b[t] = h;
    W1T[(int64_t)k * kH1 + n] = h;
  }
  GS(t, (int64_t)kH2 * kH1) {  // W2b [128,128], W2T
    const int n = (int)(t / kH1), k = (int)(t % kH1);
    const uint16_t h = to_bf16(P[kOffW2 + t]);
    W2b[t] = h;
    W2T[(int64_t)k * kH2 + n] = h;
  }
  GS(t, (int64_t)kH3 * kH2) {  // W3b [64,128], W3T [128,64]
    const int n = (int)(t / kH2), k = (int)(t % kH2);
    const uint16_t h = to_bf16(P[kOffW3 + t]);
    W3b[t] = h;
    W3T[(int64_t)k * kH3 + n] = h;
  }
}

// gather the gradients into parameter order (dW1 [128,64] -> first 20 cols,
// dW3 arrives transposed [128,64]).
__global__ void mlp_gather_grad_kernel(const float* __restrict__ dW1, const float* __restrict__ db1,
                                       const float* __restrict__ dW2, const float* __restrict__ db2,
                                       const float* __restrict__ dW3T, const float* __restrict__ db3,
                                       const float* __restrict__ dw4, const float* __restrict__ db4,
                                       float* __restrict__ g) {
  GS(i, (int64_t)(kNParams - kNormN)) {
    const int j = (int)i + kNormN;
    float v;
    if (j < kOffB1) { const int q = j - kOffW1; v = dW1[(q / kF) * kK1 + q % kF]; }
    else if (j < kOffW2) v = db1[j - kOffB1];
    else if (j < kOffB2) v = dW2[j - kOffW2];
    else if (j < kOffW3) v = db2[j - kOffB2];
    else if (j < kOffB3) { const int q = j - kOffW3; v = dW3T[(q % kH2) * kH3 + q / kH2]; }
    else if (j < kOffW4) v = db3[j - kOffB3];
    else if (j < kOffB4) v = dw4[j - kOffW4];
    else v = db4[0];
    g[i] = v;
  }
}

__global__ void sum_kernel(const float* __restrict__ a, int n, float* __restrict__ out) {
  // one warp, fixed order per lane then a fixed tree
  float s = 0.0f;
  for (int i = threadIdx.x; i < n; i += 32) s += a[i];
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) *out = s;
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
};

namespace {
size_t carve_mlp(cbmv_mlp* n, char* base) {
  size_t off = 0;
  auto take = [&](size_t bytes) -> void* {
    off = (off + 255) & ~(size_t)255;
    void* p = base ? base + off : nullptr;
    off += bytes;
    return p;
  };
  const size_t B = (size_t)n->B;
  using namespace cbmv;
  n->P = (float*)take(sizeof(float) * kNParams);
  n->m = (float*)take(sizeof(float) * kNParams);
  n->v = (float*)take(sizeof(float) * kNParams);
  n->g = (float*)take(sizeof(float) * kNParams);
  n->W1b = (uint16_t*)take(2 * kH1 * kK1);
  n->W1T = (uint16_t*)take(2 * kH1 * kK1);
  n->W2b = (uint16_t*)take(2 * kH2 * kH1);
  n->W2T = (uint16_t*)take(2 * kH2 * kH1);
  n->W3b = (uint16_t*)take(2 * kH3 * kH2);
  n->W3T = (uint16_t*)take(2 * kH3 * kH2);
  n->X0 = (uint16_t*)take(2 * B * kK1);
  n->X0T = (uint16_t*)take(2 * B * kK1);
  n->A1 = (uint16_t*)take(2 * B * kH1);
  n->A1T = (uint16_t*)take(2 * B * kH1);
  n->A2 = (uint16_t*)take(2 * B * kH2);
  n->A2T = (uint16_t*)take(2 * B * kH2);
  n->dS3 = (uint16_t*)take(2 * B * kH3);
  n->dS3T = (uint16_t*)take(2 * B * kH3);
  n->dS2 = (uint16_t*)take(2 * B * kH2);
  n->dS2T = (uint16_t*)take(2 * B * kH2);
  n->dS1 = (uint16_t*)take(2 * B * kH1);
  n->dS1T = (uint16_t*)take(2 * B * kH1);
  n->Z = (float*)take(4 * B * 128);
  n->S1 = (float*)take(4 * B * kH1);
  n->S2 = (float*)take(4 * B * kH2);
  n->S3 = (float*)take(4 * B * kH3);
  n->A3f = (float*)take(4 * B * kH3);
  n->dA = (float*)take(4 * B * 128);
  n->dSf = (float*)take(4 * B * 128);
  n->loss_i = (float*)take(4 * B);
  n->dz = (float*)take(4 * B);
  n->dw4_i = (float*)take(4 * B * kH3);
  n->dW1 = (float*)take(4 * kH1 * kK1);
  n->dW2 = (float*)take(4 * kH2 * kH1);
  n->dW3T = (float*)take(4 * kH2 * kH3);
  n->db1 = (float*)take(4 * kH1);
  n->db2 = (float*)take(4 * kH2);
  n->db3 = (float*)take(4 * kH3);
  n->dw4 = (float*)take(4 * kH3);
  n->db4 = (float*)take(4 * 4);
  n->loss = (float*)take(4 * 4);
  n->status = (int*)take(4 * 4);
  return off + 256;
}
}  // namespace

using namespace cbmv;

extern "C" int cbmv_mlp_num_params(void) { return kNParams; }

extern "C" int cbmv_mlp_create(int batch, cbmv_mlp** out) {
  CBMV_REQUIRE(out, CBMV_EINVAL, "null pointer argument");
  CBMV_REQUIRE(batch >= 128 && batch % 128 == 0 && batch <= (1 << 22), CBMV_EINVAL,
               "batch must be a multiple of 128 in [128, 4194304]");
  cbmv_mlp* n = new cbmv_mlp();
  n->B = batch;
  const size_t bytes = carve_mlp(n, nullptr);
  cudaError_t e = cudaMalloc(&n->mem, bytes);
  if (e != cudaSuccess) {
    delete n;
    return set_error(CBMV_ENOMEM, "mlp workspace: %s", cudaGetErrorString(e));
  }
  carve_mlp(n, (char*)n->mem);
  if (cudaMemset(n->mem, 0, bytes) != cudaSuccess) {
    cudaFree(n->mem);
    delete n;
    return set_error(CBMV_ECUDA, "mlp workspace clear failed");
  }
  *out = n;
  return CBMV_OK;
}

extern "C" int cbmv_mlp_destroy(cbmv_mlp* n) {
  if (!n) return CBMV_OK;
  cudaDeviceSynchronize();
  cudaFree(n->mem);
  delete n;
  return CBMV_OK;
}

// Parameters in from / out to HOST memory (kNParams floats); setting them
// resets the optimiser state.
extern "C" int cbmv_mlp_set_params(cbmv_mlp* n, const float* host) {
  CBMV_REQUIRE(n && host, CBMV_EINVAL, "null pointer argument");
  CBMV_CUDA(cudaMemcpy(n->P, host, sizeof(float) * kNParams, cudaMemcpyHostToDevice));
  CBMV_CUDA(cudaMemset(n->m, 0, sizeof(float) * kNParams));
  CBMV_CUDA(cudaMemset(n->v, 0, sizeof(float) * kNParams));
  n->step = 0;
  mlp_pack_kernel<<<64, 256>>>(n->P, n->W1b, n->W1T, n->W2b, n->W2T, n->W3b, n->W3T);
  CBMV_CUDA(cudaDeviceSynchronize());
  return check_launch("mlp_pack");
}

extern "C" int cbmv_mlp_get_params(const cbmv_mlp* n, float* host) {
  CBMV_REQUIRE(n && host, CBMV_EINVAL, "null pointer argument");
  CBMV_CUDA(cudaMemcpy(host, n->P, sizeof(float) * kNParams, cudaMemcpyDeviceToHost));
  return CBMV_OK;
}

namespace {
// forward + backward on one batch; gradients land in n->g (parameter order)
int mlp_fwd_bwd(cbmv_mlp* n, const float* X, const float* y, cudaStream_t st) {
  const int B = n->B;
  const unsigned g = grid_for((int64_t)B * 128, 256);
  int rc;
  mlp_prep_kernel<<<g, 256, 0, st>>>(X, B, n->P, n->X0, n->X0T);
  if ((rc = launch_gemm_bf16(n->X0, n->W1b, n->Z, B, kH1, kK1, n->status, st))) return rc;
  mlp_bias_relu_kernel<<<g, 256, 0, st>>>(n->Z, n->P + kOffB1, B, kH1, n->S1, n->A1, n->A1T, nullptr);
  if ((rc = launch_gemm_bf16(n->A1, n->W2b, n->Z, B, kH2, kH1, n->status, st))) return rc;
  mlp_bias_relu_kernel<<<g, 256, 0, st>>>(n->Z, n->P + kOffB2, B, kH2, n->S2, n->A2, n->A2T, nullptr);
  if ((rc = launch_gemm_bf16(n->A2, n->W3b, n->Z, B, kH3, kH2, n->status, st))) return rc;
  mlp_bias_relu_kernel<<<g, 256, 0, st>>>(n->Z, n->P + kOffB3, B, kH3, n->S3, nullptr, nullptr, n->A3f);
  mlp_head_kernel<<<grid_for((int64_t)B * 32, 256), 256, 0, st>>>(n->A3f, n->S3, y, n->P, B, n->loss_i,
                                                                  n->dz, n->dw4_i, n->dS3, n->dS3T, n->dSf);
  mlp_colsum_kernel<<<1, 64, 0, st>>>(n->dw4_i, B, kH3, n->dw4);
  mlp_colsum_kernel<<<1, 64, 0, st>>>(n->dz, B, 1, n->db4);
  mlp_colsum_kernel<<<1, 64, 0, st>>>(n->dSf, B, kH3, n->db3);
  sum_kernel<<<1, 32, 0, st>>>(n->loss_i, B, n->loss);
  // layer 3: dW3^T = A2^T dS3, dA2 = dS3 W3
  if ((rc = launch_gemm_bf16(n->A2T, n->dS3T, n->dW3T, kH2, kH3, B, n->status, st))) return rc;
  if ((rc = launch_gemm_bf16(n->dS3, n->W3T, n->dA, B, kH2, kH3, n->status, st))) return rc;
  mlp_drelu_kernel<<<g, 256, 0, st>>>(n->dA, n->S2, B, kH2, n->dS2, n->dS2T, n->dSf);
  mlp_colsum_kernel<<<1, 128, 0, st>>>(n->dSf, B, kH2, n->db2);
  // layer 2: dW2 = dS2^T A1, dA1 = dS2 W2
  if ((rc = launch_gemm_bf16(n->dS2T, n->A1T, n->dW2, kH2, kH1, B, n->status, st))) return rc;
  if ((rc = launch_gemm_bf16(n->dS2, n->W2T, n->dA, B, kH1, kH2, n->status, st))) return rc;
  mlp_drelu_kernel<<<g, 256, 0, st>>>(n->dA, n->S1, B, kH1, n->dS1, n->dS1T, n->dSf);
  mlp_colsum_kernel<<<1, 128, 0, st>>>(n->dSf, B, kH1, n->db1);
  // layer 1: dW1 = dS1^T X0
  if ((rc = launch_gemm_bf16(n->dS1T, n->X0T, n->dW1, kH1, kK1, B, n->status, st))) return rc;
  mlp_gather_grad_kernel<<<64, 256, 0, st>>>(n->dW1, n->db1, n->dW2, n->db2, n->dW3T, n->db3, n->dw4,
                                             n->db4, n->g);
  return check_launch("mlp_fwd_bwd");
}
}  // namespace

// One Adam step on a batch of B samples: X float32 [B,20] raw CBMV features,
// y float32 [B] labels (1 = correct match), device memory.  loss (device,
// may be NULL) receives the batch's mean binary cross-entropy.
extern "C" int cbmv_mlp_train_step(cbmv_mlp* n, const float* X, const float* y, float lr,
                                   float weight_decay, float* loss, void* stream) {
  CBMV_REQUIRE(n && X && y, CBMV_EINVAL, "null pointer argument");
  cudaStream_t st = as_stream(stream);
  int rc = mlp_fwd_bwd(n, X, y, st);
  if (rc) return rc;
  n->step++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float bc1 = 1.0f - powf(b1, (float)n->step), bc2 = 1.0f - powf(b2, (float)n->step);
  mlp_adam_kernel<<<64, 256, 0, st>>>(n->P, n->m, n->v, n->g, lr, b1, b2, 1e-8f, bc1, bc2, weight_decay);
  mlp_pack_kernel<<<64, 256, 0, st>>>(n->P, n->W1b, n->W1T, n->W2b, n->W2T, n->W3b, n->W3T);
  if (loss) CBMV_CUDA(cudaMemcpyAsync(loss, n->loss, sizeof(float), cudaMemcpyDeviceToDevice, st));
  return check_launch("mlp_train_step");
}

// Gradients of the batch loss without an update (for checking): grads
// float32 [num_params - 60] in parameter order (the input transform has no
// gradient), loss float32 [1]; both device memory.
extern "C" int cbmv_mlp_gradients(cbmv_mlp* n, const float* X, const float* y, float* grads, float* loss,
                                  void* stream) {
  CBMV_REQUIRE(n && X && y && grads, CBMV_EINVAL, "null pointer argument");
  cudaStream_t st = as_stream(stream);
  int rc = mlp_fwd_bwd(n, X, y, st);
  if (rc) return rc;
  CBMV_CUDA(cudaMemcpyAsync(grads, n->g, sizeof(float) * (kNParams - kNormN), cudaMemcpyDeviceToDevice, st));
  if (loss) CBMV_CUDA(cudaMemcpyAsync(loss, n->loss, sizeof(float), cudaMemcpyDeviceToDevice, st));
  return CBMV_OK;
}

// Status of the tensor-core waits since creation (0 = fine).
extern "C" int cbmv_mlp_status(const cbmv_mlp* n, int* status) {
  CBMV_REQUIRE(n && status, CBMV_EINVAL, "null pointer argument");
  CBMV_CUDA(cudaMemcpy(status, n->status, sizeof(int), cudaMemcpyDeviceToHost));
  return CBMV_OK;
}

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
// Arithmetic, per layer (the float32 accumulator in tensor memory); every
// bias enters as bf16 high + low parts multiplied by constant ones:
//   layer 1  K = 32: 20 normalised features, two constant-one columns whose
//            weights are b1's parts, zeros;
//   layers 2, 3: a first K = 16 MMA of a constant tile (ones in columns 0
//            and 1) against b2's / b3's parts (stored in the unused K
//            columns 32..63 of layer 1's weight tile) initialises the
//            accumulator, the layer's MMAs accumulate onto it;
//   hidden activations: ReLU and the bf16 rounding in one instruction
//            (cvt.rn.relu.bf16x2.f32) per pair of columns;
//   output   layer 4 is an MMA too: N = 16, rows 0 and 1 of its weight tile
//            are the high and low bf16 parts of w4, z = D[0] + D[1] + b4,
//            cost = 1 - sigmoid(z) = 1 / (1 + exp(z)).
// The features themselves are formed in float32 (they enter the network as
// bf16), from float32 cost volumes and float32 row statistics (min, 1/den),
// with one reciprocal 1/(c + e) shared by the left and right ratio.
// ====================================================================
#include "features.cuh"

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
constexpr uint32_t kBf16OneOne = 0x3F803F80u;  // two bf16 ones

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

// Two float32 values as a packed bf16 pair (low = a), round to nearest even
__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
  const __nv_bfloat162 x = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&x);
}

// ReLU of two float32 pre-activations, as a packed bf16 pair (low = a),
// round to nearest even
__device__ __forceinline__ uint32_t relu_bf16x2(float a, float b) {
  uint32_t r;
  asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(b), "f"(a));
  return r;
}

// ratio and likelihood of cost c (featextract.cpp:333 and :440) in float32
// against its row statistics st = (min, 1/den); inv_ce = 1 / (c + e).
// expf (about 1 ulp over the whole range) rather than the approximate
// exponential, whose error grows with the argument (large for the census
// and NCC likelihoods far from the row minimum).
__device__ __forceinline__ void conf_f32(float c, float inv_ce, float2 st, float e, float inv_sigma,
                                         float* ratio, float* lik) {
  const float t = c - st.x;
  *ratio = st.x == kRandMaxF ? 0.0f : (st.x + e) * inv_ce;
  *lik = expf(-(t * t) * inv_sigma) * st.y;  // 1/den = 0 on sentinel rows
}

// bf16 high part of x and the bf16 rounding of the rest: x ~ hi + lo
__device__ __forceinline__ void split_bf16(float x, float* hi, float* lo) {
  *hi = __bfloat162float(__float2bfloat16_rn(x));
  *lo = x - *hi;
}

// Stage the inference weights from the float32 parameter vector, and the
// constant tile of the bias MMAs.
__device__ void stage_inference_weights(const float* __restrict__ P, unsigned char* sW1, unsigned char* sW2,
                                        unsigned char* sW3, unsigned char* sW4, unsigned char* sOne) {
  for (int q = threadIdx.x; q < 128 * 64; q += blockDim.x) {
    const int r = q >> 6, k = q & 63;
    float v = 0.0f, hi, lo;
    if (k < kF) {
      v = P[kOffW1 + r * kF + k];
    } else if (k == kF || k == kF + 1) {
      split_bf16(P[kOffB1 + r], &hi, &lo);
      v = k == kF ? hi : lo;
    } else if (k == kColB2 || k == kColB2 + 1) {
      split_bf16(P[kOffB2 + r], &hi, &lo);
      v = k == kColB2 ? hi : lo;
    } else if (r < kH3 && (k == kColB3 || k == kColB3 + 1)) {
      split_bf16(P[kOffB3 + r], &hi, &lo);
      v = k == kColB3 ? hi : lo;
    }
    *reinterpret_cast<uint16_t*>(sW1 + umma::sw128_offset(128, r, k)) = to_bf16(v);
    *reinterpret_cast<uint16_t*>(sOne + umma::sw128_offset(128, r, k)) = to_bf16(k < 2 ? 1.0f : 0.0f);
  }
  for (int q = threadIdx.x; q < 128 * 128; q += blockDim.x) {
    const int r = q >> 7, k = q & 127;
    *reinterpret_cast<uint16_t*>(sW2 + umma::sw128_offset(128, r, k)) = to_bf16(P[kOffW2 + q]);
  }
  for (int q = threadIdx.x; q < 64 * 128; q += blockDim.x) {
    const int r = q >> 7, k = q & 127;
    *reinterpret_cast<uint16_t*>(sW3 + umma::sw128_offset(64, r, k)) = to_bf16(P[kOffW3 + q]);
  }
  for (int q = threadIdx.x; q < 16 * 64; q += blockDim.x) {
    const int r = q >> 6, k = q & 63;
    float hi, lo;
    split_bf16(P[kOffW4 + k], &hi, &lo);
    *reinterpret_cast<uint16_t*>(sW4 + umma::sw128_offset(16, r, k)) = to_bf16(r == 0 ? hi : r == 1 ? lo : 0.0f);
  }
}

// Row `row` of a K-major SW128 activation tile: 16-byte chunk j (columns
// 8j .. 8j+7 of a 64-column atom) of atom a sits at
// rowp + a * 128 * 128 + ((j << 4) ^ r7s), r7s = (row % 8) << 4.
__device__ __forceinline__ uint4* tile_chunk(unsigned char* rowp, int r7s, int a, int j) {
  return reinterpret_cast<uint4*>(rowp + a * 128 * 128 + ((j << 4) ^ r7s));
}

// ReLU of 32 loaded accumulator columns c .. c+31 -> the activation tile
__device__ __forceinline__ void epilogue_chunk(unsigned char* rowp, int r7s, int c, const uint32_t* v) {
  uint32_t h[16];
#pragma unroll
  for (int i = 0; i < 16; i++) h[i] = relu_bf16x2(__uint_as_float(v[2 * i]), __uint_as_float(v[2 * i + 1]));
#pragma unroll
  for (int q = 0; q < 4; q++)
    *tile_chunk(rowp, r7s, c >> 6, ((c & 63) >> 3) + q) = make_uint4(h[4 * q], h[4 * q + 1], h[4 * q + 2], h[4 * q + 3]);
}

// One hidden-layer epilogue of this thread's row: accumulator columns
// 0 .. NC-1 -> ReLU as bf16 into the activation tile.  The load of the
// next 32 columns is in flight while the current ones are computed.
template <int NC>
__device__ __forceinline__ void epilogue_hidden(uint32_t tlane, unsigned char* rowp, int r7s) {
  uint32_t va[32], vb[32];
  umma::tmem_ld32_issue(tlane, va);
  umma::tmem_ld32_wait(va);
#pragma unroll
  for (int c = 0; c < NC; c += 64) {
    umma::tmem_ld32_issue(tlane + c + 32, vb);
    epilogue_chunk(rowp, r7s, c, va);
    umma::tmem_ld32_wait(vb);
    if (c + 64 < NC) umma::tmem_ld32_issue(tlane + c + 64, va);
    epilogue_chunk(rowp, r7s, c + 32, vb);
    if (c + 64 < NC) umma::tmem_ld32_wait(va);
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
  stage_inference_weights(P, sW1, sW2, sW3, sW4, sOne);
  for (int i = tid; i < kF; i += kInfThreads) s_nrm[i] = make_float4(P[i], P[kF + i], P[2 * kF + i], 0.0f);
  if (tid == 0) s_b4 = P[kOffB4];
  umma::fence_async_smem();
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();

  unsigned char* sA = sTiles + g * kSmTile;
  unsigned char* rowp = sA + (row >> 3) * 1024 + (row & 7) * 128;
  const int r7s = (row & 7) << 4;
  uint64_t* bar = &bars[g];
  const uint32_t tacc = tmem_base + (uint32_t)(g * 128);
  const uint32_t tlane = tacc + ((uint32_t)(wq * 32) << 16);
  const bool leader = row == 0;
  constexpr uint32_t id128 = umma::idesc_bf16(128, 128), id64 = umma::idesc_bf16(128, 64),
                     id16 = umma::idesc_bf16(128, 16);
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
  uint32_t phase = 0;
  bool ok = true;

  FeatIn in;
  load_feat_in(fv, statsf, HW, N, t, p, d, x, in);
  for (; tile < tiles; tile += tstride) {
    // 1. the 20 features of sample t -> row of X0 (the first atom of the tile):
    //    columns 0..19 in the reference's order, 20 and 21 the bias inputs, 22..31 zero
    {
      float f[20];
      features_f32(in, f);
      uint32_t u[10];
#pragma unroll
      for (int k = 0; k < 20; k += 2) {
        const float4 na = s_nrm[k], nb = s_nrm[k + 1];
        u[k >> 1] = pack_bf16x2((fminf(f[k], na.x) - na.y) * na.z, (fminf(f[k + 1], nb.x) - nb.y) * nb.z);
      }
      *tile_chunk(rowp, r7s, 0, 0) = make_uint4(u[0], u[1], u[2], u[3]);
      *tile_chunk(rowp, r7s, 0, 1) = make_uint4(u[4], u[5], u[6], u[7]);
      *tile_chunk(rowp, r7s, 0, 2) = make_uint4(u[8], u[9], kBf16OneOne, 0u);
      *tile_chunk(rowp, r7s, 0, 3) = make_uint4(0u, 0u, 0u, 0u);
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
    umma::fence_async_smem();
    umma::tc_fence_before();
    group_sync(g);
    umma::tc_fence_after();
    // 2. layer 1 (K = 32) -> accumulator columns 0..127
    if (leader) {
      const uint64_t dA0 = DESC(sA), dW1 = DESC(sW1);
      umma::mma_bf16(tacc, dA0, dW1, id128, false);
      umma::mma_bf16(tacc, dA0 + 2, dW1 + 2, id128, true);
      umma::mma_commit(bar);
    }
    ok = group_all(g, leader ? umma::mbar_wait(bar, phase, kWaitLimit) : true);
    phase ^= 1u;
    umma::tc_fence_after();
    if (!ok) break;
    epilogue_hidden<128>(tlane, rowp, r7s);
    umma::fence_async_smem();
    umma::tc_fence_before();
    group_sync(g);
    umma::tc_fence_after();
    // 3. layer 2 (K = 128) onto the bias b2
    if (leader) {
      const uint64_t dA0 = DESC(sA), dA1 = DESC(sA + 128 * 128), dW20 = DESC(sW2), dW21 = DESC(sW2 + 128 * 128);
      umma::mma_bf16(tacc, DESC(sOne), DESC(sW1) + 2 * (kColB2 / 16), id128, false);
#pragma unroll
      for (int kk = 0; kk < 4; kk++) umma::mma_bf16(tacc, dA0 + 2 * kk, dW20 + 2 * kk, id128, true);
#pragma unroll
      for (int kk = 0; kk < 4; kk++) umma::mma_bf16(tacc, dA1 + 2 * kk, dW21 + 2 * kk, id128, true);
      umma::mma_commit(bar);
    }
    ok = group_all(g, leader ? umma::mbar_wait(bar, phase, kWaitLimit) : true);
    phase ^= 1u;
    umma::tc_fence_after();
    if (!ok) break;
    epilogue_hidden<128>(tlane, rowp, r7s);
    umma::fence_async_smem();
    umma::tc_fence_before();
    group_sync(g);
    umma::tc_fence_after();
    // 4. layer 3 (N = 64) onto the bias b3
    if (leader) {
      const uint64_t dA0 = DESC(sA), dA1 = DESC(sA + 128 * 128), dW30 = DESC(sW3), dW31 = DESC(sW3 + 64 * 128);
      umma::mma_bf16(tacc, DESC(sOne), DESC(sW1) + 2 * (kColB3 / 16), id64, false);
#pragma unroll
      for (int kk = 0; kk < 4; kk++) umma::mma_bf16(tacc, dA0 + 2 * kk, dW30 + 2 * kk, id64, true);
#pragma unroll
      for (int kk = 0; kk < 4; kk++) umma::mma_bf16(tacc, dA1 + 2 * kk, dW31 + 2 * kk, id64, true);
      umma::mma_commit(bar);
    }
    ok = group_all(g, leader ? umma::mbar_wait(bar, phase, kWaitLimit) : true);
    phase ^= 1u;
    umma::tc_fence_after();
    if (!ok) break;
    epilogue_hidden<64>(tlane, rowp, r7s);
    umma::fence_async_smem();
    umma::tc_fence_before();
    group_sync(g);
    umma::tc_fence_after();
    // 5. output layer (N = 16, rows 0/1 = high/low parts of w4) -> columns 64..79
    if (leader) {
      const uint64_t dA0 = DESC(sA), dW4 = DESC(sW4);
#pragma unroll
      for (int kk = 0; kk < 4; kk++) umma::mma_bf16(tacc + 64, dA0 + 2 * kk, dW4 + 2 * kk, id16, kk > 0);
      umma::mma_commit(bar);
    }
    ok = group_all(g, leader ? umma::mbar_wait(bar, phase, kWaitLimit) : true);
    phase ^= 1u;
    umma::tc_fence_after();
    if (!ok) break;
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
  if (!ok) {
    // let this group's MMAs still in flight finish (bounded) before the memory is freed
    if (leader) {
      atomicExch(status, 1);
      umma::mbar_wait(bar, phase ^ 1u, kWaitLimit);
    }
  }
  umma::tc_fence_before();
  __syncthreads();
  if (tid < 32) umma::tmem_dealloc(tmem_base, 128 * kGroups);
#undef DESC
}

}  // namespace

int launch_features_f32_gather(const float* const* vols, const float2* statsf, int64_t H, int64_t W, int D,
                               const int64_t* idx, int64_t n, float* out, cudaStream_t st) {
  FeatVolsF fv = {{vols[0], vols[1], vols[2], vols[3]}};
  const int64_t blocks = (n + 255) / 256;
  features_f32_gather_kernel<<<(unsigned)(blocks < 65535 * 16 ? blocks : 65535 * 16), 256, 0, st>>>(
      fv, statsf, H, W, D, idx, n, out);
  return check_launch("features_f32_gather");
}

int launch_features_mlp(const float* const* vols, const float2* statsf, int64_t H, int64_t W, int D,
                        const cbmv_mlp* m, float* prob0, cudaStream_t st, int max_ctas) {
  int dev = 0, sms = 0;
  CBMV_CUDA(cudaGetDevice(&dev));
  CBMV_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  CBMV_CUDA(cudaFuncSetAttribute(features_mlp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kSmInf));
  CBMV_REQUIRE(((uintptr_t)statsf & 7) == 0, CBMV_EINVAL, "feature statistics must be 8-byte aligned");
  const int64_t tiles = (H * W * D + 127) / 128;
  const int64_t need = (tiles + kGroups - 1) / kGroups;
  const int cap = max_ctas > 0 && max_ctas < sms ? max_ctas : sms;
  const int grid = (int)(need < cap ? need : cap);
  FeatVolsF fv = {{vols[0], vols[1], vols[2], vols[3]}};
  features_mlp_kernel<<<grid, kInfThreads, kSmInf, st>>>(fv, statsf, H, W, D, m->P, prob0, m->status);
  return check_launch("features_mlp");
}

}  // namespace cbmv
