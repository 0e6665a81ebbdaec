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
#include "mlp_net.cuh"
#include "umma.cuh"

namespace cbmv {
namespace {

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

// S = Z + b; A = act(S) as bf16 [B,N] and [N,B]; Af = act(S) float (optional)
__global__ void mlp_bias_act_kernel(const float* __restrict__ Z, const float* __restrict__ bias, int B,
                                    int N, int act, float* __restrict__ S, uint16_t* __restrict__ A,
                                    uint16_t* __restrict__ AT, float* __restrict__ Af) {
  GS(t, (int64_t)B * N) {
    const int b = (int)(t / N), n = (int)(t % N);
    const float s = Z[t] + bias[n];
    S[t] = s;
    const float a = act_t(act, s, nullptr);
    if (A) A[t] = to_bf16(a);
    if (AT) AT[(int64_t)n * B + b] = to_bf16(a);
    if (Af) Af[t] = a;
  }
}

// output layer, loss and the first backward step, one warp per sample:
// z = A3 . w4 + b4, p = sigmoid(z), loss_i = BCE; dz = (p - y) / B;
// dS3 = dz * w4 * act'(S3) -> bf16 [B,64] and [64,B]; per-sample dz and
// dz*A3 kept for the (ordered) reductions of dw4 / db4.
__global__ void mlp_head_kernel(const float* __restrict__ A3f, const float* __restrict__ S3,
                                const float* __restrict__ y, const float* __restrict__ P, int B, int act,
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
      act_t(act, S3[(int64_t)b * kH3 + k], &dg);
      const float d = g * P[kOffW4 + k] * dg;
      dS3[(int64_t)b * kH3 + k] = to_bf16(d);
      dS3T[(int64_t)k * B + b] = to_bf16(d);
      dS3f[(int64_t)b * kH3 + k] = d;
      dw4_i[(int64_t)b * kH3 + k] = g * a[k];
    }
  }
}

// dS = dA * act'(S) -> bf16 [B,N], [N,B] and float [B,N]
__global__ void mlp_dact_kernel(const float* __restrict__ dA, const float* __restrict__ S, int B, int N, int act,
                                 uint16_t* __restrict__ dS, uint16_t* __restrict__ dST,
                                 float* __restrict__ dSf) {
  GS(t, (int64_t)B * N) {
    const int b = (int)(t / N), n = (int)(t % N);
    float dg;
    act_t(act, S[t], &dg);
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
  mlp_bias_act_kernel<<<g, 256, 0, st>>>(n->Z, n->P + kOffB1, B, kH1, n->act, n->S1, n->A1, n->A1T, nullptr);
  if ((rc = launch_gemm_bf16(n->A1, n->W2b, n->Z, B, kH2, kH1, n->status, st))) return rc;
  mlp_bias_act_kernel<<<g, 256, 0, st>>>(n->Z, n->P + kOffB2, B, kH2, n->act, n->S2, n->A2, n->A2T, nullptr);
  if ((rc = launch_gemm_bf16(n->A2, n->W3b, n->Z, B, kH3, kH2, n->status, st))) return rc;
  mlp_bias_act_kernel<<<g, 256, 0, st>>>(n->Z, n->P + kOffB3, B, kH3, n->act, n->S3, nullptr, nullptr, n->A3f);
  mlp_head_kernel<<<grid_for((int64_t)B * 32, 256), 256, 0, st>>>(n->A3f, n->S3, y, n->P, B, n->act, n->loss_i,
                                                                  n->dz, n->dw4_i, n->dS3, n->dS3T, n->dSf);
  mlp_colsum_kernel<<<1, 64, 0, st>>>(n->dw4_i, B, kH3, n->dw4);
  mlp_colsum_kernel<<<1, 64, 0, st>>>(n->dz, B, 1, n->db4);
  mlp_colsum_kernel<<<1, 64, 0, st>>>(n->dSf, B, kH3, n->db3);
  sum_kernel<<<1, 32, 0, st>>>(n->loss_i, B, n->loss);
  // layer 3: dW3^T = A2^T dS3, dA2 = dS3 W3
  if ((rc = launch_gemm_bf16(n->A2T, n->dS3T, n->dW3T, kH2, kH3, B, n->status, st))) return rc;
  if ((rc = launch_gemm_bf16(n->dS3, n->W3T, n->dA, B, kH2, kH3, n->status, st))) return rc;
  mlp_dact_kernel<<<g, 256, 0, st>>>(n->dA, n->S2, B, kH2, n->act, n->dS2, n->dS2T, n->dSf);
  mlp_colsum_kernel<<<1, 128, 0, st>>>(n->dSf, B, kH2, n->db2);
  // layer 2: dW2 = dS2^T A1, dA1 = dS2 W2
  if ((rc = launch_gemm_bf16(n->dS2T, n->A1T, n->dW2, kH2, kH1, B, n->status, st))) return rc;
  if ((rc = launch_gemm_bf16(n->dS2, n->W2T, n->dA, B, kH1, kH2, n->status, st))) return rc;
  mlp_dact_kernel<<<g, 256, 0, st>>>(n->dA, n->S1, B, kH1, n->act, n->dS1, n->dS1T, n->dSf);
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

extern "C" int cbmv_mlp_set_activation(cbmv_mlp* n, int act) {
  CBMV_REQUIRE(n, CBMV_EINVAL, "null pointer argument");
  CBMV_REQUIRE(act == CBMV_ACT_RELU || act == CBMV_ACT_GELU, CBMV_EINVAL, "unknown activation %d", act);
  n->act = act;
  return CBMV_OK;
}

extern "C" int cbmv_mlp_set_precision(cbmv_mlp* n, int prec) {
  CBMV_REQUIRE(n, CBMV_EINVAL, "null pointer argument");
  CBMV_REQUIRE(prec == CBMV_PREC_F16 || prec == CBMV_PREC_BF16, CBMV_EINVAL, "unknown precision %d", prec);
  n->prec = prec;
  return CBMV_OK;
}

extern "C" int cbmv_mlp_get_precision(const cbmv_mlp* n, int* prec) {
  CBMV_REQUIRE(n && prec, CBMV_EINVAL, "null pointer argument");
  *prec = n->prec;
  return CBMV_OK;
}

extern "C" int cbmv_mlp_get_activation(const cbmv_mlp* n, int* act) {
  CBMV_REQUIRE(n && act, CBMV_EINVAL, "null pointer argument");
  *act = n->act;
  return CBMV_OK;
}

// Status of the tensor-core waits since creation (0 = fine).
extern "C" int cbmv_mlp_status(const cbmv_mlp* n, int* status) {
  CBMV_REQUIRE(n && status, CBMV_EINVAL, "null pointer argument");
  CBMV_CUDA(cudaMemcpy(status, n->status, sizeof(int), cudaMemcpyDeviceToHost));
  return CBMV_OK;
}
