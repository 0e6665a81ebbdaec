// The fused features + network kernel with ReLU hidden layers and f16
// operands, the learned path's feature read-back (cbmv_ctx_features_f32_at)
// and the dispatch on the network's activation and precision (one
// instantiation per translation unit, so that none changes how the
// compiler allocates another's registers).
#include "mlp_infer.cuh"

namespace cbmv {

int launch_features_mlp_gelu(const float* const* vols, const float2* statsf, int64_t H, int64_t W, int D,
                             const cbmv_mlp* m, float* prob0, cudaStream_t st, int max_ctas);
int launch_features_mlp_gelu_bf16(const float* const* vols, const float2* statsf, int64_t H, int64_t W, int D,
                                  const cbmv_mlp* m, float* prob0, cudaStream_t st, int max_ctas);
int launch_features_mlp_relu_bf16(const float* const* vols, const float2* statsf, int64_t H, int64_t W, int D,
                                  const cbmv_mlp* m, float* prob0, cudaStream_t st, int max_ctas);

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
  if (m->prec == CBMV_PREC_BF16) {
    if (m->act == CBMV_ACT_GELU)
      return launch_features_mlp_gelu_bf16(vols, statsf, H, W, D, m, prob0, st, max_ctas);
    return launch_features_mlp_relu_bf16(vols, statsf, H, W, D, m, prob0, st, max_ctas);
  }
  if (m->act == CBMV_ACT_GELU) return launch_features_mlp_gelu(vols, statsf, H, W, D, m, prob0, st, max_ctas);
  return launch_features_mlp_act<CBMV_ACT_RELU, true>(vols, statsf, H, W, D, m, prob0, st, max_ctas);
}

}  // namespace cbmv
