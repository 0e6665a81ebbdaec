// The fused features + network kernel with ReLU hidden layers, bf16 operands.
#include "mlp_infer.cuh"

namespace cbmv {

int launch_features_mlp_relu_bf16(const float* const* vols, const float2* statsf, int64_t H, int64_t W, int D,
                                  const cbmv_mlp* m, float* prob0, cudaStream_t st, int max_ctas) {
  return launch_features_mlp_act<CBMV_ACT_RELU, false>(vols, statsf, H, W, D, m, prob0, st, max_ctas);
}

}  // namespace cbmv
