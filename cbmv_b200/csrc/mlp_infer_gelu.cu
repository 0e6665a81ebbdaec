// The fused features + network kernel with GELU hidden layers, f16 operands.
#include "mlp_infer.cuh"

namespace cbmv {

int launch_features_mlp_gelu(const float* const* vols, const float2* statsf, int64_t H, int64_t W, int D,
                             const cbmv_mlp* m, float* prob0, cudaStream_t st, int max_ctas) {
  return launch_features_mlp_act<CBMV_ACT_GELU, true>(vols, statsf, H, W, D, m, prob0, st, max_ctas);
}

}  // namespace cbmv
