// Split-BF16 contraction on tcgen05 (placeholder until the tensor-core kernel lands).
#include "ks_common.cuh"
#include "project.cuh"

namespace ks {
int gemm_bf16x3(const __nv_bfloat16*, const __nv_bfloat16*, const __nv_bfloat16*,
                const __nv_bfloat16*, float*, int64_t, int64_t, int64_t, int64_t,
                int64_t, int64_t, bool, cudaStream_t) {
  return fail(KS_ERR_UNSUPPORTED, "split-BF16 projection not built yet");
}
}  // namespace ks
