// Mixed-precision (BF16 tensor-core) evaluation path.
#include "eval_common.cuh"

namespace dpb {
int mixed_supported(const DevModel &) { return 0; }
size_t mixed_workspace_per_atom(const DevModel &) { return 0; }
int mixed_eval(const DevModel &, const SysDesc &, const float *, const int32_t *, const float *, const int32_t *,
               double *, float *, float4 *, double *, void *, cudaStream_t) {
  return DPB_ERR_UNSUPPORTED;
}
}  // namespace dpb
