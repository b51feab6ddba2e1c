// Mixed-precision getrates (built in a later step).
#include <cuda_runtime.h>

#include "dev_mech.cuh"

namespace cg {
struct MixedPlan {
    int dummy;
};
cudaError_t mixed_prepare(const DevMech&, const cg_mech_view&, int, MixedPlan** out) {
    *out = nullptr;
    return cudaErrorNotSupported;
}
void mixed_release(MixedPlan* p) { delete p; }
cudaError_t launch_getrates_mixed(const MixedPlan*, const DevMech&, const double*, const double*, const double*,
                                  double*, int64_t, void*, size_t, cudaStream_t) {
    return cudaErrorNotSupported;
}
size_t mixed_workspace_bytes(const MixedPlan*, int64_t) { return 0; }
}  // namespace cg
