// Mixed-precision form of the two-site update (placeholder until the
// tensor-core contraction lands): reports that it is not built.
#include "mpsb_common.cuh"

namespace mpsb {
int launch_update2q_mixed(const mpsb_chain *, const mpsb_pair *, int, const double2 *, int, double, int, void *,
                          double *, int32_t *, double *, int32_t *, cudaStream_t) {
    return set_error(MPSB_EINVAL, "mixed-precision update not available in this build");
}
}  // namespace mpsb
