// Tensor-core MTTKRP (tcgen05) -- placeholder until the kernel lands.
#include "kernels.cuh"

namespace cud {

int mttkrp_tc_query(int, const long *, int, long, int, size_t *) { return CUD_ERR_UNSUPPORTED; }

int mttkrp_tc(const float *, int, const long *, const float *const *, int, long, float *, int,
              void *, cudaStream_t) {
    return CUD_ERR_UNSUPPORTED;
}

}  // namespace cud
