// Tensor-core trailing update for the FP32 LU (placeholder until the
// tcgen05 kernel lands): reports FH_ERR_UNSUPPORTED so that no caller can
// mistake the SIMT path for it.
#include "fh_lu.cuh"

namespace fhb {

fh_status gemm_tc_update(float *, int64_t, int, int64_t, int, cudaStream_t, fh_error_info *err) {
    return fail(err, FH_ERR_UNSUPPORTED, "tensor-core trailing update not built");
}

}  // namespace fhb
